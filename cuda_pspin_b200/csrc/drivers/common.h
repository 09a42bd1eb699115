// common.h -- the drop-in drivers (parallel_tempering, parallel_tempering_sparse,
// pspin24/montecarlo) on top of the C ABI.
#pragma once

#include "pspin.h"

// parallel_tempering.cu:33-529 / parallel_tempering_sparse.cu (variant)
int pt_main(int argc, char** argv, int variant);
// montecarlo.cu:23-231
int mc_main(int argc, char** argv);
// simulated_annealing.cu:30-314; extension: -batch K samples in one engine
int sa_main(int argc, char** argv);
