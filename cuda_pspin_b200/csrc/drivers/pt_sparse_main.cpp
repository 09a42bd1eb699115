// pspin_pt_sparse: drop-in for the reference's parallel_tempering_sparse
// (parallel_tempering_sparse.cu).
#include "common.h"

int main(int argc, char** argv) { return pt_main(argc, argv, PSPIN_SPARSE); }
