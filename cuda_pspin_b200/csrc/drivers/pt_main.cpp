// pspin_pt: drop-in for the reference's parallel_tempering (parallel_tempering.cu).
#include "common.h"

int main(int argc, char** argv) { return pt_main(argc, argv, PSPIN_DENSE); }
