// pspin_mc: drop-in for the reference's pspin24 (montecarlo.cu).
#include "common.h"

int main(int argc, char** argv) { return mc_main(argc, argv); }
