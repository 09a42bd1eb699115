// pspin_sa: drop-in for the reference's simulated_annealing (simulated_annealing.cu).
#include "common.h"

int main(int argc, char** argv) { return sa_main(argc, argv); }
