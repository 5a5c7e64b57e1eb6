// dsmc - the solver's command-line program (src/main.cpp:3-6), on the GPU.
#include "../../include/dsmc_reference_api.h"

int main(int argc, char **argv) { return RunSimulation(argc, argv); }
