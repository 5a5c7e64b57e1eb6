// Force-included into the reference sources when they are compiled for the
// oracle harness: Printing() (src/Sampling.cpp:55) writes below
// DSMC_RESULTS_DIRECTORY, which the harness sets at run time.
// TEST INFRASTRUCTURE ONLY.
#pragma once
const char *dsmc_ref_results_dir();
#define DSMC_RESULTS_DIRECTORY dsmc_ref_results_dir()
