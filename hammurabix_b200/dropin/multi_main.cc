// multi_main.cc -- hamx_b200_multi: runs several parameter files, one
// after another, each through a fresh Pipeline (source/pipeline/pipeline.cc)
// in one process, the way a sampling loop in C++ rebuilds the Pipeline for
// every parameter set.  The device handle of the drop-in integrator is made
// once and kept across the runs; each run's Grid_* arrays are compared with
// what the device slots hold by content (dropin_common.h), so a new
// Pipeline never integrates a previous run's grid.
//
//   hamx_b200_multi params_1.xml [params_2.xml ...]
#include <cstdlib>
#include <iostream>
#include <memory>
#include <string>

#include <pipeline.h>

int main(int argc, char **argv) {
  if (argc < 2) {
    std::cerr << "usage: hamx_b200_multi <XML parameter file> [more files ...]" << std::endl;
    return EXIT_FAILURE;
  }
  for (int i = 1; i < argc; ++i) {
    auto run = std::make_unique<Pipeline>(std::string(argv[i]));
    run->assemble_grid();
    run->assemble_tereg();
    run->assemble_breg();
    run->assemble_ternd();
    run->assemble_brnd();
    run->assemble_cre();
    run->assemble_obs();
  }
  return EXIT_SUCCESS;
}
