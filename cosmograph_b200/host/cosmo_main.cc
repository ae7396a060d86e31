// cosmo_main.cc -- config-file driver: `cosmo_b200 <config file>`, the
// reference's `cosmo <config file>` (cosmo.cc:26-96) on the B200 path.
#include <cstdlib>
#include <iostream>

#include "cosmo_b200.hpp"

int main(int argc, char** argv) {
  if (argc != 2) {
    std::cout << "Error: please supply exactly one config filename as an argument.\n";
    return EXIT_FAILURE;
  }
  return cosmo::run_config_file(argv[1]);
}
