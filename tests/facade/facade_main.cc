// facade_main.cc — drives the C++ XiEstimator facade the way h5healxi drives
// the reference's class (h5healxi.cc:279-290): read a catalogue, run with
// do_cov, save the results and subsamples.  Used by tests/test_facade_gpu.py.
//
// usage: facade_main <catalogue.bin> <grid type 0|1|2> <axis1> <axis2> <axis3>
//                    <scale> <healpix order> <output base>
// catalogue.bin: uint64 n_sightlines, then per sightline double ra, dec,
// uint32 n_pixels, then n_pixels x (float value, loglam, weight, distance).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "../../turbo-octo-spice_b200/csrc/xi_estimator.h"

int main(int argc, char** argv) {
  if (argc != 9) {
    std::cerr << "usage: facade_main cat.bin type axis1 axis2 axis3 scale order outbase\n";
    return 2;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  uint64_t n = 0;
  if (std::fread(&n, 8, 1, f) != 1) return 2;
  std::vector<tos::Forest> los(n);
  for (uint64_t s = 0; s < n; ++s) {
    uint32_t np = 0;
    if (std::fread(&los[s].ra, 8, 1, f) != 1 || std::fread(&los[s].dec, 8, 1, f) != 1 ||
        std::fread(&np, 4, 1, f) != 1)
      return 2;
    los[s].forest_id = (int)s;
    los[s].plate = 0;
    los[s].pixels.resize(np);
    if (np && std::fread(los[s].pixels.data(), sizeof(tos::ForestPixel), np, f) != np) return 2;
  }
  std::fclose(f);
  try {
    const tos::TwoPointGrid grid((tos_coord_type)std::atoi(argv[2]), tos::Axis::parse(argv[3]),
                                 tos::Axis::parse(argv[4]), tos::Axis::parse(argv[5]));
    const auto type = (tos::XiEstimator::BinningCoordinateType)std::atoi(argv[2]);
    tos::XiEstimator xi(std::atof(argv[6]), grid, type, los, std::atoi(argv[7]));
    xi.run(0, true);
    xi.save_results(argv[8]);
    xi.save_subsamples(argv[8]);
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
