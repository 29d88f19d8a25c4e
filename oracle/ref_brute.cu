// ref_brute.cu — C entry point around the reference's bruteGPU
// (gpu/brute.cu:63-225), built unchanged for sm_100a into
// oracle/_ref/libtosref_brute.so by oracle/Makefile (target `ref`).
//
// TEST INFRASTRUCTURE ONLY: bench.py's reference arm for the brute-force
// workload times it; the engine never loads it.  bruteGPU takes the five
// point columns as vectors of double, splits them into chunks of
// `chunksize` rows, and for every chunk pair (i, j <= i) copies both chunks
// to the device and runs histo_kernel with FP32 shared-memory histograms; it
// returns xi per bin (sum of w w d d over sum of w w, FP32 accumulation).
// It prints progress on stdout, which this wrapper sends to /dev/null for
// the duration of the call.  On a CUDA error the reference calls exit().
#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <iostream>
#include <vector>

#include "brute.h"

extern "C" int tosref_brute(const float* points, size_t n, double min, double max, int nbins, long chunksize,
                            double* xi_out) {
  // histo_kernel keeps nbins + 2 bins in a 256-entry histogram (gpu/brute.cu:148-150).
  if (nbins < 1 || nbins + 2 > 256 || chunksize < 1 || n == 0) return -1;
  std::vector<std::vector<double> > columns(5);
  for (int c = 0; c < 5; ++c) columns[c].reserve(n + chunksize);
  for (size_t k = 0; k < n; ++k)
    for (int c = 0; c < 5; ++c) columns[c].push_back(points[5 * k + c]);
  std::vector<double> xi;
  std::cout.flush();
  std::fflush(stdout);
  const int saved = dup(1);
  const int devnull = open("/dev/null", O_WRONLY);
  if (saved >= 0 && devnull >= 0) dup2(devnull, 1);
  bruteGPU(columns, min, max, nbins, xi, chunksize);
  std::cout.flush();
  std::fflush(stdout);
  if (saved >= 0) {
    dup2(saved, 1);
    close(saved);
  }
  if (devnull >= 0) close(devnull);
  for (int b = 0; b < nbins && b < static_cast<int>(xi.size()); ++b) xi_out[b] = xi[b];
  return static_cast<int>(xi.size());
}
