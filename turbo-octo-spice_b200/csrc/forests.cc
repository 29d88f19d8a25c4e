// forests.cc — the engine's sightlines and pixels from forests as the
// reference's loader reads them from a delta file's `lines_of_sight` group
// (HDF5Delta::loadForests, HDF5Delta.cc:40-93), for callers that read the
// groups with their own HDF5 (or other) reader.  Host code only.
//
// What the loader does with what it reads, restated:
//  - groups in increasing name order (H5Literate with H5_INDEX_NAME,
//    H5_ITER_INC: byte-wise name order);
//  - a pixel is kept when its delta and weight are finite and the weight is
//    positive, in the order stored, as ForestPixel {delta, loglam, weight,
//    r_comov} (HDF5Delta.cc:74-79);
//  - a forest with no pixel left is dropped; the others are numbered 0, 1, ...
//    in that order (forest_id; h5healxi.cc:203 bins them under that number);
//  - ra and dec go to the Forest as stored (the reference takes them as
//    radians), with the plate attribute.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/tos_b200.h"

namespace tos {
tos_status fail(tos_status s, const std::string& msg);  // engine.cu: sets tos_last_error()
}

extern "C" tos_status tos_forests_assemble(const tos_forest* forests, size_t n_forests, tos_sightline* los,
                                           size_t los_capacity, size_t* n_los, tos_pixel* pixels,
                                           size_t pixel_capacity, size_t* n_pixels) {
  if (!n_los || !n_pixels) return tos::fail(TOS_ERR_INVALID_ARG, "n_los/n_pixels is null");
  if (n_forests && !forests) return tos::fail(TOS_ERR_INVALID_ARG, "forests is null");
  for (size_t f = 0; f < n_forests; ++f) {
    const tos_forest& x = forests[f];
    if (!x.name) return tos::fail(TOS_ERR_INVALID_ARG, "forest " + std::to_string(f) + " has no name");
    if (x.n && (!x.delta || !x.weight || !x.r_comov || !x.loglam))
      return tos::fail(TOS_ERR_INVALID_ARG, "forest " + std::to_string(f) + " has a null dataset");
  }
  std::vector<size_t> order(n_forests);
  std::iota(order.begin(), order.end(), size_t(0));
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return std::strcmp(forests[a].name, forests[b].name) < 0;
  });
  auto keep = [](const tos_forest& x, uint64_t i) {
    return std::isfinite(x.delta[i]) && std::isfinite(x.weight[i]) && x.weight[i] > 0;
  };
  size_t nl = 0, np = 0;
  for (size_t f : order) {
    size_t k = 0;
    for (uint64_t i = 0; i < forests[f].n; ++i) k += keep(forests[f], i) ? 1 : 0;
    if (k > 0xFFFFFFFFull) return tos::fail(TOS_ERR_UNSUPPORTED, "a forest keeps more than 2^32 - 1 pixels");
    if (k) {
      ++nl;
      np += k;
    }
  }
  *n_los = nl;
  *n_pixels = np;
  if (!los || !pixels) return TOS_OK;  // size query
  if (los_capacity < nl || pixel_capacity < np)
    return tos::fail(TOS_ERR_INVALID_ARG, "capacity too small: need " + std::to_string(nl) + " sightlines and " +
                                              std::to_string(np) + " pixels");
  size_t s = 0, p = 0;
  for (size_t f : order) {
    const tos_forest& x = forests[f];
    const size_t first = p;
    for (uint64_t i = 0; i < x.n; ++i)
      if (keep(x, i)) pixels[p++] = tos_pixel{x.delta[i], x.loglam[i], x.weight[i], x.r_comov[i]};
    if (p == first) continue;
    tos_sightline& l = los[s];
    l.ra = x.ra;
    l.dec = x.dec;
    l.forest_id = (int32_t)s;
    l.plate = x.plate;
    l.pixel_offset = first;
    l.num_pixels = (uint32_t)(p - first);
    l.group = 0;
    ++s;
  }
  return TOS_OK;
}
