// Batched persistent launch of the fused 2D MPDATA kernel over many
// independent problems: tile candidates, work lists and the launcher's
// declaration (definition in fused_impl.cuh).
//
// A work item is one strip (the columns one warp writes) x LX rows of one
// problem; a grid of resident warps (SM count x occupancy) takes items from a
// counter in global memory until the list is exhausted.  Results do not depend
// on the tile shape: every output point goes through the same arithmetic
// whatever strip or row chunk computes it, so the tile can be chosen by timing.
#pragma once

#include <algorithm>
#include <vector>

#include "fused2d_warp.cuh"

namespace mpdx {

// candidates of the autotuner: threads per item (one warp), rows per item, and the
// share of the resident CTAs the persistent grid launches (occ_div 1: every CTA
// the SMs can hold; 2: half of them, fewer warps contending for the issue slots);
// each is timed over kTuneSteps steps
struct batch_tile {
  int nt, lx, occ_div;
};
constexpr int kNumBatchTiles = 8;
constexpr int kTuneSteps = 3;
constexpr batch_tile kBatchTiles[kNumBatchTiles] = {{32, 16, 1}, {32, 32, 1}, {32, 64, 1}, {32, 128, 1},
                                                    {32, 16, 2}, {32, 32, 2}, {32, 64, 2}, {32, 128, 2}};

// launch (or, with occ, return the resident CTAs per SM of) tile candidate
// `tile` of the persistent kernel; instantiated per real type in fused_f32.cu /
// fused_f64.cu (the FP64 one without FMA contraction)
template <class T>
int fused2d_batched(int tile, int ni, bool iga, bool fct, const f2::prob<T> *probs, const f2::item *items, int n_items,
                    int *counter, int grid, cudaStream_t s, bool occ);

// work list of tile candidate `tile` for problems of periods (P0, P1); larger
// problems first so that the tail of the list holds the small items
inline std::vector<f2::item> fused2d_batch_items(int tile, int ni, const std::vector<int> &P0, const std::vector<int> &P1) {
  const int TJ = ni == 3 ? f2w::shape<3>::WV : f2w::shape<2>::WV, LX = kBatchTiles[tile].lx;
  std::vector<int> order(P0.size());
  for (size_t p = 0; p < order.size(); ++p) order[p] = int(p);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return (long long)P0[a] * P1[a] > (long long)P0[b] * P1[b]; });
  std::vector<f2::item> items;
  for (int p : order)
    for (int x0 = 0; x0 < P0[p]; x0 += LX)
      for (int j0 = 0; j0 < P1[p]; j0 += TJ) items.push_back({p, j0, x0, std::min(x0 + LX, P0[p])});
  return items;
}

}  // namespace mpdx
