// Problem and work-item descriptors of the fused 2D MPDATA kernels
// (fused2d_warp.cuh): one 2D problem (input and output time levels, the two
// Courant-number components, periods and sizes) and one work item of the
// batched launch (problem, strip origin, row range).
#pragma once

#include "fused3d.cuh"

namespace mpdx {
namespace f2 {

template <class T>
struct prob {  // one 2D problem
  dfield<T> in, out, g0, g1;
  int P0, P1;  // periods
  int n0, n1;  // points per axis
};

// work item of the batched launch: problem, strip origin and row range
struct item {
  int prob, j0, x0, x1;
};

}  // namespace f2
}  // namespace mpdx
