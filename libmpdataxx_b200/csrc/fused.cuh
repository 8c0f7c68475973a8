// Fused MPDATA step kernels (declarations).
#pragma once

#include "state.cuh"

namespace mpdx {

template <class T>
struct fused_engine {
  void init(const mpdata_state<T> &) {}
  bool configurable(const mpdata_state<T> &) const { return false; }
  bool seams_consistent(const mpdata_state<T> &, double *) { return false; }
  void invalidate() {}
  void step(mpdata_state<T> &) { throw error(MPDX_E_UNSUPPORTED, "fused path not built"); }
};

}  // namespace mpdx
