// Fused MPDATA step: engine interface (kernels in fused3d.cuh / fused2d.cuh,
// instantiated in fused_f32.cu and fused_f64.cu).
//
// The fused kernels assume the reference's cyclic convention on every axis:
// point n-1 duplicates point 0 in the advectee and in every transverse axis of
// each advector component.  When the fields satisfy it, the fused step equals
// the reference's step bitwise (FP64) and the engine takes it; otherwise the
// solver runs the reference-structured kernels (both paths are CUDA).
#pragma once

#include "state.cuh"

namespace mpdx {

// launchers (one translation unit per real type)
template <class T> void fused3d_launch(mpdata_state<T> &st, int e, cudaStream_t s);
template <class T> void fused2d_launch(mpdata_state<T> &st, int e, cudaStream_t s);
template <class T> bool fused_seams_consistent(mpdata_state<T> &st, double *scratch);
template <class T> bool fused_configurable(const mpdata_state<T> &st);

template <class T>
struct fused_engine {
  int known = -1;  // cached seam check: -1 unknown, 0 inconsistent, 1 consistent

  void init(const mpdata_state<T> &) {}

  static bool configurable(const mpdata_state<T> &st) { return fused_configurable(st); }

  bool seams_consistent(mpdata_state<T> &st, double *scratch) {
    if (known < 0) known = fused_seams_consistent(st, scratch) ? 1 : 0;
    return known == 1;
  }
  void invalidate() { known = -1; }

  void step(mpdata_state<T> &st) {
    for (int e = 0; e < st.n_eqns; ++e) {
      if (st.nd == 3) fused3d_launch(st, e, st.stream);
      else fused2d_launch(st, e, st.stream);
      st.tl[e] ^= 1;
    }
  }
};

}  // namespace mpdx
