// Fused MPDATA step: engine interface (kernels in fused3d.cuh / fused2d.cuh,
// instantiated in fused_f32.cu and fused_f64.cu).
//
// The fused kernels assume the reference's cyclic convention on every axis:
// point n-1 duplicates point 0 in the advectee and in every transverse axis of
// each advector component.  When the fields satisfy it, the fused step equals
// the reference's step bitwise (FP64) and the engine takes it; otherwise the
// solver runs the reference-structured kernels (both paths are CUDA).
#pragma once

#include <vector>

#include "fused2d.cuh"
#include "state.cuh"

namespace mpdx {

// launchers (one translation unit per real type)
// one step of equation e with `lx` planes per CTA (0: the default of the type)
template <class T> void fused3d_launch(mpdata_state<T> &st, int e, cudaStream_t s, int lx);
template <class T> struct fused2d_plan;
template <class T> void fused2d_plan_init(const mpdata_state<T> &st, fused2d_plan<T> &p);
template <class T> void fused2d_launch(const mpdata_state<T> &st, const fused2d_plan<T> &p, int e, cudaStream_t s);
template <class T> bool fused_seams_consistent(mpdata_state<T> &st, double *scratch);
template <class T> bool fused_configurable(const mpdata_state<T> &st);

// The plane copies of the fused FP32 3D kernel, process-wide: 1 (the default)
// bulk-tensor copies in the CTAs whose tile lies inside the periods along j and
// k, 0 per-thread copies everywhere; a negative mode only queries.  Returns the
// mode before the call.
int fused3d_bulk_copies(int mode);
// The host-mapped status word of those bulk copies: a completion wait that gave
// up sets *host (both null until the first launch that uses bulk copies).
struct copy_wait_word {
  unsigned *host = nullptr, *dev = nullptr;
};
copy_wait_word &fused_copy_wait_flag();
// Planes per CTA of the fused 3D kernel, process-wide: 0 (the default) lets each
// handle tune it on its first fused steps, a positive value (a multiple of 4 from
// 8 to 512) fixes it; a negative value only queries.  Returns the setting before
// the call; an invalid value changes nothing and returns -1.
int fused3d_planes_setting(int lx);

// 2D step descriptor of equation e whose input is time level tl
template <class T>
f2::prob<T> fused2d_prob(const mpdata_state<T> &st, int e, int tl) {
  f2::prob<T> a;
  a.in = st.psi[e][tl].v;
  a.out = st.psi[e][tl ^ 1].v;
  a.g0 = st.GC[0].v; a.g1 = st.GC[1].v;
  a.P0 = st.n[0] - 1; a.P1 = st.n[1] - 1;
  a.n0 = st.n[0]; a.n1 = st.n[1];
  return a;
}

// Device-resident work plan of the 2D kernel for one solver.  The fields never
// move after setup, so descriptors and work list are written once.
template <class T>
struct fused2d_plan {
  f2::prob<T> *probs = nullptr;  // step descriptors, [equation][input time level]
  f2::item *items = nullptr;     // strips x row chunks of the problem (problem index 0)
  int *counter = nullptr;        // work counter and finished warps, re-armed by the kernel
  int n_items = 0, grid = 0;

  fused2d_plan() = default;
  fused2d_plan(const fused2d_plan &) = delete;
  fused2d_plan &operator=(const fused2d_plan &) = delete;
  ~fused2d_plan() {
    if (probs) cudaFree(probs);
    if (items) cudaFree(items);
    if (counter) cudaFree(counter);
  }
};

template <class T>
struct fused_engine {
  int known = -1;  // cached seam check: -1 unknown, 0 inconsistent, 1 consistent
  fused2d_plan<T> plan2;
  // chunk-length tuner of the 3D kernel: its first fused step runs untimed with the
  // default, then every candidate runs kTune3 timed steps (each step synchronises
  // on its end), then the fastest is kept.  The planes per CTA change only which
  // CTA computes a point, not how, so every candidate gives the same fields.
  static constexpr int kNumCand3 = 8, kTune3 = 2;
  static constexpr int kCand3[kNumCand3] = {24, 32, 40, 48, 64, 80, 96, 128};
  int lx3 = 0;        // chosen planes per CTA (0 while tuning)
  int tune_pos = -1;  // -1 before the untimed step, then timed steps so far
  float tune_ms[kNumCand3] = {};
  cudaEvent_t ev[2] = {nullptr, nullptr};

  fused_engine() = default;
  fused_engine(const fused_engine &) = delete;
  fused_engine &operator=(const fused_engine &) = delete;
  ~fused_engine() {
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
  }

  void init(const mpdata_state<T> &st) {
    if (st.nd == 2) fused2d_plan_init(st, plan2);
  }

  static bool configurable(const mpdata_state<T> &st) { return fused_configurable(st); }

  bool seams_consistent(mpdata_state<T> &st, double *scratch) {
    if (known < 0) known = fused_seams_consistent(st, scratch) ? 1 : 0;
    return known == 1;
  }
  void invalidate() { known = -1; }

  void step(mpdata_state<T> &st) {
    if (st.nd != 3) {
      for (int e = 0; e < st.n_eqns; ++e) {
        fused2d_launch(st, plan2, e, st.stream);
        st.tl[e] ^= 1;
      }
      return;
    }
    const int fixed = fused3d_planes_setting(-1);
    if (fixed > 0 || lx3 > 0 || tune_pos < 0) {
      launch3d(st, fixed > 0 ? fixed : lx3);
      if (fixed <= 0 && tune_pos < 0) tune_pos = 0;
      return;
    }
    const int c = tune_pos / kTune3;
    if (!ev[0]) {
      MPDX_CUDA(cudaEventCreate(&ev[0]));
      MPDX_CUDA(cudaEventCreate(&ev[1]));
    }
    MPDX_CUDA(cudaEventRecord(ev[0], st.stream));
    launch3d(st, kCand3[c]);
    MPDX_CUDA(cudaEventRecord(ev[1], st.stream));
    MPDX_CUDA(cudaEventSynchronize(ev[1]));
    float ms = 0.f;
    MPDX_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    tune_ms[c] += ms / float(kTune3);
    if (++tune_pos == kNumCand3 * kTune3) {
      int best = 0;
      for (int q = 1; q < kNumCand3; ++q)
        if (tune_ms[q] < tune_ms[best]) best = q;
      lx3 = kCand3[best];
    }
  }

 private:
  void launch3d(mpdata_state<T> &st, int lx) {
    for (int e = 0; e < st.n_eqns; ++e) {
      fused3d_launch(st, e, st.stream, lx);
      st.tl[e] ^= 1;
    }
  }
};

}  // namespace mpdx
