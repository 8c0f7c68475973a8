// FP32 instantiation of the fused kernels (FMA contraction allowed).
#include "fused_impl.cuh"

#include <atomic>

namespace mpdx {
int fused3d_bulk_copies(int mode) {
  static std::atomic<int> m{1};
  return mode < 0 ? m.load() : m.exchange(mode != 0 ? 1 : 0);
}
int fused3d_planes_setting(int lx) {
  static std::atomic<int> m{0};
  if (lx < 0) return m.load();
  if (lx != 0 && (lx < 8 || lx > 512 || lx % 4)) return -1;
  return m.exchange(lx);
}
copy_wait_word &fused_copy_wait_flag() {
  static copy_wait_word w;
  return w;
}

template bool fused_configurable<float>(const mpdata_state<float> &);
template void fused3d_launch<float>(mpdata_state<float> &, int, cudaStream_t, int);
template void fused2d_plan_init<float>(const mpdata_state<float> &, fused2d_plan<float> &);
template void fused2d_launch<float>(const mpdata_state<float> &, const fused2d_plan<float> &, int, cudaStream_t);
template bool fused_seams_consistent<float>(mpdata_state<float> &, double *);
template int fused2d_batched<float>(int, int, bool, bool, const f2::prob<float> *, const f2::item *, int, int *, int,
                                     cudaStream_t, bool);
}  // namespace mpdx
