// FP32 instantiation of the fused kernels (FMA contraction allowed).
#include "fused_impl.cuh"

namespace mpdx {
template bool fused_configurable<float>(const mpdata_state<float> &);
template void fused3d_launch<float>(mpdata_state<float> &, int, cudaStream_t);
template void fused2d_plan_init<float>(const mpdata_state<float> &, fused2d_plan<float> &);
template void fused2d_launch<float>(const mpdata_state<float> &, const fused2d_plan<float> &, int, cudaStream_t);
template bool fused_seams_consistent<float>(mpdata_state<float> &, double *);
template int fused2d_batched<float>(int, int, bool, bool, const f2::prob<float> *, const f2::item *, int, int *, int,
                                     cudaStream_t, bool);
}  // namespace mpdx
