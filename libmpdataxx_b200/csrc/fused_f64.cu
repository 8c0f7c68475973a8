// FP64 instantiation of the fused kernels, compiled without FMA contraction so
// that it reproduces the reference-structured path (and the reference) bitwise.
#include "fused_impl.cuh"

namespace mpdx {
template bool fused_configurable<double>(const mpdata_state<double> &);
template void fused3d_launch<double>(mpdata_state<double> &, int, cudaStream_t, int);
template void fused2d_plan_init<double>(const mpdata_state<double> &, fused2d_plan<double> &);
template void fused2d_launch<double>(const mpdata_state<double> &, const fused2d_plan<double> &, int, cudaStream_t);
template bool fused_seams_consistent<double>(mpdata_state<double> &, double *);
template int fused2d_batched<double>(int, int, bool, bool, const f2::prob<double> *, const f2::item *, int, int *, int,
                                     cudaStream_t, bool);
}  // namespace mpdx
