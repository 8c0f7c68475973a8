// Learned preconditioner for the GCR pressure solve: a linear 4-level 3D
// U-net (see precond.cu for the architecture), with its forward pass,
// backward pass and Adam training on the GPU.
#pragma once

#include <cstdint>
#include <vector>

#include "mpdx_common.cuh"

namespace mpdx {
namespace pc {

constexpr int kLevels = 4;
constexpr int kLayers = 9;  // e0 e1 e2 e3 m3 d2 d1 d0 q

struct lvl {
  int n[3];
  long long vox;
};

// One network instance: parameters (FP32 master copy + BF16 tensor-core
// fragments), Adam state and the activations of one forward pass.
class net {
 public:
  // grid: points per axis (nd = 2 or 3); wrap[d]: 1 for a cyclic axis (wrapped
  // padding), 0 for zero padding; ch: channels of levels 0..3 (multiples of 8, <= 64)
  net(int nd, const int *grid, const int *wrap, const int *ch, uint64_t seed, cudaStream_t s);
  ~net();
  net(const net &) = delete;
  net &operator=(const net &) = delete;

  int nd, ntaps, ch[kLevels], wrap[3];
  lvl L[kLevels];
  long long n_params = 0;
  cudaStream_t stream;

  // parameter layout: per layer W (cout, ntaps, cin) then b (cout), layers in order
  long long w_off[kLayers], b_off[kLayers];
  int cin[kLayers], cout[kLayers], level[kLayers];

  void set_params(const float *host);
  void get_params(float *host);
  // forward from a residual r (device): an FP64 field in halo layout (element
  // strides s0, s1, s2; q written with the same layout) or a compact FP32 array
  void forward_field(const double *r, long long s0, long long s1, long long s2, const double *unused,
                     double *q, const int *skip_flag);
  void forward_compact(const float *r, float *q);
  // gradient of sum(dq * q) for the last forward_compact(r), into grad (device, n_params)
  void backward(const float *r, const float *dq, float *grad);
  // one Adam step on the mean squared error between forward_compact(r) and target
  double train_step(const float *r, const float *target, float lr);
  void sync_weights();  // FP32 master -> BF16 fragments
  void adam_step(float lr);  // one Adam step with the gradient in `grad`

  float *params = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  long long adam_t = 0;

 private:
  uint16_t *wf[kLayers] = {}, *wtf[kLayers] = {};  // forward / adjoint fragments (tensor-core layers)
  // activations (BF16, channels-last) and gradients (FP32)
  uint16_t *a_e[4] = {}, *a_p[4] = {}, *a_m3 = nullptr, *a_d[3] = {}, *a_u[3] = {};
  float *q32 = nullptr, *dq32 = nullptr, *g_a = nullptr, *g_b = nullptr, *g_c = nullptr;
  uint16_t *g_h = nullptr;
  float *part = nullptr;
  double *loss_dev = nullptr;
  unsigned char *wmask = nullptr;
  size_t part_floats = 0;
  void alloc_all();
};

}  // namespace pc
}  // namespace mpdx
