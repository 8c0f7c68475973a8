// C ABI of the preconditioner network on its own (include/mpdx.h, mpdx_pcnet_*):
// creation, parameters, forward / backward on host arrays and training steps.
// It serves the gradient checks against the CPU oracle and users who train or
// inspect the network outside a solver.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "precond.cuh"

struct mpdx_pcnet {
  cudaStream_t stream = nullptr;
  std::unique_ptr<mpdx::pc::net> n;
  std::string err;
  float *r = nullptr, *q = nullptr, *t = nullptr;
  ~mpdx_pcnet() {
    n.reset();
    for (float *p : {r, q, t}) if (p) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {
thread_local std::string g_pc_create_error;
template <class F>
mpdx_status pc_guard(mpdx_pcnet_handle h, F f) {
  if (!h || !h->n) return MPDX_E_ARG;
  try {
    f();
    h->err.clear();
    return MPDX_OK;
  } catch (const mpdx::error &e) {
    h->err = e.what();
    return e.code;
  } catch (const std::exception &e) {
    h->err = e.what();
    return MPDX_E_ARG;
  }
}
}  // namespace

extern "C" {

mpdx_status mpdx_pcnet_create(int nd, const int *grid, const int *wrap, const int *channels, uint64_t seed,
                              mpdx_pcnet_handle *out) {
  g_pc_create_error.clear();
  if (!grid || !wrap || !channels || !out) { g_pc_create_error = "null argument"; return MPDX_E_ARG; }
  *out = nullptr;
  try {
    auto h = std::make_unique<mpdx_pcnet>();
    MPDX_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->n.reset(new mpdx::pc::net(nd, grid, wrap, channels, seed, h->stream));
    const size_t vox = size_t(h->n->L[0].vox);
    MPDX_CUDA(cudaMalloc(&h->r, vox * sizeof(float)));
    MPDX_CUDA(cudaMalloc(&h->q, vox * sizeof(float)));
    MPDX_CUDA(cudaMalloc(&h->t, vox * sizeof(float)));
    *out = h.release();
    return MPDX_OK;
  } catch (const mpdx::error &e) {
    g_pc_create_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_pc_create_error = e.what();
    return MPDX_E_ARG;
  }
}

const char *mpdx_pcnet_create_error(void) { return g_pc_create_error.c_str(); }

int64_t mpdx_pcnet_num_params(mpdx_pcnet_handle h) { return (h && h->n) ? h->n->n_params : -1; }

mpdx_status mpdx_pcnet_set_params(mpdx_pcnet_handle h, const float *host) {
  return pc_guard(h, [&] { h->n->set_params(host); });
}
mpdx_status mpdx_pcnet_get_params(mpdx_pcnet_handle h, float *host) {
  return pc_guard(h, [&] { h->n->get_params(host); });
}

mpdx_status mpdx_pcnet_forward(mpdx_pcnet_handle h, const float *r_host, float *q_host) {
  return pc_guard(h, [&] {
    const size_t vox = size_t(h->n->L[0].vox);
    MPDX_CUDA(cudaMemcpyAsync(h->r, r_host, vox * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    h->n->forward_compact(h->r, h->q);
    MPDX_CUDA(cudaMemcpyAsync(q_host, h->q, vox * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MPDX_CUDA(cudaStreamSynchronize(h->stream));
  });
}

mpdx_status mpdx_pcnet_backward(mpdx_pcnet_handle h, const float *r_host, const float *dq_host, float *grad_host) {
  return pc_guard(h, [&] {
    const size_t vox = size_t(h->n->L[0].vox);
    MPDX_CUDA(cudaMemcpyAsync(h->r, r_host, vox * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MPDX_CUDA(cudaMemcpyAsync(h->t, dq_host, vox * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    h->n->forward_compact(h->r, h->q);
    h->n->backward(h->r, h->t, h->n->grad);
    MPDX_CUDA(cudaMemcpyAsync(grad_host, h->n->grad, size_t(h->n->n_params) * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MPDX_CUDA(cudaStreamSynchronize(h->stream));
  });
}

mpdx_status mpdx_pcnet_train_step(mpdx_pcnet_handle h, const float *r_host, const float *target_host, float lr,
                                  double *loss) {
  return pc_guard(h, [&] {
    const size_t vox = size_t(h->n->L[0].vox);
    MPDX_CUDA(cudaMemcpyAsync(h->r, r_host, vox * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MPDX_CUDA(cudaMemcpyAsync(h->t, target_host, vox * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    const double l = h->n->train_step(h->r, h->t, lr);
    if (loss) *loss = l;
  });
}

const char *mpdx_pcnet_last_error(mpdx_pcnet_handle h) { return (h && h->n) ? h->err.c_str() : "invalid network"; }

void mpdx_pcnet_destroy(mpdx_pcnet_handle h) { delete h; }

}  // extern "C"
