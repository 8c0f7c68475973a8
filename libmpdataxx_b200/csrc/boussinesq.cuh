// Boussinesq solver with GCR pressure solve (declarations).
#pragma once

#include "state.cuh"

namespace mpdx {

template <class T>
struct boussinesq {
  mpdata_state<T> st;
  field<T> tht_e;
  double dt = 0;
  int ix_tht = 0;
  long long iters = 0, iters_total = 0;
  double last_residual = 0;
  boussinesq(const mpdx_config &, cudaStream_t) {
    throw error(MPDX_E_UNSUPPORTED, "Boussinesq solver not built yet");
  }
  field<T> *phi_field() { return nullptr; }
  void advance(long long) {}
};

}  // namespace mpdx
