// Reference-structured MPDATA path (declarations; kernels in general.cu).
#pragma once

#include "state.cuh"

namespace mpdx {

template <class T>
struct general {
  mpdata_state<T> *s = nullptr;

  explicit general(mpdata_state<T> *st) : s(st) {}

  // hook_ante_loop chain: along-halo fill of GC, divergence check (throws
  // MPDX_E_DIVERGENT), normal-halo fill (solver_common.hpp:191-211,
  // solver_2d.hpp:279-293, mpdata_osc_2d.hpp:40-67).  dev_scratch: one double.
  void ante_loop(double *dev_scratch);
  // G = 1 everywhere (nug option), before the user sets g_factor()
  void init_g();
  // one time step of every equation (solver_common.hpp:127-136, 321-331)
  void step();
  // nt steps of a small cyclic 1D problem (one equation; no fct, dfl, nug or
  // divergence form) in one launch of one block, with step()'s arithmetic
  bool block1d_ok() const;
  void block1d(long long nt);

  // halo exchanges (solver_{1,2,3}d.hpp)
  void xchng_sclr(field<T> &A, int ex, bool deriv = false);
  void xchng_vctr_alng(field<T> *AV, bool ad = false, bool cyclic = false);
  void xchng_vctr_nrml(field<T> *AV, int ex);
  void fill_sclr(int d, int side, field<T> &A, rng rb, rng rc, bool deriv = false);
  void fill_vctr_nrml(int d, int side, field<T> &A, rng rb, rng rc);
  void fill_vctr_alng(int d, int side, field<T> *AV, rng rb, rng rc, bool ad, bool cyclic_only);
  // pressure-solver exchanges (solver_{2,3}d.hpp xchng_pres / set_edges / xchng_flux)
  void xchng_pres(field<T> &A, int ex);
  void set_edges(field<T> *const *AV);
  void xchng_flux(field<T> *AV);
  void fill_pres(int d, int side, field<T> &A, rng rb, rng rc);
  void set_edge_pres(int d, int side, field<T> &A, rng rb, rng rc);
  void fill_flux(int d, int side, field<T> *AV, rng rb, rng rc);
  bool any_rigid() const;

 private:
  int cur_e = 0;  // equation whose advop is running (the divergence form reads its other time level)
  field<T> *GC_unco(int iter);
  field<T> *GC_corr(int iter);
  field<T> *GCit(int iter);
  template <int ND> void antidiff_nd(field<T> *res, field<T> &psi, field<T> *G);
  template <int ND> void fluxes_nd(field<T> *F, field<T> &psi, field<T> *C, bool extended);
  template <int ND> void fct_adjust_nd(int e, int iter);
  template <int ND> void advop_nd(int e);
};

extern template struct general<float>;
extern template struct general<double>;

}  // namespace mpdx
