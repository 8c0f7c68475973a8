// Device-resident state of one MPDATA solver: the fields of
// libmpdata++'s sharedmem (psi[e][tlev], GC, tmp arrays, FCT work arrays),
// allocated with the reference's halo ranges so that the reference-structured
// kernels can index them exactly as the formulae do.
#pragma once

#include <array>
#include <vector>

#include "mpdx_common.cuh"

namespace mpdx {

template <class T>
struct mpdata_state {
  int nd = 1, n[3] = {1, 1, 1}, H = 1, n_eqns = 1, n_iters = 2;
  unsigned opts = o_iga | o_fct;
  int bcs[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  T max_abs_div_eps = 0;
  rng ir[3], im[3];
  std::vector<std::array<field<T>, 2>> psi;
  std::vector<int> tl;  // time level of psi[e] holding the current state
  field<T> GC[3], tmp0[3], tmp1[3], flux[3], GC_mono[3];
  field<T> psi_min, psi_max, beta_up, beta_dn;
  field<T> G;                  // G factor with the nug option (sharedmem G); unallocated otherwise
  int upwind_filter_freq = 0;  // rt_params (mpdata_common.hpp:77): upwind-only step every n-th step
  int sptl_intrp = 0;          // ct_params_t::sptl_intrp of the div_3rd spatial terms: exact 0, aver2 1, aver4 2
  cudaStream_t stream = nullptr;
  long long timestep = 0;

  // halo depth: formulae::mpdata::halo (formulae_mpdata_common.hpp:50-59), >= 2 with fct
  static int halo_of(unsigned o) {
    int h = (o & (o_tot | o_dfl | o_div_2nd | o_div_3rd | o_div_3rd_dt)) ? 2 : 1;
    if (o & o_fct) h = h > 2 ? h : 2;
    return h;
  }
  rng sr(int d) const { return d < nd ? ext(ir[d], H) : rng{0, 0}; }
  template <class U> void alloc_sclr(field<U> &f) { rng r[3] = {sr(0), sr(1), sr(2)}; f.alloc(nd, r, stream); }
  void alloc_vctr(field<T> *v) {
    for (int c = 0; c < nd; ++c) {
      rng r[3] = {sr(0), sr(1), sr(2)};
      r[c] = ext(exh(ir[c]), H - 1);  // i^h^(halo-1)  (solver_common.hpp:370-371)
      v[c].alloc(nd, r, stream);
    }
  }

  void setup(int nd_, const int *n_, int n_eqns_, unsigned opts_, int n_iters_, const int bcs_[6]) {
    nd = nd_; n_eqns = n_eqns_; opts = opts_; n_iters = n_iters_;
    for (int d = 0; d < 3; ++d) n[d] = d < nd ? n_[d] : 1;
    for (int d = 0; d < nd; ++d) bcs[d][0] = bcs_[2 * d], bcs[d][1] = bcs_[2 * d + 1];
    H = halo_of(opts);
    for (int d = 0; d < 3; ++d) {
      ir[d] = {0, n[d] - 1};
      im[d] = d < nd ? rng{-1, n[d] - 1} : rng{0, 0};
    }
    psi.resize(n_eqns);
    tl.assign(n_eqns, 0);
    for (auto &p : psi) for (auto &a : p) alloc_sclr(a);
    alloc_vctr(GC); alloc_vctr(tmp0); alloc_vctr(flux);
    if (n_iters > 2) alloc_vctr(tmp1);
    if (opts & o_fct) {
      alloc_sclr(psi_min); alloc_sclr(psi_max); alloc_sclr(beta_up); alloc_sclr(beta_dn);
      alloc_vctr(GC_mono);
    }
    if (opts & o_nug) alloc_sclr(G);  // set to 1 by general<T>::init_g
  }

  long long cells() const { return (long long)n[0] * n[1] * n[2]; }
  // advector view extents (sharedmem.hpp:431-456, 543-577)
  void advector_extent(int d, int ex[3]) const {
    for (int q = 0; q < 3; ++q) ex[q] = n[q];
    if (d > 0) ex[0] = n[0] + 1;
  }
};

}  // namespace mpdx
