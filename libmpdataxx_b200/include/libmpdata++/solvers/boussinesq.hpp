// solvers::boussinesq<ct_params_t> (libmpdata++/solvers/boussinesq.hpp:20-52)
// with explicit buoyancy (boussinesq_expl.hpp) or, with ct_params_t::impl_tht,
// the implicit theta-perturbation form (boussinesq_impl.hpp), the velocity
// absorber ct_params_t::vip_vab (noab, expl, impl), trapezoidal right-hand-side
// coupling and the GCR pressure solve.  ct_params_t::ix names the equation
// indices (u, [v,] w, tht and vip_i/vip_j/[vip_k]).
#pragma once

#include "mpdata.hpp"

namespace libmpdataxx {
namespace solvers {

template <class ct_params_t>
struct boussinesq {
  using ct_params_t_ = ct_params_t;
  using real_t = typename ct_params_t::real_t;
  using ix = typename ct_params_t::ix;
  enum { n_dims = ct_params_t::n_dims };
  enum { n_eqns = ct_params_t::n_eqns };
  static constexpr int solver_kind = MPDX_SOLVER_BOUSSINESQ;
  static_assert(ct_params_t::rhs_scheme == trapez, "only the trapez rhs scheme is built on this backend");
  static_assert(ct_params_t::prs_scheme == cr || ct_params_t::prs_scheme == gcrk,
                "only the cr / gcrk pressure schemes are built on this backend");

  struct rt_params_t : mpdata<ct_params_t>::rt_params_t {
    real_t prs_tol = real_t(1e-7);   // mpdata_rhs_vip_prs_common.hpp:193-196
    real_t g = real_t(9.81), Tht_ref = 0, hflux_const = 0;  // boussinesq_common.hpp:32-35
    int precond = MPDX_PRECOND_IDENTITY;  // MPDX_PRECOND_LEARNED selects the learned preconditioner
    bool prs_fp64 = false;
  };

  static void fill(mpdx_config &c, const rt_params_t &p) {
    c.solver = MPDX_SOLVER_BOUSSINESQ;
    c.prs_scheme = ct_params_t::prs_scheme == cr ? MPDX_PRS_CR : MPDX_PRS_GCRK;
    c.prs_k_iters = ct_params_t::prs_k_iters;
    c.prs_tol = double(p.prs_tol);
    c.g = double(p.g);
    c.tht_ref = double(p.Tht_ref);
    c.ix_u = ix::vip_i;
    if (n_dims == 3) {
      c.ix_v = vip_j_of<ix>();
      c.ix_w = vip_k_of<ix>();
    } else {
      c.ix_v = -1;
      c.ix_w = vip_j_of<ix>();
    }
    c.ix_tht = ix::tht;
    c.precond = p.precond;
    c.prs_fp64 = p.prs_fp64 ? 1 : 0;
    c.impl_tht = ct_params_t::impl_tht ? 1 : 0;
    c.vip_vab = int(ct_params_t::vip_vab);  // noab 0, expl 1, impl 2 as MPDX_VAB_*
  }
  static constexpr bool has_vab = ct_params_t::vip_vab != 0;

 private:
  template <class I> static constexpr int vip_j_of() { return I::vip_j; }
  template <class I, class = void> struct has_k { static constexpr int v = -1; };
  template <class I> static constexpr int vip_k_of() { return k_of<I>(0); }
  template <class I> static constexpr auto k_of(int) -> decltype(int(I::vip_k)) { return I::vip_k; }
  template <class I> static constexpr int k_of(long) { return -1; }
};

}  // namespace solvers
}  // namespace libmpdataxx
