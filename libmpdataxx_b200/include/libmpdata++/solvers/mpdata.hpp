// solvers::mpdata<ct_params_t> (libmpdata++/solvers/mpdata.hpp:24-54): the
// solver type of the API.  On this backend the solver's arithmetic runs in
// the CUDA library; the type carries the compile-time parameters, the
// run-time parameter struct and the C-ABI solver kind.
#pragma once

#include <array>
#include <limits>
#include <mpdx.h>

#include "../opts.hpp"

namespace libmpdataxx {
namespace solvers {

enum rhs_scheme_t { euler_a, euler_b, trapez, mixed };  // mpdata_rhs.hpp:19-25
enum prs_scheme_t { mr, cr, pc, gcrk };                  // mpdata_rhs_vip_prs.hpp:17-30
enum vip_vab_t { noab, expl, impl };                     // mpdata_rhs_vip_common.hpp:16-21

template <class ct_params_t>
struct mpdata {
  using ct_params_t_ = ct_params_t;
  using real_t = typename ct_params_t::real_t;
  enum { n_dims = ct_params_t::n_dims };
  enum { n_eqns = ct_params_t::n_eqns };
  static constexpr int solver_kind = MPDX_SOLVER_MPDATA;
  static_assert(!ct_params_t::var_dt, "var_dt is not built on this backend");

  // solver_common.hpp:217-221 and mpdata_common.hpp:74-78
  struct rt_params_t {
    std::array<int, n_dims> grid_size;
    real_t dt = 0, max_abs_div_eps = std::numeric_limits<real_t>::epsilon(), max_courant = real_t(0.5);
    real_t di = 0, dj = 0, dk = 0;
    int n_iters = 2;
    int upwind_filter_freq = 0;
  };

  static void fill(mpdx_config &c, const rt_params_t &) { c.solver = MPDX_SOLVER_MPDATA; }
};

}  // namespace solvers
}  // namespace libmpdataxx
