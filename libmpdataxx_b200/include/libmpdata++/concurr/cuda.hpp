// concurr::cuda<solver_t, bcxl, bcxr[, bcyl, bcyr[, bczl, bczr]]>: the B200
// backend of the libmpdata++ run API (header-only; links libmpdx.so).
//
// Drop-in for concurr::{serial,openmp,threads} (concurr/detail/concurr_common.hpp:122-454):
//
//   using run_t = concurr::cuda<solvers::mpdata<ct_params_t>, bcond::cyclic, bcond::cyclic>;
//   typename run_t::rt_params_t p;  p.grid_size = {601};
//   run_t run(p);
//   run.advectee() = [](int i) { return i <= 75 || i >= 125 ? 2. : 4.; };
//   run.advector() = -.75;
//   run.advance(1200);
//
// Fields live on the device.  advectee()/advector()/sclr_array() return
// writable views of host mirrors: a mirror is downloaded when first handed
// out after a step, and a mirror handed out since the last advance() is
// uploaded before the next one, so writes through a view behave as writes
// into the reference's Blitz++ views (write through a view obtained after the
// last advance(): a mirror not handed out again is not uploaded again).
// min(0)/max(0) come from the device-side statistics.  Data otherwise leaves
// the GPU only when a view is requested.
// Hooks run on the host once per step (rank 0 only: there is one GPU).
#pragma once

#include <algorithm>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include <mpdx.h>

#include "../bcond/bcond.hpp"
#include "../opts.hpp"
#include "../output/hdf5_xdmf.hpp"
#include "any.hpp"

namespace libmpdataxx {
namespace concurr {

namespace detail {
// exception text of each status, as the reference throws them
inline void check(mpdx_handle h, mpdx_status rc) {
  if (rc == MPDX_OK) return;
  switch (rc) {
    case MPDX_E_GRID: throw std::runtime_error("libmpdata++: bogus grid size");
    case MPDX_E_DIVERGENT: throw std::runtime_error("libmpdata++: initial advector field is divergent");
    case MPDX_E_PRS_STUCK: throw std::runtime_error("libmpdata++: stuck in pressure solver");
    default: throw std::runtime_error(std::string("libmpdata++ (cuda backend): ") + (h ? mpdx_last_error(h) : mpdx_create_error()));
  }
}
// solver types wrapped in output::hdf5_xdmf carry has_output = true
template <class S, class = void>
struct has_output : std::false_type {};
template <class S>
struct has_output<S, std::void_t<decltype(S::has_output)>> : std::bool_constant<S::has_output> {};
}  // namespace detail

template <class solver_t, bcond::bcond_e bcxl, bcond::bcond_e bcxr, bcond::bcond_e bcyl = bcond::null,
          bcond::bcond_e bcyr = bcond::null, bcond::bcond_e bczl = bcond::null, bcond::bcond_e bczr = bcond::null>
class cuda : public any<typename solver_t::real_t, solver_t::n_dims> {
 public:
  using real_t = typename solver_t::real_t;
  enum { n_dims = solver_t::n_dims };
  enum { n_eqns = solver_t::n_eqns };
  using rt_params_t = typename solver_t::rt_params_t;
  using arr_t = host_view<real_t, n_dims>;
  using ct_params_t = typename solver_t::ct_params_t_;

  static_assert(n_dims >= 1 && n_dims <= 3, "n_dims must be 1, 2 or 3");
  static_assert(bcxl != bcond::null && bcxr != bcond::null, "x boundary conditions are required");
  static_assert(n_dims < 2 || (bcyl != bcond::null && bcyr != bcond::null), "y boundary conditions are required");
  static_assert(n_dims < 3 || (bczl != bcond::null && bczr != bcond::null), "z boundary conditions are required");
  // formulae_mpdata_hot_2d.hpp:147-149 (the 1D and 3D formulae never add fourth-order terms)
  static_assert(n_dims != 2 || !opts::isset(ct_params_t::opts, opts::fot) ||
                    (opts::isset(ct_params_t::opts, opts::iga) &&
                     (opts::isset(ct_params_t::opts, opts::tot) || opts::isset(ct_params_t::opts, opts::div_3rd))),
                "fot option only available with iga, and only with tot or div_3rd");

  explicit cuda(const rt_params_t &p) : p_(p) {
    mpdx_config c;
    mpdx_config_default(&c);
    c.n_dims = n_dims;
    c.n_eqns = n_eqns;
    for (int d = 0; d < 3; ++d) c.grid[d] = d < n_dims ? p.grid_size[d] : 1;
    c.opts = uint64_t(ct_params_t::opts);
    c.n_iters = p.n_iters;
    c.dtype = int(sizeof(real_t));
    const bcond::bcond_e b[6] = {bcxl, bcxr, bcyl, bcyr, bczl, bczr};
    for (int q = 0; q < 2 * n_dims; ++q) c.bcs[q] = bcond::to_c(b[q]);
    c.dt = double(p.dt);
    c.di = p.di != 0 ? double(p.di) : 1.0;
    c.dj = p.dj != 0 ? double(p.dj) : 1.0;
    c.dk = p.dk != 0 ? double(p.dk) : 1.0;
    c.max_abs_div_eps = double(p.max_abs_div_eps);
    c.upwind_filter_freq = p.upwind_filter_freq;
    c.sptl_intrp = int(ct_params_t::sptl_intrp);
    solver_t::fill(c, p);
    detail::check(nullptr, mpdx_create(&c, &h_));
  }
  ~cuda() override {
    if (h_) mpdx_destroy(h_);
  }
  cuda(const cuda &) = delete;
  cuda &operator=(const cuda &) = delete;

  // accessors (concurr_common.hpp:387-433)
  arr_t advectee(int e = 0) override { return view(MPDX_FIELD_ADVECTEE, e); }
  arr_t advector(int d = 0) override { return view(MPDX_FIELD_ADVECTOR, d); }
  // G of the nug option (sharedmem.hpp:373-380); throws without nug, as the reference does
  arr_t g_factor() override { return view(MPDX_FIELD_G, 0); }
  // advectee_global_set (concurr_common.hpp:444-453): copy a whole field into the advectee
  void advectee_global_set(const arr_t &a, int e = 0) override {
    arr_t v = advectee(e);
    std::copy(a.data(), a.data() + v.size(), v.data());
  }
  // named scalar arrays of the Boussinesq solver (boussinesq_common.hpp:20-60)
  arr_t sclr_array(const std::string &name, int = 0) override {
    if (name == "tht_e") return view(MPDX_FIELD_SCLR_ARRAY, MPDX_SCLR_THT_E);
    if (name == "tht_abs") return view(MPDX_FIELD_SCLR_ARRAY, MPDX_SCLR_THT_ABS);
    if (name == "hflux_frc") return view(MPDX_FIELD_SCLR_ARRAY, MPDX_SCLR_HFLUX_FRC);
    throw std::out_of_range("libmpdata++: unknown scalar array " + name);
  }
  // velocity absorber (concurr_common.hpp:420-428); the library throws without vip_vab
  arr_t vab_coefficient() override { return view(MPDX_FIELD_SCLR_ARRAY, MPDX_SCLR_VAB_COEFF); }
  arr_t vab_relaxed_state(int d = 0) override { return view(MPDX_FIELD_SCLR_ARRAY, MPDX_SCLR_VAB_RELAX + d); }

  // run.advance(nt) (concurr_common.hpp:380-385); hooks, if set, run after every step;
  // with output::hdf5_xdmf, records on the output steps (output_common.hpp:47-70, 150-165)
  void advance(int nt) override {
    if constexpr (detail::has_output<solver_t>::value) {
      advance_with_output(nt);
      return;
    }
    advance_steps(nt);
  }

  // run.min(e) / run.max(e) (concurr_common.hpp:392-402): equation 0 from the
  // device-side statistics after pending uploads, other equations from their view
  real_t min(int e = 0) override {
    if (e != 0) return libmpdataxx::min(advectee(e));
    flush();
    return real_t(stats().min);
  }
  real_t max(int e = 0) override {
    if (e != 0) return libmpdataxx::max(advectee(e));
    flush();
    return real_t(stats().max);
  }
  real_t time() const override { return real_t(stats().timestep) * p_.dt; }
  bool *panic_ptr() override { return &panic_; }

  // device-side statistics: timestep, FP64 mass, min/max, pressure-solver counters
  mpdx_step_stats stats() const {
    mpdx_step_stats s;
    detail::check(h_, mpdx_stats(h_, &s));
    return s;
  }
  // per-step host hook (stands in for overriding hook_post_step in a subclass)
  template <class F> void hook_post_step(F f) { hook_ = f; }
  mpdx_handle handle() const { return h_; }

 private:
  void advance_steps(int nt) {
    flush();
    if (!hook_) {
      detail::check(h_, mpdx_advance(h_, nt));
      invalidate_state();
      return;
    }
    for (int t = 0; t < nt && !panic_; ++t) {
      detail::check(h_, mpdx_advance(h_, 1));
      invalidate_state();
      hook_(*this);
      flush();
    }
  }

  // output steps: timestep % outfreq == 0 and timestep >= outstart; the fields
  // leave the device only there.  As the reference's hook_ante_loop
  // (output_common.hpp:47-64), every advance() call first rewrites const.h5 for
  // its nt and records the state it starts from, output step or not.
  void advance_with_output(int nt) {
    const long long t0 = stats().timestep, t1 = t0 + nt;
    const long long f = std::max(1, int(p_.outfreq));
    auto is_out = [&](long long t) { return t % f == 0 && t >= p_.outstart; };
    if (!rec_) {
      std::vector<int> grid(p_.grid_size.begin(), p_.grid_size.end());
      std::vector<double> dijk{double(p_.di), double(p_.dj), double(p_.dk)};
      dijk.resize(size_t(n_dims));
      rec_.reset(new output::detail::xdmf_recorder(p_.outdir, grid, double(p_.dt), dijk,
                                                     opts::opts_string(ct_params_t::opts), p_.n_iters));
    }
    // the T axis as hdf5.hpp:199-214 builds it from nt (outwindow 1): with
    // outstart = 0 the times k outfreq dt for k = 0 .. nt / outfreq; with
    // outstart > 0 t = 0 first, then outstart + k outfreq for k = 0 .. (nt - outstart) / outfreq
    // (integer division truncating toward zero, as there)
    std::vector<double> times;
    const long long os = p_.outstart;
    if (os > 0) times.push_back(0.0);
    for (long long k = 0; k <= (nt - os) / f; ++k) times.push_back(double(os + k * f) * double(p_.dt));
    rec_->start(times);
    record(t0);
    long long t = t0;
    while (t < t1) {
      long long next = t + 1;
      while (next < t1 && !is_out(next)) ++next;
      advance_steps(int(next - t));
      t = next;
      if (is_out(t)) record(t);
    }
  }
  void record(long long t) {
    std::map<std::string, std::vector<float>> fields;
    for (auto &v : p_.outvars) {
      arr_t a = view(MPDX_FIELD_ADVECTEE, v.first, false);  // read only: not re-uploaded
      fields[v.second.name] = std::vector<float>(a.data(), a.data() + a.size());
    }
    rec_->record(t, fields);
  }

  struct mirror {
    std::vector<real_t> buf;
    bool fresh = false;  // equals the device copy (downloaded after the last step)
    bool dirty = false;  // handed out since the last upload
  };

  arr_t view(int kind, int idx, bool hand_out = true) {
    std::array<int, n_dims> ext, lb;
    for (int d = 0; d < n_dims; ++d) {
      ext[d] = p_.grid_size[d];
      lb[d] = 0;
    }
    if (kind == MPDX_FIELD_ADVECTOR) {
      if (idx > 0) ext[0] += 1;  // view extents (sharedmem.hpp:431-456, 543-577)
      lb[0] = -1;
    }
    size_t n = 1;
    for (int d = 0; d < n_dims; ++d) n *= size_t(ext[d]);
    mirror &m = mirrors_[{kind, idx}];
    if (m.buf.size() != n) m.buf.assign(n, real_t(0));
    if (!m.fresh) {
      detail::check(h_, mpdx_get_field(h_, kind, idx, m.buf.data(), nullptr));
      m.fresh = true;
    }
    if (hand_out) m.dirty = true;
    return arr_t(m.buf.data(), lb, ext);
  }
  void flush() {
    for (auto &kv : mirrors_)
      if (kv.second.fresh && kv.second.dirty) {
        detail::check(h_, mpdx_set_field(h_, kv.first.first, kv.first.second, kv.second.buf.data(), nullptr));
        kv.second.dirty = false;
      }
  }
  void invalidate_state() {
    for (auto &kv : mirrors_)
      if (kv.first.first == MPDX_FIELD_ADVECTEE) kv.second.fresh = kv.second.dirty = false;
  }

  rt_params_t p_;
  mpdx_handle h_ = nullptr;
  std::map<std::pair<int, int>, mirror> mirrors_;
  std::function<void(cuda &)> hook_;
  bool panic_ = false;
  std::unique_ptr<output::detail::xdmf_recorder> rec_;
};

}  // namespace concurr
}  // namespace libmpdataxx
