// ORACLE -- test infrastructure only.
//
// CPU restatement of libmpdata++'s Boussinesq solver (solvers::boussinesq with
// the trapezoidal right-hand side and iles; explicit buoyancy, boussinesq_expl.hpp,
// or implicit theta perturbation, boussinesq_impl.hpp; no, explicit or implicit
// velocity absorber, mpdata_rhs_vip_common.hpp vip_vab) and of the GCR(k)
// pressure solve it calls every step, on top of the MPDATA restatement in
// mpdata_oracle.hpp.  Only tests/ and the CPU-baseline legs of bench.py load
// it, and only as the checker.
//
// Call order followed (file:line inside the libmpdata++ source tree):
//   hook_ante_loop   mpdata_rhs_vip_prs_common.hpp:130-160 -> mpdata_rhs_vip_common.hpp:283-302
//                    -> mpdata_rhs.hpp:154-169 -> solver_2d/3d hook_ante_loop
//   calc_gc          mpdata_rhs_vip_common.hpp:304-316, mpdata_rhs_vip.hpp (extrapolate_in_time,
//                    interpolate_in_space)
//   hook_ante_step   mpdata_rhs_vip_common.hpp:351-364, mpdata_rhs.hpp:171-193
//   hook_post_step   mpdata_rhs_vip_common.hpp:366-370, mpdata_rhs.hpp:195-214,
//                    mpdata_rhs_vip_prs_common.hpp:162-181
//   pressure solve   mpdata_rhs_vip_prs_common.hpp:47-128, mpdata_rhs_vip_prs_gcrk.hpp:39-97
//   buoyancy         boussinesq_expl.hpp:48-126 (expl), boussinesq_impl.hpp:36-141 (impl_tht)
//   absorbers        mpdata_rhs_vip_common.hpp:182-256 (vip_rhs_impl_init, vip_rhs_expl_calc,
//                    add_relax, normalize_vip), mpdata_rhs_vip_prs_common.hpp:49-84 (lap
//                    normalises the gradient unless simple), :162-181 (vip_rhs_impl_fnlz)
//
// hflux_frc and tht_abs start at zero (boussinesq_common.hpp:48-49) and are
// set, as in the reference, through sclr_array("hflux_frc") / ("tht_abs");
// vab_coefficient() and vab_relaxed_state(d) are sclr arrays "vab_coeff" and
// "vab_relax0..2" here.  Expressions keep the reference's operand order.
//
// One deliberate restatement:
//  * prs_sum() (sharedmem.hpp:115-190) is a plain per-slice Blitz++ sum in the
//    reference (Kahan with prs_khn).  Here every such sum is a compensated
//    double-double sum (TwoSum), whose value is the exact sum rounded except in
//    near-tie cases, so that it does not depend on the summation order; the
//    CUDA path computes the same quantity with a block-parallel order.
#pragma once

#include <array>
#include <vector>

#include "mpdata_oracle.hpp"

namespace mpdx_oracle {

// compensated accumulator: s + c carries the running sum to about twice the
// working precision (Knuth's TwoSum)
struct ddsum {
  double s = 0, c = 0;
  void add(double x) {
    const double t = s + x;
    const double bp = t - s;
    c += (s - (t - bp)) + (x - bp);
    s = t;
  }
  double value() const { return s + c; }
};

template <class T>
struct boussinesq : mpdata<T> {
  using B = mpdata<T>;
  using B::nd; using B::n; using B::H; using B::ir; using B::im; using B::psi; using B::tl; using B::GC;

  T dt = 1, dijk[3] = {1, 1, 1}, g = T(9.81), Tht_ref = 300, prs_tol = T(1e-7), err_tol = 0;
  int k_iters = 1, vip[3] = {0, 1, 2}, ix_w = 1, ix_tht = 2;
  int impl_tht = 0;  // ct_params_t::impl_tht
  int vab = 0;       // ct_params_t::vip_vab: 0 noab, 1 expl, 2 impl (mpdata_rhs_vip_common.hpp:16-21)
  std::array<arr<T>, 3> stash, vip_rhs, tmp_uvw, lap_tmp, vab_relax;
  std::vector<arr<T>> rhs, p_err, lap_p_err;
  arr<T> tht_e, Phi, err, lap_err, tht_abs, hflux_frc, vab_coeff, dtht_e;
  T beta = T(.25);                      // persists between solves (mpdata_rhs_vip_prs_gcrk.hpp:110-112)
  std::vector<T> alpha, tmp_den;
  T dt_stash0 = 0;
  long long iters = 0, iters_total = 0;
  bool converged = false;

  // prm = {dt, di, dj, dk, prs_tol, g, Tht_ref, max_abs_div_eps}; equations are
  // (u, [v,] w, tht) as in the reference's Boussinesq tests
  void setup_bq(int nd_, const int *n_, unsigned opts_, int n_iters_, const int *bcs_, const double *prm, int prs_k) {
    if (nd_ < 2 || nd_ > 3) throw std::runtime_error("oracle: Boussinesq needs 2 or 3 dimensions");
    for (int q = 0; q < 2 * nd_; ++q)
      if (bcs_[q] != bc_cyclic && bcs_[q] != bc_rigid) throw std::runtime_error("oracle: Boussinesq supports cyclic and rigid bconds");
    if (prs_k < 1) throw std::runtime_error("oracle: GCR k must be positive");
    B::setup(nd_, n_, nd_ + 1, opts_, n_iters_, bcs_);
    dt = T(prm[0]); dijk[0] = T(prm[1]); dijk[1] = T(prm[2]); dijk[2] = T(prm[3]);
    prs_tol = T(prm[4]); g = T(prm[5]); Tht_ref = T(prm[6]);
    if (prm[7] >= 0) this->max_abs_div_eps = T(prm[7]);
    err_tol = prs_tol / dt;
    k_iters = prs_k;
    for (int d = 0; d < nd; ++d) vip[d] = d;
    ix_w = nd - 1; ix_tht = nd;
    for (int d = 0; d < nd; ++d) {
      this->alloc_sclr(stash[d]); this->alloc_sclr(vip_rhs[d]);
      this->alloc_sclr(tmp_uvw[d]); this->alloc_sclr(lap_tmp[d]);
      this->alloc_sclr(vab_relax[d]);
    }
    this->alloc_sclr(tht_abs); this->alloc_sclr(hflux_frc); this->alloc_sclr(vab_coeff); this->alloc_sclr(dtht_e);
    // zero at construction (boussinesq_common.hpp:48-49 for hflux_frc and tht_abs)
    for (arr<T> *a : {&tht_abs, &hflux_frc, &vab_coeff, &vab_relax[0], &vab_relax[1], &vab_relax[2]})
      if (!a->v.empty()) std::fill(a->v.begin(), a->v.end(), T(0));
    rhs.resize(this->n_eqns);
    for (auto &a : rhs) this->alloc_sclr(a);
    this->alloc_sclr(tht_e); this->alloc_sclr(Phi); this->alloc_sclr(err); this->alloc_sclr(lap_err);
    p_err.resize(k_iters); lap_p_err.resize(k_iters);
    for (int v = 0; v < k_iters; ++v) { this->alloc_sclr(p_err[v]); this->alloc_sclr(lap_p_err[v]); }
    alpha.assign(k_iters, T(1)); tmp_den.assign(k_iters, T(1));
  }

  arr<T> &sclr_array(const char *name) {
    const std::string s(name);
    if (s == "tht_e") return tht_e;
    if (s == "tht_abs") return tht_abs;
    if (s == "hflux_frc") return hflux_frc;
    if (s == "vab_coeff") return vab_coeff;
    if (s.size() == 10 && s.compare(0, 9, "vab_relax") == 0 && s[9] >= '0' && s[9] < char('0' + nd)) return vab_relax[s[9] - '0'];
    throw std::runtime_error("no such scalar array");
  }
  arr<T> &vips(int d) { return this->state(vip[d]); }
  std::array<arr<T> *, 3> vips_ptrs() { return {&vips(0), nd > 1 ? &vips(1) : nullptr, nd > 2 ? &vips(2) : nullptr}; }
  std::array<arr<T> *, 3> ptrs(std::array<arr<T>, 3> &v) { return {&v[0], &v[1], &v[2]}; }

  // f(i, j, k) over the interior, memory order
  template <class F> void interior(F f) {
#pragma omp parallel for schedule(static) if (this->big())
    for (int i = 0; i < n[0]; ++i)
      for (int j = 0; j < n[1]; ++j)
        for (int k = 0; k < n[2]; ++k) f(i, j, k);
  }
  double sum1(const arr<T> &a) {
    ddsum acc;
    for (int i = 0; i < n[0]; ++i) for (int j = 0; j < n[1]; ++j) for (int k = 0; k < n[2]; ++k) acc.add(double(a(i, j, k)));
    return acc.value();
  }
  double sum2(const arr<T> &a, const arr<T> &b) {
    ddsum acc;
    for (int i = 0; i < n[0]; ++i)
      for (int j = 0; j < n[1]; ++j)
        for (int k = 0; k < n[2]; ++k) acc.add(double(T(a(i, j, k) * b(i, j, k))));
    return acc.value();
  }

  // ---- nabla operators (formulae/nabla_formulae.hpp:18-41, 149-167, 184-215) ----
  static void off(int d, int s, int &i, int &j, int &k) { i = d == 0 ? s : 0; j = d == 1 ? s : 0; k = d == 2 ? s : 0; }
  void calc_grad(std::array<arr<T>, 3> &V, arr<T> &A) {
    for (int d = 0; d < nd; ++d) {
      int pi, pj, pk; off(d, 1, pi, pj, pk);
      const T dx = dijk[d];
      arr<T> &v = V[d];
      interior([&](int i, int j, int k) { v(i, j, k) = (A(i + pi, j + pj, k + pk) - A(i - pi, j - pj, k - pk)) / dx / T(2); });
    }
  }
  void div(arr<T> &out, std::array<arr<T>, 3> &V) {
    interior([&](int i, int j, int k) {
      T r = (V[0](i + 1, j, k) - V[0](i - 1, j, k)) / dijk[0] / T(2) + (V[1](i, j + 1, k) - V[1](i, j - 1, k)) / dijk[1] / T(2);
      if (nd == 3) r = r + (V[2](i, j, k + 1) - V[2](i, j, k - 1)) / dijk[2] / T(2);
      out(i, j, k) = r;
    });
  }
  // normalize_vip (mpdata_rhs_vip_common.hpp:235-245; boussinesq_impl.hpp:61-80 with impl_tht)
  void normalize_vip(const std::array<arr<T> *, 3> &v) {
    const T hdt = T(0.5) * dt;
    if (vab == 2) {
      const int nh = impl_tht ? nd - 1 : nd;
      for (int d = 0; d < nh; ++d) {
        arr<T> &a = *v[d];
        interior([&](int i, int j, int k) { a(i, j, k) /= (1 + hdt * vab_coeff(i, j, k)); });
      }
      if (impl_tht) {
        arr<T> &a = *v[nd - 1];
        interior([&](int i, int j, int k) {
          a(i, j, k) /= (1 + hdt * vab_coeff(i, j, k)
                         + T(0.25) * dt * dt * g / Tht_ref * dtht_e(i, j, k) / (1 + hdt * tht_abs(i, j, k)));
        });
      }
    } else if (impl_tht) {
      arr<T> &a = *v[nd - 1];
      interior([&](int i, int j, int k) {
        a(i, j, k) /= (1 + T(0.25) * dt * dt * g / Tht_ref * dtht_e(i, j, k) / (1 + hdt * tht_abs(i, j, k)));
      });
    }
  }
  bool normalizes() const { return vab == 2 || impl_tht; }

  // lap() (mpdata_rhs_vip_prs_common.hpp:49-84), G = 1; simple: no normalize_vip
  void lap(arr<T> &out, arr<T> &A, bool err_init, bool simple) {
    this->xchng_pres(A, 0);
    calc_grad(lap_tmp, A);
    if (err_init)
      for (int d = 0; d < nd; ++d) { arr<T> &l = lap_tmp[d], &u = tmp_uvw[d]; interior([&](int i, int j, int k) { l(i, j, k) -= u(i, j, k); }); }
    this->set_edges(ptrs(lap_tmp));
    if (!simple) normalize_vip(ptrs(lap_tmp));
    for (int d = 0; d < nd; ++d) this->xchng_pres(lap_tmp[d], 0);
    div(out, lap_tmp);
  }

  T max_abs(const arr<T> &a) {
    T mx = a(0, 0, 0), mn = a(0, 0, 0);
    for (int i = 0; i < n[0]; ++i)
      for (int j = 0; j < n[1]; ++j)
        for (int k = 0; k < n[2]; ++k) { mx = std::max(mx, a(i, j, k)); mn = std::min(mn, a(i, j, k)); }
    return std::max(std::abs(mx), std::abs(mn));
  }

  // GCR(k) (mpdata_rhs_vip_prs_gcrk.hpp:39-97)
  bool simple = false;  // pressure_solver_update(simple) of the running solve
  void loop_init() {
    arr<T> &p0 = p_err[0];
    interior([&](int i, int j, int k) { p0(i, j, k) = err(i, j, k); });
    lap(lap_p_err[0], p_err[0], false, simple);
  }
  void loop_body() {
    for (int v = 0; v < k_iters; ++v) {
      tmp_den[v] = T(sum2(lap_p_err[v], lap_p_err[v]));
      if (tmp_den[v] != 0) beta = -T(sum2(err, lap_p_err[v])) / tmp_den[v];
      { arr<T> &p = p_err[v], &lp = lap_p_err[v]; const T b = beta;
        interior([&](int i, int j, int k) { Phi(i, j, k) += b * p(i, j, k); });
        interior([&](int i, int j, int k) { err(i, j, k) += b * lp(i, j, k); }); }
      if (max_abs(err) <= err_tol) converged = true;
      lap(lap_err, err, false, simple);
      for (int l = 0; l <= v; ++l)
        if (tmp_den[l] != 0) alpha[l] = -T(sum2(lap_err, lap_p_err[l])) / tmp_den[l];
      if (v < k_iters - 1) {
        arr<T> &pn = p_err[v + 1], &ln = lap_p_err[v + 1];
        interior([&](int i, int j, int k) { pn(i, j, k) = err(i, j, k); ln(i, j, k) = lap_err(i, j, k); });
        for (int l = 0; l <= v; ++l) {
          const T a = alpha[l]; arr<T> &pl = p_err[l], &ll = lap_p_err[l];
          interior([&](int i, int j, int k) { pn(i, j, k) += a * pl(i, j, k); ln(i, j, k) += a * ll(i, j, k); });
        }
      } else {
        arr<T> &p0 = p_err[0], &l0 = lap_p_err[0];
        const T a0 = alpha[0];
        interior([&](int i, int j, int k) {
          p0(i, j, k) = err(i, j, k) + a0 * p0(i, j, k);
          l0(i, j, k) = lap_err(i, j, k) + a0 * l0(i, j, k);
        });
        for (int l = 1; l <= v; ++l) {
          const T a = alpha[l]; arr<T> &pl = p_err[l], &ll = lap_p_err[l];
          interior([&](int i, int j, int k) { p0(i, j, k) += a * pl(i, j, k); l0(i, j, k) += a * ll(i, j, k); });
        }
      }
    }
  }

  // pressure_solver_update / _apply (mpdata_rhs_vip_prs_common.hpp:99-128)
  void pressure_solver_update(bool simple_ = false) {
    simple = simple_;
    for (int d = 0; d < nd; ++d) { arr<T> &u = tmp_uvw[d], &v = vips(d); interior([&](int i, int j, int k) { u(i, j, k) = v(i, j, k); }); }
    lap(err, Phi, true, simple);
    iters = 0;
    converged = false;
    loop_init();
    while (!converged) {
      loop_body();
      ++iters;
      if (iters > 10000) throw std::runtime_error("libmpdata++: stuck in pressure solver");
    }
    iters_total += iters;
    this->xchng_pres(Phi, 0);
    calc_grad(tmp_uvw, Phi);
  }
  void pressure_solver_apply() {
    for (int d = 0; d < nd; ++d) { arr<T> &u = tmp_uvw[d], &v = vips(d); interior([&](int i, int j, int k) { v(i, j, k) -= u(i, j, k); }); }
  }

  // update_rhs (mpdata_rhs.hpp:39-61) + boussinesq_expl.hpp:81-126 or boussinesq_impl.hpp:82-113;
  // at = 0 before the first step, 1 after each step
  void update_rhs(int at) {
    for (int e = 0; e < this->n_eqns; ++e) { arr<T> &r = rhs[e]; interior([&](int i, int j, int k) { r(i, j, k) = T(0); }); }
    for (int e = 0; e < this->n_eqns; ++e) this->xchng(e);
    arr<T> &rw = rhs[ix_w], &rt = rhs[ix_tht], &th = this->state(ix_tht), &w = vips(nd - 1);
    const T hdt = T(0.5) * dt;
    if (!impl_tht) {
      if (at == 0) {
        interior([&](int i, int j, int k) {
          rt(i, j, k) += hflux_frc(i, j, k) - tht_abs(i, j, k) * (th(i, j, k) - tht_e(i, j, k));
          rw(i, j, k) += g * (th(i, j, k) - tht_e(i, j, k)) / Tht_ref;
        });
      } else {
        interior([&](int i, int j, int k) {
          const T x = (th(i, j, k) + hdt * hflux_frc(i, j, k) + hdt * tht_abs(i, j, k) * tht_e(i, j, k)) / (1 + hdt * tht_abs(i, j, k));
          rt(i, j, k) += hflux_frc(i, j, k) - tht_abs(i, j, k) * (x - tht_e(i, j, k));
          rw(i, j, k) += g * (x - tht_e(i, j, k)) / Tht_ref;
        });
      }
    } else if (at == 0) {
      interior([&](int i, int j, int k) {
        rt(i, j, k) += -w(i, j, k) * dtht_e(i, j, k) + hflux_frc(i, j, k) - tht_abs(i, j, k) * th(i, j, k);
        rw(i, j, k) += g * th(i, j, k) / Tht_ref;
      });
    } else {
      interior([&](int i, int j, int k) {
        rt(i, j, k) += hflux_frc(i, j, k);
        rw(i, j, k) += g * (th(i, j, k) + hdt * rt(i, j, k)) / (Tht_ref * (1 + hdt * tht_abs(i, j, k)));
      });
    }
  }
  // dtht_e = d(tht_e)/dz after tht_e's scalar halo fill (boussinesq_impl.hpp:38-50)
  void calc_dtht_e() {
    this->xchng_sclr(tht_e, 0);
    const int d = nd - 1;
    int pi, pj, pk; off(d, 1, pi, pj, pk);
    const T dx = dijk[d];
    interior([&](int i, int j, int k) { dtht_e(i, j, k) = (tht_e(i + pi, j + pj, k + pk) - tht_e(i - pi, j - pj, k - pk)) / dx / T(2); });
  }
  // add_relax (mpdata_rhs_vip_common.hpp:247-254)
  void add_relax() {
    for (int d = 0; d < nd; ++d) {
      arr<T> &v = vips(d), &r = vab_relax[d];
      interior([&](int i, int j, int k) { v(i, j, k) += T(0.5) * dt * vab_coeff(i, j, k) * r(i, j, k); });
    }
  }
  void apply_rhs(T dt_arg) {  // mpdata_rhs.hpp:63-76
    for (int e = 0; e < this->n_eqns; ++e) {
      arr<T> &p = this->state(e), &r = rhs[e];
      interior([&](int i, int j, int k) { p(i, j, k) += dt_arg * r(i, j, k); });
    }
  }

  void bq_ante_loop() {
    if (impl_tht) calc_dtht_e();  // boussinesq_impl.hpp:57-61
    // correct initial velocity (mpdata_rhs_vip_prs_common.hpp:130-146)
    interior([&](int i, int j, int k) { Phi(i, j, k) = T(0); });
    this->xchng_pres(Phi, 0);
    pressure_solver_update(true);
    this->xchng_pres(Phi, 0);
    calc_grad(tmp_uvw, Phi);
    pressure_solver_apply();
    this->set_edges(vips_ptrs());
    // mpdata_rhs_vip_common.hpp:283-302
    for (int d = 0; d < nd; ++d) std::fill(GC[d].v.begin(), GC[d].v.end(), T(0));
    for (int d = 0; d < nd; ++d) { arr<T> &s = stash[d]; interior([&](int i, int j, int k) { s(i, j, k) = T(0); }); }
    B::ante_loop();
    update_rhs(0);  // trapez: update_rhs(rhs, dt / 2, 0)
    // vip_rhs_impl_init (mpdata_rhs_vip_common.hpp:182-196)
    for (int d = 0; d < nd; ++d) {
      arr<T> &r = vip_rhs[d], &v = vips(d), &rl = vab_relax[d];
      if (vab == 2) interior([&](int i, int j, int k) { r(i, j, k) = -vab_coeff(i, j, k) * (v(i, j, k) - rl(i, j, k)); });
      else interior([&](int i, int j, int k) { r(i, j, k) = T(0); });
    }
    // ini_pressure (mpdata_rhs_vip_prs_common.hpp:86-97)
    interior([&](int i, int j, int k) { Phi(i, j, k) = T(0); });
    long long npoints = 1;
    for (int d = 0; d < nd; ++d) {
      arr<T> &v = vips(d);
      interior([&](int i, int j, int k) { Phi(i, j, k) -= T(0.5) * (v(i, j, k) * v(i, j, k)); });
      npoints *= n[d];
    }
    const T mean = T(sum1(Phi)) / T(npoints);
    interior([&](int i, int j, int k) { Phi(i, j, k) -= mean; });
    this->xchng_pres(Phi, 0);
    calc_grad(tmp_uvw, Phi);
    for (int d = 0; d < nd; ++d) { arr<T> &r = vip_rhs[d], &u = tmp_uvw[d]; interior([&](int i, int j, int k) { r(i, j, k) -= u(i, j, k); }); }
  }

  void calc_gc() {
    const T b = dt_stash0 > 0 ? dt / (2 * dt_stash0) : T(0);
    for (int d = 0; d < nd; ++d) {  // extrp (mpdata_rhs_vip_common.hpp:120-153)
      arr<T> &s = stash[d], &v = vips(d);
      interior([&](int i, int j, int k) { s(i, j, k) *= -b; });
      interior([&](int i, int j, int k) { s(i, j, k) += (1 + b) * v(i, j, k); });
    }
    const int ex = H - 1;
    for (int d = 0; d < nd; ++d) this->xchng_pres(stash[d], ex);
    // intrp<d> over (m^ex along d) x (^ex across)
    const T half = T(.5);
    auto intrp = [&](int d) {
      const T c = dt / dijk[d] * half;
      rng r[3];
      for (int q = 0; q < 3; ++q) r[q] = q < nd ? ext(ir[q], ex) : rng{0, 0};
      r[d] = ext(im[d], ex);
      int pi, pj, pk; off(d, 1, pi, pj, pk);
      arr<T> &dst = GC[d], &src = stash[d];
      for (int i = r[0].f; i <= r[0].l; ++i)
        for (int j = r[1].f; j <= r[1].l; ++j)
          for (int k = r[2].f; k <= r[2].l; ++k) dst(i, j, k) = c * (src(i, j, k) + src(i + pi, j + pj, k + pk));
    };
    for (int d = 0; d < nd; ++d) intrp(d);
    this->xchng_vctr_alng(GC, false, true);
    this->xchng_vctr_nrml(GC, ex);
  }

  void step() {
    calc_gc();
    // hook_ante_step: fill_stash, vip_rhs_expl_calc, apply_rhs(dt / 2), vip_rhs_apply
    for (int d = 0; d < nd; ++d) { arr<T> &s = stash[d], &v = vips(d); interior([&](int i, int j, int k) { s(i, j, k) = v(i, j, k); }); }
    if (vab == 1)
      for (int d = 0; d < nd; ++d) {
        arr<T> &r = vip_rhs[d], &v = vips(d), &rl = vab_relax[d];
        interior([&](int i, int j, int k) { r(i, j, k) += -2 * vab_coeff(i, j, k) * (v(i, j, k) - rl(i, j, k)); });
      }
    apply_rhs(dt / 2);
    for (int d = 0; d < nd; ++d) {
      arr<T> &v = vips(d), &r = vip_rhs[d];
      interior([&](int i, int j, int k) { v(i, j, k) += T(0.5) * dt * r(i, j, k); r(i, j, k) = T(0); });
    }
    for (int e = 0; e < this->n_eqns; ++e) { this->xchng(e); this->advop(e); this->cycle(e); }
    ++this->timestep;
    dt_stash0 = dt;
    // hook_post_step: update_rhs(at = 1), apply_rhs(dt / 2), vip_rhs_impl_fnlz
    // (mpdata_rhs_vip_prs_common.hpp:162-181, then boussinesq_impl.hpp:115-125)
    update_rhs(1);
    apply_rhs(dt / 2);
    for (int d = 0; d < nd; ++d) { arr<T> &r = vip_rhs[d], &v = vips(d); interior([&](int i, int j, int k) { r(i, j, k) = -v(i, j, k); }); }
    if (vab == 2) add_relax();
    pressure_solver_update();
    pressure_solver_apply();
    normalize_vip(vips_ptrs());
    this->set_edges(vips_ptrs());
    const T hdt = T(0.5) * dt;
    for (int d = 0; d < nd; ++d) {
      arr<T> &r = vip_rhs[d], &v = vips(d);
      interior([&](int i, int j, int k) { r(i, j, k) += v(i, j, k); r(i, j, k) /= hdt; });
    }
    if (impl_tht) {
      arr<T> &th = this->state(ix_tht), &rt = rhs[ix_tht], &w = vips(nd - 1);
      interior([&](int i, int j, int k) {
        th(i, j, k) = (th(i, j, k) - T(0.5) * dt * w(i, j, k) * dtht_e(i, j, k)) / (1 + T(0.5) * dt * tht_abs(i, j, k));
        rt(i, j, k) += -w(i, j, k) * dtht_e(i, j, k) - tht_abs(i, j, k) * th(i, j, k);
      });
    }
  }

  void advance(long long nt) {
    nt += this->timestep;
    if (this->timestep == 0) bq_ante_loop();
    while (this->timestep < nt) step();
  }
};

}  // namespace mpdx_oracle
