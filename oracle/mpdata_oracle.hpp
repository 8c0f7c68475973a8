// ORACLE -- test infrastructure only.
//
// A plain C++17 CPU restatement of libmpdata++'s MPDATA advection step
// (donor-cell flux, antidiffusive corrective iterations, FCT limiter), of its
// halo fills for cyclic/open boundaries and of its time loop.  It exists to
// check the CUDA product path: only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py load it, and only as the checker.  Nothing in
// the shipped library calls it.
//
// Every function follows the reference's evaluation order (parenthesisation,
// loop ranges, halo-fill order) so that an IEEE build (-O2 -ffp-contract=off)
// reproduces the reference's FP64 arithmetic.  Arrays are NaN-filled at
// allocation (as the reference's debug builds do, libmpdata++/blitz.hpp:107-112)
// so that any read of a halo cell that the reference never fills shows up.
//
// Parity pinned against the reference's own golden data (tests/golden/*):
// 1D advscheme_opts field dumps, 2D rotating-cone stats, 3D revolving-sphere
// stats (see tests/test_oracle_golden.py).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace mpdx_oracle {

// option bits -- same values as libmpdata++/opts.hpp:34-49
enum : unsigned {
  o_fct = 1u << 0, o_abs = 1u << 1, o_tot = 1u << 2, o_pfc = 1u << 3,
  o_npa = 1u << 4, o_iga = 1u << 5, o_nug = 1u << 6, o_dfl = 1u << 7,
  o_khn = 1u << 8, o_div_2nd = 1u << 9, o_div_3rd = 1u << 10, o_div_3rd_dt = 1u << 11, o_fot = 1u << 12
};
enum { bc_cyclic = 0, bc_open = 1, bc_rigid = 2 };

struct rng { int f, l; };
// r^n (libmpdata++/formulae/arakawa_c.hpp:41-49)
inline rng ext(rng r, int n) { return {r.f - n, r.l + n}; }
// r^h: (r-h).first() .. (r+h).last()
inline rng exh(rng r) { return {r.f - 1, r.l}; }

template <class T>
struct arr {
  std::vector<T> v;
  int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  long s0 = 1, s1 = 1;
  void alloc(rng r0, rng r1, rng r2) {
    lo[0] = r0.f; lo[1] = r1.f; lo[2] = r2.f;
    hi[0] = r0.l; hi[1] = r1.l; hi[2] = r2.l;
    s1 = r2.l - r2.f + 1;
    s0 = s1 * (r1.l - r1.f + 1);
    v.assign(size_t(s0) * size_t(r0.l - r0.f + 1), std::numeric_limits<T>::quiet_NaN());
  }
  inline T &operator()(int i, int j, int k) {
#ifdef ORACLE_BOUNDS
    if (!has(i, j, k)) throw std::runtime_error("oracle: index out of bounds");
#endif
    return v[size_t((i - lo[0]) * s0 + (j - lo[1]) * s1 + (k - lo[2]))];
  }
  inline const T &operator()(int i, int j, int k) const {
#ifdef ORACLE_BOUNDS
    if (!has(i, j, k)) throw std::runtime_error("oracle: index out of bounds");
#endif
    return v[size_t((i - lo[0]) * s0 + (j - lo[1]) * s1 + (k - lo[2]))];
  }
  bool has(int i, int j, int k) const {
    return i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2];
  }
};
template <class T> using vctr = std::array<arr<T>, 3>;

// index permutation pi<d> (libmpdata++/formulae/idxperm.hpp:15-71): frame
// coordinates (a along d, b along d+1, c along d+2) -> (i, j, k)
template <int ND, int D> struct pi;
template <> struct pi<1, 0> { static inline void m(int a, int, int, int &i, int &j, int &k) { i = a; j = 0; k = 0; } };
template <> struct pi<2, 0> { static inline void m(int a, int b, int, int &i, int &j, int &k) { i = a; j = b; k = 0; } };
template <> struct pi<2, 1> { static inline void m(int a, int b, int, int &i, int &j, int &k) { i = b; j = a; k = 0; } };
template <> struct pi<3, 0> { static inline void m(int a, int b, int c, int &i, int &j, int &k) { i = a; j = b; k = c; } };
template <> struct pi<3, 1> { static inline void m(int a, int b, int c, int &i, int &j, int &k) { i = c; j = a; k = b; } };
template <> struct pi<3, 2> { static inline void m(int a, int b, int c, int &i, int &j, int &k) { i = b; j = c; k = a; } };

// inverse: physical (i, j, k) -> frame (a, b, c)
template <int ND, int D> struct ipi;
template <> struct ipi<1, 0> { static inline void m(int i, int, int, int &a, int &b, int &c) { a = i; b = 0; c = 0; } };
template <> struct ipi<2, 0> { static inline void m(int i, int j, int, int &a, int &b, int &c) { a = i; b = j; c = 0; } };
template <> struct ipi<2, 1> { static inline void m(int i, int j, int, int &a, int &b, int &c) { a = j; b = i; c = 0; } };
template <> struct ipi<3, 0> { static inline void m(int i, int j, int k, int &a, int &b, int &c) { a = i; b = j; c = k; } };
template <> struct ipi<3, 1> { static inline void m(int i, int j, int k, int &a, int &b, int &c) { a = j; b = k; c = i; } };
template <> struct ipi<3, 2> { static inline void m(int i, int j, int k, int &a, int &b, int &c) { a = k; b = i; c = j; } };

template <int ND, int D, class T>
inline T &P(arr<T> &A, int a, int b = 0, int c = 0) {
  int i, j, k; pi<ND, D>::m(a, b, c, i, j, k); return A(i, j, k);
}
template <int ND, int D, class T>
inline const T &P(const arr<T> &A, int a, int b = 0, int c = 0) {
  int i, j, k; pi<ND, D>::m(a, b, c, i, j, k); return A(i, j, k);
}

// runtime-dimension variant used by halo fills
inline void pim(int nd, int d, int a, int b, int c, int &i, int &j, int &k) {
  if (nd == 1) { i = a; j = 0; k = 0; return; }
  if (nd == 2) { if (d == 0) { i = a; j = b; } else { i = b; j = a; } k = 0; return; }
  if (d == 0) { i = a; j = b; k = c; } else if (d == 1) { i = c; j = a; k = b; } else { i = b; j = c; k = a; }
}
template <class T> inline T &PR(arr<T> &A, int nd, int d, int a, int b, int c) {
  int i, j, k; pim(nd, d, a, b, c, i, j, k); return A(i, j, k);
}

// pospart / negpart (libmpdata++/formulae/common.hpp:86-124); min/max follow
// std::min/std::max as the scalar (ix_t=int) reference paths do
template <class T> inline T pospart(unsigned o, T x) { return (o & o_npa) ? (x + std::abs(x)) / 2 : std::max(T(0), x); }
template <class T> inline T negpart(unsigned o, T x) { return (o & o_npa) ? (x - std::abs(x)) / 2 : std::min(T(0), x); }

// frac (formulae_mpdata_common.hpp:61-86) and fct_frac (:88-98)
template <class T> inline T frac(unsigned o, T nom, T den) {
  if (o & o_pfc) return den != 0 ? nom / den : T(0);
  return nom / (den + std::numeric_limits<T>::min());
}
template <class T> inline T fct_frac(T nom, T den) { return nom / (den + std::numeric_limits<T>::epsilon()); }

// donor-cell flux F (donorcell_formulae.hpp:25-34)
template <class T> inline T Fdc(unsigned o, T psi_l, T psi_r, T C) {
  return pospart(o, C) * psi_l + negpart(o, C) * psi_r;
}

template <class T>
struct mpdata {
  // configuration
  int nd = 1, n[3] = {1, 1, 1}, H = 1, n_eqns = 1, n_iters = 2;
  unsigned opts = o_iga | o_fct;
  int bcs[3][2] = {{bc_cyclic, bc_cyclic}, {bc_cyclic, bc_cyclic}, {bc_cyclic, bc_cyclic}};
  T max_abs_div_eps = std::numeric_limits<T>::epsilon();
  int upwind_filter_freq = 0;  // rt_params (mpdata_common.hpp:77): upwind-only step every n-th step

  // state
  std::vector<std::array<arr<T>, 2>> psi;  // psi[e][tlev]
  std::vector<int> tl;                     // per-eqn time level n[e] (mod 2)
  vctr<T> GC, tmp0, tmp1, flux, GC_mono;
  arr<T> psi_min, psi_max, beta_up, beta_dn;
  arr<T> Gf;  // G factor with the nug option (sharedmem G, solver_{1,2,3}d.hpp alloc); 1 elsewhere
  long long timestep = 0;

  rng ir[3];  // interior ranges
  rng im[3];  // (i.first-1 .. i.last) -- mpdata_osc_*d.hpp ctor

  static int mpdata_halo(unsigned o) {  // formulae_mpdata_common.hpp:50-59
    return (o & (o_tot | o_dfl | o_div_2nd | o_div_3rd | o_div_3rd_dt)) ? 2 : 1;
  }
  int sptl_intrp = 0;  // ct_params_t::sptl_intrp: exact, aver2, aver4 (formulae_mpdata_common.hpp:21-26)

  void setup(int nd_, const int *n_, int n_eqns_, unsigned opts_, int n_iters_, const int *bcs_) {
    nd = nd_; n_eqns = n_eqns_; opts = opts_; n_iters = n_iters_;
    if (n_iters < 1) throw std::runtime_error("n_iters must be positive");
    // divergence form with a third pass: its antidiffusive velocities read faces of GC_corr(1)
    // that no exchange fills (mpdata_osc_2d.hpp:112-121), so the reference's result is not defined
    if ((opts & (o_div_2nd | o_div_3rd | o_div_3rd_dt)) && n_iters > 2)
      throw std::runtime_error("oracle: divergence-form options need n_iters <= 2");
    // formulae_mpdata_hot_2d.hpp:147-149 (static_asserts of the 2D FOT; 1D and 3D never add it)
    if (nd == 2 && (opts & o_fot) && (!(opts & o_iga) || !(opts & (o_tot | o_div_3rd))))
      throw std::runtime_error("oracle: fot needs iga and tot or div_3rd");
    for (int d = 0; d < 3; ++d) n[d] = d < nd ? n_[d] : 1;
    for (int d = 0; d < nd; ++d) if (n[d] < 1) throw std::runtime_error("libmpdata++: bogus grid size");
    for (int d = 0; d < nd; ++d) for (int s = 0; s < 2; ++s) bcs[d][s] = bcs_[2 * d + s];
    H = mpdata_halo(opts);
    if (opts & o_fct) H = std::max(H, 2);  // fct_min_halo (mpdata_fct_common.hpp:15)
    for (int d = 0; d < 3; ++d) {
      ir[d] = {0, n[d] - 1};
      im[d] = d < nd ? rng{-1, n[d] - 1} : rng{0, 0};
    }
    psi.assign(n_eqns, {});
    tl.assign(n_eqns, 0);
    for (auto &p : psi) for (auto &a : p) alloc_sclr(a);
    alloc_vctr(GC); alloc_vctr(tmp0); alloc_vctr(flux);
    if (n_iters > 2) alloc_vctr(tmp1);  // n_tmp (mpdata_common.hpp:67-70)
    if (opts & o_fct) {
      alloc_sclr(psi_min); alloc_sclr(psi_max); alloc_sclr(beta_up); alloc_sclr(beta_dn);
      alloc_vctr(GC_mono);
    }
    if (opts & o_nug) {
      alloc_sclr(Gf);
      for (auto &v : Gf.v) v = T(1);
    }
  }

  // G and its face average G_bar_x (formulae/common.hpp:127-195, formulae_mpdata_g_{1,2,3}d.hpp);
  // the reference returns the integer 1 for both without nug
  T Gc(int i, int j, int k) const { return (opts & o_nug) ? Gf(i, j, k) : T(1); }
  template <int ND, int D> T Gbar(int a, int b, int c) const {
    if (!(opts & o_nug)) return T(1);
    return (P<ND, D>(Gf, a + 1, b, c) + P<ND, D>(Gf, a, b, c)) / T(2);
  }

  rng sr(int d) const { return d < nd ? ext(ir[d], H) : rng{0, 0}; }     // rng_sclr
  // threads pay off only on large grids; loops are elementwise, so results do not depend on it
  bool big() const { return long(n[0]) * n[1] * n[2] >= (1L << 17); }
  void alloc_sclr(arr<T> &a) { a.alloc(sr(0), sr(1), sr(2)); }
  // visit a frame box (a in ra, b in rb, c in rc) in memory order (k fastest);
  // every visit is independent, so the order does not change results
  template <int ND, int D, class F> void box(rng ra, rng rb, rng rc, F f) {
    rng ph[3] = {{0, 0}, {0, 0}, {0, 0}};
    ph[D] = ra;
    if (ND >= 2) ph[(D + 1) % ND] = rb;
    if (ND >= 3) ph[(D + 2) % ND] = rc;
#pragma omp parallel for schedule(static) if (big())
    for (int i = ph[0].f; i <= ph[0].l; ++i)
      for (int j = ph[1].f; j <= ph[1].l; ++j)
        for (int k = ph[2].f; k <= ph[2].l; ++k) {
          int a, b, c;
          ipi<ND, D>::m(i, j, k, a, b, c);
          f(a, b, c);
        }
  }
  void alloc_vctr(vctr<T> &v) {  // rng_vctr along its own axis: i^h^(halo-1)
    for (int c = 0; c < nd; ++c) {
      rng r[3] = {sr(0), sr(1), sr(2)};
      r[c] = ext(exh(ir[c]), H - 1);
      v[c].alloc(r[0], r[1], r[2]);
    }
  }

  // ---- bcond ranges (bcond_common.hpp:225-275) ----
  rng left_halo_sclr(int d) const { return {-H, -1}; }
  rng rght_halo_sclr(int d) const { return {n[d], n[d] + H - 1}; }
  rng left_intr_sclr(int d) const { return {1, H}; }
  rng rght_intr_sclr(int d) const { return {n[d] - 1 - H, n[d] - 2}; }
  rng left_halo_vctr(int d) const { return {-H, -1}; }
  rng rght_halo_vctr(int d) const { return {n[d] - 1, n[d] + H - 2}; }
  rng left_intr_vctr(int d) const { return {0, H - 1}; }
  rng rght_intr_vctr(int d) const { return {n[d] - 1 - H, n[d] - 2}; }

  // loops over the two transverse frame ranges (b along d+1, c along d+2)
  template <class F> void each(rng rb, rng rc, F f) {
    if (nd == 1) { f(0, 0); return; }
    if (nd == 2) { for (int b = rb.f; b <= rb.l; ++b) f(b, 0); return; }
    for (int b = rb.f; b <= rb.l; ++b) for (int c = rc.f; c <= rc.l; ++c) f(b, c);
  }

  // ---- halo fills: cyclic_{1,2,3}d.hpp, open_{1,2,3}d.hpp ----
  void fill_sclr(int d, int side, arr<T> &A, rng rb, rng rc, bool deriv = false) {
    const int kind = bcs[d][side];
    each(rb, rc, [&](int b, int c) {
      if (kind == bc_cyclic) {
        if (side == 0) { rng h = left_halo_sclr(d), s = rght_intr_sclr(d);
          for (int t = 0; t <= h.l - h.f; ++t) PR(A, nd, d, h.f + t, b, c) = PR(A, nd, d, s.f + t, b, c); }
        else { rng h = rght_halo_sclr(d), s = left_intr_sclr(d);
          for (int t = 0; t <= h.l - h.f; ++t) PR(A, nd, d, h.f + t, b, c) = PR(A, nd, d, s.f + t, b, c); }
      } else if (kind == bc_open) {
        rng h = side == 0 ? left_halo_sclr(d) : rght_halo_sclr(d);
        int e = side == 0 ? 0 : n[d] - 1;
        for (int i = h.f; i <= h.l; ++i) PR(A, nd, d, i, b, c) = deriv ? T(0) : PR(A, nd, d, e, b, c);
      } else if (kind == bc_rigid) {
        // mirror about the edge point (rigid_2d.hpp:16-24, 124-132; rigid_3d.hpp:30-38)
        if (side == 0) { for (int m = 1; m <= H; ++m) PR(A, nd, d, -m, b, c) = PR(A, nd, d, m, b, c); }
        else { for (int m = 1; m <= H; ++m) PR(A, nd, d, n[d] - 1 + m, b, c) = PR(A, nd, d, n[d] - 1 - m, b, c); }
      } else throw std::runtime_error("oracle: bcond kind not supported for scalars");
    });
  }
  // fill_halos_pres: cyclic as scalars; rigid one-sided-derivative extrapolation
  // (rigid_2d.hpp:26-35, 134-143; rigid_3d.hpp:40-49)
  void fill_pres(int d, int side, arr<T> &A, rng rb, rng rc) {
    const int kind = bcs[d][side];
    if (kind == bc_cyclic) { fill_sclr(d, side, A, rb, rc); return; }
    if (kind != bc_rigid) throw std::runtime_error("oracle: bcond kind not supported for pressure");
    each(rb, rc, [&](int b, int c) {
      if (side == 0) {
        for (int m = H; m >= 1; --m) PR(A, nd, d, -m, b, c) = T(2) * PR(A, nd, d, 0, b, c) - PR(A, nd, d, m, b, c);
      } else {
        const int e = n[d] - 1;
        for (int m = 1; m <= H; ++m) PR(A, nd, d, e + m, b, c) = T(2) * PR(A, nd, d, e, b, c) - PR(A, nd, d, e - m, b, c);
      }
    });
  }
  // set_edge_pres: zero on a rigid wall point, no-op otherwise (rigid_2d.hpp:52-56, 148-152)
  void set_edge_pres(int d, int side, arr<T> &A, rng rb, rng rc) {
    if (bcs[d][side] != bc_rigid) return;
    const int e = side == 0 ? 0 : n[d] - 1;
    each(rb, rc, [&](int b, int c) { PR(A, nd, d, e, b, c) = T(0); });
  }
  // fill_halos_flux: antisymmetric face next to a rigid wall, no-op otherwise
  // (rigid_2d.hpp:74-79, 170-175; rigid_3d.hpp:73-78)
  void fill_flux(int d, int side, vctr<T> &AV, rng rb, rng rc) {
    if (bcs[d][side] != bc_rigid) return;
    each(rb, rc, [&](int b, int c) {
      if (side == 0) PR(AV[d], nd, d, -1, b, c) = -PR(AV[d], nd, d, 0, b, c);
      else PR(AV[d], nd, d, n[d] - 1, b, c) = -PR(AV[d], nd, d, n[d] - 2, b, c);
    });
  }
  void fill_vctr_nrml(int d, int side, arr<T> &A, rng rb, rng rc) {
    const int kind = bcs[d][side];
    if (kind == bc_cyclic || kind == bc_rigid) { fill_sclr(d, side, A, rb, rc); return; }  // rigid: "intentional sclr"
    if (kind == bc_open) {
      rng h = side == 0 ? left_halo_sclr(d) : rght_halo_sclr(d);
      each(rb, rc, [&](int b, int c) { for (int i = h.f; i <= h.l; ++i) PR(A, nd, d, i, b, c) = T(0); });
      return;
    }
    throw std::runtime_error("oracle: bcond kind not supported for vectors");
  }
  void fill_vctr_alng(int d, int side, vctr<T> &AV, rng rb, rng rc, bool ad, bool cyclic_only = false) {
    const int kind = bcs[d][side];
    if (kind == bc_cyclic) {
      each(rb, rc, [&](int b, int c) {
        if (side == 0) { rng h = left_halo_vctr(d), s = rght_intr_vctr(d);
          for (int t = 0; t <= h.l - h.f; ++t) PR(AV[d], nd, d, h.f + t, b, c) = PR(AV[d], nd, d, s.f + t, b, c); }
        else { rng h = rght_halo_vctr(d), s = left_intr_vctr(d);
          for (int t = 0; t <= h.l - h.f; ++t) PR(AV[d], nd, d, h.f + t, b, c) = PR(AV[d], nd, d, s.f + t, b, c); }
      });
      return;
    }
    if (cyclic_only) return;  // fill_halos_vctr_alng_cyclic is a no-op for non-cyclic bconds
    if (kind == bc_rigid) {  // zero normal velocity on the wall point (rigid_2d.hpp:58-66, 154-162)
      each(rb, rc, [&](int b, int c) {
        if (side == 0) { for (int m = H; m >= (ad ? 2 : 1); --m) PR(AV[d], nd, d, -m, b, c) = -PR(AV[d], nd, d, m - 1, b, c); }
        else {  // the counter starts at 1 also when ad skips the first halo face
          const int a0 = ad ? 1 : 0;
          for (int t = 0; t < H - a0; ++t) PR(AV[d], nd, d, n[d] - 1 + a0 + t, b, c) = -PR(AV[d], nd, d, n[d] - 2 - t, b, c);
        }
      });
      return;
    }
    if (kind != bc_open) throw std::runtime_error("oracle: bcond kind not supported for vectors");
    if (nd == 1) {  // open_1d.hpp:36-40, 66-70
      if (side == 0) { rng h = left_halo_vctr(0); T v = AV[0](left_intr_vctr(0).f, 0, 0);
        for (int i = h.f; i <= h.l - (ad ? 1 : 0); ++i) AV[0](i, 0, 0) = v; }
      else { rng h = rght_halo_vctr(0); T v = AV[0](rght_intr_vctr(0).f, 0, 0);
        for (int i = h.f + (ad ? 1 : 0); i <= h.l; ++i) AV[0](i, 0, 0) = v; }
      return;
    }
    const int e = side == 0 ? 0 : n[d] - 1;
    const int d1 = (d + 1) % nd, d2 = (d + 2) % nd;
    if (nd == 2) {  // open_2d.hpp:71-91 (left), 167-186 (right)
      if (d == 0) { PR(AV[d1], nd, d, e, rb.f - 1, 0) = T(0); PR(AV[d1], nd, d, e, rb.l, 0) = T(0); }
      rng h = side == 0 ? left_halo_vctr(d) : rght_halo_vctr(d);
      int f = side == 0 ? h.f : h.f + (ad ? 1 : 0);
      int l = side == 0 ? h.l - (ad ? 1 : 0) : h.l;
      for (int ii = f; ii <= l; ++ii)
        for (int b = rb.f; b <= rb.l; ++b) {
          if (side == 0)
            PR(AV[d], nd, d, ii, b, 0) = PR(AV[d], nd, d, e, b, 0) - (PR(AV[d1], nd, d, e, b - 1, 0) - PR(AV[d1], nd, d, e, b, 0));
          else
            PR(AV[d], nd, d, ii, b, 0) = PR(AV[d], nd, d, e - 1, b, 0) + (PR(AV[d1], nd, d, e, b - 1, 0) - PR(AV[d1], nd, d, e, b, 0));
        }
      return;
    }
    // nd == 3: open_3d.hpp:66-125 (left), 197-243 (right)
    if (d == 0) {
      for (int b = rb.f; b <= rb.l; ++b) { PR(AV[d2], nd, d, e, b, rc.f - 1) = T(0); PR(AV[d2], nd, d, e, b, rc.l) = T(0); }
      for (int c = rc.f; c <= rc.l; ++c) { PR(AV[d1], nd, d, e, rb.f - 1, c) = T(0); PR(AV[d1], nd, d, e, rb.l, c) = T(0); }
    } else if (d == 1) {
      for (int c = rc.f; c <= rc.l; ++c) { PR(AV[d1], nd, d, e, rb.f - 1, c) = T(0); PR(AV[d1], nd, d, e, rb.l, c) = T(0); }
    }
    rng h = side == 0 ? left_halo_vctr(d) : rght_halo_vctr(d);
    int f = side == 0 ? h.f : h.f + (ad ? 1 : 0);
    int l = side == 0 ? h.l - (ad ? 1 : 0) : h.l;
    for (int ii = f; ii <= l; ++ii)
      for (int b = rb.f; b <= rb.l; ++b)
        for (int c = rc.f; c <= rc.l; ++c) {
          if (side == 0)
            PR(AV[d], nd, d, ii, b, c) = PR(AV[d], nd, d, e, b, c)
              - (PR(AV[d1], nd, d, e, b - 1, c) - PR(AV[d1], nd, d, e, b, c))
              - (PR(AV[d2], nd, d, e, b, c - 1) - PR(AV[d2], nd, d, e, b, c));
          else
            PR(AV[d], nd, d, ii, b, c) = PR(AV[d], nd, d, e - 1, b, c)
              + (PR(AV[d1], nd, d, e, b - 1, c) - PR(AV[d1], nd, d, e, b, c))
              + (PR(AV[d2], nd, d, e, b, c - 1) - PR(AV[d2], nd, d, e, b, c));
        }
  }

  // ---- exchange orchestration: solver_{1,2,3}d.hpp ----
  void xchng_sclr(arr<T> &A, int ex, bool deriv = false) {
    if (nd == 1) { for (int s = 0; s < 2; ++s) fill_sclr(0, s, A, {0, 0}, {0, 0}, deriv); return; }
    if (nd == 2) {  // solver_2d.hpp:40-56
      for (int s = 0; s < 2; ++s) fill_sclr(0, s, A, ext(ir[1], ex), {0, 0}, deriv);
      for (int s = 0; s < 2; ++s) fill_sclr(1, s, A, ext(ir[0], ex), {0, 0}, deriv);
      return;
    }
    // solver_3d.hpp:47-67
    for (int s = 0; s < 2; ++s) fill_sclr(1, s, A, ext(ir[2], ex), ext(ir[0], ex), deriv);
    for (int s = 0; s < 2; ++s) fill_sclr(0, s, A, ext(ir[1], ex), ext(ir[2], ex), deriv);
    for (int s = 0; s < 2; ++s) fill_sclr(2, s, A, ext(ir[0], ex), ext(ir[1], ex), deriv);
  }
  void xchng(int e) { xchng_sclr(psi[e][tl[e]], H); }
  void xchng_vctr_alng(vctr<T> &AV, bool ad = false, bool cyclic = false) {
    if (nd == 1) { for (int s = 0; s < 2; ++s) fill_vctr_alng(0, s, AV, {0, 0}, {0, 0}, ad, cyclic); return; }
    if (nd == 2) {  // solver_2d.hpp:63-88
      for (int s = 0; s < 2; ++s) fill_vctr_alng(0, s, AV, ir[1], {0, 0}, ad, cyclic);
      for (int s = 0; s < 2; ++s) fill_vctr_alng(1, s, AV, ir[0], {0, 0}, ad, cyclic);
      return;
    }
    // solver_3d.hpp:73-103
    for (int s = 0; s < 2; ++s) fill_vctr_alng(0, s, AV, ir[1], ir[2], ad, cyclic);
    for (int s = 0; s < 2; ++s) fill_vctr_alng(1, s, AV, ir[2], ir[0], ad, cyclic);
    for (int s = 0; s < 2; ++s) fill_vctr_alng(2, s, AV, ir[0], ir[1], ad, cyclic);
  }
  void xchng_vctr_nrml(vctr<T> &AV, int ex = 0) {
    if (nd == 1) return;
    if (nd == 2) {  // solver_2d.hpp:171-202
      for (int s = 0; s < 2; ++s) fill_vctr_nrml(1, s, AV[0], exh(ext(ir[0], ex)), {0, 0});
      for (int s = 0; s < 2; ++s) fill_vctr_nrml(0, s, AV[1], exh(ext(ir[1], ex)), {0, 0});
      return;
    }
    // solver_3d.hpp:207-286
    for (int s = 0; s < 2; ++s) fill_vctr_nrml(1, s, AV[0], ext(ext(ir[2], ex), 1), exh(ext(ir[0], ex)));
    for (int s = 0; s < 2; ++s) fill_vctr_nrml(2, s, AV[0], exh(ext(ir[0], ex)), ext(ext(ir[1], ex), 1));
    for (int s = 0; s < 2; ++s) fill_vctr_nrml(0, s, AV[1], exh(ext(ir[1], ex)), ext(ext(ir[2], ex), 1));
    for (int s = 0; s < 2; ++s) fill_vctr_nrml(2, s, AV[1], ext(ext(ir[0], ex), 1), exh(ext(ir[1], ex)));
    for (int s = 0; s < 2; ++s) fill_vctr_nrml(0, s, AV[2], ext(ext(ir[1], ex), 1), exh(ext(ir[2], ex)));
    for (int s = 0; s < 2; ++s) fill_vctr_nrml(1, s, AV[2], exh(ext(ir[2], ex)), ext(ext(ir[0], ex), 1));
  }

  // solver_2d.hpp:90-101, solver_3d.hpp:105-118
  void xchng_flux(vctr<T> &AV) {
    if (nd == 1) { for (int s = 0; s < 2; ++s) fill_flux(0, s, AV, {0, 0}, {0, 0}); return; }
    if (nd == 2) {
      for (int s = 0; s < 2; ++s) fill_flux(0, s, AV, ir[1], {0, 0});
      for (int s = 0; s < 2; ++s) fill_flux(1, s, AV, ir[0], {0, 0});
      return;
    }
    for (int s = 0; s < 2; ++s) fill_flux(0, s, AV, ir[1], ir[2]);
    for (int s = 0; s < 2; ++s) fill_flux(1, s, AV, ir[2], ir[0]);
    for (int s = 0; s < 2; ++s) fill_flux(2, s, AV, ir[0], ir[1]);
  }
  // solver_2d.hpp:204-220, solver_3d.hpp:288-307
  void xchng_pres(arr<T> &A, int ex = 0) {
    if (nd == 1) { for (int s = 0; s < 2; ++s) fill_pres(0, s, A, {0, 0}, {0, 0}); return; }
    if (nd == 2) {
      for (int s = 0; s < 2; ++s) fill_pres(0, s, A, ext(ir[1], ex), {0, 0});
      for (int s = 0; s < 2; ++s) fill_pres(1, s, A, ext(ir[0], ex), {0, 0});
      return;
    }
    for (int s = 0; s < 2; ++s) fill_pres(0, s, A, ext(ir[1], ex), ext(ir[2], ex));
    for (int s = 0; s < 2; ++s) fill_pres(1, s, A, ext(ir[2], ex), ext(ir[0], ex));
    for (int s = 0; s < 2; ++s) fill_pres(2, s, A, ext(ir[0], ex), ext(ir[1], ex));
  }
  // solver_2d.hpp:222-237, solver_3d.hpp:309-326 (the sign argument is unused by every bcond here)
  void set_edges(const std::array<arr<T> *, 3> &AV) {
    if (nd == 1) { for (int s = 0; s < 2; ++s) set_edge_pres(0, s, *AV[0], {0, 0}, {0, 0}); return; }
    if (nd == 2) {
      for (int s = 0; s < 2; ++s) set_edge_pres(0, s, *AV[0], ir[1], {0, 0});
      for (int s = 0; s < 2; ++s) set_edge_pres(1, s, *AV[1], ir[0], {0, 0});
      return;
    }
    for (int s = 0; s < 2; ++s) set_edge_pres(0, s, *AV[0], ir[1], ir[2]);
    for (int s = 0; s < 2; ++s) set_edge_pres(1, s, *AV[1], ir[2], ir[0]);
    for (int s = 0; s < 2; ++s) set_edge_pres(2, s, *AV[2], ir[0], ir[1]);
  }

  // ---- mpdata_common.hpp:40-60 ----
  vctr<T> &GC_unco(int iter) { return iter == 1 ? GC : (iter % 2 ? tmp1 : tmp0); }
  vctr<T> &GC_corr(int iter) { return iter % 2 ? tmp0 : tmp1; }
  vctr<T> &GCit(int iter) {  // virtual GC(iter); fct override mpdata_fct_common.hpp:31-35
    if (iter == 0) return GC;
    if (opts & o_fct) return GC_mono;
    return GC_corr(iter);
  }
  void cycle(int e) { tl[e] = (tl[e] + 1) % 2; }

  // ---- psi-derivative helpers (formulae_mpdata_psi_{1,2,3}d.hpp) ----
  // ndx_psi at (i+1/2): 1D :51-105, 2D :127-185, 3D :262-318
  template <int ND, int D> T ndx(const arr<T> &p, int a, int b, int c) const {
    const T p1 = P<ND, D>(p, a + 1, b, c), p0 = P<ND, D>(p, a, b, c);
    if (opts & o_iga) {
      if (ND == 3) return p1 - p0;
      return T(2) * (p1 - p0) / T(2);
    }
    if (opts & o_abs) return T(2) * frac(opts, std::abs(p1) - std::abs(p0), std::abs(p1) + std::abs(p0));
    return T(2) * frac(opts, p1 - p0, p1 + p0);
  }
  // ndy_psi at (i+1/2): 2D :188-240, 3D :321-392 (b is the +1 frame axis)
  template <int ND, int D> T ndy(const arr<T> &p, int a, int b, int c) const {
    T pa = P<ND, D>(p, a + 1, b + 1, c), pb = P<ND, D>(p, a, b + 1, c);
    T pc = P<ND, D>(p, a + 1, b - 1, c), pd = P<ND, D>(p, a, b - 1, c);
    if (opts & o_iga) return (pa + pb - pc - pd) / T(4);
    if (opts & o_abs) { pa = std::abs(pa); pb = std::abs(pb); pc = std::abs(pc); pd = std::abs(pd); }
    return frac(opts, pa + pb - pc - pd, pa + pb + pc + pd);
  }
  // ndz_psi at (i+1/2): 3D :395-466 (c is the +2 frame axis)
  template <int ND, int D> T ndz(const arr<T> &p, int a, int b, int c) const {
    T pa = P<ND, D>(p, a + 1, b, c + 1), pb = P<ND, D>(p, a, b, c + 1);
    T pc = P<ND, D>(p, a + 1, b, c - 1), pd = P<ND, D>(p, a, b, c - 1);
    if (opts & o_iga) return (pa + pb - pc - pd) / T(4);
    if (opts & o_abs) { pa = std::abs(pa); pb = std::abs(pb); pc = std::abs(pc); pd = std::abs(pd); }
    return frac(opts, pa + pb - pc - pd, pa + pb + pc + pd);
  }
  // ---- third-order terms (formulae_mpdata_hot_{1,2,3}d.hpp), G = 1 ----
  // four-point second derivatives at (a+1/2): 2 (pa - pb - pc + pd) / (pa + pb + pc + pd)
  // (ndxx_psi: psi_1d.hpp:110-161, psi_2d.hpp:246-300, psi_3d.hpp:469-541;
  //  ndxy_psi / ndxz_psi: psi_2d.hpp:305-359, psi_3d.hpp:545-695)
  T nd2(T pa, T pb, T pc, T pd) const {
    if (opts & o_iga) return T(2) * (pa - pb - pc + pd) / T(4);
    if (opts & o_abs) { pa = std::abs(pa); pb = std::abs(pb); pc = std::abs(pc); pd = std::abs(pd); }
    return T(2) * frac(opts, pa - pb - pc + pd, pa + pb + pc + pd);
  }
  template <int ND, int D> T ndxx(const arr<T> &p, int a, int b, int c) const {
    return nd2(P<ND, D>(p, a + 2, b, c), P<ND, D>(p, a + 1, b, c), P<ND, D>(p, a, b, c), P<ND, D>(p, a - 1, b, c));
  }
  template <int ND, int D> T ndxy(const arr<T> &p, int a, int b, int c) const {
    return nd2(P<ND, D>(p, a + 1, b + 1, c), P<ND, D>(p, a, b + 1, c), P<ND, D>(p, a + 1, b - 1, c), P<ND, D>(p, a, b - 1, c));
  }
  template <int D> T ndxz(const arr<T> &p, int a, int b, int c) const {
    return nd2(P<3, D>(p, a + 1, b, c + 1), P<3, D>(p, a, b, c + 1), P<3, D>(p, a + 1, b, c - 1), P<3, D>(p, a, b, c - 1));
  }
  // ndyz_psi (psi_3d.hpp:697-790): eight corners, no factor 2
  template <int D> T ndyz(const arr<T> &p, int a, int b, int c) const {
    T q[8] = {P<3, D>(p, a + 1, b + 1, c + 1), P<3, D>(p, a + 1, b - 1, c - 1), P<3, D>(p, a + 1, b + 1, c - 1),
              P<3, D>(p, a + 1, b - 1, c + 1), P<3, D>(p, a, b + 1, c + 1),     P<3, D>(p, a, b - 1, c - 1),
              P<3, D>(p, a, b + 1, c - 1),     P<3, D>(p, a, b - 1, c + 1)};
    const T num = q[0] + q[1] - q[2] - q[3] + q[4] + q[5] - q[6] - q[7];
    if (opts & o_iga) return num / T(8);
    if (opts & o_abs) for (T &v : q) v = std::abs(v);
    return frac(opts, q[0] + q[1] - q[2] - q[3] + q[4] + q[5] - q[6] - q[7],
                q[0] + q[1] + q[2] + q[3] + q[4] + q[5] + q[6] + q[7]);
  }
  // coefficients (hot_1d.hpp:19-40, hot_2d.hpp:21-50, hot_3d.hpp:21-95); gb = G_bar_x,
  // pow2/pow3 as products
  static T cxx(T C, T gb) { return (T(3) * C * std::abs(C) / gb - T(2) * (C * C * C) / (gb * gb) - C) / T(6); }
  static T cxy(T C, T g, T gb) { return (std::abs(C) - T(2) * (C * C) / gb) * g / (T(2) * gb); }
  static T cyz(T C, T g1, T g2, T gb) { return T(-2) * C * g1 * g2 / T(3) / (gb * gb); }
  // fourth-order terms of the 2D antidiffusive velocity, iga only
  // (formulae_mpdata_hot_2d.hpp:82-157): the third derivatives ndxxx, ndxxy, ndxyy
  // (formulae_mpdata_psi_2d.hpp:360-412) times their Courant-number coefficients;
  // cy = GC1_bar_xy, gb = G_bar_x; pow2 and pow3 as products, pow4(x) as (x x)(x x)
  // (Blitz++'s own evaluation order of pow4 cannot be checked here)
  template <int D> T fot2(const arr<T> &p, int a, int b, T C, T cy, T gb) const {
    auto ps = [&](int x, int y) { return P<2, D>(p, x, y, 0); };
    const T nxxx = (ps(a + 2, b) - T(3) * ps(a + 1, b) + T(3) * ps(a, b) - ps(a - 1, b)) / T(4);
    const T nxxy = (ps(a + 2, b + 1) - ps(a + 1, b + 1) - ps(a, b + 1) + ps(a - 1, b + 1) - ps(a + 2, b - 1)
                    + ps(a + 1, b - 1) + ps(a, b - 1) - ps(a - 1, b - 1)) / T(8);
    const T nxyy = (ps(a + 1, b + 1) - T(2) * ps(a + 1, b) + ps(a + 1, b - 1) - ps(a, b + 1) + T(2) * ps(a, b)
                    - ps(a, b - 1)) / T(6);
    const T aC = std::abs(C), C2 = C * C, C4 = (C * C) * (C * C), gb2 = gb * gb, gb3 = gb * gb * gb;
    const T acy = std::abs(cy), cy2 = cy * cy;
    const T cxxx = (T(6) * aC * C2 / gb2 - T(3) * C2 / gb - T(3) * C4 / gb3) / T(2);
    const T cxxy = T(3) * (aC - C2 / gb) * C * cy / gb2;
    const T cxyy = T(3) * (T(3) * acy * C2 / gb + T(3) * cy2 * aC / gb - T(2) * acy * aC - T(9) * cy2 * C2 / gb2) / gb / T(4);
    return nxxx * cxxx + nxxy * cxxy + nxyy * cxyy;
  }

  // ---- divergent-flow correction (formulae_mpdata_dfl_{1,2,3}d.hpp), G = 1 ----
  // -C/4/G_bar_x (div of the advector around the face) [x psi_bar_x with iga];
  // 1D: -C/2/(G(i+1)+G(i)) dC
  template <int ND, int D> T dfl(const arr<T> &p, const arr<T> &Gd, const arr<T> &G1, const arr<T> &G2, int a, int b, int c) const {
    const T C = P<ND, D>(Gd, a, b, c);
    T r;
    if (ND == 1) {
      r = T(-0.5) * C / (Gc(a + 1, 0, 0) + Gc(a, 0, 0)) * (P<ND, D>(Gd, a + 1, b, c) - P<ND, D>(Gd, a - 1, b, c));
      if (opts & o_iga) r = r * T(0.5) * (P<ND, D>(p, a + 1, b, c) + P<ND, D>(p, a, b, c));
      return r;
    }
    T s = (P<ND, D>(Gd, a + 1, b, c) - P<ND, D>(Gd, a - 1, b, c))
        + (P<ND, D>(G1, a + 1, b, c) + P<ND, D>(G1, a, b, c) - P<ND, D>(G1, a + 1, b - 1, c) - P<ND, D>(G1, a, b - 1, c));
    if (ND == 3)
      s = s + (P<ND, D>(G2, a + 1, b, c) + P<ND, D>(G2, a, b, c) - P<ND, D>(G2, a + 1, b, c - 1) - P<ND, D>(G2, a, b, c - 1));
    r = T(-0.25) * C / Gbar<ND, D>(a, b, c) * s;
    if (opts & o_iga) r = r * ((P<ND, D>(p, a + 1, b, c) + P<ND, D>(p, a, b, c)) / T(2));
    return r;
  }

  // ---- antidiffusive velocity ----
  // The reference adds TOT and DFL as integer zeros when the options are off;
  // they are left out here (x + 0 differs from x only in the sign of a zero).
  // 1D: formulae_mpdata_1d.hpp:186-210
  void antidiff1(arr<T> &res, const arr<T> &p, const vctr<T> &G) {
    for (int i = im[0].f; i <= im[0].l; ++i) {
      const T C = G[0](i, 0, 0), gb = Gbar<1, 0>(i, 0, 0);
      T r = std::abs(C) / T(2) * (T(1) - std::abs(C) / gb) * ndx<1, 0>(p, i, 0, 0);
      if (opts & o_tot) r = r + ndxx<1, 0>(p, i, 0, 0) * cxx(C, gb);
      if (opts & o_dfl) r = r + dfl<1, 0>(p, G[0], G[0], G[0], i, 0, 0);
      res(i, 0, 0) = r;
    }
  }
  // 2D: formulae_mpdata_2d.hpp:242-278 with GC1_bar_xy (formulae_mpdata_gc_2d.hpp:76-90)
  template <int D> void antidiff2(arr<T> &res, const arr<T> &p, const vctr<T> &G) {
    const arr<T> &Gd = G[D], &Gt = G[(D + 1) % 2];
    const rng ra = im[D], rb = ir[(D + 1) % 2];
    for (int a = ra.f; a <= ra.l; ++a)
      for (int b = rb.f; b <= rb.l; ++b) {
        const T C = P<2, D>(Gd, a, b), gb = Gbar<2, D>(a, b, 0);
        const T gc1 = (P<2, D>(Gt, a + 1, b) + P<2, D>(Gt, a, b) + P<2, D>(Gt, a + 1, b - 1) + P<2, D>(Gt, a, b - 1)) / T(4);
        T r = std::abs(C) / T(2) * (T(1) - std::abs(C) / gb) * ndx<2, D>(p, a, b, 0)
            - C * gc1 / (T(2) * gb) * ndy<2, D>(p, a, b, 0);
        if (opts & o_tot) r = r + (ndxx<2, D>(p, a, b, 0) * cxx(C, gb) + ndxy<2, D>(p, a, b, 0) * cxy(C, gc1, gb));
        if (opts & o_fot) r = r + fot2<D>(p, a, b, C, gc1, gb);
        if (opts & o_dfl) r = r + dfl<2, D>(p, Gd, Gt, Gt, a, b, 0);
        P<2, D>(res, a, b) = r;
      }
  }
  // 3D: formulae_mpdata_3d.hpp:254-295 with GC1_bar_xy / GC2_bar_xz (formulae_mpdata_gc_3d.hpp:100-170)
  template <int D> void antidiff3(arr<T> &res, const arr<T> &p, const vctr<T> &G) {
    const arr<T> &Gd = G[D], &G1 = G[(D + 1) % 3], &G2 = G[(D + 2) % 3];
    const rng ra = im[D], rb = ir[(D + 1) % 3], rc = ir[(D + 2) % 3];
    box<3, D>(ra, rb, rc, [&](int a, int b, int c) {
          const T C = P<3, D>(Gd, a, b, c), gb = Gbar<3, D>(a, b, c);
          const T gc1 = (P<3, D>(G1, a + 1, b, c) + P<3, D>(G1, a, b, c) + P<3, D>(G1, a + 1, b - 1, c) + P<3, D>(G1, a, b - 1, c)) / T(4);
          const T gc2 = (P<3, D>(G2, a + 1, b, c) + P<3, D>(G2, a, b, c) + P<3, D>(G2, a + 1, b, c - 1) + P<3, D>(G2, a, b, c - 1)) / T(4);
          T r = std::abs(C) / T(2) * (T(1) - std::abs(C) / gb) * ndx<3, D>(p, a, b, c)
              - C / T(2) * (gc1 * ndy<3, D>(p, a, b, c) + gc2 * ndz<3, D>(p, a, b, c)) / gb;
          if (opts & o_tot)
            r = r + (ndxx<3, D>(p, a, b, c) * cxx(C, gb) + ndxy<3, D>(p, a, b, c) * cxy(C, gc1, gb)
                     + ndxz<D>(p, a, b, c) * cxy(C, gc2, gb) + ndyz<D>(p, a, b, c) * cyz(C, gc1, gc2, gb));
          if (opts & o_dfl) r = r + dfl<3, D>(p, Gd, G1, G2, a, b, c);
          P<3, D>(res, a, b, c) = r;
        });
  }

  // ---- divergence-form antidiffusive velocity: div_2nd + div_3rd / div_3rd_dt
  // (formulae_mpdata_{1,2,3}d.hpp, helpers of formulae_mpdata_fdiv_{1,2,3}d.hpp,
  // _psi_*, _gc_*, _g_*).  p is the current iterate psi_np1 and pn the other
  // time level psi_n (psi[e][n-1]); G0 = GC[dim], G1 = GC[dim+1], G2 = GC[dim-1]
  // (= GC[dim+2] in 3D).  The advector of solvers::mpdata does not change in
  // time, so its time derivatives ndt_GC and ndtt_GC are zero
  // (mpdata_osc_{1,2,3}d.hpp hook_ante_loop) and the temporal terms that
  // multiply them are exact zeros, left out as TOT and DFL are above.  In 1D the
  // reference has no div_3rd_dt form: there it adds nothing to div_2nd.
  template <int ND, int D>
  T adiv(const arr<T> &p, const arr<T> &pn, const arr<T> &G0, const arr<T> &G1, const arr<T> &G2, int a, int b, int c) const {
    const bool iga = opts & o_iga, ab = opts & o_abs;
    auto q = [&](const arr<T> &A, int x, int y, int z) { const T v = P<ND, D>(A, x, y, z); return ab ? std::abs(v) : v; };
    auto ps = [&](int x, int y, int z) { return q(p, x, y, z); };
    auto g = [&](int x, int y, int z) { return Gc3<ND, D>(x, y, z); };
    auto G = [&](const arr<T> &A, int x, int y, int z) { return P<ND, D>(A, x, y, z); };
    // interpolated psi (psi_bar_*: abs of each value with the abs option)
    auto pbx = [&](const arr<T> &A, int x, int y, int z) { return (q(A, x + 1, y, z) + q(A, x, y, z)) / T(2); };
    auto pby = [&](const arr<T> &A, int x, int y, int z) { return (q(A, x, y, z) + q(A, x, y + 1, z)) / T(2); };
    auto pbz = [&](const arr<T> &A, int x, int y, int z) { return (q(A, x, y, z) + q(A, x, y, z + 1)) / T(2); };
    auto pbxy = [&](const arr<T> &A, int x, int y, int z) {
      return (q(A, x + 1, y, z) + q(A, x, y, z) + q(A, x, y + 1, z) + q(A, x + 1, y + 1, z)) / T(4);
    };
    auto pbxz = [&](const arr<T> &A, int x, int y, int z) {
      return (q(A, x + 1, y, z) + q(A, x, y, z) + q(A, x, y, z + 1) + q(A, x + 1, y, z + 1)) / T(4);
    };
    auto pbxyz = [&](const arr<T> &A, int x, int y, int z) {
      return (q(A, x, y, z) + q(A, x + 1, y, z) + q(A, x, y + 1, z) + q(A, x, y, z + 1) + q(A, x + 1, y + 1, z)
              + q(A, x + 1, y, z + 1) + q(A, x, y + 1, z + 1) + q(A, x + 1, y + 1, z + 1)) / T(8);
    };
    // Courant-number averages (GC0_bar_x ... GC2_bar_xz; face x+1/2 stored at x)
    auto g0bx = [&](int x, int y, int z) { return (G(G0, x, y, z) + G(G0, x - 1, y, z)) / T(2); };
    auto g1bx = [&](int x, int y, int z) { return (G(G1, x + 1, y, z) + G(G1, x, y, z)) / T(2); };
    auto g2bx = [&](int x, int y, int z) { return (G(G2, x + 1, y, z) + G(G2, x, y, z)) / T(2); };
    auto g0bxy = [&](int x, int y, int z) { return (G(G0, x, y, z) + G(G0, x - 1, y, z) + G(G0, x, y + 1, z) + G(G0, x - 1, y + 1, z)) / T(4); };
    auto g1bxy = [&](int x, int y, int z) { return (G(G1, x + 1, y, z) + G(G1, x, y, z) + G(G1, x + 1, y - 1, z) + G(G1, x, y - 1, z)) / T(4); };
    auto g2bxy = [&](int x, int y, int z) { return (G(G2, x + 1, y + 1, z) + G(G2, x, y + 1, z) + G(G2, x + 1, y, z) + G(G2, x, y, z)) / T(4); };
    auto g0bxz = [&](int x, int y, int z) { return (G(G0, x, y, z) + G(G0, x - 1, y, z) + G(G0, x, y, z + 1) + G(G0, x - 1, y, z + 1)) / T(4); };
    auto g1bxz = [&](int x, int y, int z) { return (G(G1, x + 1, y, z) + G(G1, x + 1, y, z + 1) + G(G1, x, y, z) + G(G1, x, y, z + 1)) / T(4); };
    auto g2bxz = [&](int x, int y, int z) { return (G(G2, x + 1, y, z) + G(G2, x, y, z) + G(G2, x + 1, y, z - 1) + G(G2, x, y, z - 1)) / T(4); };
    // G averages (formulae_mpdata_g_{1,2,3}d.hpp): 1 without nug
    const bool nug = opts & o_nug;
    auto gbx = [&](int x, int y, int z) { return nug ? (g(x + 1, y, z) + g(x, y, z)) / T(2) : T(1); };
    auto gbxy = [&](int x, int y, int z) { return nug ? (g(x, y, z) + g(x, y + 1, z) + g(x + 1, y, z) + g(x + 1, y + 1, z)) / T(4) : T(1); };
    auto gbxz = [&](int x, int y, int z) { return nug ? (g(x, y, z) + g(x, y, z + 1) + g(x + 1, y, z) + g(x + 1, y, z + 1)) / T(4) : T(1); };
    // flux divergences at the cell centre and at the xy / xz edges
    auto fc = [&](int x, int y, int z) {
      T r = G(G0, x, y, z) * pbx(p, x, y, z) - G(G0, x - 1, y, z) * pbx(p, x - 1, y, z);
      if (ND > 1) r = r + G(G1, x, y, z) * pby(p, x, y, z) - G(G1, x, y - 1, z) * pby(p, x, y - 1, z);
      if (ND > 2) r = r + G(G2, x, y, z) * pbz(p, x, y, z) - G(G2, x, y, z - 1) * pbz(p, x, y, z - 1);
      return r / g(x, y, z);
    };
    auto fxy = [&](int x, int y, int z) {
      T r = g0bxy(x + 1, y, z) * pby(p, x + 1, y, z) - g0bxy(x, y, z) * pby(p, x, y, z)
          + g1bxy(x, y + 1, z) * pbx(p, x, y + 1, z) - g1bxy(x, y, z) * pbx(p, x, y, z);
      if (ND > 2) r = r + g2bxy(x, y, z) * pbxyz(p, x, y, z) - g2bxy(x, y, z - 1) * pbxyz(p, x, y, z - 1);
      return r / gbxy(x, y, z);
    };
    auto fxz = [&](int x, int y, int z) {
      return (g0bxz(x + 1, y, z) * pbz(p, x + 1, y, z) - g0bxz(x, y, z) * pbz(p, x, y, z)
              + g1bxz(x, y, z) * pbxyz(p, x, y, z) - g1bxz(x, y - 1, z) * pbxyz(p, x, y - 1, z)
              + g2bxz(x, y, z + 1) * pbx(p, x, y, z + 1) - g2bxz(x, y, z) * pbx(p, x, y, z)) / gbxz(x, y, z);
    };
    // numerator of the nondimensionalised flux divergence at (a+1/2) (nfdiv)
    auto nfdiv_num = [&]() {
      T r = g0bx(a + 1, b, c) * ps(a + 1, b, c) - g0bx(a, b, c) * ps(a, b, c);
      if (ND > 1) r = r + g1bx(a, b, c) * pbxy(p, a, b, c) - g1bx(a, b - 1, c) * pbxy(p, a, b - 1, c);
      if (ND > 2) r = r + g2bx(a, b, c) * pbxz(p, a, b, c) - g2bx(a, b, c - 1) * pbxz(p, a, b, c - 1);
      return r;
    };
    // sums of psi in the denominators (their orders follow the reference)
    auto s_nfdiv = [&](const arr<T> &A) {
      if (ND == 1) return q(A, a + 1, b, c) + q(A, a, b, c);
      if (ND == 2)
        return q(A, a + 1, b, c) + q(A, a, b, c) + q(A, a, b + 1, c) + q(A, a + 1, b + 1, c) + q(A, a, b - 1, c) + q(A, a + 1, b - 1, c);
      return q(A, a + 1, b, c) + q(A, a, b, c) + q(A, a, b + 1, c) + q(A, a + 1, b + 1, c) + q(A, a, b - 1, c)
           + q(A, a + 1, b - 1, c) + q(A, a + 1, b, c + 1) + q(A, a + 1, b, c - 1) + q(A, a, b, c - 1) + q(A, a, b, c + 1);
    };
    auto s4 = [&]() { return ps(a + 2, b, c) + ps(a + 1, b, c) + ps(a, b, c) + ps(a - 1, b, c); };
    auto s_nfdiv_fdiv = [&]() {
      if (ND == 1) return s4();
      if (ND == 2) return s4() + ps(a, b + 1, c) + ps(a, b - 1, c) + ps(a + 1, b + 1, c) + ps(a + 1, b - 1, c);
      return s4() + ps(a, b + 1, c) + ps(a, b - 1, c) + ps(a + 1, b + 1, c) + ps(a + 1, b - 1, c) + ps(a, b, c + 1)
           + ps(a, b, c - 1) + ps(a + 1, b, c + 1) + ps(a + 1, b, c - 1);
    };
    auto s_ndx_fdiv = [&]() {
      if (ND < 3) return s_nfdiv_fdiv();
      return s4() + ps(a, b + 1, c) + ps(a, b - 1, c) + ps(a, b, c - 1) + ps(a, b, c + 1) + ps(a + 1, b + 1, c)
           + ps(a + 1, b - 1, c) + ps(a + 1, b, c - 1) + ps(a + 1, b, c + 1);
    };
    const T m1 = T(2 + 4 * (ND - 1)), m2 = T(4 + 4 * (ND - 1));
    const T C = G(G0, a, b, c);
    const T nfdiv = iga ? nfdiv_num() / gbx(a, b, c) : m1 * frac(opts, nfdiv_num(), gbx(a, b, c) * s_nfdiv(p));
    const T ndxp = ndx<ND, D>(p, a, b, c);
    const T d2 = std::abs(C) / 2 * ndxp - C / 2 * nfdiv;  // div_2nd
    const bool dt = (opts & o_div_3rd_dt) && ND > 1;
    if (!(opts & o_div_3rd) && !dt) return d2;
    // div_3rd: upwind-differencing correction (none with iga), spatial, mixed and temporal terms
    const T up = iga ? T(0) : std::abs(d2) / 2 * ndxp;
    const T ndxx_gc = G(G0, a + 1, b, c) + G(G0, a - 1, b, c) - 2 * G(G0, a, b, c);
    const T nxxg = iga ? ndxx_gc * pbx(p, a, b, c) : ndxx_gc;
    const T helper = sptl_intrp == 0 ? nxxg : (sptl_intrp == 1 ? 4 * nxxg : T(0));
    const T spatial = -T(1.0 / 24) * (4 * C * ndxx<ND, D>(p, a, b, c)
                                      + 2 * ndxp * ((G(G0, a + 1, b, c) - G(G0, a - 1, b, c)) / 2) + helper);
    if (!dt) {
      auto nfdiv_fdiv_num = [&]() {
        T r = g0bx(a + 1, b, c) * fc(a + 1, b, c) - g0bx(a, b, c) * fc(a, b, c);
        if (ND > 1) r = r + g1bx(a, b, c) * fxy(a, b, c) - g1bx(a, b - 1, c) * fxy(a, b - 1, c);
        if (ND > 2) r = r + g2bx(a, b, c) * fxz(a, b, c) - g2bx(a, b, c - 1) * fxz(a, b, c - 1);
        return r;
      };
      const T dfc = fc(a + 1, b, c) - fc(a, b, c);
      const T ndx_fdiv = iga ? dfc : m2 * frac(opts, dfc, s_ndx_fdiv());
      const T nfdiv_fdiv = iga ? nfdiv_fdiv_num() / gbx(a, b, c) : m2 * frac(opts, nfdiv_fdiv_num(), gbx(a, b, c) * s_nfdiv_fdiv());
      const T r3 = d2 + (up + spatial + T(0.5) * std::abs(C) * ndx_fdiv + T(1.0 / 24) * (-8 * C * nfdiv_fdiv));
      if constexpr (ND == 2)
        if (opts & o_fot) return r3 + fot_div<D>(p, G0, G1, a, b);
      return r3;
    }
    // div_3rd_dt (2D, 3D)
    auto dq = [&](int x, int y, int z) { return q(p, x, y, z) - q(pn, x, y, z); };
    T ndtx;
    {
      const T p1 = P<ND, D>(p, a + 1, b, c), n1 = P<ND, D>(pn, a + 1, b, c), p0 = P<ND, D>(p, a, b, c), n0 = P<ND, D>(pn, a, b, c);
      if (iga) ndtx = p1 - n1 - p0 + n0;
      else if (ab) ndtx = 4 * frac(opts, std::abs(p1) - std::abs(n1) - std::abs(p0) + std::abs(n0),
                                   std::abs(p1) + std::abs(n1) + std::abs(p0) + std::abs(n0));
      else ndtx = 4 * frac(opts, p1 - n1 - p0 + n0, p1 + n1 + p0 + n0);
    }
    T ndt_num = g0bx(a + 1, b, c) * dq(a + 1, b, c) - g0bx(a, b, c) * dq(a, b, c)
              + g1bx(a, b, c) * (pbxy(p, a, b, c) - pbxy(pn, a, b, c)) - g1bx(a, b - 1, c) * (pbxy(p, a, b - 1, c) - pbxy(pn, a, b - 1, c));
    if (ND > 2)
      ndt_num = ndt_num + g2bx(a, b, c) * (pbxz(p, a, b, c) - pbxz(pn, a, b, c)) - g2bx(a, b, c - 1) * (pbxz(p, a, b, c - 1) - pbxz(pn, a, b, c - 1));
    const T m4 = T(ND == 2 ? 12 : 20);
    // the denominator sums the psi_np1 values, then the psi_n values, as one chain
    T s_dt = s_nfdiv(p);
    if (!iga) {
      if (ND == 2)
        s_dt = s_dt + q(pn, a + 1, b, c) + q(pn, a, b, c) + q(pn, a, b + 1, c) + q(pn, a + 1, b + 1, c) + q(pn, a, b - 1, c)
             + q(pn, a + 1, b - 1, c);
      else
        s_dt = s_dt + q(pn, a + 1, b, c) + q(pn, a, b, c) + q(pn, a, b + 1, c) + q(pn, a + 1, b + 1, c) + q(pn, a, b - 1, c)
             + q(pn, a + 1, b - 1, c) + q(pn, a + 1, b, c + 1) + q(pn, a + 1, b, c - 1) + q(pn, a, b, c - 1) + q(pn, a, b, c + 1);
    }
    const T nfdiv_dt = iga ? ndt_num / gbx(a, b, c) : m4 * frac(opts, ndt_num, gbx(a, b, c) * s_dt);
    const T r3 = d2 + (up + spatial - T(0.5) * std::abs(C) * ndtx + T(1.0 / 24) * (8 * C * nfdiv_dt));
    if constexpr (ND == 2)
      if (opts & o_fot) return r3 + fot_div<D>(p, G0, G1, a, b);
    return r3;
  }
  // the fourth-order terms added to the 2D divergence form (formulae_mpdata_2d.hpp:300-305)
  template <int D> T fot_div(const arr<T> &p, const arr<T> &G0, const arr<T> &G1, int a, int b) const {
    const T C = P<2, D>(G0, a, b, 0), gb = Gbar<2, D>(a, b, 0);
    const T cy = (P<2, D>(G1, a + 1, b, 0) + P<2, D>(G1, a, b, 0) + P<2, D>(G1, a + 1, b - 1, 0) + P<2, D>(G1, a, b - 1, 0)) / T(4);
    return fot2<D>(p, a, b, C, cy, gb);
  }
  // res over faces im along D x interior across (formulae_mpdata_{1,2,3}d.hpp antidiff, divergence form)
  template <int ND, int D> void antidiff_div(arr<T> &res, const arr<T> &p, const arr<T> &pn, const vctr<T> &G) {
    const arr<T> &G0 = G[D], &G1 = G[(D + 1) % ND], &G2 = G[(D + 2) % ND];
    const rng ra = im[D], rb = ND > 1 ? ir[(D + 1) % ND] : rng{0, 0}, rc = ND > 2 ? ir[(D + 2) % ND] : rng{0, 0};
    box<ND, D>(ra, rb, rc, [&](int a, int b, int c) { P<ND, D>(res, a, b, c) = adiv<ND, D>(p, pn, G0, G1, G2, a, b, c); });
  }
  // G at a frame point (formulae::G; 1 without nug)
  template <int ND, int D> T Gc3(int a, int b, int c) const { return (opts & o_nug) ? P<ND, D>(Gf, a, b, c) : T(1); }

  // ---- donor-cell flux over faces ra (frame a) x rb x rc (make_flux, donorcell_formulae.hpp:36-79) ----
  template <int ND, int D> void make_flux(arr<T> &F, const arr<T> &p, const arr<T> &C, rng ra, rng rb, rng rc) {
    box<ND, D>(ra, rb, rc, [&](int a, int b, int c) {
      P<ND, D>(F, a, b, c) = Fdc(opts, P<ND, D>(p, a, b, c), P<ND, D>(p, a + 1, b, c), P<ND, D>(C, a, b, c));
    });
  }
  void fluxes(vctr<T> &F, const arr<T> &p, const vctr<T> &C, bool extended) {
    // extended: ranges im^1 x j^1 x k^1 (fct_adjust_antidiff); else im x j x k
    auto R = [&](int d) { return extended ? ext(ir[d], 1) : ir[d]; };
    auto RM = [&](int d) { return extended ? ext(im[d], 1) : im[d]; };
    if (nd == 1) make_flux<1, 0>(F[0], p, C[0], RM(0), {0, 0}, {0, 0});
    else if (nd == 2) {
      make_flux<2, 0>(F[0], p, C[0], RM(0), R(1), {0, 0});
      make_flux<2, 1>(F[1], p, C[1], RM(1), R(0), {0, 0});
    } else {
      make_flux<3, 0>(F[0], p, C[0], RM(0), R(1), R(2));
      make_flux<3, 1>(F[1], p, C[1], RM(1), R(2), R(0));
      make_flux<3, 2>(F[2], p, C[2], RM(2), R(0), R(1));
    }
  }

  // ---- donorcell_sum (donorcell_formulae.hpp:81-165), divided by G; Kahan variant with khn ----
  void donorcell_sum(arr<T> &pn, const arr<T> &po, const vctr<T> &f) {
#pragma omp parallel for schedule(static) if (big())
    for (int i = 0; i < n[0]; ++i)
      for (int j = 0; j < n[1]; ++j)
        for (int k = 0; k < n[2]; ++k) {
          const T g = Gc(i, j, k);
          if (opts & o_khn) {
            // Kahan-compensated sum (kahan_sum.hpp:14-27): psi_old, then -F(+1/2)/G and
            // F(-1/2)/G per dimension
            T sum = T(0), c = T(0);
            auto add = [&](T in) { const T y = in - c; const T t = sum + y; c = (t - sum) - y; sum = t; };
            add(po(i, j, k));
            add(-f[0](i, j, k) / g);
            add(f[0](i - 1, j, k) / g);
            if (nd > 1) { add(-f[1](i, j, k) / g); add(f[1](i, j - 1, k) / g); }
            if (nd > 2) { add(-f[2](i, j, k) / g); add(f[2](i, j, k - 1) / g); }
            pn(i, j, k) = sum;
          } else if (nd == 1)
            pn(i, j, k) = po(i, j, k) + (-f[0](i, j, k) + f[0](i - 1, j, k)) / g;
          else if (nd == 2)
            pn(i, j, k) = po(i, j, k) + ((-f[0](i, j, k) + f[0](i - 1, j, k)) + (-f[1](i, j, k) + f[1](i, j - 1, k))) / g;
          else
            pn(i, j, k) = po(i, j, k) + ((-f[0](i, j, k) + f[0](i - 1, j, k)) + (-f[1](i, j, k) + f[1](i, j - 1, k))
                                         + (-f[2](i, j, k) + f[2](i, j, k - 1))) / g;
        }
  }

  // ---- FCT: fct_init (mpdata_fct_{1,2,3}d.hpp:31-55) ----
  void fct_init(int e) {
    const arr<T> &p = psi[e][tl[e]];
    rng r0 = ext(ir[0], 1), r1 = nd > 1 ? ext(ir[1], 1) : rng{0, 0}, r2 = nd > 2 ? ext(ir[2], 1) : rng{0, 0};
#pragma omp parallel for schedule(static) if (big())
    for (int i = r0.f; i <= r0.l; ++i)
      for (int j = r1.f; j <= r1.l; ++j)
        for (int k = r2.f; k <= r2.l; ++k) {
          T mn, mx;
          if (nd == 1) {
            mn = std::min(std::min(p(i - 1, 0, 0), p(i, 0, 0)), p(i + 1, 0, 0));
            mx = std::max(std::max(p(i - 1, 0, 0), p(i, 0, 0)), p(i + 1, 0, 0));
          } else if (nd == 2) {
            mn = std::min(std::min(std::min(std::min(p(i, j + 1, 0), p(i - 1, j, 0)), p(i, j, 0)), p(i + 1, j, 0)), p(i, j - 1, 0));
            mx = std::max(std::max(std::max(std::max(p(i, j + 1, 0), p(i - 1, j, 0)), p(i, j, 0)), p(i + 1, j, 0)), p(i, j - 1, 0));
          } else {
            mn = std::min(std::min(std::min(std::min(std::min(std::min(p(i, j, k), p(i + 1, j, k)), p(i - 1, j, k)), p(i, j + 1, k)), p(i, j - 1, k)), p(i, j, k + 1)), p(i, j, k - 1));
            mx = std::max(std::max(std::max(std::max(std::max(std::max(p(i, j, k), p(i + 1, j, k)), p(i - 1, j, k)), p(i, j + 1, k)), p(i, j - 1, k)), p(i, j, k + 1)), p(i, j, k - 1));
          }
          psi_min(i, j, k) = mn;
          psi_max(i, j, k) = mx;
        }
  }

  // ---- beta_up / beta_dn (formulae_mpdata_fct_{1,2,3}d.hpp) over i^1 x j^1 x k^1 ----
  void betas(const arr<T> &p, const vctr<T> &f) {
    rng r0 = ext(ir[0], 1), r1 = nd > 1 ? ext(ir[1], 1) : rng{0, 0}, r2 = nd > 2 ? ext(ir[2], 1) : rng{0, 0};
    const unsigned o = opts;
#pragma omp parallel for schedule(static) if (big())
    for (int i = r0.f; i <= r0.l; ++i)
      for (int j = r1.f; j <= r1.l; ++j)
        for (int k = r2.f; k <= r2.l; ++k) {
          const T c = p(i, j, k);
          T mx, mn, den_up, den_dn;
          if (nd == 1) {
            mx = std::max(psi_max(i, j, k), std::max(p(i - 1, j, k), std::max(c, p(i + 1, j, k))));
            mn = std::min(psi_min(i, j, k), std::min(p(i - 1, j, k), std::min(c, p(i + 1, j, k))));
            den_up = pospart(o, f[0](i - 1, j, k)) - negpart(o, f[0](i, j, k));
            den_dn = pospart(o, f[0](i, j, k)) - negpart(o, f[0](i - 1, j, k));
          } else if (nd == 2) {
            // max(psi_max, psi(i,j+1), psi(i-1,j), psi(i,j), psi(i+1,j), psi(i,j-1)) as a right fold
            mx = std::max(psi_max(i, j, k), std::max(p(i, j + 1, k), std::max(p(i - 1, j, k), std::max(c, std::max(p(i + 1, j, k), p(i, j - 1, k))))));
            mn = std::min(psi_min(i, j, k), std::min(p(i, j + 1, k), std::min(p(i - 1, j, k), std::min(c, std::min(p(i + 1, j, k), p(i, j - 1, k))))));
            den_up = (pospart(o, f[0](i - 1, j, k)) - negpart(o, f[0](i, j, k)))
                   + (pospart(o, f[1](i, j - 1, k)) - negpart(o, f[1](i, j, k)));
            den_dn = (pospart(o, f[0](i, j, k)) - negpart(o, f[0](i - 1, j, k)))
                   + (pospart(o, f[1](i, j, k)) - negpart(o, f[1](i, j - 1, k)));
          } else {
            mx = std::max(psi_max(i, j, k), std::max(c, std::max(p(i + 1, j, k), std::max(p(i - 1, j, k),
                   std::max(p(i, j + 1, k), std::max(p(i, j - 1, k), std::max(p(i, j, k + 1), p(i, j, k - 1))))))));
            mn = std::min(psi_min(i, j, k), std::min(p(i, j + 1, k), std::min(p(i - 1, j, k), std::min(c,
                   std::min(p(i + 1, j, k), std::min(p(i, j, k + 1), std::min(p(i, j, k - 1), p(i, j - 1, k))))))));
            den_up = (pospart(o, f[0](i - 1, j, k)) - negpart(o, f[0](i, j, k)))
                   + (pospart(o, f[1](i, j - 1, k)) - negpart(o, f[1](i, j, k)))
                   + (pospart(o, f[2](i, j, k - 1)) - negpart(o, f[2](i, j, k)));
            den_dn = (pospart(o, f[0](i, j, k)) - negpart(o, f[0](i - 1, j, k)))
                   + (pospart(o, f[1](i, j, k)) - negpart(o, f[1](i, j - 1, k)))
                   + (pospart(o, f[2](i, j, k)) - negpart(o, f[2](i, j, k - 1)));
          }
          beta_up(i, j, k) = fct_frac((mx - c) * Gc(i, j, k), den_up);
          beta_dn(i, j, k) = fct_frac((c - mn) * Gc(i, j, k), den_dn);
        }
  }

  // ---- GC_mono (formulae_mpdata_fct_{1,2,3}d.hpp) over im x j x k ----
  template <int ND, int D> void gc_mono(arr<T> &out, const arr<T> &corr, const arr<T> &p) {
    const rng ra = im[D];
    const rng rb = ND > 1 ? ir[(D + 1) % ND] : rng{0, 0};
    const rng rc = ND > 2 ? ir[(D + 2) % ND] : rng{0, 0};
    const bool absv = (opts & o_abs) && !(opts & o_iga);
    box<ND, D>(ra, rb, rc, [&](int a, int b, int c) {
          const T C = P<ND, D>(corr, a, b, c);
          const T bd0 = P<ND, D>(beta_dn, a, b, c), bu1 = P<ND, D>(beta_up, a + 1, b, c);
          const T bu0 = P<ND, D>(beta_up, a, b, c), bd1 = P<ND, D>(beta_dn, a + 1, b, c);
          T lim;
          if (!absv) lim = C > 0 ? std::min(T(1), std::min(bd0, bu1)) : std::min(T(1), std::min(bu0, bd1));
          else if (C > 0) lim = P<ND, D>(p, a, b, c) > 0 ? std::min(T(1), std::min(bd0, bu1)) : std::min(T(1), std::min(bu0, bd1));
          else lim = P<ND, D>(p, a + 1, b, c) > 0 ? std::min(T(1), std::min(bu0, bd1)) : std::min(T(1), std::min(bd0, bu1));
          P<ND, D>(out, a, b, c) = C * lim;
        });
  }

  // fct_adjust_antidiff (mpdata_fct_{1,2,3}d.hpp)
  void fct_adjust_antidiff(int e, int iter) {
    const arr<T> &p = psi[e][tl[e]];
    vctr<T> &corr = GC_corr(iter);
    xchng_vctr_alng(corr, true);
    xchng_vctr_nrml(corr);
    const vctr<T> *flx = &corr;
    if (!(opts & o_iga)) { fluxes(flux, p, corr, true); flx = &flux; }
    betas(p, *flx);
    if (nd == 1) gc_mono<1, 0>(GC_mono[0], corr[0], p);
    else if (nd == 2) { gc_mono<2, 0>(GC_mono[0], corr[0], p); gc_mono<2, 1>(GC_mono[1], corr[1], p); }
    else { gc_mono<3, 0>(GC_mono[0], corr[0], p); gc_mono<3, 1>(GC_mono[1], corr[1], p); gc_mono<3, 2>(GC_mono[2], corr[2], p); }
  }

  // advop (mpdata_osc_{1,2,3}d.hpp)
  void advop(int e) {
    if (opts & o_fct) fct_init(e);
    for (int iter = 0; iter < n_iters; ++iter) {
      if (iter != 0) {
        cycle(e);
        xchng(e);
        const arr<T> &p = psi[e][tl[e]];
        vctr<T> &corr = GC_corr(iter), &unco = GC_unco(iter);
        if (opts & o_div_2nd) {
          const arr<T> &pn = psi[e][(tl[e] + 1) % 2];  // psi[e][n-1]
          if (nd == 1) antidiff_div<1, 0>(corr[0], p, pn, unco);
          else if (nd == 2) { antidiff_div<2, 0>(corr[0], p, pn, unco); antidiff_div<2, 1>(corr[1], p, pn, unco); }
          else { antidiff_div<3, 0>(corr[0], p, pn, unco); antidiff_div<3, 1>(corr[1], p, pn, unco); antidiff_div<3, 2>(corr[2], p, pn, unco); }
        } else if (nd == 1) antidiff1(corr[0], p, unco);
        else if (nd == 2) { antidiff2<0>(corr[0], p, unco); antidiff2<1>(corr[1], p, unco); }
        else { antidiff3<0>(corr[0], p, unco); antidiff3<1>(corr[1], p, unco); antidiff3<2>(corr[2], p, unco); }
        if (!(opts & o_fct) && iter != n_iters - 1) {
          xchng_vctr_nrml(corr);
          if (opts & o_dfl) xchng_vctr_alng(corr);  // mpdata_osc_1d.hpp:82-88, _2d.hpp:120-124, _3d.hpp:138-142
        }
        if (opts & o_fct) fct_adjust_antidiff(e, iter);
      }
      const arr<T> &p = psi[e][tl[e]];
      vctr<T> *flx = &flux;
      if (!(opts & o_iga) || iter == 0) fluxes(flux, p, GCit(iter), false);
      else flx = &GCit(iter);
      xchng_flux(*flx);  // mpdata_osc_2d.hpp:154-155
      donorcell_sum(psi[e][(tl[e] + 1) % 2], p, *flx);
      // upwind-only step every upwind_filter_freq steps (mpdata_osc_2d.hpp:176-179)
      if (upwind_filter_freq > 0 && timestep % upwind_filter_freq == 0) break;
    }
  }

  T max_abs_vctr_div() {
    T mx = 0;
    for (int i = 0; i < n[0]; ++i)
      for (int j = 0; j < n[1]; ++j)
        for (int k = 0; k < n[2]; ++k) {
          T v;
          if (nd == 1) v = std::abs(GC[0](i, 0, 0) - GC[0](i - 1, 0, 0)) / Gc(i, j, k);
          else if (nd == 2) v = std::abs((GC[0](i, j, 0) - GC[0](i - 1, j, 0)) + (GC[1](i, j, 0) - GC[1](i, j - 1, 0))) / Gc(i, j, k);
          else v = std::abs((GC[0](i, j, k) - GC[0](i - 1, j, k)) + (GC[1](i, j, k) - GC[1](i, j - 1, k)) + (GC[2](i, j, k) - GC[2](i, j, k - 1))) / Gc(i, j, k);
          mx = std::max(mx, v);
        }
    return mx;
  }

  // hook_ante_loop chain (solver_common.hpp:191-211, solver_2d.hpp:279-293, mpdata_osc_2d.hpp:40-67)
  void ante_loop() {
    xchng_vctr_alng(GC);
    if (nd > 1 && !(opts & o_dfl)) {
      if (max_abs_vctr_div() > max_abs_div_eps)
        throw std::runtime_error("libmpdata++: initial advector field is divergent");
    }
    if (opts & o_nug) xchng_sclr(Gf, H);  // mpdata_osc_{1,2,3}d.hpp hook_ante_loop
    if (nd > 1) xchng_vctr_nrml(GC, H - 1);
  }

  // solver_common::solve (solver_common.hpp:270-358) with solve_loop_body (:127-136)
  void advance(long long nt) {
    nt += timestep;
    if (timestep == 0) ante_loop();
    while (timestep < nt) {
      for (int e = 0; e < n_eqns; ++e) { xchng(e); advop(e); cycle(e); }
      ++timestep;
    }
  }

  // ---- accessors mirroring sharedmem::advectee()/advector() ----
  // advectee(e): interior n0 x n1 x n2, C order
  arr<T> &state(int e) { return psi[e][tl[e]]; }
  // advector(d): view with lower bound (-1, 0, 0); view element (a, b, c) maps to
  // GC[d](a-1, b-1*[d==1], c-1*[d==2]) (sharedmem.hpp:431-456, 543-577, 1D :356-372);
  // extents: d=0 (n0, n1, n2); d>=1 (n0+1, n1, n2)
  void advector_extent(int d, int ex[3]) const {
    for (int q = 0; q < 3; ++q) ex[q] = n[q];
    if (d > 0) ex[0] = n[0] + 1;
  }
  T &advector_at(int d, int a, int b, int c) {
    int i = a - 1, j = b, k = c;
    if (d == 1) j = b - 1;
    if (d == 2) k = c - 1;
    return GC[d](i, j, k);
  }
};

}  // namespace mpdx_oracle
