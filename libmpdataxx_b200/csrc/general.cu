// Reference-structured MPDATA path: one kernel per libmpdata++ formula and one
// small kernel per halo fill, launched in the order the reference's solvers call
// them.  It covers every dimension, the cyclic, open and rigid boundary conditions
// and the MPDATA options that the fused kernels do not, and it is the FP64
// parity path (this file is compiled with --fmad=false so that FP64 results
// follow the reference's rounding).
//
// Reference call structure mirrored here:
//   advop            libmpdata++/solvers/detail/mpdata_osc_{1,2,3}d.hpp
//   fct_init / fct_adjust_antidiff   mpdata_fct_{1,2,3}d.hpp
//   halo exchanges   solvers/detail/solver_{1,2,3}d.hpp, bcond/{cyclic,open,rigid}_{1,2,3}d.hpp
#include <cfloat>

#include "general.cuh"

namespace mpdx {

// ---------------------------------------------------------------------------
// frame permutation pi<d> (libmpdata++/formulae/idxperm.hpp:15-71):
// frame (a along d, b along d+1, c along d+2)  <->  physical (i, j, k)
template <int ND, int D> struct fr;
template <> struct fr<1, 0> {
  __device__ static void to(int a, int, int, int &i, int &j, int &k) { i = a; j = 0; k = 0; }
  __device__ static void from(int i, int, int, int &a, int &b, int &c) { a = i; b = 0; c = 0; }
};
template <> struct fr<2, 0> {
  __device__ static void to(int a, int b, int, int &i, int &j, int &k) { i = a; j = b; k = 0; }
  __device__ static void from(int i, int j, int, int &a, int &b, int &c) { a = i; b = j; c = 0; }
};
template <> struct fr<2, 1> {
  __device__ static void to(int a, int b, int, int &i, int &j, int &k) { i = b; j = a; k = 0; }
  __device__ static void from(int i, int j, int, int &a, int &b, int &c) { a = j; b = i; c = 0; }
};
template <> struct fr<3, 0> {
  __device__ static void to(int a, int b, int c, int &i, int &j, int &k) { i = a; j = b; k = c; }
  __device__ static void from(int i, int j, int k, int &a, int &b, int &c) { a = i; b = j; c = k; }
};
template <> struct fr<3, 1> {
  __device__ static void to(int a, int b, int c, int &i, int &j, int &k) { i = c; j = a; k = b; }
  __device__ static void from(int i, int j, int k, int &a, int &b, int &c) { a = j; b = k; c = i; }
};
template <> struct fr<3, 2> {
  __device__ static void to(int a, int b, int c, int &i, int &j, int &k) { i = b; j = c; k = a; }
  __device__ static void from(int i, int j, int k, int &a, int &b, int &c) { a = k; b = i; c = j; }
};

template <int ND, int D, class T>
__device__ __forceinline__ T &P(const dfield<T> &A, int a, int b = 0, int c = 0) {
  int i, j, k;
  fr<ND, D>::to(a, b, c, i, j, k);
  return A(i, j, k);
}

__device__ __forceinline__ void pim(int nd, int d, int a, int b, int c, int &i, int &j, int &k) {
  if (nd == 1) { i = a; j = 0; k = 0; return; }
  if (nd == 2) { if (d == 0) { i = a; j = b; } else { i = b; j = a; } k = 0; return; }
  if (d == 0) { i = a; j = b; k = c; } else if (d == 1) { i = c; j = a; k = b; } else { i = b; j = c; k = a; }
}
template <class T>
__device__ __forceinline__ T &PR(const dfield<T> &A, int nd, int d, int a, int b, int c) {
  int i, j, k;
  pim(nd, d, a, b, c, i, j, k);
  return A(i, j, k);
}

// pospart/negpart (formulae/common.hpp:86-124) follow std::max(0, x)/std::min(0, x)
template <class T> __device__ __forceinline__ T pospart(unsigned o, T x) {
  if (o & o_npa) return (x + fabs(x)) / T(2);
  return T(0) < x ? x : T(0);
}
template <class T> __device__ __forceinline__ T negpart(unsigned o, T x) {
  if (o & o_npa) return (x - fabs(x)) / T(2);
  return x < T(0) ? x : T(0);
}
template <class T> __device__ __forceinline__ T dmax(T a, T b) { return a < b ? b : a; }  // std::max
template <class T> __device__ __forceinline__ T dmin(T a, T b) { return b < a ? b : a; }  // std::min
template <class T> struct lim;
template <> struct lim<float> {
  __device__ static float tiny() { return FLT_MIN; }
  __device__ static float eps() { return FLT_EPSILON; }
};
template <> struct lim<double> {
  __device__ static double tiny() { return DBL_MIN; }
  __device__ static double eps() { return DBL_EPSILON; }
};
// frac (formulae_mpdata_common.hpp:61-86), fct_frac (:88-98)
template <class T> __device__ __forceinline__ T frac(unsigned o, T nom, T den) {
  if (o & o_pfc) return den != T(0) ? nom / den : T(0);
  return nom / (den + lim<T>::tiny());
}
template <class T> __device__ __forceinline__ T fct_frac(T nom, T den) { return nom / (den + lim<T>::eps()); }

// ---------------------------------------------------------------------------
// generic launcher: one thread per point of a physical box, op(a, b, c) in frame
template <int ND, int D, class Op>
__global__ void k_box(Op op, int i0, int j0, int k0, int ni, int nj, int nk) {
  const long long tot = (long long)ni * nj * nk;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int k = k0 + int(q % nk);
    const long long r = q / nk;
    const int j = j0 + int(r % nj);
    const int i = i0 + int(r / nj);
    int a, b, c;
    fr<ND, D>::from(i, j, k, a, b, c);
    op(a, b, c);
  }
}

template <int ND, int D, class Op>
void launch_frame(cudaStream_t s, Op op, rng ra, rng rb, rng rc) {
  // frame ranges -> physical box
  rng ph[3] = {{0, 0}, {0, 0}, {0, 0}};
  ph[D] = ra;
  if (ND >= 2) ph[(D + 1) % ND] = rb;
  if (ND >= 3) ph[(D + 2) % ND] = rc;
  const long long tot = (long long)ph[0].n() * ph[1].n() * ph[2].n();
  if (tot <= 0) return;
  const int bs = 256;
  unsigned g = ceil_div(tot, bs);
  if (g > 65535u * 8u) g = 65535u * 8u;
  k_box<ND, D><<<g, bs, 0, s>>>(op, ph[0].f, ph[1].f, ph[2].f, ph[0].n(), ph[1].n(), ph[2].n());
  MPDX_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// formulae

// nondimensional psi derivatives at (a+1/2, b, c) (formulae_mpdata_psi_{1,2,3}d.hpp)
template <int ND, int D, class T>
__device__ __forceinline__ T ndx(unsigned o, const dfield<T> &p, int a, int b, int c) {
  const T p1 = P<ND, D>(p, a + 1, b, c), p0 = P<ND, D>(p, a, b, c);
  if (o & o_iga) {
    if (ND == 3) return p1 - p0;
    return T(2) * (p1 - p0) / T(2);
  }
  if (o & o_abs) return T(2) * frac(o, fabs(p1) - fabs(p0), fabs(p1) + fabs(p0));
  return T(2) * frac(o, p1 - p0, p1 + p0);
}
template <class T>
__device__ __forceinline__ T nd4(unsigned o, T pa, T pb, T pc, T pd) {
  if (o & o_iga) return (pa + pb - pc - pd) / T(4);
  if (o & o_abs) { pa = fabs(pa); pb = fabs(pb); pc = fabs(pc); pd = fabs(pd); }
  return frac(o, pa + pb - pc - pd, pa + pb + pc + pd);
}
template <int ND, int D, class T>
__device__ __forceinline__ T ndy(unsigned o, const dfield<T> &p, int a, int b, int c) {
  return nd4(o, P<ND, D>(p, a + 1, b + 1, c), P<ND, D>(p, a, b + 1, c), P<ND, D>(p, a + 1, b - 1, c), P<ND, D>(p, a, b - 1, c));
}
template <int ND, int D, class T>
__device__ __forceinline__ T ndz(unsigned o, const dfield<T> &p, int a, int b, int c) {
  return nd4(o, P<ND, D>(p, a + 1, b, c + 1), P<ND, D>(p, a, b, c + 1), P<ND, D>(p, a + 1, b, c - 1), P<ND, D>(p, a, b, c - 1));
}

// third-order terms (formulae_mpdata_hot_{1,2,3}d.hpp): four-point second
// derivatives 2 (pa - pb - pc + pd) / (pa + pb + pc + pd) (ndxx/ndxy/ndxz_psi,
// formulae_mpdata_psi_{1,2,3}d.hpp), the eight-corner ndyz_psi (psi_3d.hpp:697-790)
// and their Courant-number coefficients
template <class T>
__device__ __forceinline__ T nd2(unsigned o, T pa, T pb, T pc, T pd) {
  if (o & o_iga) return T(2) * (pa - pb - pc + pd) / T(4);
  if (o & o_abs) { pa = fabs(pa); pb = fabs(pb); pc = fabs(pc); pd = fabs(pd); }
  return T(2) * frac(o, pa - pb - pc + pd, pa + pb + pc + pd);
}
template <int D, class T>
__device__ __forceinline__ T ndyz(unsigned o, const dfield<T> &p, int a, int b, int c) {
  T q[8] = {P<3, D>(p, a + 1, b + 1, c + 1), P<3, D>(p, a + 1, b - 1, c - 1), P<3, D>(p, a + 1, b + 1, c - 1),
            P<3, D>(p, a + 1, b - 1, c + 1), P<3, D>(p, a, b + 1, c + 1),     P<3, D>(p, a, b - 1, c - 1),
            P<3, D>(p, a, b + 1, c - 1),     P<3, D>(p, a, b - 1, c + 1)};
  if (o & o_iga) return (q[0] + q[1] - q[2] - q[3] + q[4] + q[5] - q[6] - q[7]) / T(8);
  if (o & o_abs) {
#pragma unroll
    for (int t = 0; t < 8; ++t) q[t] = fabs(q[t]);
  }
  return frac(o, q[0] + q[1] - q[2] - q[3] + q[4] + q[5] - q[6] - q[7], q[0] + q[1] + q[2] + q[3] + q[4] + q[5] + q[6] + q[7]);
}
// (gb = G_bar_x; pow2/pow3 as products)
template <class T> __device__ __forceinline__ T cxx(T C, T gb) { return (T(3) * C * fabs(C) / gb - T(2) * (C * C * C) / (gb * gb) - C) / T(6); }
template <class T> __device__ __forceinline__ T cxy(T C, T g, T gb) { return (fabs(C) - T(2) * (C * C) / gb) * g / (T(2) * gb); }
template <class T> __device__ __forceinline__ T cyz(T C, T g1, T g2, T gb) { return T(-2) * C * g1 * g2 / T(3) / (gb * gb); }

// fourth-order terms of the 2D antidiffusive velocity, iga only
// (formulae_mpdata_hot_2d.hpp:82-157): the third derivatives ndxxx, ndxxy, ndxyy
// (formulae_mpdata_psi_2d.hpp:360-412) times their Courant-number coefficients;
// cy = GC1_bar_xy, gb = G_bar_x; pow2 and pow3 as products, pow4(x) as (x x)(x x)
template <int D, class T>
__device__ __forceinline__ T fot2(const dfield<T> &p, int a, int b, T C, T cy, T gb) {
  auto ps = [&](int x, int y) { return P<2, D>(p, x, y, 0); };
  const T nxxx = (ps(a + 2, b) - T(3) * ps(a + 1, b) + T(3) * ps(a, b) - ps(a - 1, b)) / T(4);
  const T nxxy = (ps(a + 2, b + 1) - ps(a + 1, b + 1) - ps(a, b + 1) + ps(a - 1, b + 1) - ps(a + 2, b - 1)
                  + ps(a + 1, b - 1) + ps(a, b - 1) - ps(a - 1, b - 1)) / T(8);
  const T nxyy = (ps(a + 1, b + 1) - T(2) * ps(a + 1, b) + ps(a + 1, b - 1) - ps(a, b + 1) + T(2) * ps(a, b)
                  - ps(a, b - 1)) / T(6);
  const T aC = fabs(C), C2 = C * C, C4 = (C * C) * (C * C), gb2 = gb * gb, gb3 = gb * gb * gb;
  const T acy = fabs(cy), cy2 = cy * cy;
  const T cxxx = (T(6) * aC * C2 / gb2 - T(3) * C2 / gb - T(3) * C4 / gb3) / T(2);
  const T cxxy = T(3) * (aC - C2 / gb) * C * cy / gb2;
  const T cxyy = T(3) * (T(3) * acy * C2 / gb + T(3) * cy2 * aC / gb - T(2) * acy * aC - T(9) * cy2 * C2 / gb2) / gb / T(4);
  return nxxx * cxxx + nxxy * cxxy + nxyy * cxyy;
}

// antidiffusive velocity (formulae_mpdata_{1,2,3}d.hpp antidiff, standard form).
// TOT and DFL are added only when their options are set (the reference adds an
// integer zero otherwise, which changes at most the sign of a zero result).
// With nug, G_bar_x = (G(a+1) + G(a)) / 2 (formulae_mpdata_g_{1,2,3}d.hpp); 1 otherwise.
template <int ND, int D, class T>
struct op_antidiff {
  dfield<T> res, psi, G0, G1, G2;  // G0 = GC[D], G1 = GC[D+1], G2 = GC[D+2]
  unsigned o;
  dfield<T> Gf;  // G factor (nug only)
  __device__ void operator()(int a, int b, int c) const {
    const T C = P<ND, D>(G0, a, b, c);
    const T gb = (o & o_nug) ? (P<ND, D>(Gf, a + 1, b, c) + P<ND, D>(Gf, a, b, c)) / T(2) : T(1);
    T r = fabs(C) / T(2) * (T(1) - fabs(C) / gb) * ndx<ND, D>(o, psi, a, b, c);
    const T xx = (o & o_tot) ? nd2(o, P<ND, D>(psi, a + 2, b, c), P<ND, D>(psi, a + 1, b, c), P<ND, D>(psi, a, b, c),
                                   P<ND, D>(psi, a - 1, b, c)) : T(0);
    if (ND == 1) {
      if (o & o_tot) r = r + xx * cxx(C, gb);  // formulae_mpdata_hot_1d.hpp:19-52
    } else if (ND == 2) {
      // GC1_bar_xy (formulae_mpdata_gc_2d.hpp:76-90)
      const T gc1 = (P<ND, D>(G1, a + 1, b, c) + P<ND, D>(G1, a, b, c) + P<ND, D>(G1, a + 1, b - 1, c) + P<ND, D>(G1, a, b - 1, c)) / T(4);
      r = r - C * gc1 / (T(2) * gb) * ndy<ND, D>(o, psi, a, b, c);
      if (o & o_tot) {  // formulae_mpdata_hot_2d.hpp:52-80
        const T xy = nd2(o, P<ND, D>(psi, a + 1, b + 1, c), P<ND, D>(psi, a, b + 1, c), P<ND, D>(psi, a + 1, b - 1, c), P<ND, D>(psi, a, b - 1, c));
        r = r + (xx * cxx(C, gb) + xy * cxy(C, gc1, gb));
      }
      if constexpr (ND == 2)
        if (o & o_fot) r = r + fot2<D>(psi, a, b, C, gc1, gb);
    } else {
      // GC1_bar_xy, GC2_bar_xz (formulae_mpdata_gc_3d.hpp:100-170)
      const T gc1 = (P<ND, D>(G1, a + 1, b, c) + P<ND, D>(G1, a, b, c) + P<ND, D>(G1, a + 1, b - 1, c) + P<ND, D>(G1, a, b - 1, c)) / T(4);
      const T gc2 = (P<ND, D>(G2, a + 1, b, c) + P<ND, D>(G2, a, b, c) + P<ND, D>(G2, a + 1, b, c - 1) + P<ND, D>(G2, a, b, c - 1)) / T(4);
      r = r - C / T(2) * (gc1 * ndy<ND, D>(o, psi, a, b, c) + gc2 * ndz<ND, D>(o, psi, a, b, c)) / gb;
      if (o & o_tot) {  // formulae_mpdata_hot_3d.hpp:97-110
        const T xy = nd2(o, P<ND, D>(psi, a + 1, b + 1, c), P<ND, D>(psi, a, b + 1, c), P<ND, D>(psi, a + 1, b - 1, c), P<ND, D>(psi, a, b - 1, c));
        const T xz = nd2(o, P<ND, D>(psi, a + 1, b, c + 1), P<ND, D>(psi, a, b, c + 1), P<ND, D>(psi, a + 1, b, c - 1), P<ND, D>(psi, a, b, c - 1));
        r = r + (xx * cxx(C, gb) + xy * cxy(C, gc1, gb) + xz * cxy(C, gc2, gb) + ndyz<D>(o, psi, a, b, c) * cyz(C, gc1, gc2, gb));
      }
    }
    if (o & o_dfl) {  // divergent-flow correction (formulae_mpdata_dfl_{1,2,3}d.hpp)
      T d;
      if (ND == 1) {
        const T g2 = (o & o_nug) ? P<ND, D>(Gf, a + 1, b, c) + P<ND, D>(Gf, a, b, c) : T(2);
        d = T(-0.5) * C / g2 * (P<ND, D>(G0, a + 1, b, c) - P<ND, D>(G0, a - 1, b, c));
        if (o & o_iga) d = d * T(0.5) * (P<ND, D>(psi, a + 1, b, c) + P<ND, D>(psi, a, b, c));
      } else {
        T s = (P<ND, D>(G0, a + 1, b, c) - P<ND, D>(G0, a - 1, b, c))
            + (P<ND, D>(G1, a + 1, b, c) + P<ND, D>(G1, a, b, c) - P<ND, D>(G1, a + 1, b - 1, c) - P<ND, D>(G1, a, b - 1, c));
        if (ND == 3)
          s = s + (P<ND, D>(G2, a + 1, b, c) + P<ND, D>(G2, a, b, c) - P<ND, D>(G2, a + 1, b, c - 1) - P<ND, D>(G2, a, b, c - 1));
        d = T(-0.25) * C / gb * s;
        if (o & o_iga) d = d * ((P<ND, D>(psi, a + 1, b, c) + P<ND, D>(psi, a, b, c)) / T(2));
      }
      r = r + d;
    }
    P<ND, D>(res, a, b, c) = r;
  }
};

// divergence-form antidiffusive velocity: div_2nd + div_3rd / div_3rd_dt
// (formulae_mpdata_{1,2,3}d.hpp, helpers of formulae_mpdata_fdiv_{1,2,3}d.hpp,
// _psi_*, _gc_*, _g_*), in the reference's operand order.  psi is the current
// iterate psi_np1, pn the other time level psi[e][n-1]; G0 = GC[dim], G1 =
// GC[dim+1], G2 = GC[dim-1].  The advector of solvers::mpdata is constant in
// time, so ndt_GC = ndtt_GC = 0 (mpdata_osc_{1,2,3}d.hpp hook_ante_loop) and the
// temporal terms multiplying them are exact zeros, left out like TOT and DFL
// above.  1D has no div_3rd_dt form in the reference (it adds nothing there).
template <int ND, int D, class T>
struct op_antidiff_div {
  dfield<T> res, psi, pn, G0, G1, G2;
  unsigned o;
  dfield<T> Gf;
  int sptl;  // exact 0, aver2 1, aver4 2 (formulae_mpdata_common.hpp:21-26)
  __device__ T q(const dfield<T> &A, int x, int y, int z) const {
    const T v = P<ND, D>(A, x, y, z);
    return (o & o_abs) ? fabs(v) : v;
  }
  __device__ T G(const dfield<T> &A, int x, int y, int z) const { return P<ND, D>(A, x, y, z); }
  __device__ T g(int x, int y, int z) const { return (o & o_nug) ? P<ND, D>(Gf, x, y, z) : T(1); }
  __device__ T pbx(const dfield<T> &A, int x, int y, int z) const { return (q(A, x + 1, y, z) + q(A, x, y, z)) / T(2); }
  __device__ T pby(const dfield<T> &A, int x, int y, int z) const { return (q(A, x, y, z) + q(A, x, y + 1, z)) / T(2); }
  __device__ T pbz(const dfield<T> &A, int x, int y, int z) const { return (q(A, x, y, z) + q(A, x, y, z + 1)) / T(2); }
  __device__ T pbxy(const dfield<T> &A, int x, int y, int z) const {
    return (q(A, x + 1, y, z) + q(A, x, y, z) + q(A, x, y + 1, z) + q(A, x + 1, y + 1, z)) / T(4);
  }
  __device__ T pbxz(const dfield<T> &A, int x, int y, int z) const {
    return (q(A, x + 1, y, z) + q(A, x, y, z) + q(A, x, y, z + 1) + q(A, x + 1, y, z + 1)) / T(4);
  }
  __device__ T pbxyz(int x, int y, int z) const {
    return (q(psi, x, y, z) + q(psi, x + 1, y, z) + q(psi, x, y + 1, z) + q(psi, x, y, z + 1) + q(psi, x + 1, y + 1, z)
            + q(psi, x + 1, y, z + 1) + q(psi, x, y + 1, z + 1) + q(psi, x + 1, y + 1, z + 1)) / T(8);
  }
  // Courant-number averages (face x+1/2 stored at x)
  __device__ T g0bx(int x, int y, int z) const { return (G(G0, x, y, z) + G(G0, x - 1, y, z)) / T(2); }
  __device__ T g1bx(int x, int y, int z) const { return (G(G1, x + 1, y, z) + G(G1, x, y, z)) / T(2); }
  __device__ T g2bx(int x, int y, int z) const { return (G(G2, x + 1, y, z) + G(G2, x, y, z)) / T(2); }
  __device__ T g0bxy(int x, int y, int z) const { return (G(G0, x, y, z) + G(G0, x - 1, y, z) + G(G0, x, y + 1, z) + G(G0, x - 1, y + 1, z)) / T(4); }
  __device__ T g1bxy(int x, int y, int z) const { return (G(G1, x + 1, y, z) + G(G1, x, y, z) + G(G1, x + 1, y - 1, z) + G(G1, x, y - 1, z)) / T(4); }
  __device__ T g2bxy(int x, int y, int z) const { return (G(G2, x + 1, y + 1, z) + G(G2, x, y + 1, z) + G(G2, x + 1, y, z) + G(G2, x, y, z)) / T(4); }
  __device__ T g0bxz(int x, int y, int z) const { return (G(G0, x, y, z) + G(G0, x - 1, y, z) + G(G0, x, y, z + 1) + G(G0, x - 1, y, z + 1)) / T(4); }
  __device__ T g1bxz(int x, int y, int z) const { return (G(G1, x + 1, y, z) + G(G1, x + 1, y, z + 1) + G(G1, x, y, z) + G(G1, x, y, z + 1)) / T(4); }
  __device__ T g2bxz(int x, int y, int z) const { return (G(G2, x + 1, y, z) + G(G2, x, y, z) + G(G2, x + 1, y, z - 1) + G(G2, x, y, z - 1)) / T(4); }
  // G averages (formulae_mpdata_g_{1,2,3}d.hpp), 1 without nug
  __device__ T gbx(int x, int y, int z) const { return (o & o_nug) ? (g(x + 1, y, z) + g(x, y, z)) / T(2) : T(1); }
  __device__ T gbxy(int x, int y, int z) const {
    return (o & o_nug) ? (g(x, y, z) + g(x, y + 1, z) + g(x + 1, y, z) + g(x + 1, y + 1, z)) / T(4) : T(1);
  }
  __device__ T gbxz(int x, int y, int z) const {
    return (o & o_nug) ? (g(x, y, z) + g(x, y, z + 1) + g(x + 1, y, z) + g(x + 1, y, z + 1)) / T(4) : T(1);
  }
  // flux divergence at the cell centre (fdiv_centre) and at the xy / xz edges (fdiv_corner_*)
  __device__ T fc(int x, int y, int z) const {
    T r = G(G0, x, y, z) * pbx(psi, x, y, z) - G(G0, x - 1, y, z) * pbx(psi, x - 1, y, z);
    if (ND > 1) r = r + G(G1, x, y, z) * pby(psi, x, y, z) - G(G1, x, y - 1, z) * pby(psi, x, y - 1, z);
    if (ND > 2) r = r + G(G2, x, y, z) * pbz(psi, x, y, z) - G(G2, x, y, z - 1) * pbz(psi, x, y, z - 1);
    return r / g(x, y, z);
  }
  __device__ T fxy(int x, int y, int z) const {
    T r = g0bxy(x + 1, y, z) * pby(psi, x + 1, y, z) - g0bxy(x, y, z) * pby(psi, x, y, z)
        + g1bxy(x, y + 1, z) * pbx(psi, x, y + 1, z) - g1bxy(x, y, z) * pbx(psi, x, y, z);
    if (ND > 2) r = r + g2bxy(x, y, z) * pbxyz(x, y, z) - g2bxy(x, y, z - 1) * pbxyz(x, y, z - 1);
    return r / gbxy(x, y, z);
  }
  __device__ T fxz(int x, int y, int z) const {
    return (g0bxz(x + 1, y, z) * pbz(psi, x + 1, y, z) - g0bxz(x, y, z) * pbz(psi, x, y, z)
            + g1bxz(x, y, z) * pbxyz(x, y, z) - g1bxz(x, y - 1, z) * pbxyz(x, y - 1, z)
            + g2bxz(x, y, z + 1) * pbx(psi, x, y, z + 1) - g2bxz(x, y, z) * pbx(psi, x, y, z)) / gbxz(x, y, z);
  }
  // sum of psi over the six (2D) / ten (3D) points of nfdiv's denominator, continuing from s
  __device__ T s_nf(const dfield<T> &A, int a, int b, int c, T s, bool first) const {
    T r = first ? q(A, a + 1, b, c) + q(A, a, b, c) : s + q(A, a + 1, b, c) + q(A, a, b, c);
    if (ND == 1) return r;
    r = r + q(A, a, b + 1, c) + q(A, a + 1, b + 1, c) + q(A, a, b - 1, c) + q(A, a + 1, b - 1, c);
    if (ND == 3) r = r + q(A, a + 1, b, c + 1) + q(A, a + 1, b, c - 1) + q(A, a, b, c - 1) + q(A, a, b, c + 1);
    return r;
  }
  __device__ void operator()(int a, int b, int c) const {
    const bool iga = o & o_iga;
    const T C = G(G0, a, b, c);
    const T m1 = T(2 + 4 * (ND - 1)), m2 = T(4 + 4 * (ND - 1));
    // nfdiv (formulae_mpdata_fdiv_*d.hpp)
    T nn = g0bx(a + 1, b, c) * q(psi, a + 1, b, c) - g0bx(a, b, c) * q(psi, a, b, c);
    if (ND > 1) nn = nn + g1bx(a, b, c) * pbxy(psi, a, b, c) - g1bx(a, b - 1, c) * pbxy(psi, a, b - 1, c);
    if (ND > 2) nn = nn + g2bx(a, b, c) * pbxz(psi, a, b, c) - g2bx(a, b, c - 1) * pbxz(psi, a, b, c - 1);
    const T nfdiv = iga ? nn / gbx(a, b, c) : m1 * frac(o, nn, gbx(a, b, c) * s_nf(psi, a, b, c, T(0), true));
    const T ndxp = ndx<ND, D>(o, psi, a, b, c);
    const T d2 = fabs(C) / 2 * ndxp - C / 2 * nfdiv;  // div_2nd
    const bool dt = (o & o_div_3rd_dt) && ND > 1;
    if (!(o & o_div_3rd) && !dt) { P<ND, D>(res, a, b, c) = d2; return; }
    const T up = iga ? T(0) : fabs(d2) / 2 * ndxp;  // upwind-differencing correction
    const T ndxx_gc = G(G0, a + 1, b, c) + G(G0, a - 1, b, c) - 2 * G(G0, a, b, c);
    const T nxxg = iga ? ndxx_gc * pbx(psi, a, b, c) : ndxx_gc;
    const T helper = sptl == 0 ? nxxg : (sptl == 1 ? 4 * nxxg : T(0));
    const T xx = nd2(o, P<ND, D>(psi, a + 2, b, c), P<ND, D>(psi, a + 1, b, c), P<ND, D>(psi, a, b, c), P<ND, D>(psi, a - 1, b, c));
    const T spatial = -T(1.0 / 24) * (4 * C * xx + 2 * ndxp * ((G(G0, a + 1, b, c) - G(G0, a - 1, b, c)) / 2) + helper);
    T r;
    if (!dt) {
      // div_3rd: mixed (ndx_fdiv) and temporal (nfdiv_fdiv) terms
      T s4 = q(psi, a + 2, b, c) + q(psi, a + 1, b, c) + q(psi, a, b, c) + q(psi, a - 1, b, c);
      T sf = s4, sx = s4;
      if (ND > 1) {
        sf = sf + q(psi, a, b + 1, c) + q(psi, a, b - 1, c) + q(psi, a + 1, b + 1, c) + q(psi, a + 1, b - 1, c);
        if (ND == 3) {  // ndx_fdiv's denominator takes the points in another order
          sf = sf + q(psi, a, b, c + 1) + q(psi, a, b, c - 1) + q(psi, a + 1, b, c + 1) + q(psi, a + 1, b, c - 1);
          sx = s4 + q(psi, a, b + 1, c) + q(psi, a, b - 1, c) + q(psi, a, b, c - 1) + q(psi, a, b, c + 1) + q(psi, a + 1, b + 1, c)
             + q(psi, a + 1, b - 1, c) + q(psi, a + 1, b, c - 1) + q(psi, a + 1, b, c + 1);
        } else {
          sx = sf;
        }
      }
      const T f1 = fc(a + 1, b, c), f0 = fc(a, b, c);
      T nf = g0bx(a + 1, b, c) * f1 - g0bx(a, b, c) * f0;
      if (ND > 1) nf = nf + g1bx(a, b, c) * fxy(a, b, c) - g1bx(a, b - 1, c) * fxy(a, b - 1, c);
      if (ND > 2) nf = nf + g2bx(a, b, c) * fxz(a, b, c) - g2bx(a, b, c - 1) * fxz(a, b, c - 1);
      const T ndx_fdiv = iga ? f1 - f0 : m2 * frac(o, f1 - f0, sx);
      const T nfdiv_fdiv = iga ? nf / gbx(a, b, c) : m2 * frac(o, nf, gbx(a, b, c) * sf);
      r = d2 + (up + spatial + T(0.5) * fabs(C) * ndx_fdiv + T(1.0 / 24) * (-8 * C * nfdiv_fdiv));
    } else {
      // div_3rd_dt (2D, 3D): mixed term from d(psi)/dt, temporal term nfdiv_dt
      const T p1 = P<ND, D>(psi, a + 1, b, c), n1 = P<ND, D>(pn, a + 1, b, c), p0 = P<ND, D>(psi, a, b, c), n0 = P<ND, D>(pn, a, b, c);
      T ndtx;
      if (iga) ndtx = p1 - n1 - p0 + n0;
      else if (o & o_abs) ndtx = 4 * frac(o, fabs(p1) - fabs(n1) - fabs(p0) + fabs(n0), fabs(p1) + fabs(n1) + fabs(p0) + fabs(n0));
      else ndtx = 4 * frac(o, p1 - n1 - p0 + n0, p1 + n1 + p0 + n0);
      T nt = g0bx(a + 1, b, c) * (q(psi, a + 1, b, c) - q(pn, a + 1, b, c)) - g0bx(a, b, c) * (q(psi, a, b, c) - q(pn, a, b, c))
           + g1bx(a, b, c) * (pbxy(psi, a, b, c) - pbxy(pn, a, b, c)) - g1bx(a, b - 1, c) * (pbxy(psi, a, b - 1, c) - pbxy(pn, a, b - 1, c));
      if (ND > 2)
        nt = nt + g2bx(a, b, c) * (pbxz(psi, a, b, c) - pbxz(pn, a, b, c)) - g2bx(a, b, c - 1) * (pbxz(psi, a, b, c - 1) - pbxz(pn, a, b, c - 1));
      const T m4 = T(ND == 2 ? 12 : 20);
      T nfdiv_dt;
      if (iga) nfdiv_dt = nt / gbx(a, b, c);
      else nfdiv_dt = m4 * frac(o, nt, gbx(a, b, c) * s_nf(pn, a, b, c, s_nf(psi, a, b, c, T(0), true), false));
      r = d2 + (up + spatial - T(0.5) * fabs(C) * ndtx + T(1.0 / 24) * (8 * C * nfdiv_dt));
    }
    // the fourth-order terms after div_3rd (formulae_mpdata_2d.hpp:300-305; 2D only)
    if constexpr (ND == 2)
      if ((o & o_fot) && (o & (o_div_3rd | o_div_3rd_dt))) r = r + fot2<D>(psi, a, b, G(G0, a, b, c), g1bxy(a, b, c), gbx(a, b, c));
    P<ND, D>(res, a, b, c) = r;
  }
};

// donor-cell flux (donorcell_formulae.hpp:25-79)
template <int ND, int D, class T>
struct op_flux {
  dfield<T> F, psi, C;
  unsigned o;
  __device__ void operator()(int a, int b, int c) const {
    const T g = P<ND, D>(C, a, b, c);
    P<ND, D>(F, a, b, c) = pospart(o, g) * P<ND, D>(psi, a, b, c) + negpart(o, g) * P<ND, D>(psi, a + 1, b, c);
  }
};

// donorcell_sum (donorcell_formulae.hpp:81-165): divided by G (1 without nug);
// with khn a Kahan-compensated sum (kahan_sum.hpp:14-27) of psi_old, then
// -F(+1/2)/G and F(-1/2)/G per dimension
template <int ND, class T>
struct op_donorcell {
  dfield<T> pn, po, f0, f1, f2;
  unsigned o;
  dfield<T> Gf;
  __device__ void operator()(int i, int j, int k) const {
    const T g = (o & o_nug) ? Gf(i, j, k) : T(1);
    if (o & o_khn) {
      T sum = T(0), c = T(0);
      auto add = [&](T in) { const T y = in - c; const T t = sum + y; c = (t - sum) - y; sum = t; };
      add(po(i, j, k));
      add(-f0(i, j, k) / g);
      add(f0(i - 1, j, k) / g);
      if (ND > 1) { add(-f1(i, j, k) / g); add(f1(i, j - 1, k) / g); }
      if (ND > 2) { add(-f2(i, j, k) / g); add(f2(i, j, k - 1) / g); }
      pn(i, j, k) = sum;
    } else if (ND == 1) pn(i, j, k) = po(i, j, k) + (-f0(i, j, k) + f0(i - 1, j, k)) / g;
    else if (ND == 2)
      pn(i, j, k) = po(i, j, k) + ((-f0(i, j, k) + f0(i - 1, j, k)) + (-f1(i, j, k) + f1(i, j - 1, k))) / g;
    else
      pn(i, j, k) = po(i, j, k) + ((-f0(i, j, k) + f0(i - 1, j, k)) + (-f1(i, j, k) + f1(i, j - 1, k)) + (-f2(i, j, k) + f2(i, j, k - 1))) / g;
  }
};

// ---------------------------------------------------------------------------
// One-dimensional problems in one block: every step of an advance() call in a
// single launch, the fields held in shared memory, the same per-point functors
// (so the same arithmetic, bit for bit) in the order the multi-kernel path
// launches them, __syncthreads() where that path has a kernel boundary.  For
// cyclic 1D problems without FCT, dfl and nug (the 1D box of a few thousand
// points runs launch-bound otherwise).
template <class T>
struct blk1d_args {
  T *psi[2];    // global time levels (element 0 of each), halo H on both sides
  const T *gc;  // advector component 0 (element 0), valid over [-H, n-2+H]
  int n, H, n_iters, tl, uff;
  unsigned o;
  long long t0, nt;
};
template <class T>
__global__ void __launch_bounds__(1024, 1) k_block1d(blk1d_args<T> A) {
  extern __shared__ __align__(16) unsigned char raw[];
  const int n = A.n, H = A.H, L = n + 2 * H + 2, base = H + 1;  // array index 0 sits at slot base
  T *sm = reinterpret_cast<T *>(raw);
  auto arr = [&](int k) { return dfield<T>{sm + (long long)k * L + base, 1, 0, 0}; };
  dfield<T> P[2] = {arr(0), arr(1)}, GC = arr(2), T0 = arr(3), T1 = arr(4), FL = arr(5);
  const int tid = threadIdx.x, nt_ = blockDim.x;
  for (int i = -H + tid; i <= n - 1 + H; i += nt_) {
    P[0](i, 0, 0) = A.psi[0][i];
    P[1](i, 0, 0) = A.psi[1][i];
  }
  for (int i = -H + tid; i <= n - 2 + H; i += nt_) GC(i, 0, 0) = A.gc[i];
  __syncthreads();
  int tl = A.tl;
  auto fill = [&](const dfield<T> &p) {  // cyclic halo: [-H, -1] <- [n-1-H, n-2], [n, n+H-1] <- [1, H]
    for (int q = tid; q < 2 * H; q += nt_) {
      if (q < H) p(-H + q, 0, 0) = p(n - 1 - H + q, 0, 0);
      else p(n + q - H, 0, 0) = p(1 + q - H, 0, 0);
    }
  };
  const dfield<T> none{};
  for (long long s = 0; s < A.nt; ++s) {
    fill(P[tl]);  // solve_loop_body: xchng(e)
    __syncthreads();
    for (int iter = 0; iter < A.n_iters; ++iter) {
      const dfield<T> corr = iter % 2 ? T0 : T1, unco = iter == 1 ? GC : (iter % 2 ? T1 : T0);
      if (iter != 0) {
        tl ^= 1;
        fill(P[tl]);
        __syncthreads();
        const op_antidiff<1, 0, T> ad{corr, P[tl], unco, unco, unco, A.o, none};
        for (int a = -1 + tid; a <= n - 1; a += nt_) ad(a, 0, 0);
        __syncthreads();
      }
      const dfield<T> git = iter == 0 ? GC : corr;
      dfield<T> flx = git;
      if (!(A.o & o_iga) || iter == 0) {
        const op_flux<1, 0, T> fx{FL, P[tl], git, A.o};
        for (int a = -1 + tid; a <= n - 1; a += nt_) fx(a, 0, 0);
        flx = FL;
        __syncthreads();
      }
      const op_donorcell<1, T> dc{P[tl ^ 1], P[tl], flx, flx, flx, A.o, none};
      for (int i = tid; i <= n - 1; i += nt_) dc(i, 0, 0);
      __syncthreads();
      if (A.uff > 0 && (A.t0 + s) % A.uff == 0) break;  // upwind-only step (mpdata_osc_1d.hpp)
    }
    tl ^= 1;  // cycle(e)
  }
  for (int i = -H + tid; i <= n - 1 + H; i += nt_) {
    A.psi[0][i] = P[0](i, 0, 0);
    A.psi[1][i] = P[1](i, 0, 0);
  }
}

template <class T>
bool general<T>::block1d_ok() const {
  const auto &S = *s;
  if (S.nd != 1 || S.n_eqns != 1) return false;
  if (S.bcs[0][0] != MPDX_BC_CYCLIC || S.bcs[0][1] != MPDX_BC_CYCLIC) return false;
  if (S.opts & (o_fct | o_dfl | o_nug | o_div_2nd | o_div_3rd | o_div_3rd_dt)) return false;
  const size_t bytes = size_t(6) * (S.n[0] + 2 * S.H + 2) * sizeof(T);
  return S.n[0] >= 2 * S.H + 1 && bytes <= size_t(200) * 1024;
}

template <class T>
void general<T>::block1d(long long nt) {
  auto &S = *s;
  const size_t bytes = size_t(6) * (S.n[0] + 2 * S.H + 2) * sizeof(T);
  static bool attr = false;
  if (!attr) {
    MPDX_CUDA(cudaFuncSetAttribute(k_block1d<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(200 * 1024)));
    attr = true;
  }
  const long long kChunk = 1 << 16;  // steps per launch
  for (long long s0 = 0; s0 < nt; s0 += kChunk) {
    blk1d_args<T> a;
    a.psi[0] = &S.psi[0][0].v(0, 0, 0);
    a.psi[1] = &S.psi[0][1].v(0, 0, 0);
    a.gc = &S.GC[0].v(0, 0, 0);
    a.n = S.n[0]; a.H = S.H; a.n_iters = S.n_iters; a.tl = S.tl[0]; a.uff = S.upwind_filter_freq;
    a.o = S.opts;
    a.t0 = S.timestep + s0;
    a.nt = std::min(kChunk, nt - s0);
    k_block1d<T><<<1, 1024, bytes, S.stream>>>(a);
    MPDX_LAUNCH_CHECK();
    // every pass of a step flips the time level once (the cycle before each
    // corrective pass and the one ending the step): n_iters flips per step,
    // one on the upwind-only steps (timestep % upwind_filter_freq == 0)
    long long flips = a.nt * S.n_iters;
    if (a.uff > 0) {
      const long long u = a.uff, b = a.t0 + a.nt;
      flips -= ((b + u - 1) / u - (a.t0 + u - 1) / u) * (S.n_iters - 1);
    }
    if (flips & 1) S.tl[0] ^= 1;
  }
}

// fct_init (mpdata_fct_{1,2,3}d.hpp:31-55)
template <int ND, class T>
struct op_fct_init {
  dfield<T> mn, mx, p;
  __device__ void operator()(int i, int j, int k) const {
    T lo, hi;
    if (ND == 1) {
      lo = dmin(dmin(p(i - 1, j, k), p(i, j, k)), p(i + 1, j, k));
      hi = dmax(dmax(p(i - 1, j, k), p(i, j, k)), p(i + 1, j, k));
    } else if (ND == 2) {
      lo = dmin(dmin(dmin(dmin(p(i, j + 1, k), p(i - 1, j, k)), p(i, j, k)), p(i + 1, j, k)), p(i, j - 1, k));
      hi = dmax(dmax(dmax(dmax(p(i, j + 1, k), p(i - 1, j, k)), p(i, j, k)), p(i + 1, j, k)), p(i, j - 1, k));
    } else {
      lo = dmin(dmin(dmin(dmin(dmin(dmin(p(i, j, k), p(i + 1, j, k)), p(i - 1, j, k)), p(i, j + 1, k)), p(i, j - 1, k)), p(i, j, k + 1)), p(i, j, k - 1));
      hi = dmax(dmax(dmax(dmax(dmax(dmax(p(i, j, k), p(i + 1, j, k)), p(i - 1, j, k)), p(i, j + 1, k)), p(i, j - 1, k)), p(i, j, k + 1)), p(i, j, k - 1));
    }
    mn(i, j, k) = lo;
    mx(i, j, k) = hi;
  }
};

// beta_up / beta_dn (formulae_mpdata_fct_{1,2,3}d.hpp)
template <int ND, class T>
struct op_betas {
  dfield<T> bu, bd, p, pmax, pmin, f0, f1, f2;
  unsigned o;
  dfield<T> Gf;
  __device__ void operator()(int i, int j, int k) const {
    const T c = p(i, j, k);
    T mx, mn, du, dd;
    if (ND == 1) {
      mx = dmax(pmax(i, j, k), dmax(p(i - 1, j, k), dmax(c, p(i + 1, j, k))));
      mn = dmin(pmin(i, j, k), dmin(p(i - 1, j, k), dmin(c, p(i + 1, j, k))));
      du = pospart(o, f0(i - 1, j, k)) - negpart(o, f0(i, j, k));
      dd = pospart(o, f0(i, j, k)) - negpart(o, f0(i - 1, j, k));
    } else if (ND == 2) {
      mx = dmax(pmax(i, j, k), dmax(p(i, j + 1, k), dmax(p(i - 1, j, k), dmax(c, dmax(p(i + 1, j, k), p(i, j - 1, k))))));
      mn = dmin(pmin(i, j, k), dmin(p(i, j + 1, k), dmin(p(i - 1, j, k), dmin(c, dmin(p(i + 1, j, k), p(i, j - 1, k))))));
      du = (pospart(o, f0(i - 1, j, k)) - negpart(o, f0(i, j, k))) + (pospart(o, f1(i, j - 1, k)) - negpart(o, f1(i, j, k)));
      dd = (pospart(o, f0(i, j, k)) - negpart(o, f0(i - 1, j, k))) + (pospart(o, f1(i, j, k)) - negpart(o, f1(i, j - 1, k)));
    } else {
      mx = dmax(pmax(i, j, k), dmax(c, dmax(p(i + 1, j, k), dmax(p(i - 1, j, k), dmax(p(i, j + 1, k), dmax(p(i, j - 1, k), dmax(p(i, j, k + 1), p(i, j, k - 1))))))));
      mn = dmin(pmin(i, j, k), dmin(p(i, j + 1, k), dmin(p(i - 1, j, k), dmin(c, dmin(p(i + 1, j, k), dmin(p(i, j, k + 1), dmin(p(i, j, k - 1), p(i, j - 1, k))))))));
      du = (pospart(o, f0(i - 1, j, k)) - negpart(o, f0(i, j, k))) + (pospart(o, f1(i, j - 1, k)) - negpart(o, f1(i, j, k)))
         + (pospart(o, f2(i, j, k - 1)) - negpart(o, f2(i, j, k)));
      dd = (pospart(o, f0(i, j, k)) - negpart(o, f0(i - 1, j, k))) + (pospart(o, f1(i, j, k)) - negpart(o, f1(i, j - 1, k)))
         + (pospart(o, f2(i, j, k)) - negpart(o, f2(i, j, k - 1)));
    }
    const T g = (o & o_nug) ? Gf(i, j, k) : T(1);  // beta numerators times G (formulae_mpdata_fct_2d.hpp:37, 88)
    bu(i, j, k) = fct_frac((mx - c) * g, du);
    bd(i, j, k) = fct_frac((c - mn) * g, dd);
  }
};

// GC_mono (formulae_mpdata_fct_{1,2,3}d.hpp)
template <int ND, int D, class T>
struct op_gc_mono {
  dfield<T> out, corr, p, bu, bd;
  unsigned o;
  __device__ void operator()(int a, int b, int c) const {
    const T C = P<ND, D>(corr, a, b, c);
    const T bd0 = P<ND, D>(bd, a, b, c), bu1 = P<ND, D>(bu, a + 1, b, c);
    const T bu0 = P<ND, D>(bu, a, b, c), bd1 = P<ND, D>(bd, a + 1, b, c);
    T l;
    const bool absv = (o & o_abs) && !(o & o_iga);
    if (!absv) l = C > T(0) ? dmin(T(1), dmin(bd0, bu1)) : dmin(T(1), dmin(bu0, bd1));
    else if (C > T(0)) l = P<ND, D>(p, a, b, c) > T(0) ? dmin(T(1), dmin(bd0, bu1)) : dmin(T(1), dmin(bu0, bd1));
    else l = P<ND, D>(p, a + 1, b, c) > T(0) ? dmin(T(1), dmin(bu0, bd1)) : dmin(T(1), dmin(bd0, bu1));
    P<ND, D>(out, a, b, c) = C * l;
  }
};

// ---------------------------------------------------------------------------
// halo fills (runtime dimension; frame ranges b x c)
template <class T>
__global__ void k_halo_copy(dfield<T> A, int nd, int d, int dst, int src, int cnt, int bf, int nb, int cf, int nc) {
  const long long tot = (long long)cnt * nb * nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int c = cf + int(q % nc);
    const long long r = q / nc;
    const int b = bf + int(r % nb);
    const int t = int(r / nb);
    PR(A, nd, d, dst + t, b, c) = PR(A, nd, d, src + t, b, c);
  }
}
// A(pi(f + t, b, c)) = edge >= -1000000 ? A(pi(edge, b, c)) : val
template <class T>
__global__ void k_halo_set(dfield<T> A, int nd, int d, int f, int cnt, int edge, bool use_edge, T val, int bf, int nb, int cf, int nc) {
  const long long tot = (long long)cnt * nb * nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int c = cf + int(q % nc);
    const long long r = q / nc;
    const int b = bf + int(r % nb);
    const int t = int(r / nb);
    PR(A, nd, d, f + t, b, c) = use_edge ? PR(A, nd, d, edge, b, c) : val;
  }
}
// open zero-divergence fill of the along-halo (open_2d.hpp:71-91, 167-186; open_3d.hpp:101-125, 227-243)
template <class T>
__global__ void k_zero_div(dfield<T> Ad, dfield<T> A1, dfield<T> A2, int nd, int d, int side, int e, int f, int cnt,
                           int bf, int nb, int cf, int nc) {
  const long long tot = (long long)cnt * nb * nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int c = cf + int(q % nc);
    const long long r = q / nc;
    const int b = bf + int(r % nb);
    const int ii = f + int(r / nb);
    T v;
    if (side == 0) {
      v = PR(Ad, nd, d, e, b, c) - (PR(A1, nd, d, e, b - 1, c) - PR(A1, nd, d, e, b, c));
      if (nd == 3) v = v - (PR(A2, nd, d, e, b, c - 1) - PR(A2, nd, d, e, b, c));
    } else {
      v = PR(Ad, nd, d, e - 1, b, c) + (PR(A1, nd, d, e, b - 1, c) - PR(A1, nd, d, e, b, c));
      if (nd == 3) v = v + (PR(A2, nd, d, e, b, c - 1) - PR(A2, nd, d, e, b, c));
    }
    PR(Ad, nd, d, ii, b, c) = v;
  }
}

// rigid walls (bcond/rigid_{2,3}d.hpp), halo position f + t, t in [0, cnt):
//   mode 0 (scalar mirror):   A(f+t) = A(src0 + sgn*t)
//   mode 1 (pressure):        A(f+t) = 2 A(edge) - A(src0 + sgn*t)
//   mode 2 (negated mirror):  A(f+t) = -A(src0 + sgn*t)
template <class T>
__global__ void k_halo_rigid(dfield<T> A, int nd, int d, int mode, int f, int cnt, int src0, int sgn, int edge,
                             int bf, int nb, int cf, int nc) {
  const long long tot = (long long)cnt * nb * nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int c = cf + int(q % nc);
    const long long r = q / nc;
    const int b = bf + int(r % nb);
    const int t = int(r / nb);
    const T m = PR(A, nd, d, src0 + sgn * t, b, c);
    T v;
    if (mode == 0) v = m;
    else if (mode == 1) v = T(2) * PR(A, nd, d, edge, b, c) - m;
    else v = -m;
    PR(A, nd, d, f + t, b, c) = v;
  }
}

static unsigned grid_for(long long tot) {
  unsigned g = ceil_div(tot, 256);
  if (g > 65535u * 8u) g = 65535u * 8u;
  return g < 1 ? 1 : g;
}

// ---------------------------------------------------------------------------
// sequencer (host)

template <class T>
void general<T>::fill_sclr(int d, int side, field<T> &A, rng rb, rng rc, bool deriv) {
  auto &S = *s;
  const int kind = S.bcs[d][side];
  const int nd = S.nd, H = S.H, n = S.n[d];
  if (nd < 2) rb = {0, 0};
  if (nd < 3) rc = {0, 0};
  const long long tot = (long long)H * rb.n() * rc.n();
  if (kind == MPDX_BC_CYCLIC) {
    // left: [-H, -1] <- [n-1-H, n-2];  right: [n, n+H-1] <- [1, H]  (cyclic_{1,2,3}d.hpp)
    const int dst = side == 0 ? -H : n, src = side == 0 ? n - 1 - H : 1;
    k_halo_copy<T><<<grid_for(tot), 256, 0, S.stream>>>(A.v, nd, d, dst, src, H, rb.f, rb.n(), rc.f, rc.n());
  } else if (kind == MPDX_BC_OPEN) {
    // zero-gradient (open_{1,2,3}d.hpp fill_halos_sclr)
    const int f = side == 0 ? -H : n, e = side == 0 ? 0 : n - 1;
    k_halo_set<T><<<grid_for(tot), 256, 0, S.stream>>>(A.v, nd, d, f, H, e, !deriv, T(0), rb.f, rb.n(), rc.f, rc.n());
  } else if (kind == MPDX_BC_RIGID) {
    // mirror about the wall point: A(-m) = A(m), A(n-1+m) = A(n-1-m)  (rigid_2d.hpp:16-24, 124-132)
    if (side == 0) k_halo_rigid<T><<<grid_for(tot), 256, 0, S.stream>>>(A.v, nd, d, 0, -H, H, H, -1, 0, rb.f, rb.n(), rc.f, rc.n());
    else k_halo_rigid<T><<<grid_for(tot), 256, 0, S.stream>>>(A.v, nd, d, 0, n, H, n - 2, -1, 0, rb.f, rb.n(), rc.f, rc.n());
  } else {
    throw error(MPDX_E_UNSUPPORTED, "boundary condition not supported for scalars on this path");
  }
  MPDX_LAUNCH_CHECK();
}

template <class T>
void general<T>::fill_pres(int d, int side, field<T> &A, rng rb, rng rc) {
  auto &S = *s;
  const int kind = S.bcs[d][side];
  if (kind == MPDX_BC_CYCLIC) { fill_sclr(d, side, A, rb, rc); return; }
  if (kind != MPDX_BC_RIGID) throw error(MPDX_E_UNSUPPORTED, "boundary condition not supported for pressure on this path");
  const int nd = S.nd, H = S.H, n = S.n[d];
  if (nd < 2) rb = {0, 0};
  if (nd < 3) rc = {0, 0};
  const long long tot = (long long)H * rb.n() * rc.n();
  // A(-m) = 2 A(0) - A(m);  A(n-1+m) = 2 A(n-1) - A(n-1-m)  (rigid_2d.hpp:26-35, 134-143)
  if (side == 0) k_halo_rigid<T><<<grid_for(tot), 256, 0, S.stream>>>(A.v, nd, d, 1, -H, H, H, -1, 0, rb.f, rb.n(), rc.f, rc.n());
  else k_halo_rigid<T><<<grid_for(tot), 256, 0, S.stream>>>(A.v, nd, d, 1, n, H, n - 2, -1, n - 1, rb.f, rb.n(), rc.f, rc.n());
  MPDX_LAUNCH_CHECK();
}

template <class T>
void general<T>::set_edge_pres(int d, int side, field<T> &A, rng rb, rng rc) {
  auto &S = *s;
  if (S.bcs[d][side] != MPDX_BC_RIGID) return;  // no-op for cyclic (cyclic_2d.hpp:42)
  const int nd = S.nd;
  if (nd < 2) rb = {0, 0};
  if (nd < 3) rc = {0, 0};
  const int e = side == 0 ? 0 : S.n[d] - 1;  // rigid_2d.hpp:52-56, 148-152
  k_halo_set<T><<<grid_for((long long)rb.n() * rc.n()), 256, 0, S.stream>>>(A.v, nd, d, e, 1, 0, false, T(0), rb.f, rb.n(), rc.f, rc.n());
  MPDX_LAUNCH_CHECK();
}

template <class T>
void general<T>::fill_flux(int d, int side, field<T> *AV, rng rb, rng rc) {
  auto &S = *s;
  if (S.bcs[d][side] != MPDX_BC_RIGID) return;  // no-op for cyclic and open
  const int nd = S.nd, n = S.n[d];
  if (nd < 2) rb = {0, 0};
  if (nd < 3) rc = {0, 0};
  // F(-1) = -F(0);  F(n-1) = -F(n-2)  (rigid_2d.hpp:74-79, 170-175)
  const long long tot = (long long)rb.n() * rc.n();
  if (side == 0) k_halo_rigid<T><<<grid_for(tot), 256, 0, S.stream>>>(AV[d].v, nd, d, 2, -1, 1, 0, 1, 0, rb.f, rb.n(), rc.f, rc.n());
  else k_halo_rigid<T><<<grid_for(tot), 256, 0, S.stream>>>(AV[d].v, nd, d, 2, n - 1, 1, n - 2, 1, 0, rb.f, rb.n(), rc.f, rc.n());
  MPDX_LAUNCH_CHECK();
}

template <class T>
void general<T>::fill_vctr_nrml(int d, int side, field<T> &A, rng rb, rng rc) {
  auto &S = *s;
  const int kind = S.bcs[d][side];
  if (kind == MPDX_BC_CYCLIC || kind == MPDX_BC_RIGID) { fill_sclr(d, side, A, rb, rc); return; }  // rigid: as scalars
  if (kind != MPDX_BC_OPEN) throw error(MPDX_E_UNSUPPORTED, "boundary condition not supported for vectors on this path");
  const int nd = S.nd, H = S.H, n = S.n[d];
  if (nd < 2) rb = {0, 0};
  if (nd < 3) rc = {0, 0};
  const int f = side == 0 ? -H : n;
  const long long tot = (long long)H * rb.n() * rc.n();
  k_halo_set<T><<<grid_for(tot), 256, 0, S.stream>>>(A.v, nd, d, f, H, 0, false, T(0), rb.f, rb.n(), rc.f, rc.n());
  MPDX_LAUNCH_CHECK();
}

template <class T>
void general<T>::fill_vctr_alng(int d, int side, field<T> *AV, rng rb, rng rc, bool ad, bool cyclic_only) {
  auto &S = *s;
  const int kind = S.bcs[d][side];
  const int nd = S.nd, H = S.H, n = S.n[d];
  if (nd < 2) rb = {0, 0};
  if (nd < 3) rc = {0, 0};
  if (kind == MPDX_BC_CYCLIC) {
    // left: [-H, -1] <- [n-1-H, n-2];  right: [n-1, n+H-2] <- [0, H-1]
    const int dst = side == 0 ? -H : n - 1, src = side == 0 ? n - 1 - H : 0;
    const long long tot = (long long)H * rb.n() * rc.n();
    k_halo_copy<T><<<grid_for(tot), 256, 0, S.stream>>>(AV[d].v, nd, d, dst, src, H, rb.f, rb.n(), rc.f, rc.n());
    MPDX_LAUNCH_CHECK();
    return;
  }
  if (cyclic_only) return;
  if (kind == MPDX_BC_RIGID) {
    // zero normal velocity at the wall point (rigid_2d.hpp:58-66, 154-162):
    // left  GC(-m) = -GC(m-1) for m = H .. 1 (.. 2 with ad);
    // right GC(n-1+a+t) = -GC(n-2-t), t = 0 .. H-1-a, a = ad (the reference's counter starts at 1 either way)
    const int a = ad ? 1 : 0;
    const long long tot = (long long)(H - a) * rb.n() * rc.n();
    if (H - a > 0) {
      if (side == 0) k_halo_rigid<T><<<grid_for(tot), 256, 0, S.stream>>>(AV[d].v, nd, d, 2, -H, H - a, H - 1, -1, 0, rb.f, rb.n(), rc.f, rc.n());
      else k_halo_rigid<T><<<grid_for(tot), 256, 0, S.stream>>>(AV[d].v, nd, d, 2, n - 1 + a, H - a, n - 2, -1, 0, rb.f, rb.n(), rc.f, rc.n());
      MPDX_LAUNCH_CHECK();
    }
    return;
  }
  if (kind != MPDX_BC_OPEN) throw error(MPDX_E_UNSUPPORTED, "boundary condition not supported for vectors on this path");
  if (nd == 1) {  // open_1d.hpp:36-40, 66-70
    int f, cnt, src;
    if (side == 0) { f = -H; cnt = H - (ad ? 1 : 0); src = 0; }
    else { f = n - 1 + (ad ? 1 : 0); cnt = H - (ad ? 1 : 0); src = n - 1 - H; }
    if (cnt > 0) {
      k_halo_set<T><<<1, 32, 0, S.stream>>>(AV[0].v, 1, 0, f, cnt, src, true, T(0), 0, 1, 0, 1);
      MPDX_LAUNCH_CHECK();
    }
    return;
  }
  const int e = side == 0 ? 0 : n - 1;
  const int d1 = (d + 1) % nd, d2 = (d + 2) % nd;
  // zero the perpendicular components on the domain edge lines (open_2d.hpp:77-82, open_3d.hpp:72-94)
  if (nd == 2) {
    if (d == 0) {
      k_halo_set<T><<<1, 32, 0, S.stream>>>(AV[d1].v, nd, d, e, 1, 0, false, T(0), rb.f - 1, 1, 0, 1);
      k_halo_set<T><<<1, 32, 0, S.stream>>>(AV[d1].v, nd, d, e, 1, 0, false, T(0), rb.l, 1, 0, 1);
    }
  } else {
    if (d == 0) {
      k_halo_set<T><<<grid_for(rb.n()), 256, 0, S.stream>>>(AV[d2].v, nd, d, e, 1, 0, false, T(0), rb.f, rb.n(), rc.f - 1, 1);
      k_halo_set<T><<<grid_for(rb.n()), 256, 0, S.stream>>>(AV[d2].v, nd, d, e, 1, 0, false, T(0), rb.f, rb.n(), rc.l, 1);
    }
    if (d == 0 || d == 1) {
      k_halo_set<T><<<grid_for(rc.n()), 256, 0, S.stream>>>(AV[d1].v, nd, d, e, 1, 0, false, T(0), rb.f - 1, 1, rc.f, rc.n());
      k_halo_set<T><<<grid_for(rc.n()), 256, 0, S.stream>>>(AV[d1].v, nd, d, e, 1, 0, false, T(0), rb.l, 1, rc.f, rc.n());
    }
  }
  MPDX_LAUNCH_CHECK();
  int f, cnt;
  if (side == 0) { f = -H; cnt = H - (ad ? 1 : 0); }
  else { f = n - 1 + (ad ? 1 : 0); cnt = H - (ad ? 1 : 0); }
  if (cnt <= 0) return;
  const long long tot = (long long)cnt * rb.n() * rc.n();
  k_zero_div<T><<<grid_for(tot), 256, 0, S.stream>>>(AV[d].v, AV[d1].v, AV[nd == 3 ? d2 : d1].v, nd, d, side, e, f, cnt,
                                                     rb.f, rb.n(), rc.f, rc.n());
  MPDX_LAUNCH_CHECK();
}

template <class T>
void general<T>::xchng_sclr(field<T> &A, int ex, bool deriv) {
  auto &S = *s;
  const rng *ir = S.ir;
  if (S.nd == 1) { for (int q = 0; q < 2; ++q) fill_sclr(0, q, A, {0, 0}, {0, 0}, deriv); return; }
  if (S.nd == 2) {  // solver_2d.hpp:40-56
    for (int q = 0; q < 2; ++q) fill_sclr(0, q, A, ext(ir[1], ex), {0, 0}, deriv);
    for (int q = 0; q < 2; ++q) fill_sclr(1, q, A, ext(ir[0], ex), {0, 0}, deriv);
    return;
  }
  // solver_3d.hpp:47-67
  for (int q = 0; q < 2; ++q) fill_sclr(1, q, A, ext(ir[2], ex), ext(ir[0], ex), deriv);
  for (int q = 0; q < 2; ++q) fill_sclr(0, q, A, ext(ir[1], ex), ext(ir[2], ex), deriv);
  for (int q = 0; q < 2; ++q) fill_sclr(2, q, A, ext(ir[0], ex), ext(ir[1], ex), deriv);
}

template <class T>
void general<T>::xchng_vctr_alng(field<T> *AV, bool ad, bool cyclic) {
  auto &S = *s;
  const rng *ir = S.ir;
  if (S.nd == 1) { for (int q = 0; q < 2; ++q) fill_vctr_alng(0, q, AV, {0, 0}, {0, 0}, ad, cyclic); return; }
  if (S.nd == 2) {  // solver_2d.hpp:63-88
    for (int q = 0; q < 2; ++q) fill_vctr_alng(0, q, AV, ir[1], {0, 0}, ad, cyclic);
    for (int q = 0; q < 2; ++q) fill_vctr_alng(1, q, AV, ir[0], {0, 0}, ad, cyclic);
    return;
  }
  // solver_3d.hpp:73-103
  for (int q = 0; q < 2; ++q) fill_vctr_alng(0, q, AV, ir[1], ir[2], ad, cyclic);
  for (int q = 0; q < 2; ++q) fill_vctr_alng(1, q, AV, ir[2], ir[0], ad, cyclic);
  for (int q = 0; q < 2; ++q) fill_vctr_alng(2, q, AV, ir[0], ir[1], ad, cyclic);
}

template <class T>
void general<T>::xchng_vctr_nrml(field<T> *AV, int ex) {
  auto &S = *s;
  const rng *ir = S.ir;
  if (S.nd == 1) return;
  if (S.nd == 2) {  // solver_2d.hpp:171-202
    for (int q = 0; q < 2; ++q) fill_vctr_nrml(1, q, AV[0], exh(ext(ir[0], ex)), {0, 0});
    for (int q = 0; q < 2; ++q) fill_vctr_nrml(0, q, AV[1], exh(ext(ir[1], ex)), {0, 0});
    return;
  }
  // solver_3d.hpp:207-286
  for (int q = 0; q < 2; ++q) fill_vctr_nrml(1, q, AV[0], ext(ext(ir[2], ex), 1), exh(ext(ir[0], ex)));
  for (int q = 0; q < 2; ++q) fill_vctr_nrml(2, q, AV[0], exh(ext(ir[0], ex)), ext(ext(ir[1], ex), 1));
  for (int q = 0; q < 2; ++q) fill_vctr_nrml(0, q, AV[1], exh(ext(ir[1], ex)), ext(ext(ir[2], ex), 1));
  for (int q = 0; q < 2; ++q) fill_vctr_nrml(2, q, AV[1], ext(ext(ir[0], ex), 1), exh(ext(ir[1], ex)));
  for (int q = 0; q < 2; ++q) fill_vctr_nrml(0, q, AV[2], ext(ext(ir[1], ex), 1), exh(ext(ir[2], ex)));
  for (int q = 0; q < 2; ++q) fill_vctr_nrml(1, q, AV[2], exh(ext(ir[2], ex)), ext(ext(ir[0], ex), 1));
}

template <class T>
void general<T>::xchng_flux(field<T> *AV) {  // solver_2d.hpp:90-101, solver_3d.hpp:105-118
  auto &S = *s;
  const rng *ir = S.ir;
  if (S.nd == 1) { for (int q = 0; q < 2; ++q) fill_flux(0, q, AV, {0, 0}, {0, 0}); return; }
  if (S.nd == 2) {
    for (int q = 0; q < 2; ++q) fill_flux(0, q, AV, ir[1], {0, 0});
    for (int q = 0; q < 2; ++q) fill_flux(1, q, AV, ir[0], {0, 0});
    return;
  }
  for (int q = 0; q < 2; ++q) fill_flux(0, q, AV, ir[1], ir[2]);
  for (int q = 0; q < 2; ++q) fill_flux(1, q, AV, ir[2], ir[0]);
  for (int q = 0; q < 2; ++q) fill_flux(2, q, AV, ir[0], ir[1]);
}

template <class T>
void general<T>::xchng_pres(field<T> &A, int ex) {  // solver_2d.hpp:204-220, solver_3d.hpp:288-307
  auto &S = *s;
  const rng *ir = S.ir;
  if (S.nd == 1) { for (int q = 0; q < 2; ++q) fill_pres(0, q, A, {0, 0}, {0, 0}); return; }
  if (S.nd == 2) {
    for (int q = 0; q < 2; ++q) fill_pres(0, q, A, ext(ir[1], ex), {0, 0});
    for (int q = 0; q < 2; ++q) fill_pres(1, q, A, ext(ir[0], ex), {0, 0});
    return;
  }
  for (int q = 0; q < 2; ++q) fill_pres(0, q, A, ext(ir[1], ex), ext(ir[2], ex));
  for (int q = 0; q < 2; ++q) fill_pres(1, q, A, ext(ir[2], ex), ext(ir[0], ex));
  for (int q = 0; q < 2; ++q) fill_pres(2, q, A, ext(ir[0], ex), ext(ir[1], ex));
}

template <class T>
void general<T>::set_edges(field<T> *const *AV) {  // solver_2d.hpp:222-237, solver_3d.hpp:309-326
  auto &S = *s;
  const rng *ir = S.ir;
  if (S.nd == 1) { for (int q = 0; q < 2; ++q) set_edge_pres(0, q, *AV[0], {0, 0}, {0, 0}); return; }
  if (S.nd == 2) {
    for (int q = 0; q < 2; ++q) set_edge_pres(0, q, *AV[0], ir[1], {0, 0});
    for (int q = 0; q < 2; ++q) set_edge_pres(1, q, *AV[1], ir[0], {0, 0});
    return;
  }
  for (int q = 0; q < 2; ++q) set_edge_pres(0, q, *AV[0], ir[1], ir[2]);
  for (int q = 0; q < 2; ++q) set_edge_pres(1, q, *AV[1], ir[2], ir[0]);
  for (int q = 0; q < 2; ++q) set_edge_pres(2, q, *AV[2], ir[0], ir[1]);
}

template <class T>
bool general<T>::any_rigid() const {
  for (int d = 0; d < s->nd; ++d)
    for (int q = 0; q < 2; ++q)
      if (s->bcs[d][q] == MPDX_BC_RIGID) return true;
  return false;
}

template <class T>
field<T> *general<T>::GC_unco(int iter) { return iter == 1 ? s->GC : (iter % 2 ? s->tmp1 : s->tmp0); }
template <class T>
field<T> *general<T>::GC_corr(int iter) { return iter % 2 ? s->tmp0 : s->tmp1; }
template <class T>
field<T> *general<T>::GCit(int iter) {
  if (iter == 0) return s->GC;
  if (s->opts & o_fct) return s->GC_mono;
  return GC_corr(iter);
}

template <class T>
template <int ND>
void general<T>::antidiff_nd(field<T> *res, field<T> &psi, field<T> *G) {
  auto &S = *s;
  const unsigned o = S.opts;
  const rng *ir = S.ir, *im = S.im;
  if (o & o_div_2nd) {  // divergence form (formulae_mpdata_{1,2,3}d.hpp antidiff with div_2nd)
    const dfield<T> pn = S.psi[cur_e][S.tl[cur_e] ^ 1].v;  // psi[e][n-1]
    const int sp = S.sptl_intrp;
    if (ND == 1) {
      launch_frame<1, 0>(S.stream, op_antidiff_div<1, 0, T>{res[0].v, psi.v, pn, G[0].v, G[0].v, G[0].v, o, S.G.v, sp}, im[0], {0, 0}, {0, 0});
    } else if (ND == 2) {
      launch_frame<2, 0>(S.stream, op_antidiff_div<2, 0, T>{res[0].v, psi.v, pn, G[0].v, G[1].v, G[1].v, o, S.G.v, sp}, im[0], ir[1], {0, 0});
      launch_frame<2, 1>(S.stream, op_antidiff_div<2, 1, T>{res[1].v, psi.v, pn, G[1].v, G[0].v, G[0].v, o, S.G.v, sp}, im[1], ir[0], {0, 0});
    } else {
      launch_frame<3, 0>(S.stream, op_antidiff_div<3, 0, T>{res[0].v, psi.v, pn, G[0].v, G[1].v, G[2].v, o, S.G.v, sp}, im[0], ir[1], ir[2]);
      launch_frame<3, 1>(S.stream, op_antidiff_div<3, 1, T>{res[1].v, psi.v, pn, G[1].v, G[2].v, G[0].v, o, S.G.v, sp}, im[1], ir[2], ir[0]);
      launch_frame<3, 2>(S.stream, op_antidiff_div<3, 2, T>{res[2].v, psi.v, pn, G[2].v, G[0].v, G[1].v, o, S.G.v, sp}, im[2], ir[0], ir[1]);
    }
    return;
  }
  if (ND == 1) {
    launch_frame<1, 0>(S.stream, op_antidiff<1, 0, T>{res[0].v, psi.v, G[0].v, G[0].v, G[0].v, o, S.G.v}, im[0], {0, 0}, {0, 0});
  } else if (ND == 2) {
    launch_frame<2, 0>(S.stream, op_antidiff<2, 0, T>{res[0].v, psi.v, G[0].v, G[1].v, G[1].v, o, S.G.v}, im[0], ir[1], {0, 0});
    launch_frame<2, 1>(S.stream, op_antidiff<2, 1, T>{res[1].v, psi.v, G[1].v, G[0].v, G[0].v, o, S.G.v}, im[1], ir[0], {0, 0});
  } else {
    launch_frame<3, 0>(S.stream, op_antidiff<3, 0, T>{res[0].v, psi.v, G[0].v, G[1].v, G[2].v, o, S.G.v}, im[0], ir[1], ir[2]);
    launch_frame<3, 1>(S.stream, op_antidiff<3, 1, T>{res[1].v, psi.v, G[1].v, G[2].v, G[0].v, o, S.G.v}, im[1], ir[2], ir[0]);
    launch_frame<3, 2>(S.stream, op_antidiff<3, 2, T>{res[2].v, psi.v, G[2].v, G[0].v, G[1].v, o, S.G.v}, im[2], ir[0], ir[1]);
  }
}

template <class T>
template <int ND>
void general<T>::fluxes_nd(field<T> *F, field<T> &psi, field<T> *C, bool extended) {
  auto &S = *s;
  const unsigned o = S.opts;
  auto R = [&](int d) { return extended ? ext(S.ir[d], 1) : S.ir[d]; };
  auto RM = [&](int d) { return extended ? ext(S.im[d], 1) : S.im[d]; };
  if (ND == 1) {
    launch_frame<1, 0>(S.stream, op_flux<1, 0, T>{F[0].v, psi.v, C[0].v, o}, RM(0), {0, 0}, {0, 0});
  } else if (ND == 2) {
    launch_frame<2, 0>(S.stream, op_flux<2, 0, T>{F[0].v, psi.v, C[0].v, o}, RM(0), R(1), {0, 0});
    launch_frame<2, 1>(S.stream, op_flux<2, 1, T>{F[1].v, psi.v, C[1].v, o}, RM(1), R(0), {0, 0});
  } else {
    launch_frame<3, 0>(S.stream, op_flux<3, 0, T>{F[0].v, psi.v, C[0].v, o}, RM(0), R(1), R(2));
    launch_frame<3, 1>(S.stream, op_flux<3, 1, T>{F[1].v, psi.v, C[1].v, o}, RM(1), R(2), R(0));
    launch_frame<3, 2>(S.stream, op_flux<3, 2, T>{F[2].v, psi.v, C[2].v, o}, RM(2), R(0), R(1));
  }
}

template <class T>
template <int ND>
void general<T>::fct_adjust_nd(int e, int iter) {
  auto &S = *s;
  field<T> &p = S.psi[e][S.tl[e]];
  field<T> *corr = GC_corr(iter);
  xchng_vctr_alng(corr, true);
  xchng_vctr_nrml(corr, 0);
  field<T> *flx = corr;
  if (!(S.opts & o_iga)) { fluxes_nd<ND>(S.flux, p, corr, true); flx = S.flux; }
  rng r0 = ext(S.ir[0], 1), r1 = ND > 1 ? ext(S.ir[1], 1) : rng{0, 0}, r2 = ND > 2 ? ext(S.ir[2], 1) : rng{0, 0};
  const dfield<T> z = flx[0].v;
  launch_frame<ND, 0>(S.stream, op_betas<ND, T>{S.beta_up.v, S.beta_dn.v, p.v, S.psi_max.v, S.psi_min.v, flx[0].v,
                                                ND > 1 ? flx[1].v : z, ND > 2 ? flx[2].v : z, S.opts, S.G.v},
                      r0, r1, r2);
  const rng *ir = S.ir, *im = S.im;
  if (ND == 1) {
    launch_frame<1, 0>(S.stream, op_gc_mono<1, 0, T>{S.GC_mono[0].v, corr[0].v, p.v, S.beta_up.v, S.beta_dn.v, S.opts}, im[0], {0, 0}, {0, 0});
  } else if (ND == 2) {
    launch_frame<2, 0>(S.stream, op_gc_mono<2, 0, T>{S.GC_mono[0].v, corr[0].v, p.v, S.beta_up.v, S.beta_dn.v, S.opts}, im[0], ir[1], {0, 0});
    launch_frame<2, 1>(S.stream, op_gc_mono<2, 1, T>{S.GC_mono[1].v, corr[1].v, p.v, S.beta_up.v, S.beta_dn.v, S.opts}, im[1], ir[0], {0, 0});
  } else {
    launch_frame<3, 0>(S.stream, op_gc_mono<3, 0, T>{S.GC_mono[0].v, corr[0].v, p.v, S.beta_up.v, S.beta_dn.v, S.opts}, im[0], ir[1], ir[2]);
    launch_frame<3, 1>(S.stream, op_gc_mono<3, 1, T>{S.GC_mono[1].v, corr[1].v, p.v, S.beta_up.v, S.beta_dn.v, S.opts}, im[1], ir[2], ir[0]);
    launch_frame<3, 2>(S.stream, op_gc_mono<3, 2, T>{S.GC_mono[2].v, corr[2].v, p.v, S.beta_up.v, S.beta_dn.v, S.opts}, im[2], ir[0], ir[1]);
  }
}

template <class T>
template <int ND>
void general<T>::advop_nd(int e) {
  auto &S = *s;
  if (S.opts & o_fct) {  // fct_init over i^1 x j^1 x k^1
    rng r0 = ext(S.ir[0], 1), r1 = ND > 1 ? ext(S.ir[1], 1) : rng{0, 0}, r2 = ND > 2 ? ext(S.ir[2], 1) : rng{0, 0};
    launch_frame<ND, 0>(S.stream, op_fct_init<ND, T>{S.psi_min.v, S.psi_max.v, S.psi[e][S.tl[e]].v}, r0, r1, r2);
  }
  for (int iter = 0; iter < S.n_iters; ++iter) {
    if (iter != 0) {
      S.tl[e] ^= 1;  // cycle(e)
      xchng_sclr(S.psi[e][S.tl[e]], S.H);
      field<T> *corr = GC_corr(iter);
      cur_e = e;
      antidiff_nd<ND>(corr, S.psi[e][S.tl[e]], GC_unco(iter));
      if (!(S.opts & o_fct) && iter != S.n_iters - 1) {
        xchng_vctr_nrml(corr, 0);
        if (S.opts & o_dfl) xchng_vctr_alng(corr, false);  // mpdata_osc_1d.hpp:82-88, _2d.hpp:120-124, _3d.hpp:138-142
      }
      if (S.opts & o_fct) fct_adjust_nd<ND>(e, iter);
    }
    field<T> &p = S.psi[e][S.tl[e]];
    field<T> *flx = S.flux;
    if (!(S.opts & o_iga) || iter == 0) fluxes_nd<ND>(S.flux, p, GCit(iter), false);
    else flx = GCit(iter);
    if (any_rigid()) xchng_flux(flx);  // mpdata_osc_2d.hpp:154-155 (a no-op without rigid walls)
    const dfield<T> z = flx[0].v;
    launch_frame<ND, 0>(S.stream, op_donorcell<ND, T>{S.psi[e][S.tl[e] ^ 1].v, p.v, flx[0].v, ND > 1 ? flx[1].v : z, ND > 2 ? flx[2].v : z, S.opts, S.G.v},
                        S.ir[0], ND > 1 ? S.ir[1] : rng{0, 0}, ND > 2 ? S.ir[2] : rng{0, 0});
    // upwind-only step every upwind_filter_freq steps (mpdata_osc_2d.hpp:176-179)
    if (S.upwind_filter_freq > 0 && S.timestep % S.upwind_filter_freq == 0) break;
  }
}

// divergence of the advector: max |div GC| / G over the interior (solver_{2,3}d.hpp max_abs_vctr_div)
template <class T>
__global__ void k_max_abs_div(int nd, int n0, int n1, int n2, dfield<T> g0, dfield<T> g1, dfield<T> g2, bool nug, dfield<T> G,
                              double *out) {
  double m = 0;
  const long long tot = (long long)n0 * n1 * n2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int k = int(q % n2);
    const long long r = q / n2;
    const int j = int(r % n1), i = int(r / n1);
    T v;
    if (nd == 1) v = fabs(g0(i, j, k) - g0(i - 1, j, k));
    else if (nd == 2) v = fabs((g0(i, j, k) - g0(i - 1, j, k)) + (g1(i, j, k) - g1(i, j - 1, k)));
    else v = fabs((g0(i, j, k) - g0(i - 1, j, k)) + (g1(i, j, k) - g1(i, j - 1, k)) + (g2(i, j, k) - g2(i, j, k - 1)));
    if (nug) v = v / G(i, j, k);
    m = fmax(m, double(v));
  }
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) {
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long *>(out), (unsigned long long)__double_as_longlong(m));
  }
}

template <class T>
void general<T>::ante_loop(double *dev_scratch) {
  auto &S = *s;
  xchng_vctr_alng(S.GC);
  if (S.nd > 1 && !(S.opts & o_dfl)) {
    MPDX_CUDA(cudaMemsetAsync(dev_scratch, 0, sizeof(double), S.stream));
    const dfield<T> z = S.GC[0].v;
    k_max_abs_div<T><<<grid_for(S.cells()), 256, 0, S.stream>>>(S.nd, S.n[0], S.n[1], S.n[2], S.GC[0].v,
                                                                S.nd > 1 ? S.GC[1].v : z, S.nd > 2 ? S.GC[2].v : z,
                                                                (S.opts & o_nug) != 0, S.G.v, dev_scratch);
    MPDX_LAUNCH_CHECK();
    double m = 0;
    MPDX_CUDA(cudaMemcpyAsync(&m, dev_scratch, sizeof(double), cudaMemcpyDeviceToHost, S.stream));
    MPDX_CUDA(cudaStreamSynchronize(S.stream));
    if (T(m) > S.max_abs_div_eps) throw error(MPDX_E_DIVERGENT, "libmpdata++: initial advector field is divergent");
  }
  if (S.opts & o_nug) xchng_sclr(S.G, S.H);  // mpdata_osc_{1,2,3}d.hpp hook_ante_loop
  if (S.nd > 1) xchng_vctr_nrml(S.GC, S.H - 1);
}

template <class T>
__global__ void k_fill(T *p, size_t n, T v) {
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) p[q] = v;
}

template <class T>
void general<T>::init_g() {
  auto &S = *s;
  if (!(S.opts & o_nug)) return;
  const size_t n = S.G.bytes / sizeof(T);
  k_fill<T><<<grid_for((long long)n), 256, 0, S.stream>>>(static_cast<T *>(S.G.base), n, T(1));
  MPDX_LAUNCH_CHECK();
}

template <class T>
void general<T>::step() {
  auto &S = *s;
  for (int e = 0; e < S.n_eqns; ++e) {
    xchng_sclr(S.psi[e][S.tl[e]], S.H);  // solve_loop_body: xchng(e)
    if (S.nd == 1) advop_nd<1>(e);
    else if (S.nd == 2) advop_nd<2>(e);
    else advop_nd<3>(e);
    S.tl[e] ^= 1;  // cycle(e)
  }
}

template struct general<float>;
template struct general<double>;

}  // namespace mpdx
