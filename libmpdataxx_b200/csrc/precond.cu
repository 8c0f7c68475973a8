// Learned preconditioner network for the GCR pressure solve.
//
// Architecture (a linear 4-level U-net; tests/test_precond_oracle.py pins
// the float64 restatement oracle/precond_oracle.py that the kernels follow):
//
//   e0 = conv(r, 1 -> C0)                     level 0 (the pressure grid)
//   e1 = conv(pool(e0), C0 -> C1)             level 1 (ceil(n/2) points per axis)
//   e2 = conv(pool(e1), C1 -> C2)             level 2
//   e3 = conv(pool(e2), C2 -> C3)             level 3
//   m3 = conv(e3, C3 -> C3)                   level 3
//   d2 = conv(up(m3), C3 -> C2) + e2          level 2
//   d1 = conv(up(d2), C2 -> C1) + e1          level 1
//   d0 = conv(up(d1), C1 -> C0) + e0          level 0
//   q  = conv(d0, C0 -> 1)                    level 0
//
// conv: 3^d-point stencil with bias; cyclic axes wrap (modulo the level's
// size), rigid axes pad with zeros.  pool: average of the fine points of a
// coarse point; up: coarse point floor(p/2).
//
// Tensors are BF16, channels-last ([point][channel]).  The seven convolutions
// with C_in, C_out >= 8 run on the tensor cores as implicit GEMMs
// (mma.sync m16n8k16 BF16 -> FP32): a CTA stages a halo tile of the input in
// shared memory, each warp owns 16 consecutive output points along the
// contiguous axis and all output channels, and every K-step of 16 pairs two
// 8-channel groups (a group = 8 channels of one stencil tap) fetched with
// ldmatrix; the weights come pre-arranged in fragment order.  The 1 -> C0 and
// C0 -> 1 end layers are per-point FMA loops.  Backward: the input gradient of
// a tensor-core convolution is the same kernel with the adjoint weights (taps
// mirrored, channels transposed); weight gradients are per-tap GEMMs over the
// points (ldmatrix.trans fragments) with a fixed-order reduction.
#include <cmath>
#include <cstring>
#include <random>

#include "precond.cuh"

namespace mpdx {
namespace pc {

// ---------------------------------------------------------------------------
// helpers

__device__ __forceinline__ uint16_t f2bf(float x) {  // round to nearest even
  unsigned u = __float_as_uint(x);
  if ((u & 0x7f800000u) == 0x7f800000u) return uint16_t(u >> 16);  // inf / nan
  u += 0x7fffu + ((u >> 16) & 1u);
  return uint16_t(u >> 16);
}
__device__ __forceinline__ float bf2f(uint16_t h) { return __uint_as_float(unsigned(h) << 16); }
struct grid3 {
  int n[3], wrap[3];
  long long vox;
};
// coordinate x of an axis with n points under the padding rule (one point of
// padding per side; farther points, which only partial tiles touch, read as zero)
__device__ __forceinline__ int padx(int x, int n, int w) {
  if (x >= 0 && x < n) return x;
  if (!w || x < -1 || x > n) return -1;
  return x < 0 ? n - 1 : 0;
}
// tap t -> offsets (i slowest, k fastest); 2D uses only c = 0
template <int ND>
__device__ __forceinline__ void tap_off(int t, int &a, int &b, int &c) {
  if (ND == 3) { a = t / 9 - 1; b = (t / 3) % 3 - 1; c = t % 3 - 1; }
  else { a = t / 3 - 1; b = t % 3 - 1; c = 0; }
}
__device__ __forceinline__ long long vindex(const grid3 &g, int i, int j, int k) {
  return ((long long)i * g.n[1] + j) * g.n[2] + k;
}
// neighbour (i+a, j+b, k+c) under the padding rule, -1 for a zero pad
__device__ __forceinline__ long long nbr(const grid3 &g, int i, int j, int k, int a, int b, int c) {
  const int x = padx(i + a, g.n[0], g.wrap[0]), y = padx(j + b, g.n[1], g.wrap[1]), z = padx(k + c, g.n[2], g.wrap[2]);
  if (x < 0 || y < 0 || z < 0) return -1;
  return vindex(g, x, y, z);
}

// ---------------------------------------------------------------------------
// tensor-core convolution (forward, or input gradient with adjoint weights)

template <int ND> struct tile;
template <> struct tile<3> { static constexpr int T0 = 2, T1 = 4, T2 = 16; };
template <> struct tile<2> { static constexpr int T0 = 8, T1 = 16, T2 = 1; };

// the convolution's tile: R rows of 16 points per warp (8 warps); R = 4 on the fine
// 3D levels, where every weight fragment then serves four MMAs
template <int ND, int R> struct ctile;
template <> struct ctile<3, 1> { static constexpr int T0 = 2, T1 = 4, T2 = 16; };
template <> struct ctile<3, 4> { static constexpr int T0 = 4, T1 = 8, T2 = 16; };
template <> struct ctile<2, 1> { static constexpr int T0 = 8, T1 = 16, T2 = 1; };

template <int CIN>
struct sv {  // bytes per point in the shared tile (padded against bank conflicts)
  static constexpr int v = CIN >= 16 ? CIN * 2 + 16 : 16;
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return unsigned(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

struct conv_out {
  uint16_t *bf;         // BF16 output (or null)
  float *f32;           // FP32 output (or null)
  const float *bias;    // (cout) or null
  const uint16_t *skip; // BF16 tensor added to the output (or null)
};

// X: [vox][CIN] BF16 on grid g; Wf: fragments [chunk][COUT/8][32] x uint2.
// UP = 1: X lives on the coarse grid cg and the input is its nearest up-sampling,
// X(p) = X_coarse(floor(p / 2)) (k_up), read straight into the halo tile.
// UP = 2: the same for a fine grid of even sides (padding and wrapping then agree
// between the fine and the coarse grid): the CTA stages the coarse points its halo
// tile covers, (T/2 + 2) per axis, and each lane's ldmatrix row points at the
// coarse point of its fine point.
template <int CIN, int COUT, int ND, int UP, int R>
__global__ void __launch_bounds__(256) k_conv_tc(grid3 g, grid3 cg, const uint16_t *__restrict__ X, const uint2 *__restrict__ Wf,
                                                 conv_out o, const int *skip_flag) {
  if (skip_flag && *skip_flag) return;
  using TL = ctile<ND, R>;
  constexpr int T0 = TL::T0, T1 = TL::T1, T2 = TL::T2;
  constexpr bool CO = UP == 2;  // coarse staging
  constexpr int H0 = CO ? T0 / 2 + 2 : T0 + 2, H1 = CO ? T1 / 2 + 2 : T1 + 2;
  constexpr int H2 = ND == 3 ? (CO ? T2 / 2 + 2 : T2 + 2) : 1;
  constexpr int CB = CIN / 8, SV = sv<CIN>::v, NTAPS = ND == 3 ? 27 : 9;
  constexpr int NG = NTAPS * CB, NCH = (NG + 1) / 2, NT = COUT / 8;
  extern __shared__ __align__(16) unsigned char sm[];

  const int nt1 = (g.n[1] + T1 - 1) / T1, nt2 = (g.n[2] + T2 - 1) / T2;
  const int tb = blockIdx.x;
  const int i0 = (tb / (nt1 * nt2)) * T0, j0 = ((tb / nt2) % nt1) * T1, k0 = (tb % nt2) * T2;
  // stage the halo tile
  for (int q = threadIdx.x; q < H0 * H1 * H2 * CB; q += blockDim.x) {
    const int hv = q / CB, cb = q % CB;
    const int hk = hv % H2, hj = (hv / H2) % H1, hi = hv / (H2 * H1);
    long long v;
    if constexpr (CO) {
      // coarse coordinates i0/2 - 1 + hi (i0 even), padded on the coarse grid
      v = nbr(cg, i0 / 2 - 1 + hi, j0 / 2 - 1 + hj, ND == 3 ? k0 / 2 - 1 + hk : 0, 0, 0, 0);
    } else if constexpr (UP == 1) {
      const int x = padx(i0 - 1 + hi, g.n[0], g.wrap[0]), y = padx(j0 - 1 + hj, g.n[1], g.wrap[1]);
      const int z = ND == 3 ? padx(k0 - 1 + hk, g.n[2], g.wrap[2]) : 0;
      v = (x < 0 || y < 0 || z < 0) ? -1
                                    : vindex(cg, min(x / 2, cg.n[0] - 1), min(y / 2, cg.n[1] - 1), min(z / 2, cg.n[2] - 1));
    } else {
      v = nbr(g, i0 - 1 + hi, j0 - 1 + hj, ND == 3 ? k0 - 1 + hk : 0, 0, 0, 0);
    }
    // asynchronous 16-byte copy; a padding point copies no bytes and is zero-filled
    const uint16_t *src = v >= 0 ? X + v * CIN + cb * 8 : X;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(sm + hv * SV + cb * 16)), "l"(src),
                 "r"(v >= 0 ? 16 : 0)
                 : "memory");
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();

  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // the warp's rows of the tile (ND = 3: rows (ti, tj) of 16 points along k; ND = 2: row ti along j)
  int ti[R], tj[R];
#pragma unroll
  for (int rr = 0; rr < R; ++rr) {
    const int row = w * R + rr;
    ti[rr] = ND == 3 ? row / T1 : row;
    tj[rr] = ND == 3 ? row % T1 : 0;
  }
  // ldmatrix row of this lane: point m, group slot gs (0: k 0-7, 1: k 8-15)
  const int lm = (lane & 7) + ((lane >> 3) & 1) * 8, gs = lane >> 4;
  float acc[R][NT][4];
#pragma unroll
  for (int rr = 0; rr < R; ++rr)
#pragma unroll
    for (int n = 0; n < NT; ++n) acc[rr][n][0] = acc[rr][n][1] = acc[rr][n][2] = acc[rr][n][3] = 0.f;
  const unsigned sbase = smem_u32(sm);
  // fully unrolled: every chunk's taps and channel groups are constants (a lane's
  // group slot gs selects between two of them)
#pragma unroll
  for (int ch = 0; ch < NCH; ++ch) {
    int gidx = 2 * ch + gs;
    if (gidx >= NG) gidx = 2 * ch;  // zero weights pair with any valid address
    const int tap = gidx / CB, cb = gidx % CB;
    int a, b, c;
    tap_off<ND>(tap, a, b, c);
    uint2 bw[NT];
#pragma unroll
    for (int n = 0; n < NT; ++n) bw[n] = __ldg(Wf + (size_t(ch) * NT + n) * 32 + lane);
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      int hv;
      if constexpr (CO) {  // fine tile coordinate f in [-1, T] -> staged coarse row (f + 2) / 2
        if (ND == 3) hv = (((ti[rr] + a + 2) >> 1) * H1 + ((tj[rr] + b + 2) >> 1)) * H2 + ((lm + c + 2) >> 1);
        else hv = ((ti[rr] + a + 2) >> 1) * H1 + ((lm + b + 2) >> 1);
      } else {
        if (ND == 3) hv = ((ti[rr] + 1 + a) * H1 + (tj[rr] + 1 + b)) * H2 + (lm + 1 + c);
        else hv = (ti[rr] + 1 + a) * H1 + (lm + 1 + b);
      }
      unsigned af[4];
      asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                   : "=r"(af[0]), "=r"(af[1]), "=r"(af[2]), "=r"(af[3])
                   : "r"(sbase + hv * SV + cb * 16));
#pragma unroll
      for (int n = 0; n < NT; ++n) mma16816(acc[rr][n], af, bw[n].x, bw[n].y);
    }
  }
  // epilogue: rows lane/4 and lane/4 + 8, columns 2 (lane % 4) + {0, 1} of each 8-channel tile
#pragma unroll
  for (int rr = 0; rr < R; ++rr)
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int m = lane / 4 + 8 * h;
    int gi, gj, gk;
    if (ND == 3) { gi = i0 + ti[rr]; gj = j0 + tj[rr]; gk = k0 + m; }
    else { gi = i0 + ti[rr]; gj = j0 + m; gk = 0; }
    if (gi >= g.n[0] || gj >= g.n[1] || gk >= g.n[2]) continue;
    const long long v = vindex(g, gi, gj, gk);
#pragma unroll
    for (int n = 0; n < NT; ++n) {
      const int co = n * 8 + 2 * (lane % 4);
      float y0 = acc[rr][n][2 * h], y1 = acc[rr][n][2 * h + 1];
      if (o.bias) { y0 += o.bias[co]; y1 += o.bias[co + 1]; }
      if (o.skip) {
        const unsigned s2 = *reinterpret_cast<const unsigned *>(o.skip + v * COUT + co);
        y0 += bf2f(uint16_t(s2 & 0xffffu));
        y1 += bf2f(uint16_t(s2 >> 16));
      }
      if (o.bf) *reinterpret_cast<unsigned *>(o.bf + v * COUT + co) = unsigned(f2bf(y0)) | (unsigned(f2bf(y1)) << 16);
      if (o.f32) *reinterpret_cast<float2 *>(o.f32 + v * COUT + co) = make_float2(y0, y1);
    }
  }
}

// weight gradient of a tensor-core layer, one tap per blockIdx.y:
// part[(tap * gridDim.x + bx) * COUT * CIN + co * CIN + ci] = sum over this CTA's points of dY[p][co] X[p + tap][ci]
template <int CIN, int COUT, int ND>
__global__ void __launch_bounds__(256) k_conv_dw(grid3 g, const uint16_t *__restrict__ dY, const uint16_t *__restrict__ X,
                                                 float *part) {
  using TL = tile<ND>;
  constexpr int T0 = TL::T0, T1 = TL::T1, T2 = TL::T2, TP = T0 * T1 * T2;  // 128 points
  constexpr int COUTP = COUT < 16 ? 16 : COUT;                          // rows of the M dimension
  constexpr int SY = COUTP * 2 + 16, SX = sv<CIN>::v;
  constexpr int MT = COUTP / 16, NTn = CIN / 8, PAIRS = MT * NTn, PPW = (PAIRS + 7) / 8;
  extern __shared__ __align__(16) unsigned char sm[];
  unsigned char *sy = sm, *sx = sm + TP * SY;
  const int tap = blockIdx.y;
  int ta, tbo, tc;
  tap_off<ND>(tap, ta, tbo, tc);
  const int nt1 = (g.n[1] + T1 - 1) / T1, nt2 = (g.n[2] + T2 - 1) / T2;
  const long long ntiles = (long long)((g.n[0] + T0 - 1) / T0) * nt1 * nt2;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float acc[PPW][4];
#pragma unroll
  for (int q = 0; q < PPW; ++q) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = 0.f;

  for (long long tb = blockIdx.x; tb < ntiles; tb += gridDim.x) {
    const int i0 = int(tb / (nt1 * nt2)) * T0, j0 = int((tb / nt2) % nt1) * T1, k0 = int(tb % nt2) * T2;
    __syncthreads();
    for (int q = threadIdx.x; q < TP * (COUTP / 8); q += blockDim.x) {
      const int p = q / (COUTP / 8), cb = q % (COUTP / 8);
      const int pk = p % T2, pj = (p / T2) % T1, pi = p / (T2 * T1);
      const int gi = i0 + pi, gj = j0 + pj, gk = ND == 3 ? k0 + pk : 0;
      uint4 val = make_uint4(0, 0, 0, 0);
      if (gi < g.n[0] && gj < g.n[1] && gk < g.n[2] && cb * 8 < COUT)
        val = *reinterpret_cast<const uint4 *>(dY + vindex(g, gi, gj, gk) * COUT + cb * 8);
      *reinterpret_cast<uint4 *>(sy + p * SY + cb * 16) = val;
    }
    for (int q = threadIdx.x; q < TP * (CIN / 8); q += blockDim.x) {
      const int p = q / (CIN / 8), cb = q % (CIN / 8);
      const int pk = p % T2, pj = (p / T2) % T1, pi = p / (T2 * T1);
      const int gi = i0 + pi, gj = j0 + pj, gk = ND == 3 ? k0 + pk : 0;
      uint4 val = make_uint4(0, 0, 0, 0);
      if (gi < g.n[0] && gj < g.n[1] && gk < g.n[2]) {
        const long long v = nbr(g, gi, gj, gk, ta, tbo, tc);
        if (v >= 0) val = *reinterpret_cast<const uint4 *>(X + v * CIN + cb * 8);
      }
      *reinterpret_cast<uint4 *>(sx + p * SX + cb * 16) = val;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PPW; ++q) {
      const int pr = w + 8 * q;
      if (pr >= PAIRS) break;
      const int mt = pr / NTn, nt = pr % NTn;
#pragma unroll
      for (int ks = 0; ks < TP / 16; ++ks) {
        unsigned af[4], b0, b1;
        {  // A = dY^T (co x points): matrices (co 0-7, p 0-7), (co 8-15, p 0-7), (co 0-7, p 8-15), (co 8-15, p 8-15)
          const int mi = lane >> 3, r = lane & 7;
          const int co0 = mt * 16 + (mi & 1) * 8, p0 = ks * 16 + (mi >> 1) * 8;
          asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                       : "=r"(af[0]), "=r"(af[1]), "=r"(af[2]), "=r"(af[3])
                       : "r"(smem_u32(sy + (p0 + r) * SY + co0 * 2)));
        }
        {  // B = X (points x ci): matrices (p 0-7, ci 0-7), (p 8-15, ci 0-7)
          const int mi = (lane >> 3) & 1, r = lane & 7;
          asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                       : "=r"(b0), "=r"(b1)
                       : "r"(smem_u32(sx + (ks * 16 + mi * 8 + r) * SX + nt * 16)));
        }
        mma16816(acc[q], af, b0, b1);
      }
    }
  }
  float *out = part + (size_t(tap) * gridDim.x + blockIdx.x) * COUT * CIN;
#pragma unroll
  for (int q = 0; q < PPW; ++q) {
    const int pr = w + 8 * q;
    if (pr >= PAIRS) break;
    const int mt = pr / NTn, nt = pr % NTn;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int co = mt * 16 + lane / 4 + 8 * h, ci = nt * 8 + 2 * (lane % 4);
      if (co < COUT) {
        out[co * CIN + ci] = acc[q][2 * h];
        out[co * CIN + ci + 1] = acc[q][2 * h + 1];
      }
    }
  }
}

// grad[w_off + (co * ntaps + t) * cin + ci] = sum over blocks of part (fixed order)
__global__ void k_dw_reduce(const float *part, int nblk, int ntaps, int cout, int cin, float *grad) {
  const int tot = ntaps * cout * cin;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) {
    const int ci = q % cin, co = (q / cin) % cout, t = q / (cin * cout);
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += part[(size_t(t) * nblk + b) * cout * cin + co * cin + ci];
    grad[(size_t(co) * ntaps + t) * cin + ci] = s;
  }
}

// bias gradient: grad_b[c] = sum over points of dY[p][c] (FP32 dY), fixed-order block partials
__global__ void k_db(const float *dY, long long vox, int C, float *part) {
  extern __shared__ float red[];
  for (int c = 0; c < C; ++c) {
    float s = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < vox; p += (long long)gridDim.x * blockDim.x)
      s += dY[p * C + c];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[size_t(c) * gridDim.x + blockIdx.x] = red[0];
    __syncthreads();
  }
}
__global__ void k_db_reduce(const float *part, int nblk, int C, float *grad_b) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (int b = 0; b < nblk; ++b) s += part[size_t(c) * nblk + b];
  grad_b[c] = s;
}

// ---------------------------------------------------------------------------
// end layers (per-point loops)

// Tiles of the per-point end layers: 512 points, 128 threads, each thread a column
// of four points along i (ND = 3: 4 x 8 x 16; ND = 2: 4 x 128), even sizes at even
// origins so that every 2^d block of the pooling lies inside one tile.  A thread
// reads the six halo values of its column once per (j, k) tap offset and uses
// them for the three i offsets of all four points.
template <int ND> struct etile;
template <> struct etile<3> { static constexpr int T0 = 4, T1 = 8, T2 = 16, H0 = 6, H1 = 10, H2 = 18; };
template <> struct etile<2> { static constexpr int T0 = 4, T1 = 128, T2 = 1, H0 = 6, H1 = 130, H2 = 1; };
constexpr int kEndThreads = 128;

template <int ND>
__device__ __forceinline__ void etile_origin(const grid3 &g, int b, int &i0, int &j0, int &k0) {
  using E = etile<ND>;
  const int n1 = (g.n[1] + E::T1 - 1) / E::T1, n2 = (g.n[2] + E::T2 - 1) / E::T2;
  i0 = (b / (n1 * n2)) * E::T0; j0 = ((b / n2) % n1) * E::T1; k0 = (b % n2) * E::T2;
}
template <int ND>
inline long long etile_count(const grid3 &g) {
  using E = etile<ND>;
  return (long long)((g.n[0] + E::T0 - 1) / E::T0) * ((g.n[1] + E::T1 - 1) / E::T1) * ((g.n[2] + E::T2 - 1) / E::T2);
}
// tap index of offsets (ta, tb, tc) in tap_off's order
template <int ND>
__device__ __forceinline__ constexpr int tap_of(int ta, int tb, int tc) {
  return ND == 3 ? (ta + 1) * 9 + (tb + 1) * 3 + (tc + 1) : (ta + 1) * 3 + (tb + 1);
}

// e0[p][co] = b[co] + sum_t W[co][t] r(p + tap_t), r from an FP64 halo'ed field or a
// compact FP32 array, staged with its halo in shared memory; with POOL the CTA also
// writes the pooled level-1 input p1 = pool(e0) of its tile (k_pool's average of the
// BF16 values, in k_pool's order)
template <int C0, int ND, bool FIELD, bool POOL>
__global__ void __launch_bounds__(kEndThreads) k_conv_in(grid3 g, grid3 cg, const double *rf, long long s0, long long s1,
                                                         long long s2, const float *rc, const float *W, const float *b,
                                                         uint16_t *e0, uint16_t *p1, const int *skip_flag) {
  if (skip_flag && *skip_flag) return;
  using E = etile<ND>;
  constexpr int NTAPS = ND == 3 ? 27 : 9, NH = E::H0 * E::H1 * E::H2, NP = E::T0 * E::T1 * E::T2;
  constexpr int TC = ND == 3 ? 1 : 0;  // k offsets -TC..TC
  __shared__ float rs[NH];
  __shared__ __align__(16) float ws[NTAPS * C0];  // tap-major: ws[t][co]
  __shared__ float bs[C0];
  __shared__ float es[POOL ? NP * C0 : 1];
  int i0, j0, k0;
  etile_origin<ND>(g, blockIdx.x, i0, j0, k0);
  for (int q = threadIdx.x; q < C0 * NTAPS; q += blockDim.x) ws[(q % NTAPS) * C0 + q / NTAPS] = W[q];
  if (threadIdx.x < C0) bs[threadIdx.x] = b[threadIdx.x];
  for (int q = threadIdx.x; q < NH; q += blockDim.x) {
    const int hk = q % E::H2, hj = (q / E::H2) % E::H1, hi = q / (E::H2 * E::H1);
    const int x = padx(i0 - 1 + hi, g.n[0], g.wrap[0]), y = padx(j0 - 1 + hj, g.n[1], g.wrap[1]);
    const int z = ND == 3 ? padx(k0 - 1 + hk, g.n[2], g.wrap[2]) : 0;
    float r = 0.f;
    if (x >= 0 && y >= 0 && z >= 0) r = FIELD ? float(rf[x * s0 + y * s1 + z * s2]) : rc[vindex(g, x, y, z)];
    rs[q] = r;
  }
  __syncthreads();
  const int c = threadIdx.x % E::T2, bb = threadIdx.x / E::T2;
  float acc[4][C0];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int co = 0; co < C0; ++co) acc[a][co] = bs[co];
#pragma unroll
  for (int tb = -1; tb <= 1; ++tb)
#pragma unroll
    for (int tc = -TC; tc <= TC; ++tc) {
      float col[6];
#pragma unroll
      for (int h = 0; h < 6; ++h) col[h] = rs[(h * E::H1 + (bb + 1 + tb)) * E::H2 + (ND == 3 ? c + 1 + tc : 0)];
#pragma unroll
      for (int ta = -1; ta <= 1; ++ta) {
        const int t = tap_of<ND>(ta, tb, tc);
        float w[C0];
#pragma unroll
        for (int q = 0; q < C0 / 4; ++q) {
          const float4 v = reinterpret_cast<const float4 *>(ws + t * C0)[q];
          w[4 * q] = v.x; w[4 * q + 1] = v.y; w[4 * q + 2] = v.z; w[4 * q + 3] = v.w;
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int co = 0; co < C0; ++co) acc[a][co] = fmaf(w[co], col[a + 1 + ta], acc[a][co]);
      }
    }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + a, j = j0 + bb, k = k0 + c;
    unsigned pk[C0 / 2];
#pragma unroll
    for (int co = 0; co < C0; co += 2) pk[co / 2] = unsigned(f2bf(acc[a][co])) | (unsigned(f2bf(acc[a][co + 1])) << 16);
    if (i < g.n[0] && j < g.n[1] && k < g.n[2]) {
      uint4 *dst = reinterpret_cast<uint4 *>(e0 + vindex(g, i, j, k) * C0);
#pragma unroll
      for (int h = 0; h < C0 / 8; ++h) dst[h] = make_uint4(pk[4 * h], pk[4 * h + 1], pk[4 * h + 2], pk[4 * h + 3]);
    }
    if constexpr (POOL) {
      const int lin = (a * E::T1 + bb) * E::T2 + c;
#pragma unroll
      for (int co = 0; co < C0; co += 2) {
        es[lin * C0 + co] = bf2f(uint16_t(pk[co / 2] & 0xffffu));
        es[lin * C0 + co + 1] = bf2f(uint16_t(pk[co / 2] >> 16));
      }
    }
  }
  if constexpr (POOL) {
    __syncthreads();
    constexpr int Q0 = E::T0 / 2, Q1 = E::T1 / 2, Q2 = ND == 3 ? E::T2 / 2 : 1;
    for (int q = threadIdx.x; q < Q0 * Q1 * Q2 * C0; q += blockDim.x) {
      const int co = q % C0, V = q / C0;
      const int K = V % Q2, J = (V / Q2) % Q1, I = V / (Q2 * Q1);
      const int gI = i0 / 2 + I, gJ = j0 / 2 + J, gK = ND == 3 ? k0 / 2 + K : 0;
      if (gI >= cg.n[0] || gJ >= cg.n[1] || gK >= cg.n[2]) continue;
      float sum = 0.f;
      int cnt = 0;
      const int l0 = ((2 * gI - i0) * E::T1 + (2 * gJ - j0)) * E::T2 + (ND == 3 ? 2 * gK - k0 : 0);
      const bool full = 2 * gI + 1 < g.n[0] && 2 * gJ + 1 < g.n[1] && (ND == 2 || 2 * gK + 1 < g.n[2]);
      if (full) {  // the whole 2^d block exists: k_pool's order without the checks
        constexpr int DK = ND == 3 ? 1 : 0;
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int bb = 0; bb < 2; ++bb)
#pragma unroll
            for (int d = 0; d <= DK; ++d) sum += es[(l0 + (a * E::T1 + bb) * E::T2 + d) * C0 + co];
        cnt = ND == 3 ? 8 : 4;
      } else {
        for (int a = 0; a < 2; ++a)
          for (int bb = 0; bb < 2; ++bb)
            for (int d = 0; d < 2; ++d) {
              const int i = 2 * gI + a, j = 2 * gJ + bb, k = 2 * gK + d;
              if (i >= g.n[0] || j >= g.n[1] || k >= g.n[2]) continue;
              if ((g.n[0] == 1 && a) || (g.n[1] == 1 && bb) || (g.n[2] == 1 && d)) continue;
              const int lin = ((i - i0) * E::T1 + (j - j0)) * E::T2 + (ND == 3 ? k - k0 : 0);
              sum += es[lin * C0 + co];
              ++cnt;
            }
      }
      p1[vindex(cg, gI, gJ, gK) * C0 + co] = f2bf(sum / float(cnt));
    }
  }
}

// q(p) = b + sum_t sum_ci W[t][ci] d0[p + tap_t][ci], to an FP64 halo'ed field or a
// compact FP32 array; d0 (BF16) is staged with its halo in shared memory
template <int C0, int ND, bool FIELD>
__global__ void __launch_bounds__(kEndThreads) k_conv_outl(grid3 g, const uint16_t *d0, const float *W, const float *b,
                                                           double *qf, long long s0, long long s1, long long s2, float *qc,
                                                           const int *skip_flag) {
  if (skip_flag && *skip_flag) return;
  using E = etile<ND>;
  constexpr int NTAPS = ND == 3 ? 27 : 9, NH = E::H0 * E::H1 * E::H2, CB = C0 / 8;
  constexpr int TC = ND == 3 ? 1 : 0;
  __shared__ uint4 ds[NH * CB];
  __shared__ __align__(16) float ws[NTAPS * C0];  // W[t][ci]
  __shared__ float b0;
  int i0, j0, k0;
  etile_origin<ND>(g, blockIdx.x, i0, j0, k0);
  for (int q = threadIdx.x; q < NTAPS * C0; q += blockDim.x) ws[q] = W[q];
  if (threadIdx.x == 0) b0 = b[0];
  for (int q = threadIdx.x; q < NH * CB; q += blockDim.x) {
    const int hv = q / CB, cb = q % CB;
    const int hk = hv % E::H2, hj = (hv / E::H2) % E::H1, hi = hv / (E::H2 * E::H1);
    const int x = padx(i0 - 1 + hi, g.n[0], g.wrap[0]), y = padx(j0 - 1 + hj, g.n[1], g.wrap[1]);
    const int z = ND == 3 ? padx(k0 - 1 + hk, g.n[2], g.wrap[2]) : 0;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (x >= 0 && y >= 0 && z >= 0) v = *reinterpret_cast<const uint4 *>(d0 + vindex(g, x, y, z) * C0 + cb * 8);
    ds[q] = v;
  }
  __syncthreads();
  const int c = threadIdx.x % E::T2, bb = threadIdx.x / E::T2;
  float acc[4] = {b0, b0, b0, b0};
#pragma unroll
  for (int tb = -1; tb <= 1; ++tb)
#pragma unroll
    for (int tc = -TC; tc <= TC; ++tc)
#pragma unroll
      for (int cb = 0; cb < CB; ++cb) {
        float col[6][8];
#pragma unroll
        for (int h = 0; h < 6; ++h) {
          const uint4 u = ds[((h * E::H1 + (bb + 1 + tb)) * E::H2 + (ND == 3 ? c + 1 + tc : 0)) * CB + cb];
          const unsigned w4[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            col[h][2 * e] = bf2f(uint16_t(w4[e] & 0xffffu));
            col[h][2 * e + 1] = bf2f(uint16_t(w4[e] >> 16));
          }
        }
#pragma unroll
        for (int ta = -1; ta <= 1; ++ta) {
          const int t = tap_of<ND>(ta, tb, tc);
          const float4 wa = reinterpret_cast<const float4 *>(ws + t * C0 + cb * 8)[0];
          const float4 wb = reinterpret_cast<const float4 *>(ws + t * C0 + cb * 8)[1];
          const float w[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int e = 0; e < 8; ++e) acc[a] = fmaf(w[e], col[a + 1 + ta][e], acc[a]);
        }
      }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + a, j = j0 + bb, k = k0 + c;
    if (i < g.n[0] && j < g.n[1] && k < g.n[2]) {
      if (FIELD) qf[i * s0 + j * s1 + k * s2] = double(acc[a]);
      else qc[vindex(g, i, j, k)] = acc[a];
    }
  }
}

// q layer backward: dd0[p][ci] = sum_t W[t][ci] dq(p - tap_t) (adjoint), FP32
template <int C0, int ND>
__global__ void k_outl_adj(grid3 g, const float *dq, const float *W, float *dd0) {
  constexpr int NTAPS = ND == 3 ? 27 : 9;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.vox; p += (long long)gridDim.x * blockDim.x) {
    const int k = int(p % g.n[2]), j = int((p / g.n[2]) % g.n[1]), i = int(p / ((long long)g.n[2] * g.n[1]));
    float acc[C0];
#pragma unroll
    for (int c = 0; c < C0; ++c) acc[c] = 0.f;
#pragma unroll
    for (int t = 0; t < NTAPS; ++t) {
      int a, bb, c;
      tap_off<ND>(t, a, bb, c);
      const long long v = nbr(g, i, j, k, -a, -bb, -c);
      if (v < 0) continue;
      const float d = dq[v];
#pragma unroll
      for (int ci = 0; ci < C0; ++ci) acc[ci] = fmaf(W[t * C0 + ci], d, acc[ci]);
    }
#pragma unroll
    for (int c = 0; c < C0; ++c) dd0[p * C0 + c] = acc[c];
  }
}

// dW of an end layer, one tap per blockIdx.y: sum_p dY[p][y] X[p + tap][x] for every pair
// (y, x) (at most 16 pairs); Y is FP32 [p][cy]; X is a compact FP32 scalar (e0) or BF16 [p][cx] (q)
template <int ND>
__global__ void k_endl_dw(grid3 g, const float *dY, int cy, const float *xs, const uint16_t *xb, int cx, float *part) {
  extern __shared__ float red[];
  const int t = blockIdx.y;
  int a, bb, c;
  tap_off<ND>(t, a, bb, c);
  const int npair = cy * cx;
  float acc[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) acc[q] = 0.f;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.vox; p += (long long)gridDim.x * blockDim.x) {
    const int k = int(p % g.n[2]), j = int((p / g.n[2]) % g.n[1]), i = int(p / ((long long)g.n[2] * g.n[1]));
    const long long v = nbr(g, i, j, k, a, bb, c);
    if (v < 0) continue;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      if (q >= npair) break;
      const int yc = q / cx, xc = q % cx;
      const float xv = xs ? xs[v] : bf2f(xb[v * cx + xc]);
      acc[q] = fmaf(dY[p * cy + yc], xv, acc[q]);
    }
  }
  for (int q = 0; q < npair; ++q) {
    red[threadIdx.x] = acc[q];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t(t) * npair + q) * gridDim.x + blockIdx.x] = red[0];
    __syncthreads();
  }
}
// grad[(co * ntaps + t) * cin + ci] from part[(t * npair + pr) * nblk + b], pr = (y, x) = (co, ci)
__global__ void k_endl_reduce(const float *part, int nblk, int ntaps, int cy, int cx, int cout, int cin, bool y_is_out,
                              float *grad) {
  const int tot = ntaps * cy * cx;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) {
    const int pr = q % (cy * cx), t = q / (cy * cx);
    const int yc = pr / cx, xc = pr % cx;
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += part[(size_t(t) * cy * cx + pr) * nblk + b];
    (void)cout; (void)y_is_out;
    grad[(size_t(yc) * ntaps + t) * cin + xc] = s;  // pair (y, x) = (output channel, input channel)
  }
}

// ---------------------------------------------------------------------------
// pooling / up-sampling and their adjoints, conversions

// coarse[P][c] = mean over fine p with floor(p/2) = P; a thread per coarse point and
// group of 8 channels (16-byte loads and stores; C is a multiple of 8)
__global__ void k_pool(grid3 f, grid3 cg, int C, const uint16_t *x, uint16_t *y, const int *skip_flag) {
  if (skip_flag && *skip_flag) return;
  const int CB = C / 8;
  for (long long P = blockIdx.x * (long long)blockDim.x + threadIdx.x; P < cg.vox * CB; P += (long long)gridDim.x * blockDim.x) {
    const int cb = int(P % CB);
    const long long V = P / CB;
    const int K = int(V % cg.n[2]), J = int((V / cg.n[2]) % cg.n[1]), I = int(V / ((long long)cg.n[2] * cg.n[1]));
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int cnt = 0;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 2; ++d) {
          const int i = 2 * I + a, j = 2 * J + b, k = 2 * K + d;
          if (i >= f.n[0] || j >= f.n[1] || k >= f.n[2]) continue;
          if ((f.n[0] == 1 && a) || (f.n[1] == 1 && b) || (f.n[2] == 1 && d)) continue;
          const uint4 u = *reinterpret_cast<const uint4 *>(x + vindex(f, i, j, k) * C + cb * 8);
          const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
          for (int h = 0; h < 4; ++h) {
            s[2 * h] += bf2f(uint16_t(w[h] & 0xffffu));
            s[2 * h + 1] += bf2f(uint16_t(w[h] >> 16));
          }
          ++cnt;
        }
    unsigned o[4];
#pragma unroll
    for (int h = 0; h < 4; ++h)
      o[h] = unsigned(f2bf(s[2 * h] / float(cnt))) | (unsigned(f2bf(s[2 * h + 1] / float(cnt))) << 16);
    *reinterpret_cast<uint4 *>(y + V * C + cb * 8) = make_uint4(o[0], o[1], o[2], o[3]);
  }
}
// fine[p][c] = coarse[floor(p/2)][c]
__global__ void k_up(grid3 f, grid3 cg, int C, const uint16_t *x, uint16_t *y, const int *skip_flag) {
  if (skip_flag && *skip_flag) return;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < f.vox * C; q += (long long)gridDim.x * blockDim.x) {
    const int c = int(q % C);
    const long long v = q / C;
    const int k = int(v % f.n[2]), j = int((v / f.n[2]) % f.n[1]), i = int(v / ((long long)f.n[2] * f.n[1]));
    const int I = min(i / 2, cg.n[0] - 1), J = min(j / 2, cg.n[1] - 1), K = min(k / 2, cg.n[2] - 1);
    y[q] = x[vindex(cg, I, J, K) * C + c];
  }
}
// coarse grad[P][c] = sum of fine grads with floor(p/2) = P (adjoint of up); add: accumulate
__global__ void k_up_adj(grid3 f, grid3 cg, int C, const float *dx, float *dy, bool add) {
  for (long long P = blockIdx.x * (long long)blockDim.x + threadIdx.x; P < cg.vox * C; P += (long long)gridDim.x * blockDim.x) {
    const int c = int(P % C);
    const long long V = P / C;
    const int K = int(V % cg.n[2]), J = int((V / cg.n[2]) % cg.n[1]), I = int(V / ((long long)cg.n[2] * cg.n[1]));
    float s = 0.f;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 2; ++d) {
          const int i = 2 * I + a, j = 2 * J + b, k = 2 * K + d;
          if (i >= f.n[0] || j >= f.n[1] || k >= f.n[2]) continue;
          if ((f.n[0] == 1 && a) || (f.n[1] == 1 && b) || (f.n[2] == 1 && d)) continue;
          s += dx[vindex(f, i, j, k) * C + c];
        }
    dy[P] = add ? dy[P] + s : s;
  }
}
// fine grad[p][c] += coarse grad[floor(p/2)][c] / count (adjoint of pool)
__global__ void k_pool_adj(grid3 f, grid3 cg, int C, const float *dc, float *df) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < f.vox * C; q += (long long)gridDim.x * blockDim.x) {
    const int c = int(q % C);
    const long long v = q / C;
    const int k = int(v % f.n[2]), j = int((v / f.n[2]) % f.n[1]), i = int(v / ((long long)f.n[2] * f.n[1]));
    const int I = min(i / 2, cg.n[0] - 1), J = min(j / 2, cg.n[1] - 1), K = min(k / 2, cg.n[2] - 1);
    const int cnt = (2 * I + 1 < f.n[0] && f.n[0] > 1 ? 2 : 1) * (2 * J + 1 < f.n[1] && f.n[1] > 1 ? 2 : 1) *
                    (2 * K + 1 < f.n[2] && f.n[2] > 1 ? 2 : 1);
    df[q] += dc[vindex(cg, I, J, K) * C + c] / float(cnt);
  }
}
__global__ void k_to_bf16(const float *x, uint16_t *y, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) y[q] = f2bf(x[q]);
}
__global__ void k_copy(const float *x, float *y, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) y[q] = x[q];
}

// loss = sum((q - t)^2) / n, dq = 2 (q - t) / n
__global__ void k_mse(const float *q, const float *t, long long n, float *dq, double *loss) {
  double s = 0.0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const float d = q[p] - t[p];
    dq[p] = 2.f * d / float(n);
    s += double(d) * double(d);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s / double(n));
}

// Adam (Kingma & Ba 2015); `mask` zeroes the update of the biases (the
// preconditioner stays a linear map)
__global__ void k_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2, float eps,
                       float c1, float c2, const unsigned char *mask) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    if (mask && !mask[q]) continue;
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq, vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
  }
}

// fragment layout of a tensor-core layer's weights (W: (cout, ntaps, cin) FP32):
//   frag[(ch * (COUT/8) + nt) * 32 + lane] = {b0, b1}, b0 = W[co][g0 taps][2 (lane % 4) + {0,1}],
//   b1 = the same for group g1, co = nt * 8 + lane / 4; groups g0 = 2 ch, g1 = 2 ch + 1 (zero past the end).
// adj: the adjoint weights Wt[ci][tap'][co] = W[co][ntaps - 1 - tap'][ci] (cin and cout swapped)
__global__ void k_pack(const float *W, int cout, int cin, int ntaps, bool adj, uint2 *frag) {
  const int CO = adj ? cin : cout, CI = adj ? cout : cin;
  const int CB = CI / 8, NG = ntaps * CB, NCH = (NG + 1) / 2, NT = CO / 8;
  const int tot = NCH * NT * 32;
  auto w = [&](int co, int tap, int ci) -> float {
    if (!adj) return W[(size_t(co) * ntaps + tap) * cin + ci];
    return W[(size_t(ci) * ntaps + (ntaps - 1 - tap)) * cin + co];
  };
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) {
    const int lane = q % 32, nt = (q / 32) % NT, ch = q / (32 * NT);
    const int co = nt * 8 + lane / 4, kk = 2 * (lane % 4);
    unsigned half[2];
    for (int s = 0; s < 2; ++s) {
      const int gidx = 2 * ch + s;
      float x0 = 0.f, x1 = 0.f;
      if (gidx < NG) {
        const int tap = gidx / CB, ci = (gidx % CB) * 8 + kk;
        x0 = w(co, tap, ci);
        x1 = w(co, tap, ci + 1);
      }
      half[s] = unsigned(f2bf(x0)) | (unsigned(f2bf(x1)) << 16);
    }
    frag[q] = make_uint2(half[0], half[1]);
  }
}

// ---------------------------------------------------------------------------
// host

namespace {
unsigned gsz(long long n, int bs = 256) {
  long long b = (n + bs - 1) / bs;
  return unsigned(std::max(1LL, std::min<long long>(b, 148LL * 16)));
}
template <class T> void dalloc(T *&p, size_t n) { MPDX_CUDA(cudaMalloc(&p, n * sizeof(T))); }
}  // namespace

net::net(int nd_, const int *grid, const int *wrap_, const int *ch_, uint64_t seed, cudaStream_t s)
    : nd(nd_), stream(s) {
  if (nd != 2 && nd != 3) throw error(MPDX_E_ARG, "the preconditioner network is built for 2D and 3D grids");
  ntaps = nd == 3 ? 27 : 9;
  for (int l = 0; l < kLevels; ++l) {
    ch[l] = ch_[l];
    if (ch[l] != 8 && ch[l] != 16 && ch[l] != 32 && ch[l] != 64)
      throw error(MPDX_E_ARG, "preconditioner channels must be 8, 16, 32 or 64");
  }
  for (int d = 0; d < 3; ++d) wrap[d] = d < nd ? wrap_[d] : 1;
  int g[3] = {grid[0], grid[1], nd == 3 ? grid[2] : 1};
  for (int l = 0; l < kLevels; ++l) {
    for (int d = 0; d < 3; ++d) L[l].n[d] = g[d];
    L[l].vox = (long long)g[0] * g[1] * g[2];
    for (int d = 0; d < 3; ++d) g[d] = g[d] > 1 ? (g[d] + 1) / 2 : 1;
  }
  const int dims[kLayers][3] = {{1, ch[0], 0},     {ch[0], ch[1], 1}, {ch[1], ch[2], 2},
                                {ch[2], ch[3], 3}, {ch[3], ch[3], 3}, {ch[3], ch[2], 2},
                                {ch[2], ch[1], 1}, {ch[1], ch[0], 0}, {ch[0], 1, 0}};
  long long off = 0;
  for (int q = 0; q < kLayers; ++q) {
    cin[q] = dims[q][0]; cout[q] = dims[q][1]; level[q] = dims[q][2];
    w_off[q] = off; off += (long long)cout[q] * ntaps * cin[q];
    b_off[q] = off; off += cout[q];
  }
  n_params = off;
  alloc_all();
  // initialisation: N(0, 1 / fan-in) weights, zero biases, and a zero output
  // layer, so that an untrained network returns 0 and training starts from
  // "no correction" (relative residual 1)
  std::vector<float> h(n_params, 0.f);
  std::mt19937_64 rng(seed);
  for (int q = 0; q < kLayers - 1; ++q) {
    std::normal_distribution<double> nd01(0.0, 1.0 / std::sqrt(double(ntaps * cin[q])));
    for (long long x = 0; x < (long long)cout[q] * ntaps * cin[q]; ++x) h[w_off[q] + x] = float(nd01(rng));
  }
  set_params(h.data());
}

void net::alloc_all() {
  dalloc(params, n_params); dalloc(grad, n_params); dalloc(adam_m, n_params); dalloc(adam_v, n_params);
  MPDX_CUDA(cudaMemsetAsync(adam_m, 0, n_params * sizeof(float), stream));
  MPDX_CUDA(cudaMemsetAsync(adam_v, 0, n_params * sizeof(float), stream));
  for (int q = 1; q < kLayers - 1; ++q) {
    const int NG = ntaps * cin[q] / 8, NCH = (NG + 1) / 2;
    uint16_t *p = nullptr;
    dalloc(p, size_t(NCH) * (cout[q] / 8) * 32 * 4);
    wf[q] = p;
    const int NGt = ntaps * cout[q] / 8, NCHt = (NGt + 1) / 2;
    dalloc(p, size_t(NCHt) * (cin[q] / 8) * 32 * 4);
    wtf[q] = p;
  }
  for (int l = 0; l < 4; ++l) dalloc(a_e[l], size_t(L[l].vox) * ch[l]);
  for (int l = 1; l < 4; ++l) dalloc(a_p[l], size_t(L[l].vox) * ch[l - 1]);
  dalloc(a_m3, size_t(L[3].vox) * ch[3]);
  for (int l = 0; l < 3; ++l) dalloc(a_d[l], size_t(L[l].vox) * ch[l]);
  for (int l = 0; l < 3; ++l) dalloc(a_u[l], size_t(L[l].vox) * ch[l + 1]);
  dalloc(q32, L[0].vox); dalloc(dq32, L[0].vox);
  size_t big = 0;
  for (int l = 0; l < 4; ++l) {
    big = std::max(big, size_t(L[l].vox) * ch[l]);
    if (l < 3) big = std::max(big, size_t(L[l].vox) * ch[l + 1]);
    if (l > 0) big = std::max(big, size_t(L[l].vox) * ch[l - 1]);
  }
  dalloc(g_a, big * 4);  // four level accumulators share one block (offsets below)
  dalloc(g_b, big); dalloc(g_c, big); dalloc(g_h, big);
  part_floats = size_t(1184 + 27) * 64 * 64;
  dalloc(part, part_floats);
  dalloc(loss_dev, 1);
  // Adam updates the weights only: the biases stay zero, so the network is a linear map
  std::vector<unsigned char> mask(n_params, 1);
  for (int q = 0; q < kLayers; ++q)
    for (int c = 0; c < cout[q]; ++c) mask[b_off[q] + c] = 0;
  dalloc(wmask, n_params);
  MPDX_CUDA(cudaMemcpy(wmask, mask.data(), n_params, cudaMemcpyHostToDevice));
}

net::~net() {
  cudaStreamSynchronize(stream);
  for (float *p : {params, grad, adam_m, adam_v, q32, dq32, g_a, g_b, g_c, part}) if (p) cudaFree(p);
  for (int q = 0; q < kLayers; ++q) { if (wf[q]) cudaFree(wf[q]); if (wtf[q]) cudaFree(wtf[q]); }
  for (int l = 0; l < 4; ++l) { if (a_e[l]) cudaFree(a_e[l]); if (a_p[l]) cudaFree(a_p[l]); }
  for (int l = 0; l < 3; ++l) { if (a_d[l]) cudaFree(a_d[l]); if (a_u[l]) cudaFree(a_u[l]); }
  if (a_m3) cudaFree(a_m3);
  if (g_h) cudaFree(g_h);
  if (loss_dev) cudaFree(loss_dev);
  if (wmask) cudaFree(wmask);
}

void net::set_params(const float *host) {
  MPDX_CUDA(cudaMemcpyAsync(params, host, n_params * sizeof(float), cudaMemcpyHostToDevice, stream));
  sync_weights();
  MPDX_CUDA(cudaStreamSynchronize(stream));
}
void net::get_params(float *host) {
  MPDX_CUDA(cudaMemcpyAsync(host, params, n_params * sizeof(float), cudaMemcpyDeviceToHost, stream));
  MPDX_CUDA(cudaStreamSynchronize(stream));
}
void net::sync_weights() {
  for (int q = 1; q < kLayers - 1; ++q) {
    k_pack<<<64, 256, 0, stream>>>(params + w_off[q], cout[q], cin[q], ntaps, false, reinterpret_cast<uint2 *>(wf[q]));
    k_pack<<<64, 256, 0, stream>>>(params + w_off[q], cout[q], cin[q], ntaps, true, reinterpret_cast<uint2 *>(wtf[q]));
  }
  MPDX_LAUNCH_CHECK();
}

namespace {
grid3 g3(const lvl &l, const int *wrap) {
  grid3 g;
  for (int d = 0; d < 3; ++d) { g.n[d] = l.n[d]; g.wrap[d] = wrap[d]; }
  g.vox = l.vox;
  return g;
}

template <int ND, int R>
long long ctile_count(const grid3 &g) {
  using TL = ctile<ND, R>;
  return (long long)((g.n[0] + TL::T0 - 1) / TL::T0) * ((g.n[1] + TL::T1 - 1) / TL::T1) * ((g.n[2] + TL::T2 - 1) / TL::T2);
}
template <int CIN, int COUT, int ND, int UP, int R>
void conv_tc_launch_r(const grid3 &g, const grid3 &cg, const uint16_t *X, const uint16_t *Wf, conv_out o, const int *skip,
                      cudaStream_t s) {
  using TL = ctile<ND, R>;
  constexpr bool CO = UP == 2;
  constexpr int H0 = CO ? TL::T0 / 2 + 2 : TL::T0 + 2, H1 = CO ? TL::T1 / 2 + 2 : TL::T1 + 2;
  constexpr int H2 = ND == 3 ? (CO ? TL::T2 / 2 + 2 : TL::T2 + 2) : 1;
  const size_t smem = size_t(H0) * H1 * H2 * sv<CIN>::v;
  auto kern = k_conv_tc<CIN, COUT, ND, UP, R>;
  static bool attr = false;
  if (!attr) { MPDX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))); attr = true; }
  kern<<<unsigned(ctile_count<ND, R>(g)), 256, smem, s>>>(g, cg, X, reinterpret_cast<const uint2 *>(Wf), o, skip);
  MPDX_LAUNCH_CHECK();
}
// four rows per warp where the grid still gives every SM four or more tiles (and
// the tile fits shared memory comfortably), one row per warp otherwise
template <int CIN, int COUT, int ND, int UP>
void conv_tc_launch3(const grid3 &g, const grid3 &cg, const uint16_t *X, const uint16_t *Wf, conv_out o, const int *skip,
                     cudaStream_t s) {
  if constexpr (ND == 3 && CIN <= 32) {
    if (ctile_count<3, 4>(g) >= 4 * 148) return conv_tc_launch_r<CIN, COUT, ND, UP, 4>(g, cg, X, Wf, o, skip, s);
  }
  conv_tc_launch_r<CIN, COUT, ND, UP, 1>(g, cg, X, Wf, o, skip, s);
}
// the coarse staging of the up-sampled input where every axis of the fine grid
// has an even number of points (or one point)
template <int CIN, int COUT, int ND, bool UP>
void conv_tc_launch2(const grid3 &g, const grid3 &cg, const uint16_t *X, const uint16_t *Wf, conv_out o, const int *skip,
                     cudaStream_t s) {
  if constexpr (!UP) {
    conv_tc_launch3<CIN, COUT, ND, 0>(g, cg, X, Wf, o, skip, s);
  } else {
    bool even = true;
    for (int d = 0; d < ND; ++d) even = even && (g.n[d] % 2 == 0) && cg.n[d] * 2 == g.n[d];
    if (even) conv_tc_launch3<CIN, COUT, ND, 2>(g, cg, X, Wf, o, skip, s);
    else conv_tc_launch3<CIN, COUT, ND, 1>(g, cg, X, Wf, o, skip, s);
  }
}
template <int CIN, int COUT, int ND>
void conv_tc_launch(const grid3 &g, const uint16_t *X, const uint16_t *Wf, conv_out o, const int *skip, cudaStream_t s) {
  conv_tc_launch2<CIN, COUT, ND, false>(g, g, X, Wf, o, skip, s);
}
template <int CIN, int COUT, int ND>
void conv_tc_up_launch(const grid3 &g, const grid3 &cg, const uint16_t *X, const uint16_t *Wf, conv_out o, const int *skip,
                       cudaStream_t s) {
  conv_tc_launch2<CIN, COUT, ND, true>(g, cg, X, Wf, o, skip, s);
}
template <int CIN, int COUT, int ND>
int conv_dw_launch(const grid3 &g, const uint16_t *dY, const uint16_t *X, float *part, size_t part_floats, cudaStream_t s) {
  using TL = tile<ND>;
  constexpr int TP = TL::T0 * TL::T1 * TL::T2, COUTP = COUT < 16 ? 16 : COUT;
  const size_t smem = size_t(TP) * (COUTP * 2 + 16) + size_t(TP) * sv<CIN>::v;
  auto kern = k_conv_dw<CIN, COUT, ND>;
  static bool attr = false;
  if (!attr) { MPDX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))); attr = true; }
  const int ntaps = ND == 3 ? 27 : 9;
  const long long ntiles = (long long)((g.n[0] + TL::T0 - 1) / TL::T0) * ((g.n[1] + TL::T1 - 1) / TL::T1) * ((g.n[2] + TL::T2 - 1) / TL::T2);
  long long gx = std::min<long long>(ntiles, 1184 / ntaps + 1);
  while (size_t(gx) * ntaps * COUT * CIN > part_floats && gx > 1) --gx;
  kern<<<dim3(unsigned(gx), ntaps), 256, smem, s>>>(g, dY, X, part);
  MPDX_LAUNCH_CHECK();
  return int(gx);
}

// dispatch over the channel pairs the U-net uses
template <int ND>
void conv_tc(int cin, int cout, const grid3 &g, const uint16_t *X, const uint16_t *Wf, conv_out o, const int *skip, cudaStream_t s) {
#define MPDX_PC_TC(A, B) if (cin == A && cout == B) return conv_tc_launch<A, B, ND>(g, X, Wf, o, skip, s);
  MPDX_PC_TC(8, 8) MPDX_PC_TC(8, 16) MPDX_PC_TC(16, 8) MPDX_PC_TC(16, 16) MPDX_PC_TC(16, 32) MPDX_PC_TC(32, 16)
  MPDX_PC_TC(32, 32) MPDX_PC_TC(32, 64) MPDX_PC_TC(64, 32) MPDX_PC_TC(64, 64) MPDX_PC_TC(8, 32) MPDX_PC_TC(32, 8)
  MPDX_PC_TC(16, 64) MPDX_PC_TC(64, 16) MPDX_PC_TC(8, 64) MPDX_PC_TC(64, 8)
#undef MPDX_PC_TC
  throw error(MPDX_E_ARG, "unsupported channel pair");
}
// the decoder's convolutions of the nearest up-sampling of a coarse tensor (C_in > C_out)
template <int ND>
void conv_tc_up(int cin, int cout, const grid3 &g, const grid3 &cg, const uint16_t *X, const uint16_t *Wf, conv_out o,
                const int *skip, cudaStream_t s) {
#define MPDX_PC_TCU(A, B) if (cin == A && cout == B) return conv_tc_up_launch<A, B, ND>(g, cg, X, Wf, o, skip, s);
  MPDX_PC_TCU(16, 8) MPDX_PC_TCU(32, 16) MPDX_PC_TCU(64, 32) MPDX_PC_TCU(64, 64) MPDX_PC_TCU(32, 32) MPDX_PC_TCU(16, 16)
  MPDX_PC_TCU(32, 8) MPDX_PC_TCU(64, 16) MPDX_PC_TCU(64, 8) MPDX_PC_TCU(8, 8)
#undef MPDX_PC_TCU
  throw error(MPDX_E_ARG, "unsupported channel pair");
}
template <int ND>
int conv_dw(int cin, int cout, const grid3 &g, const uint16_t *dY, const uint16_t *X, float *part, size_t pf, cudaStream_t s) {
#define MPDX_PC_DW(A, B) if (cin == A && cout == B) return conv_dw_launch<A, B, ND>(g, dY, X, part, pf, s);
  MPDX_PC_DW(8, 8) MPDX_PC_DW(8, 16) MPDX_PC_DW(16, 8) MPDX_PC_DW(16, 16) MPDX_PC_DW(16, 32) MPDX_PC_DW(32, 16)
  MPDX_PC_DW(32, 32) MPDX_PC_DW(32, 64) MPDX_PC_DW(64, 32) MPDX_PC_DW(64, 64) MPDX_PC_DW(8, 32) MPDX_PC_DW(32, 8)
  MPDX_PC_DW(16, 64) MPDX_PC_DW(64, 16) MPDX_PC_DW(8, 64) MPDX_PC_DW(64, 8)
#undef MPDX_PC_DW
  throw error(MPDX_E_ARG, "unsupported channel pair");
}
}  // namespace

// forward pass with the residual source selected by the caller
template <int ND>
static void forward_impl(net &N, const double *rf, long long s0, long long s1, long long s2, const float *rc, double *qf,
                         float *qc, const int *skip, uint16_t **a_e, uint16_t **a_p, uint16_t *a_m3, uint16_t **a_d,
                         uint16_t **a_u, uint16_t **wf) {
  cudaStream_t s = N.stream;
  grid3 G[4];
  for (int l = 0; l < 4; ++l) G[l] = g3(N.L[l], N.wrap);
  const float *P = N.params;
  const int c0 = N.ch[0];
  // e0, and the level-1 input pool(e0) in the same pass
  const float *W0 = P + N.w_off[0], *B0 = P + N.b_off[0];
  const unsigned EB = unsigned(etile_count<ND>(G[0]));
  if (c0 == 8) {
    if (rf) k_conv_in<8, ND, true, true><<<EB, kEndThreads, 0, s>>>(G[0], G[1], rf, s0, s1, s2, nullptr, W0, B0, a_e[0], a_p[1], skip);
    else k_conv_in<8, ND, false, true><<<EB, kEndThreads, 0, s>>>(G[0], G[1], nullptr, 0, 0, 0, rc, W0, B0, a_e[0], a_p[1], skip);
  } else if (c0 == 16) {
    if (rf) k_conv_in<16, ND, true, true><<<EB, kEndThreads, 0, s>>>(G[0], G[1], rf, s0, s1, s2, nullptr, W0, B0, a_e[0], a_p[1], skip);
    else k_conv_in<16, ND, false, true><<<EB, kEndThreads, 0, s>>>(G[0], G[1], nullptr, 0, 0, 0, rc, W0, B0, a_e[0], a_p[1], skip);
  } else throw error(MPDX_E_ARG, "level-0 channels must be 8 or 16");
  MPDX_LAUNCH_CHECK();
  // encoder
  for (int l = 1; l < 4; ++l) {
    if (l > 1) k_pool<<<gsz(G[l].vox * N.ch[l - 1] / 8), 256, 0, s>>>(G[l - 1], G[l], N.ch[l - 1], a_e[l - 1], a_p[l], skip);
    conv_tc<ND>(N.cin[l], N.cout[l], G[l], a_p[l], wf[l], conv_out{a_e[l], nullptr, P + N.b_off[l], nullptr}, skip, s);
  }
  conv_tc<ND>(N.cin[4], N.cout[4], G[3], a_e[3], wf[4], conv_out{a_m3, nullptr, P + N.b_off[4], nullptr}, skip, s);
  // decoder: layer 5 -> level 2, 6 -> 1, 7 -> 0
  const uint16_t *coarse = a_m3;
  for (int q = 5; q <= 7; ++q) {
    const int l = N.level[q];
    // up-sampling read by the convolution's tile load (not written out)
    conv_tc_up<ND>(N.cin[q], N.cout[q], G[l], G[l + 1], coarse, wf[q], conv_out{a_d[l], nullptr, P + N.b_off[q], a_e[l]}, skip, s);
    coarse = a_d[l];
  }
  MPDX_LAUNCH_CHECK();
  const float *W8 = P + N.w_off[8], *B8 = P + N.b_off[8];
  if (c0 == 8) {
    if (qf) k_conv_outl<8, ND, true><<<EB, kEndThreads, 0, s>>>(G[0], a_d[0], W8, B8, qf, s0, s1, s2, nullptr, skip);
    else k_conv_outl<8, ND, false><<<EB, kEndThreads, 0, s>>>(G[0], a_d[0], W8, B8, nullptr, 0, 0, 0, qc, skip);
  } else {
    if (qf) k_conv_outl<16, ND, true><<<EB, kEndThreads, 0, s>>>(G[0], a_d[0], W8, B8, qf, s0, s1, s2, nullptr, skip);
    else k_conv_outl<16, ND, false><<<EB, kEndThreads, 0, s>>>(G[0], a_d[0], W8, B8, nullptr, 0, 0, 0, qc, skip);
  }
  MPDX_LAUNCH_CHECK();
}

void net::forward_field(const double *r, long long s0, long long s1, long long s2, const double *, double *q,
                        const int *skip_flag) {
  if (nd == 3) forward_impl<3>(*this, r, s0, s1, s2, nullptr, q, nullptr, skip_flag, a_e, a_p, a_m3, a_d, a_u, wf);
  else forward_impl<2>(*this, r, s0, s1, s2, nullptr, q, nullptr, skip_flag, a_e, a_p, a_m3, a_d, a_u, wf);
}
void net::forward_compact(const float *r, float *q) {
  if (nd == 3) forward_impl<3>(*this, nullptr, 0, 0, 0, r, nullptr, q, nullptr, a_e, a_p, a_m3, a_d, a_u, wf);
  else forward_impl<2>(*this, nullptr, 0, 0, 0, r, nullptr, q, nullptr, a_e, a_p, a_m3, a_d, a_u, wf);
}

template <int ND>
static void backward_impl(net &N, const float *r, const float *dq, float *gr, uint16_t **a_e, uint16_t **a_p,
                          uint16_t *a_m3, uint16_t **a_d, uint16_t **a_u, uint16_t **wtf, float *g_acc_base, float *g_b,
                          float *g_c, uint16_t *g_h, float *part, size_t pf) {
  cudaStream_t s = N.stream;
  grid3 G[4];
  for (int l = 0; l < 4; ++l) G[l] = g3(N.L[l], N.wrap);
  const int nt = N.ntaps, c0 = N.ch[0];
  // level accumulators dE_l (FP32, L_l x ch[l]) inside g_acc_base
  float *dE[4];
  {
    size_t off = 0;
    for (int l = 0; l < 4; ++l) { dE[l] = g_acc_base + off; off += size_t(N.L[l].vox) * N.ch[l]; }
  }
  const unsigned RB = 296;
  auto bias_grad = [&](const float *dY, long long vox, int C, float *gb) {
    k_db<<<RB, 256, 256 * sizeof(float), s>>>(dY, vox, C, part);
    k_db_reduce<<<1, 64, 0, s>>>(part, RB, C, gb);
  };
  // ---- q layer (C0 -> 1) ----
  if (c0 == 8) k_outl_adj<8, ND><<<gsz(G[0].vox), 256, 0, s>>>(G[0], dq, N.params + N.w_off[8], dE[0]);
  else k_outl_adj<16, ND><<<gsz(G[0].vox), 256, 0, s>>>(G[0], dq, N.params + N.w_off[8], dE[0]);
  k_endl_dw<ND><<<dim3(RB, nt), 256, 256 * sizeof(float), s>>>(G[0], dq, 1, nullptr, a_d[0], c0, part);
  k_endl_reduce<<<8, 256, 0, s>>>(part, RB, nt, 1, c0, 1, c0, true, gr + N.w_off[8]);
  bias_grad(dq, G[0].vox, 1, gr + N.b_off[8]);
  MPDX_LAUNCH_CHECK();
  // ---- decoder: layers 7 (level 0), 6 (1), 5 (2); dE[l] holds d(d_l) on entry ----
  for (int q = 7; q >= 5; --q) {
    const int l = N.level[q], ci = N.cin[q], co = N.cout[q];
    // the forward pass reads the up-sampled input inside its convolution; the weight
    // gradient needs it written out
    k_up<<<gsz(G[l].vox * ci), 256, 0, s>>>(G[l], G[l + 1], ci, l == 2 ? a_m3 : a_d[l + 1], a_u[l], nullptr);
    k_to_bf16<<<gsz(G[l].vox * co), 256, 0, s>>>(dE[l], g_h, G[l].vox * co);
    const int gx = conv_dw<ND>(ci, co, G[l], g_h, a_u[l], part, pf, s);
    k_dw_reduce<<<64, 256, 0, s>>>(part, gx, nt, co, ci, gr + N.w_off[q]);
    bias_grad(dE[l], G[l].vox, co, gr + N.b_off[q]);
    // d(u_l) = conv^T(d(d_l)), then up adjoint into level l+1
    conv_tc<ND>(co, ci, G[l], g_h, wtf[q], conv_out{nullptr, g_b, nullptr, nullptr}, nullptr, s);
    k_up_adj<<<gsz(G[l + 1].vox * ci), 256, 0, s>>>(G[l], G[l + 1], ci, g_b, dE[l + 1], false);
    MPDX_LAUNCH_CHECK();
  }
  // dE[3] now holds d(m3); the skip connections add d(d_l) to d(e_l): keep copies
  // (dE[0..2] were consumed by k_to_bf16 but still hold d(d_l) = the skip part of d(e_l))
  // ---- m3 (level 3, input e3) ----
  {
    const int ci = N.cin[4], co = N.cout[4];
    k_to_bf16<<<gsz(G[3].vox * co), 256, 0, s>>>(dE[3], g_h, G[3].vox * co);
    const int gx = conv_dw<ND>(ci, co, G[3], g_h, a_e[3], part, pf, s);
    k_dw_reduce<<<64, 256, 0, s>>>(part, gx, nt, co, ci, gr + N.w_off[4]);
    bias_grad(dE[3], G[3].vox, co, gr + N.b_off[4]);
    conv_tc<ND>(co, ci, G[3], g_h, wtf[4], conv_out{nullptr, g_c, nullptr, nullptr}, nullptr, s);  // d(e3)
    k_copy<<<gsz(G[3].vox * ci), 256, 0, s>>>(g_c, dE[3], G[3].vox * ci);
  }
  // ---- encoder: layers 3, 2, 1 (input p_l = pool(e_{l-1})); dE[l] holds d(e_l) ----
  for (int q = 3; q >= 1; --q) {
    const int l = q, ci = N.cin[q], co = N.cout[q];
    k_to_bf16<<<gsz(G[l].vox * co), 256, 0, s>>>(dE[l], g_h, G[l].vox * co);
    const int gx = conv_dw<ND>(ci, co, G[l], g_h, a_p[l], part, pf, s);
    k_dw_reduce<<<64, 256, 0, s>>>(part, gx, nt, co, ci, gr + N.w_off[q]);
    bias_grad(dE[l], G[l].vox, co, gr + N.b_off[q]);
    conv_tc<ND>(co, ci, G[l], g_h, wtf[q], conv_out{nullptr, g_b, nullptr, nullptr}, nullptr, s);  // d(p_l)
    k_pool_adj<<<gsz(G[l - 1].vox * ci), 256, 0, s>>>(G[l - 1], G[l], ci, g_b, dE[l - 1]);
    MPDX_LAUNCH_CHECK();
  }
  // ---- e0 (1 -> C0, input r) ----
  k_endl_dw<ND><<<dim3(RB, nt), 256, 256 * sizeof(float), s>>>(G[0], dE[0], c0, r, nullptr, 1, part);
  k_endl_reduce<<<8, 256, 0, s>>>(part, RB, nt, c0, 1, c0, 1, true, gr + N.w_off[0]);
  bias_grad(dE[0], G[0].vox, c0, gr + N.b_off[0]);
  MPDX_LAUNCH_CHECK();
}

void net::backward(const float *r, const float *dq, float *gr) {
  if (nd == 3) backward_impl<3>(*this, r, dq, gr, a_e, a_p, a_m3, a_d, a_u, wtf, g_a, g_b, g_c, g_h, part, part_floats);
  else backward_impl<2>(*this, r, dq, gr, a_e, a_p, a_m3, a_d, a_u, wtf, g_a, g_b, g_c, g_h, part, part_floats);
}

double net::train_step(const float *r, const float *target, float lr) {
  cudaStream_t s = stream;
  forward_compact(r, q32);
  MPDX_CUDA(cudaMemsetAsync(loss_dev, 0, sizeof(double), s));
  k_mse<<<gsz(L[0].vox), 256, 0, s>>>(q32, target, L[0].vox, dq32, loss_dev);
  backward(r, dq32, grad);
  adam_step(lr);
  double loss = 0;
  MPDX_CUDA(cudaMemcpyAsync(&loss, loss_dev, sizeof(double), cudaMemcpyDeviceToHost, s));
  MPDX_CUDA(cudaStreamSynchronize(s));
  return loss;
}

void net::adam_step(float lr) {
  cudaStream_t s = stream;
  ++adam_t;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, float(adam_t)), c2 = 1.f - std::pow(b2, float(adam_t));
  k_adam<<<gsz(n_params), 256, 0, s>>>(params, grad, adam_m, adam_v, n_params, lr, b1, b2, 1e-8f, c1, c2, wmask);
  MPDX_LAUNCH_CHECK();
  sync_weights();
}

}  // namespace pc
}  // namespace mpdx
