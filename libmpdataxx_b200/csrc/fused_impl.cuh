// Launchers of the fused MPDATA kernels and the periodic-seam check.
// Included once per real type (fused_f32.cu, fused_f64.cu) so that each type
// gets its own compiler flags.
#pragma once

#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>
#include <type_traits>

#include "fused.cuh"
#include "fused3d.cuh"
#include "fused3d_f32.cuh"
#include "fused2d_batch.cuh"

namespace mpdx {

#ifndef MPDX_LX3
#define MPDX_LX3 64  // planes per CTA of the 3D kernel (4 warm-up planes per chunk)
#endif
template <class T> struct tiles;
template <> struct tiles<float> {
  static constexpr int CR = 32, LX3 = MPDX_LX3;   // 3D canvas rows (x 64 columns), planes per CTA
};
template <> struct tiles<double> {
  static constexpr int CR = 16, LX3 = 64;
};

template <class T>
bool fused_configurable(const mpdata_state<T> &st) {
  for (int d = 0; d < st.nd; ++d)
    if (st.bcs[d][0] != MPDX_BC_CYCLIC || st.bcs[d][1] != MPDX_BC_CYCLIC) return false;
  if (st.opts & ~(o_fct | o_iga)) return false;
  if (st.upwind_filter_freq > 0) return false;
  if (st.nd == 3) return st.n_iters == 2 && st.n[0] - 1 >= 2 && st.n[1] - 1 >= 2 && st.n[2] - 1 >= 2;
  if (st.nd == 2) {
    const bool ok_iters = st.n_iters == 2 || (st.n_iters == 3 && !(st.opts & o_iga));
    return ok_iters && st.n[0] - 1 >= 2 && st.n[1] - 1 >= 2;
  }
  return false;
}

template <class K>
static void set_smem(K kernel, size_t bytes) {
  MPDX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
}

template <class T, bool IGA, bool FCT>
static void launch3(const f3::args<T> &a, cudaStream_t s, dim3 grid) {
  constexpr int CR = tiles<T>::CR;
  using C = f3::canvas<CR>;
  auto kern = f3::k_fused3d<T, IGA, FCT, CR>;
  const size_t bytes = size_t(C::total) * C::N * sizeof(T);
  static bool attr = false;
  if (!attr) { set_smem(kern, bytes); attr = true; }
  kern<<<grid, C::NT, bytes, s>>>(a);
  MPDX_LAUNCH_CHECK();
}

// the driver's tensor-map encoder, found through the runtime's entry-point query
// (so that the library links no driver library); null where the query fails
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      (void)cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// the tiled map of one FP32 field over (k, j, x) with extents (P2, P1, P0) and a
// box of one canvas plane (64 columns x `rows` rows); false where the field's
// layout does not meet the copy's rules (16-byte aligned origin and strides)
inline bool plane_map(CUtensorMap &m, const dfield<float> &f, const f3::args<float> &a, int rows) {
  const auto enc = tensor_map_encoder();
  if (!enc || f.s2 != 1 || (reinterpret_cast<std::uintptr_t>(f.o) & 15u) || f.s1 <= 0 || f.s0 <= 0 || (f.s1 % 4) ||
      (f.s0 % 4))
    return false;
  const cuuint64_t dims[3] = {cuuint64_t(a.P2), cuuint64_t(a.P1), cuuint64_t(a.P0)};
  const cuuint64_t strides[2] = {cuuint64_t(f.s1) * 4u, cuuint64_t(f.s0) * 4u};
  const cuuint32_t box[3] = {64u, cuuint32_t(rows), 1u}, elem[3] = {1u, 1u, 1u};
  return enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(f.o), dims, strides, box, elem,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the host-mapped word that a bulk-copy wait which gives up sets (allocated at the
// first launch that uses bulk copies; null where that allocation fails)
inline unsigned *copy_wait_flag_device() {
  auto &f = fused_copy_wait_flag();
  static std::once_flag once;
  std::call_once(once, [&] {
    unsigned *h = nullptr, *d = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void **>(&h), sizeof(unsigned), cudaHostAllocMapped) != cudaSuccess) {
      (void)cudaGetLastError();
      return;
    }
    *h = 0u;
    if (cudaHostGetDevicePointer(reinterpret_cast<void **>(&d), h, 0) != cudaSuccess) {
      (void)cudaGetLastError();
      cudaFreeHost(h);
      return;
    }
    f.dev = d;
    f.host = h;
  });
  return f.dev;
}

// the FP32 kernel with the regrouped single-precision arithmetic (iga variants)
template <bool FCT>
static void launch3s(const f3::args<float> &a, cudaStream_t s, dim3 grid) {
  constexpr int CR = tiles<float>::CR;
  using C = f3s::canvas_s<CR>;
  auto kern = f3s::k_fused3d_s<FCT, CR>;
  // the planes, then two mbarriers and the warp counter
  const size_t bytes = size_t(C::total) * C::N * sizeof(float) + 32;
  static bool attr = false;
  if (!attr) { set_smem(kern, bytes); attr = true; }
  f3s::tma_planes m{};
  // bulk copies only where some tile lies inside the periods along j and k
  if (fused3d_bulk_copies(-1) == 1 && a.P2 >= 64 && a.P1 >= CR) {
    m.timeout = copy_wait_flag_device();
    m.on = m.timeout && plane_map(m.in, a.in, a, CR) && plane_map(m.g0, a.g0, a, CR) && plane_map(m.g1, a.g1, a, CR) &&
           plane_map(m.g2, a.g2, a, CR);
  }
  kern<<<grid, C::NT, bytes, s>>>(a, m);
  MPDX_LAUNCH_CHECK();
}

template <class T>
void fused3d_launch(mpdata_state<T> &st, int e, cudaStream_t s, int lx) {
  using C = f3::canvas<tiles<T>::CR>;
  const int LX = lx > 0 ? lx : tiles<T>::LX3;
  f3::args<T> a;
  a.in = st.psi[e][st.tl[e]].v;
  a.out = st.psi[e][st.tl[e] ^ 1].v;
  a.g0 = st.GC[0].v; a.g1 = st.GC[1].v; a.g2 = st.GC[2].v;
  a.P0 = st.n[0] - 1; a.P1 = st.n[1] - 1; a.P2 = st.n[2] - 1;
  a.n0 = st.n[0]; a.n1 = st.n[1]; a.n2 = st.n[2];
  a.LX = LX;
  a.tiles_z = (a.P2 + C::TZ - 1) / C::TZ;
  const int tiles_y = (a.P1 + C::TY - 1) / C::TY;
  dim3 grid(tiles_y * a.tiles_z, (a.P0 + LX - 1) / LX);
  const bool iga = st.opts & o_iga, fct = st.opts & o_fct;
  if constexpr (std::is_same<T, float>::value) {
    if (iga) {
      if (fct) launch3s<true>(a, s, grid);
      else launch3s<false>(a, s, grid);
      return;
    }
  }
  if (iga && fct) launch3<T, true, true>(a, s, grid);
  else if (iga) launch3<T, true, false>(a, s, grid);
  else if (fct) launch3<T, false, true>(a, s, grid);
  else launch3<T, false, false>(a, s, grid);
}

// 2D: one warp per item of one strip (128 columns) x LX rows; the rows per item
// are chosen so that small problems still spread over the GPU (the warm-up rows
// of every chunk are recomputed, so chunks stay at 16 rows or more)
template <class T>
void fused2d_plan_init(const mpdata_state<T> &st, fused2d_plan<T> &p) {
  int dev = 0, n_sm = 0;
  MPDX_CUDA(cudaGetDevice(&dev));
  MPDX_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  const int P0 = st.n[0] - 1, P1 = st.n[1] - 1;
  const int WV = st.n_iters == 3 ? f2w::shape<3>::WV : f2w::shape<2>::WV;
  const int n_strips = (P1 + WV - 1) / WV;
  int LX = 64;
  while (LX > 16 && (long long)n_strips * ((P0 + LX - 1) / LX) < 8LL * n_sm) LX /= 2;
  std::vector<f2::item> items;
  for (int x0 = 0; x0 < P0; x0 += LX)
    for (int j0 = 0; j0 < P1; j0 += WV) items.push_back({0, j0, x0, std::min(x0 + LX, P0)});
  std::vector<f2::prob<T>> pr(2 * st.n_eqns);
  for (int e = 0; e < st.n_eqns; ++e)
    for (int tl = 0; tl < 2; ++tl) pr[2 * e + tl] = fused2d_prob(st, e, tl);
  MPDX_CUDA(cudaMalloc(&p.probs, pr.size() * sizeof(f2::prob<T>)));
  MPDX_CUDA(cudaMalloc(&p.items, items.size() * sizeof(f2::item)));
  MPDX_CUDA(cudaMalloc(&p.counter, 2 * sizeof(int)));
  MPDX_CUDA(cudaMemcpy(p.probs, pr.data(), pr.size() * sizeof(f2::prob<T>), cudaMemcpyHostToDevice));
  MPDX_CUDA(cudaMemcpy(p.items, items.data(), items.size() * sizeof(f2::item), cudaMemcpyHostToDevice));
  MPDX_CUDA(cudaMemset(p.counter, 0, 2 * sizeof(int)));
  MPDX_CUDA(cudaDeviceSynchronize());
  p.n_items = int(items.size());
  p.grid = (p.n_items + 3) / 4;  // one warp per item, blocks of 4 warps
}

// ---------------------------------------------------------------------------
// the 2D kernel for given options: launch it (or, with occupancy_only, return
// its resident CTAs per SM)
template <class T, int NI, bool IGA, bool FCT>
static int launch2(const f2::prob<T> *probs, const f2::item *items, int n_items, int *counter, int grid,
                   cudaStream_t s, bool occupancy_only) {
  auto kern = f2w::k_fused2d_w<T, NI, IGA, FCT>;
  if (occupancy_only) {
    int occ = 0;
    MPDX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 128, 0));
    return occ;
  }
  kern<<<grid, 128, 0, s>>>(probs, items, n_items, counter);
  MPDX_LAUNCH_CHECK();
  return 0;
}

template <class T>
static int launch2_opts(int ni, bool iga, bool fct, const f2::prob<T> *probs, const f2::item *items, int n_items,
                        int *counter, int grid, cudaStream_t s, bool occ) {
  if (ni == 3) {
    if (fct) return launch2<T, 3, false, true>(probs, items, n_items, counter, grid, s, occ);
    return launch2<T, 3, false, false>(probs, items, n_items, counter, grid, s, occ);
  }
  if (iga && fct) return launch2<T, 2, true, true>(probs, items, n_items, counter, grid, s, occ);
  if (iga) return launch2<T, 2, true, false>(probs, items, n_items, counter, grid, s, occ);
  if (fct) return launch2<T, 2, false, true>(probs, items, n_items, counter, grid, s, occ);
  return launch2<T, 2, false, false>(probs, items, n_items, counter, grid, s, occ);
}

template <class T>
void fused2d_launch(const mpdata_state<T> &st, const fused2d_plan<T> &p, int e, cudaStream_t s) {
  launch2_opts<T>(st.n_iters, st.opts & o_iga, st.opts & o_fct, p.probs + 2 * e + st.tl[e], p.items, p.n_items,
                  p.counter, p.grid, s, false);
}

// batched persistent launch (fused2d_batch.cuh): the same kernel over the work
// list of many problems
template <class T>
int fused2d_batched(int tile, int ni, bool iga, bool fct, const f2::prob<T> *probs, const f2::item *items, int n_items,
                    int *counter, int grid, cudaStream_t s, bool occ) {
  (void)tile;  // the rows per item are in the work list
  return launch2_opts<T>(ni, iga, fct, probs, items, n_items, counter, grid, s, occ);
}

// ---------------------------------------------------------------------------
// seam check: the duplicate point n-1 must equal point 0 along every periodic
// axis, for the advectees and for the transverse axes of the advector faces.
template <class T>
__device__ __forceinline__ bool same_bits(T a, T b) {
  if (sizeof(T) == 8) return __double_as_longlong(double(a)) == __double_as_longlong(double(b));
  return __float_as_int(float(a)) == __float_as_int(float(b));
}

// compare f(.., n_ax-1, ..) with f(.., 0, ..) over the box e0 x e1 x e2 (axis ax collapsed)
template <class T>
__global__ void k_seam(dfield<T> f, int ax, int last, int e0, int e1, int e2, unsigned *flag) {
  const long long tot = (long long)e0 * e1 * e2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    int c = int(q % e2);
    const long long r = q / e2;
    int b = int(r % e1), a = int(r / e1);
    int i0 = a, j0 = b, k0 = c, i1 = a, j1 = b, k1 = c;
    if (ax == 0) { i0 = 0; i1 = last; }
    if (ax == 1) { j0 = 0; j1 = last; }
    if (ax == 2) { k0 = 0; k1 = last; }
    if (!same_bits(f(i0, j0, k0), f(i1, j1, k1))) atomicOr(flag, 1u);
  }
}

template <class T>
bool fused_seams_consistent(mpdata_state<T> &st, double *scratch) {
  unsigned *flag = reinterpret_cast<unsigned *>(scratch);
  MPDX_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned), st.stream));
  auto check = [&](const field<T> &f, int ax, int face_ax) {
    int e[3];
    for (int d = 0; d < 3; ++d) e[d] = d < st.nd ? st.n[d] : 1;
    if (face_ax >= 0) e[face_ax] = st.n[face_ax] - 1;  // unique faces 0..n-2
    e[ax] = 1;
    const long long tot = (long long)e[0] * e[1] * e[2];
    unsigned g = ceil_div(tot, 256);
    if (g > 4096) g = 4096;
    k_seam<T><<<g, 256, 0, st.stream>>>(f.v, ax, st.n[ax] - 1, e[0], e[1], e[2], flag);
    MPDX_LAUNCH_CHECK();
  };
  for (int q = 0; q < st.n_eqns; ++q)
    for (int ax = 0; ax < st.nd; ++ax) check(st.psi[q][st.tl[q]], ax, -1);
  for (int d = 0; d < st.nd; ++d)
    for (int ax = 0; ax < st.nd; ++ax)
      if (ax != d) check(st.GC[d], ax, d);
  unsigned h = 0;
  MPDX_CUDA(cudaMemcpyAsync(&h, flag, sizeof(h), cudaMemcpyDeviceToHost, st.stream));
  MPDX_CUDA(cudaStreamSynchronize(st.stream));
  return h == 0;
}

}  // namespace mpdx
