// Solver handles and the C ABI (include/mpdx.h).
//
// A handle owns the device fields of one solver (libmpdata++'s sharedmem),
// a CUDA stream, and small scratch buffers.  Host data enters and leaves only
// through mpdx_set_field / mpdx_get_field / mpdx_stats.
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "boussinesq.cuh"
#include "fused.cuh"
#include "fused2d_batch.cuh"
#include "general.cuh"
#include "stats.cuh"

namespace mpdx {

// ---------------------------------------------------------------------------
// host <-> field transfers: contiguous staging buffer on the device, then a
// gather/scatter kernel between C-ordered views and the padded halo'ed field.
template <class T>
__global__ void k_view_copy(dfield<T> f, T *buf, int e0, int e1, int e2, int o0, int o1, int o2, bool to_field) {
  const long long tot = (long long)e0 * e1 * e2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int c = int(q % e2);
    const long long r = q / e2;
    const int b = int(r % e1), a = int(r / e1);
    T &x = f(a + o0, b + o1, c + o2);
    if (to_field) x = buf[q];
    else buf[q] = x;
  }
}

// device address and element strides of a field view (element (0, 0, 0) of the view)
struct view_desc {
  int nd, ex[3];
  void *base;
  long long st[3];
};

// Asynchronous pinned-memory transfers (mpdx_set_field_async / mpdx_get_field_async):
// uploads run on their own stream, downloads on another, each after the compute
// enqueued so far and after the last transfer of the same field; compute and the
// synchronous entry points wait for every transfer issued before them (join).
struct async_xfer {
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_compute = nullptr, ev_h2d = nullptr, ev_d2h = nullptr;
  std::map<std::pair<int, int>, cudaEvent_t> last;
  bool pending = false;
  ~async_xfer() {
    if (h2d) cudaStreamSynchronize(h2d);
    if (d2h) cudaStreamSynchronize(d2h);
    for (auto &kv : last) cudaEventDestroy(kv.second);
    for (cudaEvent_t e : {ev_compute, ev_h2d, ev_d2h}) if (e) cudaEventDestroy(e);
    if (h2d) cudaStreamDestroy(h2d);
    if (d2h) cudaStreamDestroy(d2h);
  }
  void ensure() {
    if (h2d) return;
    MPDX_CUDA(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking));
    MPDX_CUDA(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&ev_compute, &ev_h2d, &ev_d2h}) MPDX_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  // one pitched copy between a C-ordered host array and the view
  static void copy(const view_desc &v, void *host, int es, bool up, cudaStream_t s) {
    cudaMemcpy3DParms p;
    std::memset(&p, 0, sizeof(p));
    size_t w = 0, rows = 1, planes = 1, dpitch = 0, dslice_rows = 1;
    if (v.nd == 3) { w = v.ex[2]; rows = v.ex[1]; planes = v.ex[0]; dpitch = v.st[1]; dslice_rows = size_t(v.st[0] / v.st[1]); }
    else if (v.nd == 2) { w = v.ex[1]; rows = v.ex[0]; dpitch = v.st[0]; dslice_rows = rows; }
    else { w = v.ex[0]; dpitch = w; }
    const cudaPitchedPtr dev = make_cudaPitchedPtr(v.base, dpitch * es, w, dslice_rows);
    const cudaPitchedPtr hst = make_cudaPitchedPtr(host, w * es, w, rows);
    p.srcPtr = up ? hst : dev;
    p.dstPtr = up ? dev : hst;
    p.extent = make_cudaExtent(w * es, rows, planes);
    p.kind = up ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    MPDX_CUDA(cudaMemcpy3DAsync(&p, s));
  }
  void transfer(cudaStream_t compute, int kind, int idx, const view_desc &v, void *host, int es, bool up) {
    ensure();
    cudaStream_t s = up ? h2d : d2h;
    MPDX_CUDA(cudaEventRecord(ev_compute, compute));
    MPDX_CUDA(cudaStreamWaitEvent(s, ev_compute, 0));
    cudaEvent_t &e = last[{kind, idx}];
    if (e) MPDX_CUDA(cudaStreamWaitEvent(s, e, 0));
    else MPDX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    copy(v, host, es, up, s);
    MPDX_CUDA(cudaEventRecord(e, s));
    MPDX_CUDA(cudaEventRecord(up ? ev_h2d : ev_d2h, s));
    pending = true;
  }
  void join(cudaStream_t compute) {
    if (!pending) return;
    MPDX_CUDA(cudaStreamWaitEvent(compute, ev_h2d, 0));
    MPDX_CUDA(cudaStreamWaitEvent(compute, ev_d2h, 0));
    pending = false;
  }
  void sync() {
    if (h2d) MPDX_CUDA(cudaStreamSynchronize(h2d));
    if (d2h) MPDX_CUDA(cudaStreamSynchronize(d2h));
  }
};

struct solver_base {
  virtual ~solver_base() {
    xfer_async.reset();
    if (stream) cudaStreamDestroy(stream);
  }
  cudaStream_t stream = nullptr;
  std::string err;
  int dtype = 8;
  std::unique_ptr<async_xfer> xfer_async{new async_xfer};
  virtual void set_field(int kind, int idx, const void *src, bool device) = 0;
  virtual void get_field(int kind, int idx, void *dst, bool device) = 0;
  virtual void view_extent(int kind, int idx, int ex[3]) = 0;
  virtual view_desc describe(int kind, int idx) = 0;
  virtual void invalidate_fused() {}
  virtual void advance(long long nt) = 0;
  virtual void stats(mpdx_step_stats *out) = 0;
  // learned GCR preconditioner (Boussinesq solvers only)
  virtual void precond_record(long long) { throw error(MPDX_E_UNSUPPORTED, "no pressure solve in this solver"); }
  virtual double precond_train(long long, double, unsigned long long) { throw error(MPDX_E_UNSUPPORTED, "no pressure solve in this solver"); }
  virtual void precond_enable(bool) { throw error(MPDX_E_UNSUPPORTED, "no pressure solve in this solver"); }
  virtual long long precond_pairs() { return 0; }
  virtual long long precond_directions() { return -1; }
  virtual void precond_set_directions(long long) { throw error(MPDX_E_UNSUPPORTED, "no pressure solve in this solver"); }
  virtual long long precond_num_params() { return 0; }
  virtual void precond_params(float *, const float *) { throw error(MPDX_E_UNSUPPORTED, "no pressure solve in this solver"); }
  virtual double precond_loss_grad(const double *, const double *, double, float *) {
    throw error(MPDX_E_UNSUPPORTED, "no pressure solve in this solver");
  }
  // the fused 3D kernel's chunk-length tuner (MPDATA solvers only)
  virtual void tuning3d(mpdx_tuning3d *out) { std::memset(out, 0, sizeof(*out)); }
};

// common transfer machinery for solvers built on mpdata_state<T>
template <class T>
struct transfer {
  T *staging = nullptr;
  size_t cap = 0;
  ~transfer() { if (staging) cudaFree(staging); }
  void ensure(size_t n) {
    if (n <= cap) return;
    if (staging) cudaFree(staging);
    staging = nullptr;
    MPDX_CUDA(cudaMalloc(&staging, n * sizeof(T)));
    cap = n;
  }
  // view (e0 x e1 x e2) at field offset (o0, o1, o2)
  void put(cudaStream_t s, field<T> &f, const void *src, bool device, const int ex[3], const int off[3]) {
    const size_t n = size_t(ex[0]) * ex[1] * ex[2];
    const T *dsrc = static_cast<const T *>(src);
    if (!device) {
      ensure(n);
      MPDX_CUDA(cudaMemcpyAsync(staging, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
      dsrc = staging;
    }
    k_view_copy<T><<<std::max(1u, std::min(ceil_div(n, 256), 65535u * 4)), 256, 0, s>>>(
        f.v, const_cast<T *>(dsrc), ex[0], ex[1], ex[2], off[0], off[1], off[2], true);
    MPDX_LAUNCH_CHECK();
    MPDX_CUDA(cudaStreamSynchronize(s));
  }
  void get(cudaStream_t s, field<T> &f, void *dst, bool device, const int ex[3], const int off[3]) {
    const size_t n = size_t(ex[0]) * ex[1] * ex[2];
    T *ddst = static_cast<T *>(dst);
    if (!device) { ensure(n); ddst = staging; }
    k_view_copy<T><<<std::max(1u, std::min(ceil_div(n, 256), 65535u * 4)), 256, 0, s>>>(
        f.v, ddst, ex[0], ex[1], ex[2], off[0], off[1], off[2], false);
    MPDX_LAUNCH_CHECK();
    if (!device) MPDX_CUDA(cudaMemcpyAsync(dst, staging, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    MPDX_CUDA(cudaStreamSynchronize(s));
  }
};

template <class T>
struct mpdata_solver : solver_base {
  mpdata_state<T> st;
  general<T> gen{&st};
  transfer<T> xfer;
  stats_engine<T> stat;
  fused_engine<T> fus;
  int path = MPDX_PATH_AUTO, last_path = MPDX_PATH_GENERAL;
  double *scratch = nullptr;

  mpdata_solver(const mpdx_config &c) {
    dtype = sizeof(T);
    MPDX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    st.stream = stream;
    st.setup(c.n_dims, c.grid, c.n_eqns, unsigned(c.opts), c.n_iters, c.bcs);
    st.max_abs_div_eps = c.max_abs_div_eps < 0 ? std::numeric_limits<T>::epsilon() : T(c.max_abs_div_eps);
    st.upwind_filter_freq = c.upwind_filter_freq;
    st.sptl_intrp = c.sptl_intrp;
    gen.init_g();
    path = c.path;
    MPDX_CUDA(cudaMalloc(&scratch, 64));
    fus.init(st);
    if (path == MPDX_PATH_FUSED && !fus.configurable(st))
      throw error(MPDX_E_UNSUPPORTED, "fused path requested but not available for this configuration");
  }
  ~mpdata_solver() override { if (scratch) cudaFree(scratch); }

  void view(int kind, int idx, int ex[3], int off[3], field<T> *&f) {
    if (kind == MPDX_FIELD_ADVECTEE) {
      if (idx < 0 || idx >= st.n_eqns) throw error(MPDX_E_ARG, "equation index out of range");
      for (int q = 0; q < 3; ++q) { ex[q] = st.n[q]; off[q] = 0; }
      f = &st.psi[idx][st.tl[idx]];
      return;
    }
    if (kind == MPDX_FIELD_ADVECTOR) {
      if (idx < 0 || idx >= st.nd) throw error(MPDX_E_ARG, "advector component out of range");
      st.advector_extent(idx, ex);
      off[0] = -1; off[1] = idx == 1 ? -1 : 0; off[2] = idx == 2 ? -1 : 0;
      f = &st.GC[idx];
      return;
    }
    if (kind == MPDX_FIELD_G) {
      if (!(st.opts & o_nug)) throw error(MPDX_E_ARG, "libmpdata++: g_factor() called with nug option unset?");
      for (int q = 0; q < 3; ++q) { ex[q] = st.n[q]; off[q] = 0; }
      f = &st.G;
      return;
    }
    throw error(MPDX_E_ARG, "field kind not available for this solver");
  }
  void view_extent(int kind, int idx, int ex[3]) override {
    int off[3]; field<T> *f; view(kind, idx, ex, off, f);
  }
  view_desc describe(int kind, int idx) override {
    view_desc d;
    int off[3]; field<T> *f;
    view(kind, idx, d.ex, off, f);
    d.nd = st.nd;
    d.base = &f->v(off[0], off[1], off[2]);
    d.st[0] = f->v.s0; d.st[1] = f->v.s1; d.st[2] = f->v.s2;
    return d;
  }
  void invalidate_fused() override { fus.invalidate(); }
  void set_field(int kind, int idx, const void *src, bool device) override {
    int ex[3], off[3]; field<T> *f;
    view(kind, idx, ex, off, f);
    xfer.put(stream, *f, src, device, ex, off);
    fus.invalidate();
  }
  void get_field(int kind, int idx, void *dst, bool device) override {
    int ex[3], off[3]; field<T> *f;
    view(kind, idx, ex, off, f);
    xfer.get(stream, *f, dst, device, ex, off);
  }
  void advance(long long nt) override {
    if (nt <= 0) return;
    if (st.timestep == 0) gen.ante_loop(scratch);
    if (path != MPDX_PATH_GENERAL && gen.block1d_ok()) {
      gen.block1d(nt);
      st.timestep += nt;
      last_path = MPDX_PATH_FUSED;
      return;
    }
    bool use_fused = false;
    if (path != MPDX_PATH_GENERAL && fus.configurable(st)) {
      use_fused = fus.seams_consistent(st, scratch);
      if (!use_fused && path == MPDX_PATH_FUSED)
        throw error(MPDX_E_UNSUPPORTED, "fused path requested but the periodic seams of the fields are inconsistent");
    }
    last_path = use_fused ? MPDX_PATH_FUSED : MPDX_PATH_GENERAL;
    for (long long t = 0; t < nt; ++t) {
      if (use_fused) fus.step(st);
      else gen.step();
      ++st.timestep;
    }
  }
  void stats(mpdx_step_stats *out) override {
    std::memset(out, 0, sizeof(*out));
    out->timestep = st.timestep;
    stat.reduce(st, st.psi[0][st.tl[0]], out);
    out->path = last_path;
  }
  void tuning3d(mpdx_tuning3d *out) override {
    std::memset(out, 0, sizeof(*out));
    const int fixed = fused3d_planes_setting(-1);
    out->chosen = fixed > 0 ? fixed : fus.lx3;
    out->n_candidates = fused_engine<T>::kNumCand3;
    for (int q = 0; q < fused_engine<T>::kNumCand3; ++q) {
      out->lx[q] = fused_engine<T>::kCand3[q];
      out->ms[q] = fus.lx3 > 0 ? fus.tune_ms[q] : 0.f;
    }
  }
};

// Boussinesq handle (solvers::boussinesq with GCR pressure solve); P is the
// type of the pressure solve (T, or double under FP32 advection with prs_fp64)
template <class T, class P>
struct boussinesq_solver : solver_base {
  std::unique_ptr<boussinesq<T, P>> b;
  transfer<T> xfer;
  stats_engine<T> stat;
  explicit boussinesq_solver(const mpdx_config &c) {
    dtype = sizeof(T);
    MPDX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    b.reset(new boussinesq<T, P>(c, stream));
  }
  void view(int kind, int idx, int ex[3], int off[3], field<T> *&f) {
    auto &st = b->st;
    for (int q = 0; q < 3; ++q) { ex[q] = st.n[q]; off[q] = 0; }
    if (kind == MPDX_FIELD_ADVECTEE) {
      if (idx < 0 || idx >= st.n_eqns) throw error(MPDX_E_ARG, "equation index out of range");
      f = &st.psi[idx][st.tl[idx]];
      return;
    }
    if (kind == MPDX_FIELD_SCLR_ARRAY) {
      if (idx == MPDX_SCLR_THT_E) f = &b->tht_e;
      else if (idx == MPDX_SCLR_THT_ABS) f = &b->tht_abs;
      else if (idx == MPDX_SCLR_HFLUX_FRC) f = &b->hflux_frc;
      else if (idx == MPDX_SCLR_VAB_COEFF || (idx >= MPDX_SCLR_VAB_RELAX && idx < MPDX_SCLR_VAB_RELAX + st.nd)) {
        // vab_coefficient() / vab_relaxed_state(d) throw without the option (sharedmem.hpp:471-494)
        if (b->vab == MPDX_VAB_NONE)
          throw error(MPDX_E_ARG, "libmpdata++: vab_coeff() called with option vip_vab unset?");
        f = idx == MPDX_SCLR_VAB_COEFF ? &b->vab_coeff : &b->vab_relax[idx - MPDX_SCLR_VAB_RELAX];
      } else throw error(MPDX_E_ARG, "unknown scalar array");
      return;
    }
    if (kind == MPDX_FIELD_PRESSURE) {
      if constexpr (std::is_same<T, P>::value) { f = b->phi_field(); return; }
      throw error(MPDX_E_ARG, "the pressure is held in FP64 in this configuration and has no real_t view");
    }
    throw error(MPDX_E_ARG, "field kind not available for this solver");
  }
  void view_extent(int kind, int idx, int ex[3]) override {
    int off[3]; field<T> *f; view(kind, idx, ex, off, f);
  }
  view_desc describe(int kind, int idx) override {
    view_desc d;
    int off[3]; field<T> *f;
    view(kind, idx, d.ex, off, f);
    d.nd = b->st.nd;
    d.base = &f->v(off[0], off[1], off[2]);
    d.st[0] = f->v.s0; d.st[1] = f->v.s1; d.st[2] = f->v.s2;
    return d;
  }
  void set_field(int kind, int idx, const void *src, bool device) override {
    int ex[3], off[3]; field<T> *f;
    view(kind, idx, ex, off, f);
    xfer.put(stream, *f, src, device, ex, off);
  }
  void get_field(int kind, int idx, void *dst, bool device) override {
    int ex[3], off[3]; field<T> *f;
    view(kind, idx, ex, off, f);
    xfer.get(stream, *f, dst, device, ex, off);
  }
  void advance(long long nt) override { b->advance(nt); }
  void precond_record(long long n) override { b->precond_record(n); }
  double precond_train(long long steps, double lr, unsigned long long seed) override { return b->precond_train(steps, lr, seed); }
  void precond_enable(bool on) override { b->precond_enable(on); }
  long long precond_directions() override { return b->nl_used; }
  void precond_set_directions(long long nl) override {
    if (nl < -1 || nl > 64) throw error(MPDX_E_ARG, "learned corrections per solve must be -1 (tuned) or 0..64");
    b->nl_fixed = int(nl);
  }
  long long precond_pairs() override { return b->n_pairs; }
  long long precond_num_params() override {
    b->ensure_net();
    return b->net->n_params;
  }
  double precond_loss_grad(const double *r, const double *t, double c, float *g) override {
    return b->precond_loss_grad(r, t, c, g);
  }
  void precond_params(float *get, const float *set) override {
    b->ensure_net();
    if (get) b->net->get_params(get);
    if (set) b->net->set_params(set);
  }
  void stats(mpdx_step_stats *out) override {
    std::memset(out, 0, sizeof(*out));
    auto &st = b->st;
    out->timestep = st.timestep;
    out->time = double(st.timestep) * b->dt;
    stat.reduce(st, st.psi[b->ix_tht][st.tl[b->ix_tht]], out);
    out->gcr_iters = b->iters;
    out->gcr_iters_total = b->iters_total;
    out->gcr_residual = b->last_residual;
    out->gcr_ms = b->last_solve_ms;
    out->gcr_fallback = b->restarted ? 2 : (b->fell_back ? 1 : 0);
    out->path = MPDX_PATH_GENERAL;
  }
};

// ---------------------------------------------------------------------------
// Batched advance of independent 2D problems (one persistent launch per step)

struct batch_base {
  virtual ~batch_base() = default;
  virtual void advance(long long nt) = 0;
  virtual void info(mpdx_batch_info *out) = 0;
  virtual void sync() = 0;
  std::string err;
};

template <class T>
struct batch_impl : batch_base {
  std::vector<mpdata_solver<T> *> hs;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_done = nullptr, ev_a = nullptr, ev_b = nullptr;
  int mode = MPDX_BATCH_PERSISTENT, ni = 2;
  bool iga = false, fct = false;
  int tile = -1, items_tile = -1, n_items = 0, grid = 0, n_sm = 0, next_candidate = 0;
  double tune_ms[kNumBatchTiles] = {};
  f2::prob<T> *probs_dev = nullptr;  // [2][n]: step parity 0 and 1
  f2::item *items_dev = nullptr;
  size_t items_cap = 0;
  int *counter = nullptr;            // work counter and finished warps, re-armed by the kernel
  cudaGraphExec_t graph = nullptr;   // two steps (parity 0, then 1)
  long long cells = 0;

  batch_impl(const std::vector<mpdata_solver<T> *> &v, int mode_) : hs(v), mode(mode_) {
    const auto &s0 = hs[0]->st;
    ni = s0.n_iters; iga = s0.opts & o_iga; fct = s0.opts & o_fct;
    for (size_t p = 0; p < hs.size(); ++p) {
      const auto &st = hs[p]->st;
      if (st.nd != 2) throw error(MPDX_E_UNSUPPORTED, "batched advance is built for 2D problems");
      if (st.opts != s0.opts || st.n_iters != s0.n_iters)
        throw error(MPDX_E_ARG, "all problems of a batch need the same opts and n_iters");
      if (st.n_eqns != 1) throw error(MPDX_E_UNSUPPORTED, "batched problems advect one equation each");
      if (!fused_configurable(st))
        throw error(MPDX_E_UNSUPPORTED, "batched advance needs cyclic boundaries, opts within {fct, iga} (n_iters 2, or 3 without iga) and no upwind filter");
      for (size_t q = 0; q < p; ++q)
        if (hs[q] == hs[p]) throw error(MPDX_E_ARG, "a problem appears twice in the batch");
      cells += st.cells();
    }
    MPDX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    MPDX_CUDA(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
    MPDX_CUDA(cudaEventCreate(&ev_a));
    MPDX_CUDA(cudaEventCreate(&ev_b));
    MPDX_CUDA(cudaMalloc(&probs_dev, 2 * hs.size() * sizeof(f2::prob<T>)));
    MPDX_CUDA(cudaMalloc(&counter, 2 * sizeof(int)));
    MPDX_CUDA(cudaMemsetAsync(counter, 0, 2 * sizeof(int), stream));
    int dev = 0;
    MPDX_CUDA(cudaGetDevice(&dev));
    MPDX_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  }
  ~batch_impl() override {
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    if (probs_dev) cudaFree(probs_dev);
    if (items_dev) cudaFree(items_dev);
    if (counter) cudaFree(counter);
    if (ev_done) cudaEventDestroy(ev_done);
    if (ev_a) cudaEventDestroy(ev_a);
    if (ev_b) cudaEventDestroy(ev_b);
    if (stream) cudaStreamDestroy(stream);
  }

  void use_tile(int t) {
    if (t == items_tile) return;
    const bool same_items = items_tile >= 0 && kBatchTiles[items_tile].lx == kBatchTiles[t].lx;
    const int occ = fused2d_batched<T>(t, ni, iga, fct, nullptr, nullptr, 0, nullptr, 0, stream, true);
    grid = std::max(1, std::max(1, occ) / kBatchTiles[t].occ_div) * n_sm;
    if (same_items) { items_tile = t; return; }
    std::vector<int> P0(hs.size()), P1(hs.size());
    for (size_t p = 0; p < hs.size(); ++p) { P0[p] = hs[p]->st.n[0] - 1; P1[p] = hs[p]->st.n[1] - 1; }
    const auto items = fused2d_batch_items(t, ni, P0, P1);
    if (items.size() > items_cap) {
      if (items_dev) cudaFree(items_dev);
      items_dev = nullptr;
      MPDX_CUDA(cudaMalloc(&items_dev, items.size() * sizeof(f2::item)));
      items_cap = items.size();
    }
    MPDX_CUDA(cudaMemcpyAsync(items_dev, items.data(), items.size() * sizeof(f2::item), cudaMemcpyHostToDevice, stream));
    MPDX_CUDA(cudaStreamSynchronize(stream));
    n_items = int(items.size());
    items_tile = t;
  }
  void one_step(int parity) {
    fused2d_batched<T>(items_tile, ni, iga, fct, probs_dev + parity * hs.size(), items_dev, n_items, counter, grid,
                       stream, false);
  }
  void capture() {
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    cudaGraph_t g = nullptr;
    MPDX_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    one_step(0);
    one_step(1);
    MPDX_CUDA(cudaStreamEndCapture(stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    MPDX_CUDA(e);
  }

  void advance(long long nt) override {
    if (nt <= 0) return;
    for (size_t p = 0; p < hs.size(); ++p) {
      auto *h = hs[p];
      // transfers issued with the asynchronous entry points on this member come
      // first: the seam check and the batched kernel read the uploaded fields
      h->xfer_async->join(h->stream);
      MPDX_CUDA(cudaStreamSynchronize(h->stream));
      try {
        if (h->st.timestep == 0) h->gen.ante_loop(h->scratch);
      } catch (const error &e) {
        throw error(e.code, std::string(e.what()) + " (batch problem " + std::to_string(p) + ")");
      }
      if (!h->fus.seams_consistent(h->st, h->scratch))
        throw error(MPDX_E_UNSUPPORTED, "batched advance: the periodic seams of the fields of problem " + std::to_string(p) +
                                            " are inconsistent");
    }
    // problem descriptors for both step parities, from the current time levels
    std::vector<f2::prob<T>> pr(2 * hs.size());
    for (size_t p = 0; p < hs.size(); ++p) {
      auto &st = hs[p]->st;
      for (int par = 0; par < 2; ++par) {
        pr[par * hs.size() + p] = fused2d_prob(st, 0, st.tl[0] ^ par);
      }
    }
    MPDX_CUDA(cudaMemcpyAsync(probs_dev, pr.data(), pr.size() * sizeof(f2::prob<T>), cudaMemcpyHostToDevice, stream));
    long long s = 0;
    if (mode == MPDX_BATCH_PER_PROBLEM) {
      for (; s < nt; ++s)
        for (auto *h : hs) {
          fused2d_launch(h->st, h->fus.plan2, 0, stream);
          h->st.tl[0] ^= 1;
        }
    } else {
      // autotuning: every candidate timed over kTuneSteps consecutive steps (fewer if the
      // call ends first; the next call times a candidate afresh), then the fastest in a graph
      while (s < nt && tile < 0) {
        const int c = next_candidate;
        use_tile(c);
        const long long k = std::min<long long>(kTuneSteps, nt - s);
        MPDX_CUDA(cudaEventRecord(ev_a, stream));
        for (long long q = 0; q < k; ++q) one_step(int((s + q) & 1));
        MPDX_CUDA(cudaEventRecord(ev_b, stream));
        MPDX_CUDA(cudaEventSynchronize(ev_b));
        float ms = 0;
        MPDX_CUDA(cudaEventElapsedTime(&ms, ev_a, ev_b));
        s += k;
        if (k < kTuneSteps) continue;  // too few steps for a measurement
        tune_ms[c] = ms / double(k);
        ++next_candidate;
        if (next_candidate == kNumBatchTiles) {
          int best = 0;
          for (int q = 1; q < kNumBatchTiles; ++q)
            if (tune_ms[q] < tune_ms[best]) best = q;
          tile = best;
          use_tile(best);
          capture();
        }
      }
      if (s < nt && (s & 1)) one_step(1), ++s;
      for (; s + 2 <= nt; s += 2) MPDX_CUDA(cudaGraphLaunch(graph, stream));
      if (s < nt) one_step(0), ++s;
      for (auto *h : hs) h->st.tl[0] ^= int(nt & 1);
    }
    for (auto *h : hs) {
      h->st.timestep += nt;
      h->last_path = MPDX_PATH_FUSED;
    }
    MPDX_CUDA(cudaEventRecord(ev_done, stream));
    for (auto *h : hs) MPDX_CUDA(cudaStreamWaitEvent(h->stream, ev_done, 0));
  }

  void sync() override { MPDX_CUDA(cudaStreamSynchronize(stream)); }

  void info(mpdx_batch_info *out) override {
    std::memset(out, 0, sizeof(*out));
    out->n_problems = int(hs.size());
    out->cells = cells;
    out->mode = mode;
    if (tile >= 0) { out->tile_nt = kBatchTiles[tile].nt; out->tile_lx = kBatchTiles[tile].lx; out->grid = grid; }
    out->n_candidates = kNumBatchTiles;
    for (int q = 0; q < kNumBatchTiles && q < 8; ++q) out->tune_ms[q] = tune_ms[q];
  }
};

}  // namespace mpdx

struct mpdx_solver {
  std::unique_ptr<mpdx::solver_base> impl;
};

namespace {
thread_local std::string g_create_error;

// the bounds-checked build reports an out-of-range field access of the call's
// kernels as the call's error (after waiting for the device)
inline void check_bounds() {
#ifdef MPDX_BOUNDS_CHECK
  mpdx::oob_info *r = mpdx::oob_record();
  if (!r) return;
  MPDX_CUDA(cudaDeviceSynchronize());
  mpdx::oob_info h;
  MPDX_CUDA(cudaMemcpy(&h, r, sizeof(h), cudaMemcpyDeviceToHost));
  if (h.hit) {
    MPDX_CUDA(cudaMemset(r, 0, sizeof(h)));
    throw mpdx::error(MPDX_E_CUDA, "bounds-checked build: a field was indexed at (" + std::to_string(h.i) + ", " +
                                       std::to_string(h.j) + ", " + std::to_string(h.k) + "), outside its allocation");
  }
#endif
}

// a bulk plane copy of the fused 3D kernel whose completion wait gave up (a
// host-mapped word that the kernel sets; read without waiting for the device)
inline void check_copy_waits() {
  auto &w = mpdx::fused_copy_wait_flag();
  if (!w.host) return;
  volatile unsigned *v = w.host;
  if (*v) {
    *v = 0u;
    throw mpdx::error(MPDX_E_CUDA, "fused 3D kernel: a bulk plane copy did not complete within its wait limit; "
                                   "the results of the steps since the previous call are invalid");
  }
}

template <class F>
mpdx_status guarded(mpdx_handle h, F f) {
  if (!h || !h->impl) return MPDX_E_ARG;
  try {
    f();
    check_bounds();
    check_copy_waits();
    h->impl->err.clear();
    return MPDX_OK;
  } catch (const mpdx::error &e) {
    h->impl->err = e.what();
    return e.code;
  } catch (const std::exception &e) {
    h->impl->err = e.what();
    return MPDX_E_ARG;
  }
}

void validate(const mpdx_config &c) {
  using namespace mpdx;
  if (c.n_dims < 1 || c.n_dims > 3) throw error(MPDX_E_ARG, "n_dims must be 1, 2 or 3");
  for (int d = 0; d < c.n_dims; ++d)
    if (c.grid[d] < 1) throw error(MPDX_E_GRID, "libmpdata++: bogus grid size");
  if (c.dtype != 4 && c.dtype != 8) throw error(MPDX_E_ARG, "dtype must be 4 or 8");
  if (c.n_eqns < 1) throw error(MPDX_E_ARG, "n_eqns must be positive");
  if (c.n_iters < 1) throw error(MPDX_E_ARG, "n_iters must be positive");
  const unsigned o = unsigned(c.opts);
  const unsigned built = o_fct | o_abs | o_tot | o_pfc | o_npa | o_iga | o_dfl | o_nug | o_khn | o_div_2nd | o_div_3rd | o_div_3rd_dt | o_fot;
  if (o & ~built)
    throw error(MPDX_E_UNSUPPORTED, "MPDATA option not built on this backend (supported: fct abs tot pfc npa iga dfl nug khn div_2nd div_3rd div_3rd_dt fot)");
  // fot: the 2D FOT's static_asserts (formulae_mpdata_hot_2d.hpp:147-149); the 1D and 3D
  // antidiffusive velocities never add fourth-order terms, so there the option changes nothing
  if ((o & o_fot) && c.n_dims == 2 && (!(o & o_iga) || !(o & (o_tot | o_div_3rd))))
    throw error(MPDX_E_ARG, "fot option only available with iga, and only with tot or div_3rd");
  // the divergence form (formulae_mpdata_{1,2,3}d.hpp): div_3rd / div_3rd_dt extend div_2nd,
  // exclude each other and tot / dfl (static_asserts and enable_ifs there)
  if (o & (o_div_2nd | o_div_3rd | o_div_3rd_dt)) {
    if (!(o & o_div_2nd)) throw error(MPDX_E_ARG, "div_3rd and div_3rd_dt need div_2nd");
    if ((o & o_div_3rd) && (o & o_div_3rd_dt)) throw error(MPDX_E_ARG, "div_3rd and div_3rd_dt are mutually exclusive");
    if (o & (o_tot | o_dfl)) throw error(MPDX_E_ARG, "div_2nd & div_3rd options are incompatible with tot and dfl");
    if (c.solver == MPDX_SOLVER_BOUSSINESQ)
      throw error(MPDX_E_UNSUPPORTED, "the divergence-form options are built for solvers::mpdata (constant advector) only");
    // a third pass reads its base velocity GC_unco(2) = GC_corr(1) (mpdata_common.hpp:40-60) at halo
    // faces that no exchange of the second pass fills (mpdata_osc_2d.hpp:112-121 fills only the
    // normal halos over the interior; the fdiv and ndx terms reach two faces along and the corners),
    // so the reference's result there depends on uninitialised memory
    if (c.n_iters > 2)
      throw error(MPDX_E_UNSUPPORTED, "the divergence-form options are built for n_iters <= 2 (a third pass reads halo faces the reference never fills)");
  }
  if (c.sptl_intrp < 0 || c.sptl_intrp > 2) throw error(MPDX_E_ARG, "sptl_intrp must be exact (0), aver2 (1) or aver4 (2)");
  if ((o & o_nug) && c.solver == MPDX_SOLVER_BOUSSINESQ)
    throw error(MPDX_E_UNSUPPORTED, "nug option is built for solvers::mpdata only on this backend");
  if (c.upwind_filter_freq < 0) throw error(MPDX_E_ARG, "upwind_filter_freq must be non-negative");
  if ((o & o_iga) && (o & o_abs)) throw error(MPDX_E_ARG, "abs & iga options are mutually exclusive");
  for (int q = 0; q < 2 * c.n_dims; ++q) {
    const int k = c.bcs[q];
    if (k != MPDX_BC_CYCLIC && k != MPDX_BC_OPEN && k != MPDX_BC_RIGID && k != MPDX_BC_GNDSKY) throw error(MPDX_E_ARG, "unknown boundary kind");
    if (k == MPDX_BC_GNDSKY && c.n_dims != 3) throw error(MPDX_E_UNSUPPORTED, "gndsky is a 3D boundary condition (bcond/gndsky_3d.hpp)");
  }
  if (c.solver != MPDX_SOLVER_BOUSSINESQ && (c.impl_tht || c.vip_vab))
    throw error(MPDX_E_ARG, "impl_tht and vip_vab are options of the Boussinesq solver");
  if (c.vip_vab < MPDX_VAB_NONE || c.vip_vab > MPDX_VAB_IMPL) throw error(MPDX_E_ARG, "unknown velocity absorber");
}
}  // namespace

extern "C" {

void mpdx_config_default(mpdx_config *c) {
  std::memset(c, 0, sizeof(*c));
  c->solver = MPDX_SOLVER_MPDATA;
  c->n_dims = 1;
  c->n_eqns = 1;
  c->grid[0] = c->grid[1] = c->grid[2] = 1;
  c->opts = mpdx::o_iga | mpdx::o_fct;  // ct_params_default_t::opts (opts.hpp:83)
  c->n_iters = 2;                       // mpdata_common.hpp:77
  c->dtype = 8;
  c->dt = 0;
  c->di = c->dj = c->dk = 1;
  c->max_abs_div_eps = -1;
  c->path = MPDX_PATH_AUTO;
  c->prs_scheme = MPDX_PRS_CR;
  c->prs_k_iters = 4;                   // ct_params_default_t::prs_k_iters (opts.hpp:91)
  c->prs_tol = 1e-7;
  c->g = 9.81;                          // boussinesq_common.hpp:34
  c->tht_ref = 0;
  c->ix_u = 0; c->ix_v = -1; c->ix_w = 1; c->ix_tht = 2;
  c->precond = MPDX_PRECOND_IDENTITY;
  c->prs_fp64 = 0;
}

mpdx_status mpdx_create(const mpdx_config *cfg, mpdx_handle *out) {
  g_create_error.clear();
  if (!cfg || !out) { g_create_error = "null argument"; return MPDX_E_ARG; }
  *out = nullptr;
  try {
    validate(*cfg);
    // gndsky (bcond/gndsky_3d.hpp) is the rigid condition for every field filled here
    mpdx_config cc = *cfg;
    for (int q = 0; q < 2 * cc.n_dims; ++q)
      if (cc.bcs[q] == MPDX_BC_GNDSKY) cc.bcs[q] = MPDX_BC_RIGID;
    cfg = &cc;
    auto h = std::make_unique<mpdx_solver>();
    if (cfg->solver == MPDX_SOLVER_BOUSSINESQ) {
      if (cfg->dtype == 8) h->impl.reset(new mpdx::boussinesq_solver<double, double>(*cfg));
      else if (cfg->prs_fp64) h->impl.reset(new mpdx::boussinesq_solver<float, double>(*cfg));
      else h->impl.reset(new mpdx::boussinesq_solver<float, float>(*cfg));
    } else {
      if (cfg->dtype == 8) h->impl.reset(new mpdx::mpdata_solver<double>(*cfg));
      else h->impl.reset(new mpdx::mpdata_solver<float>(*cfg));
    }
    *out = h.release();
    return MPDX_OK;
  } catch (const mpdx::error &e) {
    g_create_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_create_error = e.what();
    return MPDX_E_ARG;
  }
}

const char *mpdx_create_error(void) { return g_create_error.c_str(); }

static void strided_pack(const void *src, void *dst, const int ex[3], const int64_t *st, int es, bool pack) {
  // pack: strided src -> C-ordered dst;  !pack: C-ordered src -> strided dst
  size_t q = 0;
  const char *s = static_cast<const char *>(src);
  char *d = static_cast<char *>(dst);
  for (int a = 0; a < ex[0]; ++a)
    for (int b = 0; b < ex[1]; ++b)
      for (int c = 0; c < ex[2]; ++c, ++q) {
        const int64_t o = (int64_t(a) * st[0] + int64_t(b) * st[1] + int64_t(c) * st[2]) * es;
        if (pack) std::memcpy(d + q * es, s + o, es);
        else std::memcpy(d + o, s + q * es, es);
      }
}

mpdx_status mpdx_set_field(mpdx_handle h, int kind, int idx, const void *host, const int64_t *strides) {
  const mpdx::trace_range tr("mpdx_set_field");
  return guarded(h, [&] {
    if (!host) throw mpdx::error(MPDX_E_ARG, "null host buffer");
    h->impl->xfer_async->join(h->impl->stream);
    if (!strides) { h->impl->set_field(kind, idx, host, false); return; }
    int ex[3];
    h->impl->view_extent(kind, idx, ex);
    const int es = h->impl->dtype;
    std::vector<char> tmp(size_t(ex[0]) * ex[1] * ex[2] * es);
    strided_pack(host, tmp.data(), ex, strides, es, true);
    h->impl->set_field(kind, idx, tmp.data(), false);
  });
}

mpdx_status mpdx_get_field(mpdx_handle h, int kind, int idx, void *host, const int64_t *strides) {
  const mpdx::trace_range tr("mpdx_get_field");
  return guarded(h, [&] {
    if (!host) throw mpdx::error(MPDX_E_ARG, "null host buffer");
    h->impl->xfer_async->join(h->impl->stream);
    if (!strides) { h->impl->get_field(kind, idx, host, false); return; }
    int ex[3];
    h->impl->view_extent(kind, idx, ex);
    const int es = h->impl->dtype;
    std::vector<char> tmp(size_t(ex[0]) * ex[1] * ex[2] * es);
    h->impl->get_field(kind, idx, tmp.data(), false);
    strided_pack(tmp.data(), host, ex, strides, es, false);
  });
}

// the handle's stream waits for the work issued so far to the legacy default stream
static void after_legacy_stream(cudaStream_t s) {
  cudaEvent_t e;
  MPDX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  MPDX_CUDA(cudaEventRecord(e, cudaStreamLegacy));
  const cudaError_t w = cudaStreamWaitEvent(s, e, 0);
  cudaEventDestroy(e);
  MPDX_CUDA(w);
}

mpdx_status mpdx_set_field_device(mpdx_handle h, int kind, int idx, const void *dev) {
  return guarded(h, [&] {
    if (!dev) throw mpdx::error(MPDX_E_ARG, "null device buffer");
    after_legacy_stream(h->impl->stream);
    h->impl->xfer_async->join(h->impl->stream);
    h->impl->set_field(kind, idx, dev, true);
  });
}

mpdx_status mpdx_get_field_device(mpdx_handle h, int kind, int idx, void *dev) {
  return guarded(h, [&] {
    if (!dev) throw mpdx::error(MPDX_E_ARG, "null device buffer");
    after_legacy_stream(h->impl->stream);  // the buffer may still be in use there
    h->impl->xfer_async->join(h->impl->stream);
    h->impl->get_field(kind, idx, dev, true);
  });
}

mpdx_status mpdx_set_field_async(mpdx_handle h, int kind, int idx, const void *host) {
  return guarded(h, [&] {
    if (!host) throw mpdx::error(MPDX_E_ARG, "null host buffer");
    const auto v = h->impl->describe(kind, idx);
    h->impl->xfer_async->transfer(h->impl->stream, kind, idx, v, const_cast<void *>(host), h->impl->dtype, true);
    h->impl->invalidate_fused();
  });
}

mpdx_status mpdx_get_field_async(mpdx_handle h, int kind, int idx, void *host) {
  return guarded(h, [&] {
    if (!host) throw mpdx::error(MPDX_E_ARG, "null host buffer");
    const auto v = h->impl->describe(kind, idx);
    h->impl->xfer_async->transfer(h->impl->stream, kind, idx, v, host, h->impl->dtype, false);
  });
}

mpdx_status mpdx_advance(mpdx_handle h, int64_t nt) {
  const mpdx::trace_range tr("mpdx_advance");
  return guarded(h, [&] {
    h->impl->xfer_async->join(h->impl->stream);
    h->impl->advance(nt);
  });
}

mpdx_status mpdx_sync(mpdx_handle h) {
  return guarded(h, [&] {
    MPDX_CUDA(cudaStreamSynchronize(h->impl->stream));
    h->impl->xfer_async->sync();
  });
}

mpdx_status mpdx_stats(mpdx_handle h, mpdx_step_stats *out) {
  const mpdx::trace_range tr("mpdx_stats");
  return guarded(h, [&] {
    if (!out) throw mpdx::error(MPDX_E_ARG, "null output");
    h->impl->xfer_async->join(h->impl->stream);
    h->impl->stats(out);
  });
}

void *mpdx_stream(mpdx_handle h) { return (h && h->impl) ? (void *)h->impl->stream : nullptr; }

int mpdx_fused3d_bulk_copies(int mode) { return mpdx::fused3d_bulk_copies(mode); }

int mpdx_fused3d_planes_per_cta(int lx) { return mpdx::fused3d_planes_setting(lx); }

mpdx_status mpdx_fused3d_tuning(mpdx_handle h, mpdx_tuning3d *out) {
  if (!out) return MPDX_E_ARG;
  return guarded(h, [&] { h->impl->tuning3d(out); });
}

const char *mpdx_last_error(mpdx_handle h) { return (h && h->impl) ? h->impl->err.c_str() : "invalid handle"; }

}  // extern "C"

struct mpdx_batch {
  std::unique_ptr<mpdx::batch_base> impl;
};

extern "C" {

mpdx_status mpdx_batch_create(const mpdx_handle *handles, int n, int mode, mpdx_batch_handle *out) {
  g_create_error.clear();
  if (!handles || !out || n < 1) { g_create_error = "null argument or empty batch"; return MPDX_E_ARG; }
  *out = nullptr;
  try {
    if (mode != MPDX_BATCH_PERSISTENT && mode != MPDX_BATCH_PER_PROBLEM) throw mpdx::error(MPDX_E_ARG, "unknown batch mode");
    const int dtype = handles[0] && handles[0]->impl ? handles[0]->impl->dtype : 0;
    auto collect = [&](auto *tag) {
      using S = std::remove_pointer_t<decltype(tag)>;
      std::vector<S *> v;
      for (int p = 0; p < n; ++p) {
        if (!handles[p] || !handles[p]->impl) throw mpdx::error(MPDX_E_ARG, "null handle in batch");
        auto *sp = dynamic_cast<S *>(handles[p]->impl.get());
        if (!sp) throw mpdx::error(MPDX_E_ARG, "batch members must be MPDATA solvers of the same dtype");
        v.push_back(sp);
      }
      return v;
    };
    auto b = std::make_unique<mpdx_batch>();
    if (dtype == 8) b->impl.reset(new mpdx::batch_impl<double>(collect((mpdx::mpdata_solver<double> *)nullptr), mode));
    else if (dtype == 4) b->impl.reset(new mpdx::batch_impl<float>(collect((mpdx::mpdata_solver<float> *)nullptr), mode));
    else throw mpdx::error(MPDX_E_ARG, "null handle in batch");
    *out = b.release();
    return MPDX_OK;
  } catch (const mpdx::error &e) {
    g_create_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_create_error = e.what();
    return MPDX_E_ARG;
  }
}

static mpdx_status batch_guarded(mpdx_batch_handle b, const std::function<void()> &f) {
  if (!b || !b->impl) return MPDX_E_ARG;
  try {
    f();
    check_bounds();
    check_copy_waits();
    b->impl->err.clear();
    return MPDX_OK;
  } catch (const mpdx::error &e) {
    b->impl->err = e.what();
    return e.code;
  } catch (const std::exception &e) {
    b->impl->err = e.what();
    return MPDX_E_ARG;
  }
}

mpdx_status mpdx_batch_advance(mpdx_batch_handle b, int64_t nt) {
  const mpdx::trace_range tr("mpdx_batch_advance");
  return batch_guarded(b, [&] { b->impl->advance(nt); });
}

mpdx_status mpdx_batch_get_info(mpdx_batch_handle b, mpdx_batch_info *out) {
  return batch_guarded(b, [&] {
    if (!out) throw mpdx::error(MPDX_E_ARG, "null output");
    b->impl->info(out);
  });
}

mpdx_status mpdx_batch_sync(mpdx_batch_handle b) {
  return batch_guarded(b, [&] { b->impl->sync(); });
}

const char *mpdx_batch_last_error(mpdx_batch_handle b) { return (b && b->impl) ? b->impl->err.c_str() : "invalid batch"; }

void mpdx_batch_destroy(mpdx_batch_handle b) { delete b; }

mpdx_status mpdx_precond_record(mpdx_handle h, int64_t max_pairs) {
  return guarded(h, [&] { h->impl->precond_record(max_pairs); });
}

mpdx_status mpdx_precond_train(mpdx_handle h, int64_t steps, double lr, uint64_t seed, double *final_loss) {
  const mpdx::trace_range tr("mpdx_precond_train");
  return guarded(h, [&] {
    const double l = h->impl->precond_train(steps, lr, seed);
    if (final_loss) *final_loss = l;
  });
}

mpdx_status mpdx_precond_set_directions(mpdx_handle h, int64_t nl) {
  return guarded(h, [&] { h->impl->precond_set_directions(nl); });
}

int64_t mpdx_precond_directions(mpdx_handle h) {
  return (h && h->impl) ? h->impl->precond_directions() : -1;
}

mpdx_status mpdx_precond_enable(mpdx_handle h, int on) {
  return guarded(h, [&] { h->impl->precond_enable(on != 0); });
}

int64_t mpdx_precond_pairs(mpdx_handle h) { return (h && h->impl) ? h->impl->precond_pairs() : -1; }

int64_t mpdx_precond_num_params(mpdx_handle h) {
  if (!h || !h->impl) return -1;
  try { return h->impl->precond_num_params(); } catch (const std::exception &e) { h->impl->err = e.what(); return -1; }
}

mpdx_status mpdx_precond_get_params(mpdx_handle h, float *host) {
  return guarded(h, [&] {
    if (!host) throw mpdx::error(MPDX_E_ARG, "null buffer");
    h->impl->precond_params(host, nullptr);
  });
}

mpdx_status mpdx_precond_loss_grad(mpdx_handle h, const double *r, const double *t, double c, double *loss, float *grad) {
  return guarded(h, [&] {
    if (!r || !t || !loss) throw mpdx::error(MPDX_E_ARG, "null buffer");
    *loss = h->impl->precond_loss_grad(r, t, c, grad);
  });
}

mpdx_status mpdx_precond_set_params(mpdx_handle h, const float *host) {
  return guarded(h, [&] {
    if (!host) throw mpdx::error(MPDX_E_ARG, "null buffer");
    h->impl->precond_params(nullptr, host);
  });
}

void mpdx_destroy(mpdx_handle h) {
  if (!h) return;
  if (h->impl && h->impl->stream) cudaStreamSynchronize(h->impl->stream);
  delete h;
}

}  // extern "C"
