// ORACLE -- test infrastructure only.
// C entry points over mpdata_oracle.hpp so that the Python tests (ctypes) and
// the CPU-baseline leg of bench.py can drive the CPU restatement.  Buffers are
// C-ordered doubles; the oracle converts to its own real type (float/double).
#include <cstring>
#include <memory>
#include <string>

#include "mpdata_oracle.hpp"
#include "boussinesq_oracle.hpp"

using namespace mpdx_oracle;

namespace {

struct base_t {
  virtual ~base_t() = default;
  virtual void set_advectee(int e, const double *src) = 0;
  virtual void get_advectee(int e, double *dst) = 0;
  virtual void set_advector(int d, const double *src) = 0;
  virtual void get_advector(int d, double *dst) = 0;
  virtual void advance(long long nt) = 0;
  virtual long long timestep() const = 0;
  virtual void set_sclr(const char *, const double *) { throw std::runtime_error("no such scalar array"); }
  virtual void set_param(const char *, double) { throw std::runtime_error("no such parameter"); }
  virtual long long last_iters() const { return -1; }
  std::string err;
};

template <class S, class T>
struct wrap_t : base_t {
  S s;
  void set_advectee(int e, const double *src) override {
    auto &a = s.state(e);
    size_t q = 0;
    for (int i = 0; i < s.n[0]; ++i) for (int j = 0; j < s.n[1]; ++j) for (int k = 0; k < s.n[2]; ++k) a(i, j, k) = T(src[q++]);
  }
  void get_advectee(int e, double *dst) override {
    auto &a = s.state(e);
    size_t q = 0;
    for (int i = 0; i < s.n[0]; ++i) for (int j = 0; j < s.n[1]; ++j) for (int k = 0; k < s.n[2]; ++k) dst[q++] = double(a(i, j, k));
  }
  void set_advector(int d, const double *src) override {
    int ex[3]; s.advector_extent(d, ex);
    size_t q = 0;
    for (int a = 0; a < ex[0]; ++a) for (int b = 0; b < ex[1]; ++b) for (int c = 0; c < ex[2]; ++c) s.advector_at(d, a, b, c) = T(src[q++]);
  }
  void get_advector(int d, double *dst) override {
    int ex[3]; s.advector_extent(d, ex);
    size_t q = 0;
    for (int a = 0; a < ex[0]; ++a) for (int b = 0; b < ex[1]; ++b) for (int c = 0; c < ex[2]; ++c) dst[q++] = double(s.advector_at(d, a, b, c));
  }
  void advance(long long nt) override { s.advance(nt); }
  long long timestep() const override { return s.timestep; }
  // g_factor() (sharedmem.hpp:373-380, 458-465, 579-586): interior values of G
  void set_sclr(const char *name, const double *src) override {
    if (std::strcmp(name, "G") != 0) throw std::runtime_error("no such scalar array");
    if (!(s.opts & o_nug)) throw std::runtime_error("libmpdata++: g_factor() called with nug option unset?");
    size_t q = 0;
    for (int i = 0; i < s.n[0]; ++i) for (int j = 0; j < s.n[1]; ++j) for (int k = 0; k < s.n[2]; ++k) s.Gf(i, j, k) = T(src[q++]);
  }
  void set_param(const char *name, double v) override {
    if (std::strcmp(name, "upwind_filter_freq") == 0) s.upwind_filter_freq = int(v);
    else if (std::strcmp(name, "sptl_intrp") == 0) s.sptl_intrp = int(v);
    else throw std::runtime_error("no such parameter");
  }
};

template <class T>
struct bq_wrap_t : wrap_t<boussinesq<T>, T> {
  void set_sclr(const char *name, const double *src) override {
    auto &a = this->s.sclr_array(name);
    size_t q = 0;
    for (int i = 0; i < this->s.n[0]; ++i) for (int j = 0; j < this->s.n[1]; ++j) for (int k = 0; k < this->s.n[2]; ++k) a(i, j, k) = T(src[q++]);
  }
  long long last_iters() const override { return this->s.iters; }
  // compile-time options of the reference's ct_params_t, set before the first advance
  void set_param(const char *name, double v) override {
    if (std::strcmp(name, "impl_tht") == 0) this->s.impl_tht = int(v);
    else if (std::strcmp(name, "vip_vab") == 0) this->s.vab = int(v);
    else wrap_t<boussinesq<T>, T>::set_param(name, v);
  }
};

}  // namespace

#include <omp.h>

extern "C" {

void *orc_mpdata_create(int dtype, int nd, const int *n, int n_eqns, unsigned opts, int n_iters,
                        const int *bcs, double max_abs_div_eps, char *err, int errlen) {
  try {
    if (dtype == 8) {
      auto *w = new wrap_t<mpdata<double>, double>();
      w->s.setup(nd, n, n_eqns, opts, n_iters, bcs);
      if (max_abs_div_eps >= 0) w->s.max_abs_div_eps = max_abs_div_eps;
      return w;
    }
    if (dtype == 4) {
      auto *w = new wrap_t<mpdata<float>, float>();
      w->s.setup(nd, n, n_eqns, opts, n_iters, bcs);
      if (max_abs_div_eps >= 0) w->s.max_abs_div_eps = float(max_abs_div_eps);
      return w;
    }
    throw std::runtime_error("dtype must be 4 or 8");
  } catch (const std::exception &e) {
    if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
    return nullptr;
  }
}

// Boussinesq with GCR pressure solve; prm = {dt, di, dj, dk, prs_tol, g, Tht_ref, max_abs_div_eps}
void *orc_boussinesq_create(int dtype, int nd, const int *n, unsigned opts, int n_iters, const int *bcs,
                            const double *prm, int prs_k, char *err, int errlen) {
  try {
    if (dtype == 8) {
      auto *w = new bq_wrap_t<double>();
      w->s.setup_bq(nd, n, opts, n_iters, bcs, prm, prs_k);
      return w;
    }
    if (dtype == 4) {
      auto *w = new bq_wrap_t<float>();
      w->s.setup_bq(nd, n, opts, n_iters, bcs, prm, prs_k);
      return w;
    }
    throw std::runtime_error("dtype must be 4 or 8");
  } catch (const std::exception &e) {
    if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
    return nullptr;
  }
}

void orc_destroy(void *h) { delete static_cast<base_t *>(h); }

#define ORC_TRY(body)                                                              \
  try { body; return 0; } catch (const std::exception &e) {                        \
    auto *b = static_cast<base_t *>(h); b->err = e.what(); return 1; }

int orc_set_advectee(void *h, int e, const double *src) { ORC_TRY(static_cast<base_t *>(h)->set_advectee(e, src)) }
int orc_get_advectee(void *h, int e, double *dst) { ORC_TRY(static_cast<base_t *>(h)->get_advectee(e, dst)) }
int orc_set_advector(void *h, int d, const double *src) { ORC_TRY(static_cast<base_t *>(h)->set_advector(d, src)) }
int orc_get_advector(void *h, int d, double *dst) { ORC_TRY(static_cast<base_t *>(h)->get_advector(d, dst)) }
int orc_set_sclr_array(void *h, const char *name, const double *src) { ORC_TRY(static_cast<base_t *>(h)->set_sclr(name, src)) }
int orc_set_param(void *h, const char *name, double v) { ORC_TRY(static_cast<base_t *>(h)->set_param(name, v)) }
int orc_advance(void *h, long long nt) { ORC_TRY(static_cast<base_t *>(h)->advance(nt)) }
long long orc_timestep(void *h) { return static_cast<base_t *>(h)->timestep(); }
long long orc_last_iters(void *h) { return static_cast<base_t *>(h)->last_iters(); }
const char *orc_last_error(void *h) { return static_cast<base_t *>(h)->err.c_str(); }

// OpenMP threads of the parallel loops that follow (the timed CPU baseline runs
// with one thread and with all host threads in one process)
void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int orc_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
