// Boussinesq solver with GCR(k) pressure solve (solvers::boussinesq, iles,
// trapezoidal right-hand side, explicit buoyancy) on the device.
#pragma once

#include <vector>

#include <memory>

#include "general.cuh"
#include "precond.cuh"

namespace mpdx {

namespace bq {
struct geom;
template <class T> struct forcing;
}  // namespace bq

constexpr int kGcrMaxK = 8;        // largest k of GCR(k) built
constexpr int kRedBlocks = 1184;   // largest reduction grid: 8 x 148 SMs (a fixed shape per grid size => reproducible sums)
constexpr int kRedThreads = 256;
constexpr int kRedSlots = kGcrMaxK + 2;

// GCR scalars that live on the device.  beta, alpha and tmp_den persist from
// solve to solve as the reference's members do (mpdata_rhs_vip_prs_gcrk.hpp:25-27).
template <class T>
struct gcr_dev {
  T beta;
  T alpha[kGcrMaxK];
  T tmp_den[kGcrMaxK];
  T pend_den, pend_num;  // sums produced with a new search direction, consumed by the next update
  T mean;                // ini_pressure: mean of Phi
  double residual;       // max|err| at the last convergence check
  int converged, done, stuck, cur;
  int bad;               // a learned direction gave non-finite sums: nothing was updated with it
  long long iters;
  unsigned int arrive;   // last-block ticket of the running reduction
};

// T: type of the advected state (real_t); P: type of the pressure solve
// (Phi, the GCR fields and scalars) -- T itself, or double under FP32 advection.
template <class T, class P>
struct boussinesq {
  mpdata_state<T> st;
  general<T> gen{&st};
  field<T> stash[3], vip_rhs[3], rhs[4], tht_e;
  // theta absorber and heat flux (sclr_array "tht_abs", "hflux_frc"), velocity
  // absorber (vab_coefficient(), vab_relaxed_state(d)), d(tht_e)/dz (impl_tht)
  field<T> tht_abs, hflux_frc, vab_coeff, vab_relax[3], dtht_e;
  int impl_tht = 0, vab = MPDX_VAB_NONE;
  bool normalizes() const { return vab == MPDX_VAB_IMPL || impl_tht; }
  field<P> Phi, err[2], lap_err, den[3];  // den: normalize_vip denominators per velocity component
  std::vector<field<P>> p_err, lap_p_err;
  double dt = 0;
  T dtT = 0, g = 0, tht_ref = 0;
  double dijk[3] = {1, 1, 1};
  P err_tol = 0;
  int k_iters = 1, vip[3] = {0, 1, 2}, ix_w = 1, ix_tht = 2;
  T dt_stash0 = 0;
  long long iters = 0, iters_total = 0, predicted = 8;
  double last_residual = 0, last_solve_ms = 0;
  cudaEvent_t ev_solve[2] = {nullptr, nullptr};
  gcr_dev<P> *dev = nullptr;
  gcr_dev<P> *hdev = nullptr;  // pinned host copy for the convergence read-back
  double *part = nullptr;      // per-block partial results of the running reduction
  double *scratch = nullptr;
  int *vip_dev = nullptr;      // vip[] on the device

  // learned preconditioner (FP64 pressure solve only): the network, whether GCR
  // uses it, and the recorded (initial residual, correction) pairs of solves
  std::unique_ptr<pc::net> net;
  bool use_net = false;
  static constexpr int kSnaps = 3;  // recorded pairs per solve beyond the initial one (iterations 16, 32, 64)
  field<P> snap[1 + kSnaps], phi_start;  // phi_start: Phi when a learned solve began
  float *pairs = nullptr, *tr_r = nullptr, *tr_t = nullptr, *tr_q = nullptr, *tr_z = nullptr, *tr_dq = nullptr;
  float *tr_a = nullptr, *tr_b = nullptr;
  double out_scale = 0, last_train_loss = -1;
  double *tr_loss = nullptr;
  long long last_plain_iters = 250;
  float last_plain_ms = 0;  // device time of the last plain solve (0: none yet)
  bool fell_back = false;
  bool restarted = false;   // the last learned solve was redone from its start with plain GCR
  // learned solves: the first nl search directions come from the network, the rest
  // are plain GCR's; nl is chosen among the candidates by the measured solve times
  static constexpr int kNlCand = 4;
  int nl_cand[kNlCand] = {1, 2, 4, 0};
  double nl_ms[kNlCand] = {0, 0, 0, 0};
  int nl_tries[kNlCand] = {0, 0, 0, 0};
  int nl_fixed = 1;          // >= 0: every learned solve takes this many learned corrections; -1: tuned
  long long nl_used = -1;    // learned corrections of the last learned solve
  long long n_learned = 0;   // learned solves so far
  int pick_nl();
  long long max_pairs = 0, n_pairs = 0;
  int pc_channels[4] = {8, 16, 32, 64};

  void precond_record(long long max_pairs);
  // Adam on the energy-norm loss with a cosine learning-rate schedule; returns the
  // held-out loss of the weights kept (the best seen, never worse than the start)
  double precond_train(long long steps, double lr, unsigned long long seed);
  // energy-norm loss (and its parameter gradient, if grad_host) of one pair given by
  // the caller (interior, C order), with output scale c
  double precond_loss_grad(const double *r, const double *t, double c, float *grad_host);
  void precond_enable(bool on);
  void ensure_net();

  boussinesq(const mpdx_config &c, cudaStream_t s);
  ~boussinesq();
  boussinesq(const boussinesq &) = delete;
  boussinesq &operator=(const boussinesq &) = delete;
  field<P> *phi_field() { return &Phi; }
  void advance(long long nt);

 private:
  field<T> &vips(int d) { return st.psi[vip[d]][st.tl[vip[d]]]; }
  void ante_loop();
  void step();
  // pressure_solver_update up to the final gradient; simple: no normalize_vip in lap()
  void pressure_solve(bool simple);
  void ensure_training();
  double pair_energy(float c, bool grad);
  void load_pair(long long k);
  bq::forcing<T> forcing();
  bq::geom norm_geom(bq::geom g) const;
};

extern template struct boussinesq<float, float>;
extern template struct boussinesq<float, double>;
extern template struct boussinesq<double, double>;

}  // namespace mpdx
