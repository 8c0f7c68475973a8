// The 4_revolving_sphere_3d set-up of the reference's test suite (59^3 open
// grid, 556 steps, rotation about (1,1,1)/sqrt(3)) written against the
// header-only concurr::cuda API, for the opts given on the command line
// (0 | iga | fct | iga|fct and n_iters).  Prints max, min, Linf, L2, L1 as in
// revolving_sphere_stats.hpp:46-64.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <libmpdata++/concurr/cuda.hpp>
#include <libmpdata++/solvers/mpdata.hpp>

using namespace libmpdataxx;

template <int opts_arg>
int run_case(int n_iters) {
  struct ct_params_t : ct_params_default_t {
    using real_t = double;
    enum { n_dims = 3 };
    enum { n_eqns = 1 };
    enum { opts = opts_arg };
  };
  using run_t = concurr::cuda<solvers::mpdata<ct_params_t>, bcond::open, bcond::open, bcond::open, bcond::open,
                              bcond::open, bcond::open>;
  const int nt = 556, nx = 59;
  typename run_t::rt_params_t p;
  p.n_iters = n_iters;
  p.grid_size = {nx, nx, nx};
  const double pi = std::acos(-1.0);
  const double dt = 0.018 * 2 * pi, L = 100, dx = L / (nx - 1), dy = dx, dz = dx, h = 4, r = 15,
               d = 25 / std::sqrt(3.0), x0 = 50 - d, y0 = 50 + d, z0 = 50 + d;
  p.di = dx; p.dj = dy; p.dk = dz; p.dt = dt;
  run_t slv(p);
  slv.advectee() = [&](int i, int j, int k) {
    const double t = std::pow(i * dx - x0, 2) + std::pow(j * dx - y0, 2) + std::pow(k * dx - z0, 2);
    return t - std::pow(r, 2) <= 0 ? h : 0.;
  };
  const double omega = 0.1, xc = 50, yc = 50, zc = 50;
  slv.advector(0) = [&](int i, int j, int k) { return omega / std::sqrt(3.) * (-(j * dy - yc) + (k * dz - zc)) * dt / dx; };
  slv.advector(1) = [&](int i, int j, int k) { return omega / std::sqrt(3.) * ((i * dx - xc) - (k * dz - zc)) * dt / dy; };
  slv.advector(2) = [&](int i, int j, int k) { return omega / std::sqrt(3.) * (-(i * dx - xc) + (j * dy - yc)) * dt / dz; };
  auto ic0 = slv.advectee();
  std::vector<double> ic(ic0.data(), ic0.data() + ic0.size());
  slv.advance(nt);
  auto fc = slv.advectee();
  double mx = -1e300, mn = 1e300, linf = 0, l2 = 0, l1 = 0;
  for (size_t q = 0; q < fc.size(); ++q) {
    const double v = fc.data()[q], e = v - ic[q];
    mx = std::max(mx, v);
    mn = std::min(mn, v);
    linf = std::max(linf, std::abs(e));
    l2 += e * e;
    l1 += std::abs(e);
  }
  const double n3 = std::pow(double(nx), 3);
  std::printf("%.10f %.10f %.10f %.10f %.10f\n", mx, mn, linf, 1.0 / (nt * dt) * std::sqrt(l2 / n3),
              1.0 / (nt * dt) * (l1 / n3));
  return 0;
}

int main(int argc, char **argv) {
  const int o = argc > 1 ? std::atoi(argv[1]) : 0, it = argc > 2 ? std::atoi(argv[2]) : 2;
  if (o == 0) return run_case<0>(it);
  if (o == int(opts::iga)) return run_case<opts::iga>(it);
  if (o == int(opts::fct)) return run_case<opts::fct>(it);
  return run_case<opts::iga | opts::fct>(it);
}
