// 4_revolving_sphere_3d (fct, n_iters 2) with output::hdf5_xdmf<slv_t>, as the
// reference's revolving_sphere_3d.cpp declares it (outfreq = nt, outvars[0] =
// "psi", outdir from the command line), on concurr::cuda.
#include <cmath>
#include <cstdio>
#include <string>

#include <libmpdata++/concurr/cuda.hpp>
#include <libmpdata++/output/hdf5_xdmf.hpp>
#include <libmpdata++/solvers/mpdata.hpp>

using namespace libmpdataxx;

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  struct ct_params_t : ct_params_default_t {
    using real_t = double;
    enum { n_dims = 3 };
    enum { n_eqns = 1 };
    enum { opts = opts::fct };
  };
  using slv_out_t = output::hdf5_xdmf<solvers::mpdata<ct_params_t>>;
  using run_t = concurr::cuda<slv_out_t, bcond::open, bcond::open, bcond::open, bcond::open, bcond::open, bcond::open>;
  const int nt = 556, nx = 59;
  typename run_t::rt_params_t p;
  p.n_iters = 2;
  p.grid_size = {nx, nx, nx};
  p.outfreq = nt;
  p.outvars[0].name = "psi";
  p.outdir = argv[1];
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
  slv.advance(nt);
  return 0;
}
