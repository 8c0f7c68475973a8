// The output writer of the header-only API alone (no GPU): const.h5 and the
// records at timesteps 0 and 556 of the 4_revolving_sphere_3d set-up (59^3,
// dt = 0.018 * 2 pi, dx = 100 / 58, opts fct, n_iters 2), into the directory
// given on the command line; the advectee written is the initial sphere.
#include <cmath>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include <libmpdata++/opts.hpp>
#include <libmpdata++/output/hdf5_xdmf.hpp>

using namespace libmpdataxx;

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  const int nx = 59, nt = 556;
  const double pi = std::acos(-1.0), dt = 0.018 * 2 * pi, dx = 100.0 / (nx - 1), h = 4, r = 15,
               d = 25 / std::sqrt(3.0), x0 = 50 - d, y0 = 50 + d, z0 = 50 + d;
  output::detail::xdmf_recorder rec(argv[1], {nx, nx, nx}, dt, {dx, dx, dx}, opts::opts_string(opts::fct), 2);
  rec.start({0.0, nt * dt});
  std::vector<float> psi(size_t(nx) * nx * nx);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < nx; ++j)
      for (int k = 0; k < nx; ++k) {
        const double t = std::pow(i * dx - x0, 2) + std::pow(j * dx - y0, 2) + std::pow(k * dx - z0, 2);
        psi[(size_t(i) * nx + j) * nx + k] = float(t - std::pow(r, 2) <= 0 ? h : 0.);
      }
  rec.record(0, {{"psi", psi}});
  rec.record(nt, {{"psi", psi}});
  return 0;
}
