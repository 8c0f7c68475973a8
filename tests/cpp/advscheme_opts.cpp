// The 1_advscheme_opts set-up of the reference's test suite (601-cell cyclic
// grid, Courant -0.75, 1200 steps, two equations), written against the
// header-only concurr::cuda API.  Prints both advectees after the run, one
// value per line, for comparison with the reference's golden field dumps.
#include <cstdio>

#include <libmpdata++/concurr/cuda.hpp>
#include <libmpdata++/solvers/mpdata.hpp>

using namespace libmpdataxx;

template <int opts_arg>
void test() {
  struct ct_params_t : ct_params_default_t {
    using real_t = double;
    enum { n_dims = 1 };
    enum { n_eqns = 2 };
    enum { opts = opts_arg };
  };
  using run_t = concurr::cuda<solvers::mpdata<ct_params_t>, bcond::cyclic, bcond::cyclic>;
  typename run_t::rt_params_t p;
  const int nx = 601, nt = 1200;
  p.grid_size = {nx};
  run_t run(p);
  run.advectee(0) = [](int i) { return (i <= 75 || i >= 125) ? 2. : 4.; };
  run.advectee(1) = [](int i) { return (i <= 75 || i >= 125) ? -1. : 1.; };
  run.advector() = -.75;
  run.advance(nt);
  for (int e = 0; e < 2; ++e) {
    auto a = run.advectee(e);
    for (int i = 0; i < nx; ++i) std::printf("%.17g\n", a(i));
  }
}

int main() {
  test<opts::abs>();
  test<opts::iga>();
  test<opts::iga | opts::tot>();
  test<opts::iga | opts::fct>();
  test<opts::iga | opts::tot | opts::fct>();
  return 0;
}
