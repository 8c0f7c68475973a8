// output::hdf5_xdmf<slv_t> with outstart > 0 on concurr::cuda: a 2D cyclic
// run of nt = 10 steps with outfreq = 2 and outstart = 4.  As the reference's
// hook_ante_loop does, the state at the start of the advance() call is recorded
// although step 0 is not an output step, and the T axis of const.h5 holds t = 0
// before the output times 4, 6, 8, 10 (output/hdf5.hpp, "for outstart>0 we
// still want to store t=0").  A second advance() of 3 steps records its own
// starting state (step 10) again and then step 12.
#include <cstdio>
#include <string>

#include <libmpdata++/concurr/cuda.hpp>
#include <libmpdata++/output/hdf5_xdmf.hpp>
#include <libmpdata++/solvers/mpdata.hpp>

using namespace libmpdataxx;

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  struct ct_params_t : ct_params_default_t {
    using real_t = double;
    enum { n_dims = 2 };
    enum { n_eqns = 1 };
    enum { opts = opts::fct };
  };
  using slv_out_t = output::hdf5_xdmf<solvers::mpdata<ct_params_t>>;
  using run_t = concurr::cuda<slv_out_t, bcond::cyclic, bcond::cyclic, bcond::cyclic, bcond::cyclic>;
  typename run_t::rt_params_t p;
  p.n_iters = 2;
  p.grid_size = {16, 12};
  p.outfreq = 2;
  p.outstart = 4;
  p.outvars[0].name = "psi";
  p.outdir = argv[1];
  p.dt = 0.5;
  run_t slv(p);
  slv.advectee() = [](int i, int j) { return 1.0 + ((i % 15) > 4 && (i % 15) < 9 ? 1.0 : 0.0) + 0.0 * j; };
  slv.advector(0) = 0.25;
  slv.advector(1) = 0.0;
  slv.advance(10);
  if (std::string(argv[2]) == "2") slv.advance(3);
  return 0;
}
