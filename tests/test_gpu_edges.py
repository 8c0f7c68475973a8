"""Edge cases of the general (reference-structured) path against the oracle, FP64:

  * the smallest grids whose halo fills stay within the grid (n = 2 halo + 1
    points per axis: 3 without, 5 with the halo-2 options fct / tot);
  * ragged 3D grids (every extent different, odd and even) with different
    boundary conditions on the axes and on the two sides of an axis;
  * a zero advector (nothing moves, bit for bit) and a zero advectee (stays
    zero, bit for bit);
  * several equations advected by one advector (n_eqns 3), each equal to its own
    single-equation run.
The divergence check is switched off (random advectors are divergent)."""
import numpy as np
import pytest

from libmpdataxx_b200 import opts as o
from oracle import Oracle
from runners import load
from test_gpu_parity import make_run, rel_err

pytestmark = pytest.mark.gpu
RTOL64 = 1e-12
NO_DIV = 1e30


def random_problem(grid, seed, n_eqns=1, cmax=0.3):
    rng = np.random.default_rng(seed)
    nd = len(grid)
    psi = [rng.uniform(0.5, 2.0, size=grid) for _ in range(n_eqns)]
    adv = []
    for d in range(nd):
        shape = list(grid)
        if d > 0:
            shape[0] += 1
        adv.append(rng.uniform(-cmax, cmax, size=shape))
    return {"grid": tuple(grid), "advectee": psi, "advector": adv}


def run_both(s, bcs, opts, iters, steps, n_eqns=1):
    orc = Oracle(s["grid"], opts, n_iters=iters, n_eqns=n_eqns, bcs=bcs, max_abs_div_eps=NO_DIV)
    load(orc, s)
    run = make_run(s["grid"], opts, n_iters=iters, n_eqns=n_eqns, bcs=bcs, max_abs_div_eps=NO_DIV)
    for e, a in enumerate(s["advectee"]):
        run.set_advectee(a, e)
    for d, a in enumerate(s["advector"]):
        run.set_advector(a, d)
    orc.advance(steps)
    run.advance(steps)
    return run, orc


SMALLEST = []
for nd in (1, 2, 3):
    for bc in ("cyclic", "open", "rigid"):
        SMALLEST.append((nd, bc, 0, 2, 3))        # halo 1
        SMALLEST.append((nd, bc, o.fct, 2, 5))    # halo 2
        SMALLEST.append((nd, bc, o.iga | o.tot, 2, 5))


@pytest.mark.parametrize("nd,bc,opts,iters,n", SMALLEST)
def test_smallest_grid_matches_oracle(nd, bc, opts, iters, n):
    grid = (n,) * nd
    bcs = [bc] * (2 * nd)
    s = random_problem(grid, seed=nd * 10 + n)
    run, orc = run_both(s, bcs, opts, iters, 5)
    assert rel_err(run.advectee(), orc.advectee()) <= RTOL64


# (left, right) per axis; a cyclic side is paired with a cyclic side
MIXED = [["cyclic", "cyclic", "open", "rigid", "rigid", "open"],
         ["open", "open", "cyclic", "cyclic", "rigid", "rigid"],
         ["rigid", "open", "rigid", "rigid", "cyclic", "cyclic"],
         ["open", "rigid", "open", "open", "open", "rigid"]]


@pytest.mark.parametrize("bcs", MIXED, ids=["".join(b[:1] for b in bc) for bc in MIXED])
@pytest.mark.parametrize("opts,iters", [(o.fct, 2), (o.iga | o.fct, 2), (o.tot, 3)])
def test_ragged_3d_mixed_boundaries(bcs, opts, iters):
    s = random_problem((7, 12, 9), seed=len("".join(bcs)) + iters)
    run, orc = run_both(s, bcs, opts, iters, 4)
    assert rel_err(run.advectee(), orc.advectee()) <= RTOL64


@pytest.mark.parametrize("nd", [1, 2, 3])
def test_zero_advector_leaves_advectee_unchanged(nd):
    grid = {1: (17,), 2: (9, 11), 3: (6, 7, 8)}[nd]
    s = random_problem(grid, seed=nd)
    s["advector"] = [np.zeros_like(a) for a in s["advector"]]
    for opts in (0, o.fct, o.iga | o.fct | o.tot):
        run, _ = run_both(s, ["open"] * (2 * nd), opts, 2, 3)
        np.testing.assert_array_equal(run.advectee(), s["advectee"][0])


@pytest.mark.parametrize("nd", [1, 2, 3])
def test_zero_advectee_stays_zero(nd):
    grid = {1: (17,), 2: (9, 11), 3: (6, 7, 8)}[nd]
    s = random_problem(grid, seed=nd + 40)
    s["advectee"] = [np.zeros(grid)]
    for opts in (0, o.fct, o.iga | o.fct):
        run, _ = run_both(s, ["cyclic"] * (2 * nd), opts, 2, 3)
        assert not np.any(run.advectee())


def test_several_equations_match_single_runs():
    grid = (11, 10, 9)
    s = random_problem(grid, seed=5, n_eqns=3)
    bcs = ["cyclic", "cyclic", "open", "open", "rigid", "rigid"]
    run, orc = run_both(s, bcs, o.iga | o.fct, 2, 4, n_eqns=3)
    for e in range(3):
        assert rel_err(run.advectee(e), orc.advectee(e)) <= RTOL64
        one = {"grid": grid, "advectee": [s["advectee"][e]], "advector": s["advector"]}
        r1, _ = run_both(one, bcs, o.iga | o.fct, 2, 4)
        np.testing.assert_array_equal(r1.advectee(), run.advectee(e))
