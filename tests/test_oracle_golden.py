"""Pins the CPU oracle to the reference's own golden data (tests/golden/*,
extracted from libmpdata++ tests/paper_2015_GMD/*/refdata by make_golden.py).
The oracle is trusted as the parity checker for the CUDA path only because it
reproduces these numbers."""
import json
import math
import os

import numpy as np
import pytest

from libmpdataxx_b200 import opts as o
from libmpdataxx_b200 import setups
from oracle import Oracle
from runners import check_sphere_fields, run_oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def golden():
    with open(os.path.join(GOLD, "golden_stats.json")) as f:
        return json.load(f)


# 1_advscheme_opts: 601-cell cyclic, C = -0.75, 1200 steps; values printed with 5 decimals
@pytest.mark.parametrize("case", ["abs", "iga", "iga_tot", "iga_fct", "iga_tot_fct"])
def test_advscheme_opts_1d(case):
    ref = np.load(os.path.join(GOLD, "advscheme_opts.npz"))[case]
    s = setups.advscheme_opts()
    np.testing.assert_allclose(ref[0], s["advectee"][0], atol=6e-6)
    np.testing.assert_allclose(ref[1], s["advectee"][1], atol=6e-6)
    out = run_oracle(s, setups.ADVSCHEME_CASES[case])
    np.testing.assert_allclose(out[0], ref[2], rtol=0, atol=6e-6)
    np.testing.assert_allclose(out[1], ref[3], rtol=0, atol=6e-6)


# 0_basic_example: 101-cell open, iga|fct (default opts), records every 20 steps
def test_basic_example_1d():
    ref = np.load(os.path.join(GOLD, "basic_example.npz"))
    s = setups.basic_example()
    orc = Oracle(s["grid"], s["opts"], n_iters=2, bcs=s["bcs"])
    orc.set_advectee(s["advectee"][0])
    orc.set_advector(s["advector"][0])
    np.testing.assert_allclose(orc.advectee(), ref["records"][0], atol=6e-6)
    for rec in ref["records"][1:]:
        orc.advance(20)
        np.testing.assert_allclose(orc.advectee(), rec, rtol=0, atol=6e-6)


def _check_stats(got, want, keys, atol=6e-9):
    for k in keys:
        assert abs(got[k] - want["tN:" + k]) <= atol, (k, got[k], want["tN:" + k])


# 2_convergence_1d: error norms printed with 4 significant digits; the oracle runs
# the four coarsest grid steps (every Courant number and solver), the GPU all eight
def within_4_digits(got, want):
    return abs(got - want) <= 0.5e-4 * 10 ** math.floor(math.log10(abs(want))) * 1.01


@pytest.mark.parametrize("key", list(setups.CONVERGENCE_SOLVERS))
def test_convergence_1d_coarse(key):
    opts, iters = setups.CONVERGENCE_SOLVERS[key]
    rows = golden()["convergence_1d"][key]
    checked = 0
    for dx, cour, want in rows:
        if dx < 0.125:
            continue
        s = setups.convergence_1d(dx, cour)
        out = run_oracle(s, opts, n_iters=iters)[0]
        got = setups.convergence_error(out, s["exact"], s["nt"], s["dt"])
        assert within_4_digits(got, want), (key, dx, cour, got, want)
        checked += 1
    assert checked == 4 * 19


# 3_rotating_cone_2d: 101^2 open, 3768 steps; stats with 8 decimals
@pytest.mark.parametrize("case", list(setups.CONE_CASES))
def test_rotating_cone_2d(case):
    s = setups.rotating_cone()
    opts, iters = setups.CONE_CASES[case]
    out = run_oracle(s, opts, n_iters=iters)[0]
    st = setups.cone_stats(s["advectee"][0], out, s["nt"], s["dt"])
    _check_stats(st, golden()["rotating_cone_2d"][case], ["min(psi)", "max(psi)", "rms error"])


# 4_revolving_sphere_3d: 59^3 open, 556 steps; stats with 8 decimals, and the
# float32 output fields (HDF5 refdata: planes through the sphere and block sums)
@pytest.mark.parametrize("case", list(setups.SPHERE_CASES))
def test_revolving_sphere_3d(case):
    s = setups.revolving_sphere()
    opts, iters = setups.SPHERE_CASES[case]
    out = run_oracle(s, opts, n_iters=iters)[0]
    st = setups.sphere_stats(s["advectee"][0], out, s["nt"], s["dt"])
    _check_stats(st, golden()["revolving_sphere_3d"][case], ["max(solution)", "min(solution)", "Linf", "L2", "L1"])
    check_sphere_fields(case, out)


def test_revolving_sphere_fields_fixture_catches_a_change():
    """The field check is not vacuous: one cell of the sphere moved by 1e-6 fails it."""
    s = setups.revolving_sphere()
    opts, iters = setups.SPHERE_CASES["fct"]
    out = run_oracle(s, opts, n_iters=iters)[0]
    ref = np.load(os.path.join(GOLD, "revolving_sphere_fields.npz"))
    c = ref["centre"]
    out[c[0], c[1], c[2]] += 1e-6
    with pytest.raises(AssertionError):
        check_sphere_fields("fct", out)
    out[c[0], c[1], c[2]] -= 1e-6
    out[3, 50, 7] += 1e-5  # off every plane: caught by the block sums
    with pytest.raises(AssertionError):
        check_sphere_fields("fct", out)


# tests/unit/cone_bugs: FP32 fct never undershoots the background (exact)
def test_cone_bugs_fp32_exact_min():
    s = setups.cone_bugs()
    out = run_oracle(s, s["opts"], n_iters=2, dtype=np.float32)[0]
    assert out.min() - 1 == 0


def test_divergent_advector_raises():
    s = setups.cone_bugs()
    s["advector"][0] = s["advector"][0] + np.linspace(0, 0.1, s["grid"][0])[:, None]
    with pytest.raises(RuntimeError, match="initial advector field is divergent"):
        run_oracle(s, o.fct)


def test_bogus_grid_raises():
    with pytest.raises(RuntimeError, match="bogus grid size"):
        Oracle((0, 4), o.fct)


# --- tests/paper_2015_GMD/8_boussinesq_2d: stats.txt.gz every 10 steps ---------
def _bq_golden_check(orc, s, rows):
    from libmpdataxx_b200.setups import boussinesq_stats
    init = s["advectee"][2]
    for row in rows:
        orc.advance(row["timestep"] - orc.timestep)
        st = boussinesq_stats(orc.advectee(2), orc.advectee(0), orc.advectee(1), s["tht_ref"], init)
        for key, v in st.items():
            # stats.txt prints std::scientific with 6 digits after the point
            assert float("%.6e" % v) == row[key], (row["timestep"], key, v, row[key])


def test_boussinesq_2d_golden_first_steps():
    from libmpdataxx_b200.setups import boussinesq_2d
    from runners import bq_oracle
    s = boussinesq_2d()
    rows = golden()["boussinesq_2d"]["rows"]
    _bq_golden_check(bq_oracle(s), s, [r for r in rows if r["timestep"] <= 30])


@pytest.mark.slow
def test_boussinesq_2d_golden_800_steps():
    from libmpdataxx_b200.setups import boussinesq_2d
    from runners import bq_oracle
    s = boussinesq_2d()
    _bq_golden_check(bq_oracle(s), s, golden()["boussinesq_2d"]["rows"])


def test_boussinesq_pressure_solver_stuck():
    """More than 10000 GCR iterations throw the reference's error (mpdata_rhs_vip_prs_common.hpp:118-122)."""
    from libmpdataxx_b200.setups import boussinesq_2d
    from runners import bq_oracle
    s = boussinesq_2d(nx=17, ny=17, r0=30.0)
    s["prs_tol"] = 1e-300
    orc = bq_oracle(s)
    with pytest.raises(RuntimeError, match="stuck in pressure solver"):
        orc.advance(1)


def test_oracle_boussinesq_zero_forcings_equal_plain():
    """With the velocity absorber's coefficient and the theta absorber at zero, the
    implicit absorber (normalisation by 1 + 0, relaxation by 0) gives the plain
    solver's fields bit for bit."""
    from runners import bq_oracle
    from test_gpu_boussinesq import random_bq
    s = random_bq((19, 17), ["cyclic", "cyclic", "rigid", "rigid"], seed=9)
    a = bq_oracle(s)
    t = dict(s)
    t["vip_vab"] = 2
    t["vab_coeff"] = np.zeros(s["grid"])
    t["vab_relax"] = [np.zeros(s["grid"]), np.zeros(s["grid"])]
    b = bq_oracle(t)
    a.advance(3)
    b.advance(3)
    for e in range(3):
        np.testing.assert_array_equal(a.advectee(e), b.advectee(e))


def test_oracle_impl_tht_close_to_expl_with_uniform_environment():
    """With a uniform tht_e (dtht_e = 0) and no absorbers, the implicit form
    (theta as the perturbation, boussinesq_impl.hpp) and the explicit form
    (full theta, boussinesq_expl.hpp) describe the same flow.  They agree to the
    pressure solver's tolerance: the upwind flux of the constant 300 K part of the
    full theta cancels only where the discrete divergence of the Courant field,
    which the solve drives below prs_tol / dt, is zero."""
    from runners import bq_oracle
    from test_gpu_boussinesq import random_bq
    s = random_bq((19, 17), ["cyclic"] * 4, seed=4)
    a = bq_oracle(s)
    t = dict(s)
    t["advectee"] = list(s["advectee"])
    t["advectee"][2] = s["advectee"][2] - s["tht_e"]
    t["impl_tht"] = True
    b = bq_oracle(t)
    a.advance(4)
    b.advance(4)
    for e in range(2):
        np.testing.assert_allclose(b.advectee(e), a.advectee(e), rtol=0, atol=1e-5)
    np.testing.assert_allclose(b.advectee(2) + s["tht_e"], a.advectee(2), rtol=0, atol=1e-4)
