"""Fused MPDATA kernels (2D strip and 3D column streaming) against the oracle.

The fused path applies to all-cyclic grids whose periodic seams are consistent
(point n-1 duplicates point 0).  In FP64 it must reproduce the oracle to 1e-12
relative (it is compiled without FMA contraction and follows the reference's
operand order); FP32 results are bounded against the FP64 oracle with the
tolerance written in each test, and exact properties (positivity, FCT bounds)
are checked bit-for-bit."""
import numpy as np
import pytest

from libmpdataxx_b200 import opts as o, setups
from oracle import Oracle
from runners import load
from test_gpu_parity import make_run, rel_err

pytestmark = pytest.mark.gpu
FUSED = 2


def periodic_setup(grid, seed, cmax=0.45):
    rng = np.random.default_rng(seed)
    u = rng.uniform(0.2, 3.0, size=tuple(g - 1 for g in grid))
    psi = setups.wrap_periodic(u)
    if len(grid) == 2:
        adv = list(setups.periodic_curl_2d(grid[0], grid[1], seed, cmax=cmax))
    else:
        adv = list(setups.periodic_curl_3d(grid, seed, cmax=cmax, dtype=np.float64))
    return {"grid": tuple(grid), "bcs": ["cyclic"] * (2 * len(grid)), "advectee": [psi], "advector": adv}


def run_both(s, opts, iters, dtype, steps, path="auto"):
    run = make_run(s["grid"], opts, n_iters=iters, bcs=s["bcs"], dtype=dtype, path=path, max_abs_div_eps=1e-6)
    run.set_advectee(s["advectee"][0])
    for d, a in enumerate(s["advector"]):
        run.set_advector(a, d)
    orc = Oracle(s["grid"], opts, n_iters=iters, bcs=s["bcs"], max_abs_div_eps=1e-6)
    load(orc, s)
    return run, orc


CASES_3D = [((24, 22, 41), o.iga | o.fct), ((24, 22, 41), o.fct), ((24, 22, 41), o.iga), ((24, 22, 41), 0),
            ((40, 40, 40), o.iga | o.fct), ((19, 30, 70), o.iga | o.fct)]
CASES_2D = [((40, 300), o.fct, 3), ((40, 300), o.fct, 2), ((40, 300), o.iga | o.fct, 2), ((40, 300), o.iga, 2),
            ((40, 300), 0, 2), ((40, 300), 0, 3), ((67, 33), o.fct, 3), ((9, 7), o.fct, 2), ((130, 600), o.iga | o.fct, 2)]


@pytest.mark.parametrize("grid,opts", CASES_3D)
def test_fused3d_fp64_matches_oracle(grid, opts):
    s = periodic_setup(grid, seed=sum(grid))
    run, orc = run_both(s, opts, 2, np.float64, 3)
    for chunk in (1, 2):
        run.advance(chunk)
        orc.advance(chunk)
        assert run.stats()["path"] == FUSED
        assert rel_err(run.advectee(), orc.advectee()) <= 1e-12


@pytest.mark.parametrize("grid,opts,iters", CASES_2D)
def test_fused2d_fp64_matches_oracle(grid, opts, iters):
    s = periodic_setup(grid, seed=sum(grid) + iters)
    run, orc = run_both(s, opts, iters, np.float64, 3)
    for chunk in (1, 3):
        run.advance(chunk)
        orc.advance(chunk)
        assert run.stats()["path"] == FUSED
        assert rel_err(run.advectee(), orc.advectee()) <= 1e-12


@pytest.mark.parametrize("grid,opts,iters", [((48, 40, 70), o.iga | o.fct, 2), ((60, 300), o.fct, 3), ((60, 300), o.fct, 2)])
def test_fused_fp32_against_fp64_oracle(grid, opts, iters):
    """FP32 fused step vs the FP64 oracle: max-abs and L2 error after 10 steps.
    Tolerance: 1e-5 of max|psi| (FP32 rounding accumulated over 10 steps)."""
    s = periodic_setup(grid, seed=3)
    run, orc = run_both(s, opts, iters, np.float32, 10)
    run.advance(10)
    orc.advance(10)
    assert run.stats()["path"] == FUSED
    a, b = run.advectee().astype(np.float64), orc.advectee()
    err_max = np.abs(a - b).max() / np.abs(b).max()
    err_l2 = np.sqrt(((a - b) ** 2).mean()) / np.sqrt((b ** 2).mean())
    print(f"FP32 vs FP64 oracle: max-abs {err_max:.2e}, L2 {err_l2:.2e}")
    assert err_max <= 1e-5 and err_l2 <= 1e-6


@pytest.mark.parametrize("grid", [(48, 40, 70), (60, 300)])
def test_fused_fp32_fct_bounds_exact(grid):
    """FCT on nonnegative input: every value stays inside [min, max] of the
    initial field exactly (monotonicity), and nothing goes negative."""
    s = periodic_setup(grid, seed=11)
    lo, hi = s["advectee"][0].min(), s["advectee"][0].max()
    run, _ = run_both(s, o.iga | o.fct if len(grid) == 3 else o.fct, 2, np.float32, 0)
    run.advance(25)
    psi = run.advectee()
    assert run.stats()["path"] == FUSED
    assert psi.min() >= np.float32(lo) and psi.max() <= np.float32(hi)


def test_inconsistent_seam_uses_general_path():
    s = periodic_setup((24, 22, 41), seed=5)
    s["advectee"][0][-1, 3, 4] += 0.5  # break psi(n-1) == psi(0)
    run, orc = run_both(s, o.iga | o.fct, 2, np.float64, 2)
    run.advance(2)
    orc.advance(2)
    assert run.stats()["path"] == 1
    assert rel_err(run.advectee(), orc.advectee()) <= 1e-12


@pytest.mark.parametrize("grid,opts", [((24, 120, 240), o.iga | o.fct), ((24, 120, 240), o.iga), ((70, 64, 130), o.iga | o.fct)])
def test_fused3d_fp32_bulk_copies_bitwise(grid, opts):
    """The FP32 3D kernel's plane copies: bulk-tensor copies (the CTAs whose tile
    lies inside the periods along j and k; 9 of 25 tiles on 24 x 120 x 240, 1 of 9
    on 70 x 64 x 130) and per-thread copies everywhere give bitwise-identical
    fields, and both stay within 1e-5 of max|psi| of the FP64 oracle."""
    from libmpdataxx_b200 import _lib
    L = _lib.lib()
    s = periodic_setup(grid, seed=17)
    res = {}
    try:
        for mode in (1, 0):
            L.mpdx_fused3d_bulk_copies(mode)
            run, orc = run_both(s, opts, 2, np.float32, 6)
            run.advance(6)
            assert run.stats()["path"] == FUSED
            res[mode] = run.advectee()
    finally:
        L.mpdx_fused3d_bulk_copies(1)
    assert np.array_equal(res[0], res[1])
    orc.advance(6)
    b = orc.advectee()
    assert np.abs(res[1].astype(np.float64) - b).max() / np.abs(b).max() <= 1e-5


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_fused3d_planes_per_cta_bitwise(dtype):
    """The planes per CTA of the fused 3D kernel (the x-chunk one CTA marches
    through, after its warm-up planes) change only which CTA computes a point:
    chunks of 8 to 512 planes give bitwise-identical fields (130 x 64 x 130,
    iga|fct, 5 steps; 17 chunks of 8 down to one chunk of 512), so tuning the chunk
    length never changes a result."""
    from libmpdataxx_b200 import _lib
    L = _lib.lib()
    s = periodic_setup((130, 64, 130), seed=23)
    res = {}
    try:
        for lx in (64, 8, 32, 96, 128, 512):
            assert L.mpdx_fused3d_planes_per_cta(lx) >= 0
            run, _ = run_both(s, o.iga | o.fct, 2, dtype, 5)
            run.advance(5)
            assert run.stats()["path"] == FUSED
            assert run.tuning3d()["chosen"] == lx
            res[lx] = run.advectee()
    finally:
        L.mpdx_fused3d_planes_per_cta(0)
    for lx, a in res.items():
        assert np.array_equal(a, res[64]), lx


def test_fused3d_tuner_keeps_fastest():
    """With the process-wide setting at 0 a handle tunes its planes per CTA on its
    first fused steps (one untimed step, two timed steps per candidate), keeps the
    fastest candidate, reports every candidate's time, and its fields equal those
    of a run with the chosen chunk length fixed."""
    from libmpdataxx_b200 import _lib
    L = _lib.lib()
    assert L.mpdx_fused3d_planes_per_cta(-1) == 0
    s = periodic_setup((130, 64, 130), seed=29)
    run, _ = run_both(s, o.iga | o.fct, 2, np.float32, 19)
    run.advance(3)
    assert run.tuning3d()["chosen"] == 0
    run.advance(14)
    t = run.tuning3d()
    lxs = [c[0] for c in t["candidates"]]
    ms = [c[1] for c in t["candidates"]]
    assert lxs == [24, 32, 40, 48, 64, 80, 96, 128]
    assert all(m > 0 for m in ms)
    assert t["chosen"] == lxs[int(np.argmin(ms))]
    run.advance(2)
    tuned = run.advectee()
    try:
        L.mpdx_fused3d_planes_per_cta(t["chosen"])
        ref, _ = run_both(s, o.iga | o.fct, 2, np.float32, 19)
        ref.advance(19)
    finally:
        L.mpdx_fused3d_planes_per_cta(0)
    assert np.array_equal(tuned, ref.advectee())
