"""GPU parity of the Boussinesq solver and its GCR(k) pressure solve.

FP64 fields must match the CPU oracle to 1e-12 relative after every step and
the pressure solver must take the same number of iterations; the 2D buoyant
thermal must reproduce the reference's stats.txt (7 significant digits) at
every one of its 80 records."""
import numpy as np
import pytest

from libmpdataxx_b200 import _lib, opts as o, setups, solvers
from runners import bq_oracle, bq_run

pytestmark = pytest.mark.gpu

RTOL64 = 1e-12


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def random_bq(grid, bcs, seed, prs_k=1, wind=0.5):
    """Thermal bubble plus noise in a stratified state, with a random initial
    wind (so that the initial projection does work)."""
    rng = np.random.default_rng(seed)
    nd = len(grid)
    dx = (10.0,) * 3
    idx = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in grid], indexing="ij")
    z = idx[-1] * dx[nd - 1]
    # stratified only along a rigid vertical axis: along a cyclic axis every field,
    # tht_e included, must be periodic or the pressure problem has no solution
    tht_e = 300.0 * np.exp(1e-4 * z / 9.81) if bcs[-1] == "rigid" else np.full(grid, 300.0)
    r2 = sum(((idx[d] - 0.5 * (grid[d] - 1)) / (0.25 * grid[d])) ** 2 for d in range(nd))
    tht = tht_e + np.where(r2 <= 1.0, 0.5, 0.0) + rng.uniform(-0.01, 0.01, size=grid)
    vel = [rng.uniform(-wind, wind, size=grid) for _ in range(nd)]
    fields = vel + [tht]
    for d in range(nd):  # duplicated-endpoint convention along cyclic axes
        if bcs[2 * d] == "cyclic":
            for f in fields:
                sl_last = [slice(None)] * nd
                sl_first = [slice(None)] * nd
                sl_last[d], sl_first[d] = -1, 0
                f[tuple(sl_last)] = f[tuple(sl_first)]
    return {"grid": tuple(grid), "bcs": bcs, "advectee": fields, "tht_e": tht_e, "dt": 0.75, "dx": dx,
            "tht_ref": 300.0, "g": 9.81, "prs_tol": 1e-7, "prs_k": prs_k}


CASES = [
    ((33, 29), ["cyclic"] * 4, 1),
    ((31, 27), ["cyclic", "cyclic", "rigid", "rigid"], 1),
    ((25, 23), ["rigid"] * 4, 4),
    ((26, 21), ["cyclic", "cyclic", "rigid", "rigid"], 3),
    ((17, 15, 13), ["cyclic"] * 4 + ["rigid"] * 2, 1),
    ((13, 14, 15), ["cyclic"] * 6, 2),
]


@pytest.mark.parametrize("grid,bcs,prs_k", CASES)
def test_boussinesq_fp64_matches_oracle(grid, bcs, prs_k):
    s = random_bq(grid, bcs, seed=len(grid) * 10 + prs_k, prs_k=prs_k)
    orc = bq_oracle(s)
    run = bq_run(s)
    for step in range(6):
        orc.advance(1)
        run.advance(1)
        st = run.stats()
        assert st["gcr_iters"] == orc.last_iters, (step, st["gcr_iters"], orc.last_iters)
        for e in range(len(grid) + 1):
            assert rel_err(run.advectee(e), orc.advectee(e)) <= RTOL64, (step, e)
    assert st["timestep"] == 6 and st["gcr_iters_total"] > 0


def test_boussinesq_2d_reproduces_reference_stats():
    """tests/paper_2015_GMD/8_boussinesq_2d (201 x 201, cr, 800 steps) against refdata/stats.txt."""
    import json
    import os
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden_stats.json")))["boussinesq_2d"]
    s = setups.boussinesq_2d()
    run = bq_run(s)
    init = s["advectee"][2]
    for row in gold["rows"]:
        run.advance(row["timestep"] - run.stats()["timestep"])
        st = setups.boussinesq_stats(run.advectee(2), run.advectee(0), run.advectee(1), s["tht_ref"], init)
        for key, v in st.items():
            assert float("%.6e" % v) == row[key], (row["timestep"], key, v, row[key])
    # the reference's own acceptance check (boussinesq_2d.cpp:114-116)
    tht = run.advectee(2)
    assert tht.min() >= 300 - 0.01 and tht.max() <= 300.5 + 0.01


@pytest.mark.parametrize("prs_fp64", [False, True])
def test_boussinesq_fp32_close_to_fp64_oracle(prs_fp64):
    """FP32 advection with an FP32 or an FP64 pressure solve, against the FP64 oracle."""
    s = random_bq((41, 37), ["cyclic", "cyclic", "rigid", "rigid"], seed=5)
    orc = bq_oracle(s)
    run = bq_run(s, dtype=np.float32, prs_fp64=prs_fp64)
    orc.advance(20)
    run.advance(20)
    for e in range(3):
        ref = orc.advectee(e)
        err = np.abs(run.advectee(e).astype(np.float64) - ref)
        scale = max(np.abs(ref).max(), 1e-30) if e < 2 else 1.0
        print(f"eqn {e}: max-abs {err.max():.3e}  L2 {np.sqrt((err ** 2).mean()):.3e}")
        # velocities: 1e-3 of their range; theta (~300 K, FP32 ulp 3e-5 K): 2e-3 K
        assert err.max() <= (1e-3 * scale if e < 2 else 2e-3)


def test_boussinesq_stuck_pressure_solver_raises():
    s = random_bq((17, 17), ["cyclic"] * 4, seed=3)
    s["prs_tol"] = 1e-300
    run = bq_run(s)
    with pytest.raises(RuntimeError, match="stuck in pressure solver"):
        run.advance(1)


def test_boussinesq_rejects_unbuilt_configurations():
    s = random_bq((17, 17), ["open"] * 4, seed=3)
    with pytest.raises(RuntimeError, match="cyclic and rigid"):
        bq_run(s)


def test_boussinesq_fp64_pressure_is_not_viewed_as_fp32():
    s = random_bq((17, 15), ["cyclic"] * 4, seed=2)
    run = bq_run(s, dtype=np.float32, prs_fp64=True)
    out = np.empty((17, 15), dtype=np.float32)
    rc = run.L.mpdx_get_field(run.h, _lib.FIELD_PRESSURE, 0, out.ctypes.data, None)
    assert rc == _lib.MPDX_E_ARG


def test_reciprocal_division_matches_cuda_division(tmp_path):
    """The pressure operators divide by the grid spacing with mpdx::qdiv
    (reciprocal + Markstein correction) and the FP32 quad kernels divide with
    mpdx::rdivf (refined reciprocal + Markstein correction); both must return
    the IEEE quotient."""
    import os
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    exe = str(tmp_path / "qdiv_check")
    subprocess.run(["nvcc", "-std=c++17", "-O3", "--fmad=false", "-gencode", "arch=compute_100a,code=sm_100a",
                    os.path.join(here, "cuda", "qdiv_check.cu"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr


def forced_bq(grid, bcs, seed, impl_tht, vip_vab):
    """random_bq plus the forcings of boussinesq_common.hpp / boussinesq_impl.hpp and
    the velocity absorber of mpdata_rhs_vip_common.hpp, all non-zero: a theta
    absorber and a velocity absorber in the upper third, a heat flux decaying with
    height, non-zero relaxed velocities.  With impl_tht the advected theta is the
    perturbation from tht_e (boussinesq_impl.hpp:8-10)."""
    s = random_bq(grid, bcs, seed)
    nd = len(grid)
    rng = np.random.default_rng(seed + 100)
    z = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in grid], indexing="ij")[-1] / (grid[-1] - 1)
    top = np.where(z >= 2.0 / 3.0, (z - 2.0 / 3.0) * 3.0, 0.0)
    s["tht_abs"] = 0.05 * top
    s["hflux_frc"] = 1e-3 * np.exp(-4 * z)
    s["impl_tht"] = impl_tht
    s["vip_vab"] = vip_vab
    if vip_vab:
        s["vab_coeff"] = 0.08 * top
        s["vab_relax"] = [rng.uniform(-0.2, 0.2, size=grid) for _ in range(nd)]
    if impl_tht:
        s["advectee"][nd] = s["advectee"][nd] - s["tht_e"]
    for d in range(nd):  # duplicated-endpoint convention along cyclic axes
        if bcs[2 * d] == "cyclic":
            for f in [s["tht_abs"], s["hflux_frc"]] + s.get("vab_relax", []) + ([s["vab_coeff"]] if vip_vab else []):
                sl_last = [slice(None)] * nd
                sl_first = [slice(None)] * nd
                sl_last[d], sl_first[d] = -1, 0
                f[tuple(sl_last)] = f[tuple(sl_first)]
    return s


FORCED = [
    ((29, 25), ["cyclic", "cyclic", "rigid", "rigid"], True, solvers.noab, 1),
    ((29, 25), ["cyclic", "cyclic", "rigid", "rigid"], False, solvers.expl, 1),
    ((27, 23), ["cyclic", "cyclic", "rigid", "rigid"], False, solvers.impl, 1),
    ((27, 23), ["cyclic", "cyclic", "rigid", "rigid"], True, solvers.impl, 3),
    ((15, 13, 17), ["cyclic"] * 4 + ["gndsky"] * 2, True, solvers.impl, 1),
    ((13, 15, 14), ["cyclic"] * 4 + ["gndsky"] * 2, False, solvers.expl, 2),
]


@pytest.mark.parametrize("grid,bcs,impl_tht,vab,prs_k", FORCED)
def test_boussinesq_forcings_fp64_match_oracle(grid, bcs, impl_tht, vab, prs_k):
    """impl_tht (boussinesq_impl.hpp), the velocity absorber in its explicit and
    implicit forms (mpdata_rhs_vip_common.hpp:182-256, normalised Laplacian of
    mpdata_rhs_vip_prs_common.hpp:49-84), the theta absorber and heat flux, and the
    3D ground/sky boundary (gndsky_3d.hpp): FP64 against the oracle after every step
    with identical GCR iteration counts."""
    s = forced_bq(grid, bcs, seed=len(grid) * 7 + prs_k, impl_tht=impl_tht, vip_vab=vab)
    s["prs_k"] = prs_k
    orc = bq_oracle(s)
    run = bq_run(s)
    for step in range(5):
        orc.advance(1)
        run.advance(1)
        st = run.stats()
        assert st["gcr_iters"] == orc.last_iters, (step, st["gcr_iters"], orc.last_iters)
        for e in range(len(grid) + 1):
            assert rel_err(run.advectee(e), orc.advectee(e)) <= RTOL64, (step, e)


def test_vab_accessors_need_the_option():
    s = random_bq((17, 15), ["cyclic", "cyclic", "rigid", "rigid"], seed=3)
    run = bq_run(s)
    with pytest.raises(_lib.MpdxError, match="vip_vab unset"):
        run.vab_coefficient()
