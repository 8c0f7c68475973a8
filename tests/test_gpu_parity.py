"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

FP64 results must match the oracle to 1e-12 relative (max |gpu - oracle| /
max |oracle|), as the reference's own solver would on the same inputs; FP32
results are compared with a tolerance stated per test and their error
against an FP64 run is reported."""
import numpy as np
import pytest

from libmpdataxx_b200 import bcond, concurr, opts as o, setups, solvers
from oracle import Oracle
from runners import load

pytestmark = pytest.mark.gpu

RTOL64 = 1e-12


def make_run(grid, opts, n_iters=2, n_eqns=1, bcs=None, dtype=np.float64, path="general", max_abs_div_eps=None,
             upwind_filter_freq=0, sptl_intrp=0):
    nd = len(grid)

    class ct(solvers.ct_params_default_t):
        pass

    ct.sptl_intrp = sptl_intrp
    ct.real_t = dtype
    ct.n_dims = nd
    ct.n_eqns = n_eqns
    ct.opts = opts
    p = solvers.mpdata.rt_params_t(grid_size=list(grid), n_iters=n_iters, max_abs_div_eps=max_abs_div_eps,
                                   upwind_filter_freq=upwind_filter_freq)
    bcs = bcs or ["cyclic"] * (2 * nd)
    return concurr.cuda(solvers.mpdata(ct), *[getattr(bcond, b) for b in bcs], p=p, path=path)


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def random_setup(grid, bcs, seed, signed=False):
    rng = np.random.default_rng(seed)
    nd = len(grid)
    psi = rng.uniform(0.5, 2.0, size=grid)
    if signed:
        psi = psi * np.where(rng.uniform(size=grid) < 0.3, -1.0, 1.0)
    if nd == 1:
        adv = [np.full(grid, 0.4)]
    elif nd == 2:
        adv = list(setups.periodic_curl_2d(grid[0], grid[1], seed, cmax=0.45))
    else:
        assert grid[0] == grid[1] == grid[2]
        adv = list(setups.periodic_curl_3d(grid[0], seed, cmax=0.3, dtype=np.float64))
    if all(b == "cyclic" for b in bcs):
        psi = setups.wrap_periodic(psi[tuple(slice(0, g - 1) for g in grid)])
    return {"grid": tuple(grid), "bcs": bcs, "advectee": [psi], "advector": adv}


CASES = []
for nd, grid in [(1, (37,)), (2, (19, 23)), (3, (13, 13, 13))]:
    for bc in ("cyclic", "open", "rigid"):
        for opts, iters in [(0, 1), (0, 2), (o.fct, 2), (o.iga, 2), (o.iga | o.fct, 2), (o.fct, 3), (0, 3),
                            (o.abs, 2), (o.abs | o.fct, 2), (o.pfc, 2), (o.npa | o.fct, 2)]:
            CASES.append((nd, grid, bc, opts, iters))
CASES.append((1, (37,), "cyclic", o.iga | o.tot, 2))
CASES.append((1, (37,), "open", o.iga | o.tot | o.fct, 2))
CASES.append((1, (37,), "cyclic", o.tot, 3))
# third-order terms in 2D and 3D (formulae_mpdata_hot_{2,3}d.hpp)
for nd, grid in [(2, (19, 23)), (3, (13, 13, 13))]:
    for bc in ("cyclic", "open", "rigid"):
        for opts, iters in [(o.iga | o.tot, 2), (o.tot, 2), (o.abs | o.tot, 2), (o.iga | o.tot | o.fct, 2),
                            (o.tot | o.fct, 3)]:
            CASES.append((nd, grid, bc, opts, iters))

# divergent-flow correction (formulae_mpdata_dfl_{1,2,3}d.hpp) on a divergent advector
DFL_CASES = []
for nd, grid in [(1, (37,)), (2, (19, 23)), (3, (13, 13, 13))]:
    for bc in ("cyclic", "open", "rigid"):
        for opts, iters in [(o.dfl, 2), (o.iga | o.dfl, 2), (o.dfl | o.fct, 2), (o.iga | o.dfl | o.fct, 2),
                            (o.dfl, 3), (o.iga | o.tot | o.dfl | o.fct, 3)]:
            DFL_CASES.append((nd, grid, bc, opts, iters))


@pytest.mark.parametrize("nd,grid,bc,opts,iters", DFL_CASES)
def test_dfl_fp64_matches_oracle(nd, grid, bc, opts, iters):
    bcs = [bc] * (2 * nd)
    s = random_setup(grid, bcs, seed=nd * 100 + iters + 7, signed=bool(opts & o.iga))
    rng = np.random.default_rng(nd * 10 + iters)
    s["advector"] = [a + 0.05 * rng.uniform(-1.0, 1.0, np.shape(a)) for a in s["advector"]]
    _check_parity(s, grid, bcs, opts, iters, eps=None)


# non-unit G (nug, with a spatially varying G), Kahan donor-cell sums (khn) and the upwind filter
NUG_CASES = []
for nd, grid in [(1, (37,)), (2, (19, 23)), (3, (13, 13, 13))]:
    for bc in ("cyclic", "open", "rigid"):
        for opts, iters in [(o.nug, 2), (o.nug | o.iga | o.fct, 2), (o.nug | o.fct, 3), (o.nug | o.tot | o.fct, 2),
                            (o.nug | o.iga | o.tot, 3), (o.khn, 2), (o.khn | o.nug | o.fct, 2)]:
            NUG_CASES.append((nd, grid, bc, opts, iters))


@pytest.mark.parametrize("nd,grid,bc,opts,iters", NUG_CASES)
def test_nug_khn_fp64_matches_oracle(nd, grid, bc, opts, iters):
    bcs = [bc] * (2 * nd)
    s = random_setup(grid, bcs, seed=nd * 100 + iters + 3, signed=bool(opts & o.iga))
    rng = np.random.default_rng(nd + iters)
    G = rng.uniform(0.7, 1.3, grid)
    if bc == "cyclic":
        G = setups.wrap_periodic(G[tuple(slice(0, g - 1) for g in grid)])
    if opts & o.nug:
        s["G"] = G
    _check_parity(s, grid, bcs, opts, iters, eps=1e30 if bc == "rigid" else 1e-10)


@pytest.mark.parametrize("nd,grid", [(1, (37,)), (2, (19, 23)), (3, (13, 13, 13))])
@pytest.mark.parametrize("opts,iters,uff", [(o.iga | o.fct, 2, 2), (o.fct, 3, 3), (0, 2, 1)])
def test_upwind_filter_fp64_matches_oracle(nd, grid, opts, iters, uff):
    bcs = ["cyclic"] * (2 * nd)
    s = random_setup(grid, bcs, seed=nd * 100 + iters + 5, signed=bool(opts & o.iga))
    _check_parity(s, grid, bcs, opts, iters, eps=1e-10, uff=uff)


def test_g_factor_needs_nug():
    run = make_run((8, 8), o.fct)
    with pytest.raises(RuntimeError, match="g_factor"):
        run.set_g_factor(np.ones((8, 8)))


@pytest.mark.parametrize("nd,grid,bc,opts,iters", CASES)
def test_general_path_fp64_matches_oracle(nd, grid, bc, opts, iters):
    bcs = [bc] * (2 * nd)
    s = random_setup(grid, bcs, seed=nd * 100 + iters, signed=bool(opts & (o.abs | o.iga)))
    # rigid walls mirror the normal Courant number with a sign flip, so a field that
    # is not zero on the wall faces fails the reference's divergence guard; the
    # guard is lifted for those cases (the numerics under test do not depend on it)
    _check_parity(s, grid, bcs, opts, iters, eps=1e30 if bc == "rigid" else 1e-10)


def _check_parity(s, grid, bcs, opts, iters, eps, uff=0, sptl=0):
    orc = Oracle(grid, opts, n_iters=iters, bcs=bcs, max_abs_div_eps=eps, upwind_filter_freq=uff)
    if sptl:
        orc.set_param("sptl_intrp", sptl)
    load(orc, s)
    run = make_run(grid, opts, n_iters=iters, bcs=bcs, max_abs_div_eps=eps, upwind_filter_freq=uff, sptl_intrp=sptl)
    run.set_advectee(s["advectee"][0])
    for d, a in enumerate(s["advector"]):
        run.set_advector(a, d)
    if "G" in s:
        orc.set_g_factor(s["G"])
        run.set_g_factor(s["G"])
    for chunk in (1, 4):
        orc.advance(chunk)
        run.advance(chunk)
        assert rel_err(run.advectee(), orc.advectee()) <= RTOL64


def test_advector_view_roundtrip():
    grid = (6, 7, 5)
    run = make_run(grid, o.fct, max_abs_div_eps=1.0)
    rng = np.random.default_rng(0)
    for d in range(3):
        a = rng.normal(size=run._shape(1, d))
        run.set_advector(a, d)
        np.testing.assert_array_equal(run.advector(d), a)


def test_mirror_semantics():
    """advectee() is a writable mirror: writes are seen by the next advance."""
    s = setups.cone_bugs()
    run = make_run(s["grid"], o.fct)
    run.advectee()[...] = s["advectee"][0]
    run.advector(0)[...] = s["advector"][0]
    run.advector(1)[...] = s["advector"][1]
    run.advance(2)
    orc = Oracle(s["grid"], o.fct, bcs=s["bcs"])
    load(orc, s)
    orc.advance(2)
    assert rel_err(run.advectee(), orc.advectee()) <= RTOL64


def test_divergent_advector_raises():
    s = setups.cone_bugs()
    run = make_run(s["grid"], o.fct)
    run.set_advectee(s["advectee"][0])
    run.set_advector(s["advector"][0] + np.linspace(0, 0.1, s["grid"][0])[:, None], 0)
    run.set_advector(s["advector"][1], 1)
    with pytest.raises(RuntimeError, match="initial advector field is divergent"):
        run.advance(1)


def test_cone_bugs_fp32_exact_min():
    """tests/unit/cone_bugs: FP32 fct never goes below the background."""
    s = setups.cone_bugs()
    run = make_run(s["grid"], o.fct, dtype=np.float32)
    run.set_advectee(s["advectee"][0])
    for d, a in enumerate(s["advector"]):
        run.set_advector(a, d)
    run.advance(s["nt"])
    assert run.advectee().min() - 1 == 0


def test_stats_mass_conserved():
    grid = (33, 33)
    s = random_setup(grid, ["cyclic"] * 4, seed=7)
    run = make_run(grid, o.iga | o.fct, max_abs_div_eps=1e-10)
    run.set_advectee(s["advectee"][0])
    for d, a in enumerate(s["advector"]):
        run.set_advector(a, d)
    m0 = run.stats()["mass"]
    run.advance(20)
    st = run.stats()
    assert st["timestep"] == 20
    assert abs(st["mass"] - m0) <= 1e-12 * abs(m0)
    psi = run.advectee()
    assert st["min"] == psi.min() and st["max"] == psi.max()


# divergence-form MPDATA: div_2nd, div_3rd, div_3rd_dt (formulae_mpdata_{1,2,3}d.hpp,
# formulae_mpdata_fdiv_{1,2,3}d.hpp), with the gauges, FCT, nug and the spatial helpers
DIV_CASES = []
for nd, grid in [(1, (37,)), (2, (19, 23)), (3, (13, 13, 13))]:
    for bc in ("cyclic", "open", "rigid"):
        for opts, iters, sptl in [(o.div_2nd, 2, 0), (o.div_2nd | o.div_3rd, 2, 0), (o.iga | o.div_2nd | o.div_3rd, 2, 1),
                                  (o.abs | o.div_2nd | o.div_3rd, 2, 2), (o.div_2nd | o.div_3rd_dt, 2, 0),
                                  (o.iga | o.fct | o.div_2nd | o.div_3rd_dt, 2, 0), (o.fct | o.div_2nd | o.div_3rd, 2, 1),
                                  (o.nug | o.div_2nd | o.div_3rd, 2, 0), (o.nug | o.iga | o.div_2nd | o.div_3rd_dt, 2, 1)]:
            DIV_CASES.append((nd, grid, bc, opts, iters, sptl))


@pytest.mark.parametrize("nd,grid,bc,opts,iters,sptl", DIV_CASES)
def test_div_fp64_matches_oracle(nd, grid, bc, opts, iters, sptl):
    bcs = [bc] * (2 * nd)
    s = random_setup(grid, bcs, seed=nd * 100 + iters + 11, signed=bool(opts & (o.abs | o.iga)))
    if opts & o.nug:
        rng = np.random.default_rng(nd + iters + 1)
        G = rng.uniform(0.7, 1.3, grid)
        if bc == "cyclic":
            G = setups.wrap_periodic(G[tuple(slice(0, g - 1) for g in grid)])
        s["G"] = G
    _check_parity(s, grid, bcs, opts, iters, eps=1e30 if bc == "rigid" else 1e-10, sptl=sptl)


def test_div_options_validated():
    from libmpdataxx_b200 import _lib
    for opts in (o.div_3rd, o.div_2nd | o.div_3rd | o.div_3rd_dt, o.div_2nd | o.tot):
        with pytest.raises(_lib.MpdxError):
            make_run((9, 9), opts)
    # a third pass would read halo faces of the second pass's velocities that the reference
    # never fills (its result there depends on uninitialised memory)
    for opts in (o.div_2nd, o.fct | o.div_2nd | o.div_3rd):
        with pytest.raises(_lib.MpdxError):
            make_run((9, 9), opts, n_iters=3)


@pytest.mark.parametrize("opts,iters,uff", [(0, 2, 0), (o.iga, 2, 0), (0, 3, 0), (o.abs, 2, 0), (o.tot, 2, 0),
                                            (o.iga | o.tot, 3, 0), (o.npa | o.pfc, 2, 0), (o.khn, 2, 0), (0, 2, 3)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_block1d_equals_general_path(opts, iters, uff, dtype):
    """Cyclic 1D problems advance in one launch of one block (all steps of an
    advance() call, fields in shared memory) with the per-point arithmetic of the
    multi-kernel path: equal to it bit for bit, and to the oracle in FP64."""
    grid = (2000,)
    s = setups.box_1d()
    s["advectee"][0] = s["advectee"][0].astype(dtype)
    runs = {}
    for path in ("general", "auto"):
        r = make_run(grid, opts, n_iters=iters, dtype=dtype, path=path, upwind_filter_freq=uff)
        r.set_advectee(s["advectee"][0])
        r.set_advector(s["advector"][0].astype(dtype), 0)
        runs[path] = r
    for chunk in (13, 7):
        for r in runs.values():
            r.advance(chunk)
        np.testing.assert_array_equal(runs["auto"].advectee(), runs["general"].advectee())
    from libmpdataxx_b200 import _lib
    assert runs["auto"].stats()["path"] == _lib.PATH_FUSED and runs["general"].stats()["path"] == _lib.PATH_GENERAL
    if dtype == np.float64:
        orc = Oracle(grid, opts, n_iters=iters, bcs=["cyclic"] * 2, upwind_filter_freq=uff)
        load(orc, s)
        orc.advance(20)
        assert rel_err(runs["auto"].advectee(), orc.advectee()) <= RTOL64


FOT_CASES = [(bc, opts, iters) for bc in ("cyclic", "open", "rigid")
             for opts, iters in ((o.iga | o.tot | o.fot, 2), (o.iga | o.tot | o.fot, 3), (o.iga | o.tot | o.fot | o.fct, 2),
                                 (o.iga | o.div_2nd | o.div_3rd | o.fot, 2))]


@pytest.mark.parametrize("bc,opts,iters", FOT_CASES)
def test_fot_fp64_matches_oracle(bc, opts, iters):
    """Fourth-order terms (2D, iga with tot or div_3rd): the general path against the oracle."""
    grid = (23, 19)
    bcs = [bc] * 4
    s = random_setup(grid, bcs, seed=iters + 7, signed=True)
    _check_parity(s, grid, bcs, opts, iters, eps=1e30 if bc == "rigid" else 1e-10)


def test_fot_convergence_order_on_gpu():
    """The reference's convergence check of fot (tests/sandbox/convergence_2d_3d/convergence_2d.cpp)
    through the GPU path: order 4 for iga|tot|fot, 3 for iga|tot."""
    def err(opts, np_):
        dx = 1.0 / (np_ - 1)
        dt = 0.2 * dx
        i, j = np.meshgrid(np.arange(np_), np.arange(np_), indexing="ij")
        psi = 2 + np.sin(2 * np.pi * i * dx) * np.sin(2 * np.pi * j * dx)
        run = make_run((np_, np_), opts, n_iters=2, bcs=["cyclic"] * 4)
        run.set_advectee(psi)
        run.set_advector(np.full(run._shape(1, 0), 1.0 * dt / dx), 0)
        run.set_advector(np.full(run._shape(1, 1), 2.0 * dt / dx), 1)
        run.advance(int(1.0 / dt))
        return float(np.sqrt(((run.advectee() - psi) ** 2).sum() / (np_ * np_)))
    for opts, order in ((o.iga | o.tot, 3), (o.iga | o.tot | o.fot, 4)):
        assert round(np.log2(err(opts, 33) / err(opts, 65))) == order
