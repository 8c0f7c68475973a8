"""The oracle's third-order terms (tot) and divergent-flow correction (dfl)
across dimensions.

No golden data of the reference pins dfl, nor tot in 3D (the rotating-cone
goldens pin tot in 2D, test_oracle_golden.py).  These restatements are checked
for consistency instead: a problem that is uniform along y (and z), with zero
transverse Courant numbers, must evolve exactly as the 1D problem does -- the
2D/3D formulae (formulae_mpdata_{hot,dfl}_{2,3}d.hpp) reduce to the 1D ones
(formulae_mpdata_{hot,dfl}_1d.hpp) when every transverse difference vanishes,
and they do so bit for bit because the extra terms are exact zeros and the
constant factors (-0.5/2 against -0.25/1, 0.5 (a + b) against (a + b)/2) round
identically.  The transverse boundaries are cyclic: an open boundary fills its
halo faces by the zero-divergence condition (open_2d.hpp fill_halos_vctr_alng),
which makes the transverse Courant numbers of a divergent flow non-zero there.
Along x an open boundary fills 1D and 2D halos differently as well (open_1d.hpp
copies the boundary face, open_2d.hpp the first inner face), so with open x
boundaries only rows out of the boundaries' reach are compared."""
import numpy as np
import pytest

from libmpdataxx_b200 import opts as o
from oracle import Oracle

NX = 29
CASES = [(o.dfl, 2), (o.iga | o.dfl, 2), (o.dfl | o.fct, 2), (o.iga | o.dfl | o.fct, 2), (o.dfl, 3),
         (o.tot, 2), (o.iga | o.tot, 2), (o.abs | o.tot, 2), (o.tot | o.fct, 3), (o.iga | o.tot | o.dfl | o.fct, 2)]


def _problem(seed, signed):
    rng = np.random.default_rng(seed)
    psi = rng.uniform(0.5, 2.0, NX)
    if signed:
        psi *= np.where(rng.uniform(size=NX) < 0.3, -1.0, 1.0)
    x = np.arange(NX) / (NX - 1)
    gc = 0.25 + 0.1 * np.sin(2 * np.pi * x) + 0.05 * rng.uniform(-1, 1, NX)  # divergent
    return psi, gc


def _run(grid, bc, opts, iters, psi1, gc1, nt):
    nd = len(grid)
    orc = Oracle(grid, opts, n_iters=iters, bcs=[bc] * 2 + ["cyclic"] * (2 * nd - 2), max_abs_div_eps=1e30)
    orc.set_advectee(np.broadcast_to(psi1.reshape((NX,) + (1,) * (nd - 1)), grid))
    orc.set_advector(np.broadcast_to(gc1.reshape((NX,) + (1,) * (nd - 1)), grid), 0)
    for d in range(1, nd):
        orc.set_advector(np.zeros(orc.advector_shape(d)), d)
    orc.advance(nt)
    out = orc.advectee()
    return out.reshape(NX, -1) if nd > 1 else out.reshape(NX, 1)


@pytest.mark.parametrize("bc", ["open", "cyclic"])
@pytest.mark.parametrize("opts,iters", CASES)
def test_uniform_transverse_reduces_to_1d(opts, iters, bc):
    psi, gc = _problem(seed=iters * 31 + opts % 97, signed=bool(opts & (o.abs | o.iga)))
    nt, rows = (6, slice(None)) if bc == "cyclic" else (2, slice(12, NX - 12))
    ref = _run((NX,), bc, opts, iters, psi, gc, nt=nt)
    for grid in [(NX, 5), (NX, 4, 5)]:
        got = _run(grid, bc, opts, iters, psi, gc, nt=nt)
        for col in range(got.shape[1]):
            np.testing.assert_array_equal(got[rows, col], ref[rows, 0])


def test_dfl_changes_the_result():
    """The correction is active: a divergent flow gives a different answer with dfl."""
    psi, gc = _problem(seed=5, signed=False)
    a = _run((NX, 5), "open", o.iga, 2, psi, gc, nt=6)
    b = _run((NX, 5), "open", o.iga | o.dfl, 2, psi, gc, nt=6)
    assert np.abs(a - b).max() > 1e-6


def test_tot_changes_the_result():
    psi, gc = _problem(seed=6, signed=False)
    a = _run((NX, 4, 5), "cyclic", o.fct, 2, psi, gc, nt=6)
    b = _run((NX, 4, 5), "cyclic", o.tot | o.fct, 2, psi, gc, nt=6)
    assert np.abs(a - b).max() > 1e-6


# ---- nug: non-unit G (formulae_mpdata_g_{1,2,3}d.hpp, donorcell_sum / G, betas * G) ----
def _run_g(grid, opts, iters, psi, adv, G=None, nt=4, bcs=None):
    nd = len(grid)
    orc = Oracle(grid, opts, n_iters=iters, bcs=bcs or ["cyclic"] * (2 * nd), max_abs_div_eps=1e30)
    orc.set_advectee(psi)
    for d, a in enumerate(adv):
        orc.set_advector(a, d)
    if G is not None:
        orc.set_g_factor(G)
    orc.advance(nt)
    return orc.advectee()


def _random_2d(seed, grid=(17, 19)):
    rng = np.random.default_rng(seed)
    psi = rng.uniform(0.5, 2.0, grid)
    adv = [rng.uniform(-0.3, 0.3, (grid[0], grid[1])), rng.uniform(-0.3, 0.3, (grid[0] + 1, grid[1]))]
    return psi, adv


@pytest.mark.parametrize("opts,iters", [(0, 2), (o.iga | o.fct, 2), (o.tot | o.fct, 3), (o.iga | o.dfl, 2), (o.khn, 2)])
def test_nug_with_unit_g_is_plain(opts, iters):
    """G = 1 everywhere gives the no-nug result bit for bit (every G factor is an exact 1)."""
    psi, adv = _random_2d(1)
    a = _run_g(psi.shape, opts, iters, psi, adv)
    b = _run_g(psi.shape, opts | o.nug, iters, psi, adv, G=np.ones(psi.shape))
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("opts,iters", [(0, 2), (o.iga, 2), (o.tot, 2), (o.iga | o.tot, 3), (o.dfl, 2),
                                        (o.iga | o.dfl, 2), (o.abs | o.tot, 2), (o.npa, 2), (o.pfc, 3)])
@pytest.mark.parametrize("nd", [1, 2, 3])
def test_nug_constant_g_scales_courant_numbers(opts, iters, nd):
    """With G = 2 everywhere the scheme equals the no-nug scheme on the advector C/2, bit
    for bit: every G factor then rescales by an exact power of two.  (Not with fct, whose
    beta denominators add an unscaled epsilon.)"""
    rng = np.random.default_rng(nd * 7 + iters)
    grid = {1: (23,), 2: (13, 15), 3: (9, 10, 11)}[nd]
    psi = rng.uniform(0.5, 2.0, grid)
    if opts & o.abs:
        psi *= np.where(rng.uniform(size=grid) < 0.3, -1.0, 1.0)
    adv = []
    for d in range(nd):
        s = list(grid)
        if d > 0:
            s[0] += 1
        adv.append(rng.uniform(-0.6, 0.6, s))
    a = _run_g(grid, opts, iters, psi, [x / 2 for x in adv])
    b = _run_g(grid, opts | o.nug, iters, psi, adv, G=np.full(grid, 2.0))
    np.testing.assert_array_equal(a, b)


# ---- khn: Kahan-compensated donor-cell sums (donorcell_formulae.hpp:81-165) ----
def test_khn_close_to_plain_and_different():
    psi, adv = _random_2d(2)
    a = _run_g(psi.shape, o.iga | o.fct, 2, psi, adv)
    b = _run_g(psi.shape, o.iga | o.fct | o.khn, 2, psi, adv)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
    assert np.abs(a - b).max() > 0


# ---- upwind_filter_freq (mpdata_osc_2d.hpp:176-179) ----
def test_upwind_filter_every_step_is_upwind():
    psi, adv = _random_2d(3)
    grid = psi.shape
    ref = Oracle(grid, o.fct, n_iters=1, max_abs_div_eps=1e30)
    uf = Oracle(grid, o.fct, n_iters=2, max_abs_div_eps=1e30, upwind_filter_freq=1)
    mp = Oracle(grid, o.fct, n_iters=2, max_abs_div_eps=1e30, upwind_filter_freq=2)
    for r in (ref, uf, mp):
        r.set_advectee(psi)
        for d, a in enumerate(adv):
            r.set_advector(a, d)
    for r in (ref, uf, mp):
        r.advance(1)
    np.testing.assert_array_equal(uf.advectee(), ref.advectee())
    np.testing.assert_array_equal(mp.advectee(), ref.advectee())  # timestep 0 is filtered
    for r in (ref, uf, mp):
        r.advance(1)
    np.testing.assert_array_equal(uf.advectee(), ref.advectee())
    assert np.abs(mp.advectee() - ref.advectee()).max() > 1e-6      # timestep 1 is full MPDATA


# ---- divergence-form MPDATA (div_2nd, div_3rd, div_3rd_dt) ----
# No golden data of the reference pins these options on a plain MPDATA set-up
# (its mp3 tests run them with var_dt and the nug geometry of the sphere).  The
# restatement of formulae_mpdata_{1,2,3}d.hpp / formulae_mpdata_fdiv_{1,2,3}d.hpp
# is checked against two properties instead:
#  * for a uniform flow the divergence form of the second-order antidiffusive
#    velocity is the standard one: in 1D for every gauge, and in 2D / 3D with
#    iga (where nfdiv's transverse psi averages are the ndy / ndz numerators);
#  * the third-order corrections reduce the error of a smooth translated field
#    several times against second order (third-order accuracy in space and time).
from libmpdataxx_b200 import setups  # noqa: E402

D2, D3, DT = o.div_2nd, o.div_3rd, o.div_3rd_dt


def _div_run(grid, opts, adv, psi, nt, sptl=None):
    orc = Oracle(grid, opts, n_iters=2, bcs=["cyclic"] * (2 * len(grid)), max_abs_div_eps=1e-6)
    if sptl is not None:
        orc.set_param("sptl_intrp", sptl)
    orc.set_advectee(psi)
    for d, a in enumerate(adv):
        orc.set_advector(a, d)
    orc.advance(nt)
    return orc.advectee()


@pytest.mark.parametrize("grid,base", [((41,), 0), ((41,), o.iga), ((41,), o.abs), ((23, 19), o.iga),
                                       ((13, 12, 11), o.iga), ((23, 19), o.iga | o.fct)])
def test_div_2nd_equals_standard_form_for_uniform_flow(grid, base):
    rng = np.random.default_rng(len(grid))
    psi = setups.wrap_periodic(rng.uniform(0.5, 2.0, size=tuple(g - 1 for g in grid)))
    adv = []
    for d in range(len(grid)):
        shp = list(grid)
        if d > 0:
            shp[0] += 1
        adv.append(np.full(shp, [0.3, -0.2, 0.15][d]))
    a = _div_run(grid, base, adv, psi, 3)
    b = _div_run(grid, base | D2, adv, psi, 3)
    np.testing.assert_allclose(b, a, rtol=0, atol=4e-15)


def _smooth_translation(n=65, nt=64, c=(0.25, 0.125)):
    P = n - 1
    X, Y = np.meshgrid(np.arange(P), np.arange(P), indexing="ij")

    def blob(sx, sy):
        d2 = np.minimum(np.abs(X - sx), P - np.abs(X - sx)) ** 2 + np.minimum(np.abs(Y - sy), P - np.abs(Y - sy)) ** 2
        return 1 + np.exp(-d2 / (2 * 6.0 ** 2))

    psi = setups.wrap_periodic(blob(20, 20))
    exact = setups.wrap_periodic(blob(20 + c[0] * nt, 20 + c[1] * nt))
    adv = [np.full((n, n), c[0]), np.full((n + 1, n), c[1])]
    return (n, n), adv, psi, exact, nt


@pytest.mark.parametrize("base", [0, o.iga])
def test_div_3rd_is_more_accurate_than_second_order(base):
    grid, adv, psi, exact, nt = _smooth_translation()
    err = lambda r: float(np.sqrt(((r - exact) ** 2).mean()))
    e2 = err(_div_run(grid, base | D2, adv, psi, nt))
    e3 = err(_div_run(grid, base | D2 | D3, adv, psi, nt))
    edt = err(_div_run(grid, base | D2 | DT, adv, psi, nt))
    assert e3 < 0.35 * e2 and edt < 0.2 * e2, (e2, e3, edt)
    # the spatial helper (exact, aver2, aver4) multiplies ndxx_GC0, zero in a uniform flow
    for sp in (1, 2):
        assert err(_div_run(grid, base | D2 | D3, adv, psi, nt, sptl=sp)) == e3


def test_div_third_pass_refused():
    """With n_iters = 3 the third pass of the divergence form reads faces of the second
    pass's velocities GC_corr(1) that no exchange fills (mpdata_osc_2d.hpp:112-121), so
    the reference's result would depend on uninitialised memory: the oracle refuses."""
    for opts in (D2, D2 | D3, o.fct | D2 | DT):
        with pytest.raises(RuntimeError, match="n_iters"):
            Oracle((9, 9), opts, n_iters=3, bcs=["cyclic"] * 4)


def _convergence_2d(opts, iters, np_):
    """The reference's 2D convergence set-up (tests/sandbox/convergence_2d_3d/convergence_2d.cpp:18-64):
    np x np cyclic points, dx = dy = 1 / (np - 1), dt = 0.2 dx, psi = 2 + sin(2 pi i dx) sin(2 pi j dy),
    velocity (1, 2) (Courant numbers 0.2, 0.4), int(1 / dt) steps; the L2 error against the start
    divided by the time (1)."""
    dx = 1.0 / (np_ - 1)
    dt = 0.2 * dx
    nt = int(1.0 / dt)
    i, j = np.meshgrid(np.arange(np_), np.arange(np_), indexing="ij")
    psi = 2 + np.sin(2 * np.pi * i * dx) * np.sin(2 * np.pi * j * dx)
    orc = Oracle((np_, np_), opts, n_iters=iters, bcs=["cyclic"] * 4)
    orc.set_advectee(psi)
    orc.set_advector(np.full(orc.advector_shape(0), 1.0 * dt / dx), 0)
    orc.set_advector(np.full(orc.advector_shape(1), 2.0 * dt / dx), 1)
    orc.advance(nt)
    return float(np.sqrt(((orc.advectee() - psi) ** 2).sum() / (np_ * np_)))


@pytest.mark.parametrize("opts,iters,order", [(0, 2, 2), (o.iga | o.fct, 2, 2), (o.tot, 3, 3), (o.abs | o.tot, 3, 3),
                                              (o.iga | o.tot, 2, 3), (o.iga | o.tot | o.fot, 2, 4)])
def test_convergence_order_2d(opts, iters, order):
    """The reference's own check of the fourth-order terms (fot) and of the lower
    orders (tests/sandbox/convergence_2d_3d/convergence_2d.cpp:66-124): the order
    round(log2(err(33) / err(65))) of each option set."""
    assert round(np.log2(_convergence_2d(opts, iters, 33) / _convergence_2d(opts, iters, 65))) == order


def test_fot_rules():
    """fot needs iga and tot or div_3rd in 2D (formulae_mpdata_hot_2d.hpp:147-149);
    the 1D and 3D formulae never add fourth-order terms."""
    for bad in (o.fot, o.fot | o.tot, o.fot | o.iga):
        with pytest.raises(RuntimeError, match="fot"):
            Oracle((9, 9), bad, n_iters=2, bcs=["cyclic"] * 4)
    rng = np.random.default_rng(3)
    psi = rng.uniform(0.5, 2.0, 20)
    psi[-1] = psi[0]
    runs = []
    for opts in (o.iga | o.tot, o.iga | o.tot | o.fot):
        orc = Oracle((20,), opts, n_iters=2, bcs=["cyclic"] * 2)
        orc.set_advectee(psi)
        orc.set_advector(np.full(orc.advector_shape(0), 0.3), 0)
        orc.advance(5)
        runs.append(orc.advectee())
    np.testing.assert_array_equal(runs[0], runs[1])
