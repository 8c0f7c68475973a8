"""GCR with the learned preconditioner inside the Boussinesq solver.

Pairs recorded from plain solves train the network on the GPU; with it
enabled every pressure solve stops at the same tolerance and the flow stays the
one plain GCR produces (to the solver tolerance).  A learned solve that has run
as long as the last plain solve hands over to plain directions."""
import numpy as np
import pytest

from libmpdataxx_b200 import setups
from runners import bq_run

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def bubble(n=(48, 48, 24)):
    return setups.boussinesq_bubble_3d(*n)


@pytest.mark.parametrize("dtype,prs_fp64", [(np.float64, False), (np.float32, True)])
def test_learned_gcr_reaches_same_tolerance_and_flow(dtype, prs_fp64):
    """Record pairs from plain solves, train on the GPU, enable: every learned
    solve must end at the reference's stopping test (max|err| <= prs_tol / dt)
    and give the flow plain GCR gives.  The held-out training loss of the weights
    kept must fall below that of no correction."""
    s = bubble()
    plain = bq_run(s, dtype=dtype, prs_fp64=prs_fp64)
    learn = bq_run(s, dtype=dtype, prs_fp64=prs_fp64)
    learn.precond_record(40)
    plain.advance(12)
    learn.advance(12)
    assert 12 < learn.precond_pairs() <= 40  # initial residuals plus later iterations of each solve
    loss = learn.precond_train(300, lr=2e-3)
    print("held-out training loss (relative energy of the error, 1 = no correction)", loss)
    assert loss < 1.0  # the weights kept improve on the zero-output start
    learn.precond_enable(True)
    tol = s["prs_tol"] / s["dt"]
    it_p, it_l, ms_p, ms_l = [], [], [], []
    for _ in range(4):
        plain.advance(1)
        learn.advance(1)
        sp, sl = plain.stats(), learn.stats()
        it_p.append(sp["gcr_iters"]); ms_p.append(sp["gcr_ms"])
        it_l.append(sl["gcr_iters"]); ms_l.append(sl["gcr_ms"])
        assert sl["gcr_residual"] <= tol * (1 + 1e-6) and sp["gcr_residual"] <= tol * (1 + 1e-6)
    print("iterations plain", it_p, "learned", it_l, "ms plain", ms_p, "learned", ms_l)
    for e in range(4):
        a, b = learn.advectee(e).astype(np.float64), plain.advectee(e).astype(np.float64)
        scale = np.abs(b).max() if e < 3 else 1.0
        # velocities within 1e-3 of their scale, theta (about 300 K; an FP32 ulp is
        # 3e-5 K) within 5e-4 K: both runs stop at the same tolerance, not at the same bits
        assert np.abs(a - b).max() <= (1e-3 * max(scale, 1e-3) if e < 3 else 5e-4), e


def test_learned_corrections_keep_cyclic_duplicates():
    """On a cyclic axis point n-1 duplicates point 0; the learned corrections
    (whose network pads cyclic axes with period n) must keep Phi's duplicate
    planes equal, as plain GCR's directions do, or the projected velocity differs
    across the seam (the flow then loses its FCT bounds over a few hundred steps)."""
    s = bubble((24, 20, 12))
    run = bq_run(s, dtype=np.float64)
    run.precond_record(20)
    run.advance(5)
    run.precond_train(60, lr=2e-3)
    run.precond_enable(True)
    run.precond_set_directions(2)
    run.advance(3)
    assert run.precond_directions() == 2
    from libmpdataxx_b200 import _lib
    phi = np.empty(tuple(s["grid"]), dtype=np.float64)
    assert run.L.mpdx_get_field(run.h, _lib.FIELD_PRESSURE, 0, phi.ctypes.data, None) == 0
    np.testing.assert_array_equal(phi[-1], phi[0])
    np.testing.assert_array_equal(phi[:, -1], phi[:, 0])
    # the count chosen by solve time: the first solves try the candidates in turn
    run.precond_set_directions(-1)
    run.advance(2)
    assert run.precond_directions() == 1
    with pytest.raises(RuntimeError):
        run.precond_set_directions(-2)


def test_learned_corrections_reduce_iterations():
    """What the trained network gains: on the 3D bubble (96 x 96 x 48, FP32
    advection, FP64 GCR to prs_tol / dt), one learned correction at the start of
    every solve, after 60 recorded plain solves and 300 Adam steps, needs fewer
    GCR iterations per solve (learned correction included) than plain GCR over
    the same steps; device times are printed."""
    s = setups.boussinesq_bubble_3d(96, 96, 48)
    plain = bq_run(s, dtype=np.float32, prs_fp64=True)
    learn = bq_run(s, dtype=np.float32, prs_fp64=True)
    learn.precond_record(240)
    plain.advance(60)
    learn.advance(60)
    loss = learn.precond_train(300, lr=1e-3)
    learn.precond_enable(True)  # one learned correction per solve (the default)
    it_p, it_l, ms_p, ms_l = [], [], [], []
    tol = s["prs_tol"] / s["dt"]
    for _ in range(40):
        plain.advance(1)
        learn.advance(1)
        sp, sl = plain.stats(), learn.stats()
        assert sl["gcr_residual"] <= tol * (1 + 1e-6)
        it_p.append(sp["gcr_iters"]); ms_p.append(sp["gcr_ms"])
        it_l.append(sl["gcr_iters"]); ms_l.append(sl["gcr_ms"])
    mp, ml = float(np.mean(it_p[-20:])), float(np.mean(it_l[-20:]))
    print(f"held-out loss {loss:.3f}; last 20 solves: plain {mp:.1f} iterations {np.mean(ms_p[-20:]):.2f} ms, "
          f"learned {ml:.1f} iterations {np.mean(ms_l[-20:]):.2f} ms")
    assert ml < 0.9 * mp


def test_training_loss_and_gradient_match_oracle():
    """The energy-norm training loss and its gradient with respect to every layer,
    the pressure operator and its exact adjoint on the rigid walls included,
    against the float64 oracle (BF16 activations: 3e-2 on the loss, 5e-2 on the
    gradients, as for the network alone)."""
    import precond_oracle as po
    from libmpdataxx_b200.precond import pack, unpack
    s = bubble((24, 20, 12))
    run = bq_run(s)
    ch = (8, 16, 32, 64)
    P = unpack(run.precond_params(), 3, ch)
    rng = np.random.default_rng(6)
    P["W_q"] = rng.normal(size=P["W_q"].shape) / np.sqrt(P["W_q"].shape[1] * P["W_q"].shape[2])
    run.set_precond_params(pack(P, 3, ch))
    P = unpack(run.precond_params(), 3, ch)
    grid = s["grid"]
    r = rng.normal(size=grid)
    t = rng.normal(size=grid)
    c = 0.8
    loss, g = run.precond_loss_grad(r, t, c)
    rigid = ((False, False), (False, False), (True, True))
    E, G = po.energy_loss(P, r, t, c, grid, (True, True, False), rigid, s["dx"], ch)
    print("loss", loss, E)
    assert abs(loss - E) <= 3e-2 * abs(E)
    gu = unpack(g, 3, ch)
    for name in ["W_e0", "W_e2", "W_m3", "W_d1", "W_d0", "W_q"]:
        print(name, "grad rel err", rel(gu[name], G[name]))
        assert rel(gu[name], G[name]) <= 5e-2, name
    # a zero output gives loss 1 exactly (up to FP32 sums)
    P0 = dict(P)
    P0["W_q"] = np.zeros_like(P["W_q"])
    run.set_precond_params(pack(P0, 3, ch))
    l0, _ = run.precond_loss_grad(r, t, c, grad=False)
    assert abs(l0 - 1.0) <= 1e-5


def test_precond_params_roundtrip_and_requires_fp64():
    s = bubble((24, 24, 12))
    run = bq_run(s)
    p = run.precond_params()
    p2 = p * 0.5
    run.set_precond_params(p2)
    np.testing.assert_array_equal(run.precond_params(), p2)
    r32 = bq_run(s, dtype=np.float32)  # FP32 pressure solve: no learned preconditioner
    with pytest.raises(RuntimeError, match="FP64 pressure"):
        r32.precond_record(2)
    with pytest.raises(RuntimeError, match="no recorded"):
        run.precond_train(5)
