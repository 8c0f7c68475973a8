"""The preconditioner network's CPU oracle: its analytic gradients must agree
with finite differences (this pins the oracle before it checks the GPU)."""
import numpy as np
import pytest

import precond_oracle as po


@pytest.mark.parametrize("grid,wrap", [((9, 7, 6), (True, True, False)), ((11, 10), (True, False, False))])
def test_gradients_match_finite_differences(grid, wrap):
    nd = len(grid)
    ch = (2, 3, 4, 5)
    P = po.init_params(nd, ch, seed=1)
    rng = np.random.default_rng(2)
    for k in P:
        if k.startswith("b_"):
            P[k] = rng.normal(size=P[k].shape) * 0.1
    r = rng.normal(size=grid)
    w = rng.normal(size=grid)  # loss = sum(w * q)
    wrap3 = tuple(wrap) + (False,) * (3 - len(wrap))
    q, c = po.forward(r, P, grid, wrap3, ch)
    G = po.backward(w, c, P, grid, wrap3)

    def loss(P2, r2):
        return float((w * po.forward(r2, P2, grid, wrap3, ch)[0]).sum())

    eps = 1e-6
    for name in ["W_e0", "W_e3", "W_m3", "W_d2", "W_d0", "W_q", "b_e1", "b_d1", "b_q"]:
        flat = P[name].reshape(-1)
        for idx in rng.choice(flat.size, size=min(4, flat.size), replace=False):
            Pp = {k: v.copy() for k, v in P.items()}
            Pm = {k: v.copy() for k, v in P.items()}
            Pp[name].reshape(-1)[idx] += eps
            Pm[name].reshape(-1)[idx] -= eps
            fd = (loss(Pp, r) - loss(Pm, r)) / (2 * eps)
            assert abs(fd - G[name].reshape(-1)[idx]) <= 1e-6 * max(1.0, abs(fd)), (name, idx, fd, G[name].reshape(-1)[idx])
    for idx in rng.choice(r.size, size=4, replace=False):
        rp, rm = r.copy(), r.copy()
        rp.reshape(-1)[idx] += eps
        rm.reshape(-1)[idx] -= eps
        fd = (loss(P, rp) - loss(P, rm)) / (2 * eps)
        assert abs(fd - G["r"].reshape(-1)[idx]) <= 1e-6 * max(1.0, abs(fd))


def test_network_is_linear_and_shapes():
    grid = (12, 9, 5)
    P = po.init_params(3, seed=0)
    r = np.random.default_rng(0).normal(size=grid)
    q1, _ = po.forward(r, P, grid, (True, True, False))
    q2, _ = po.forward(3.0 * r, P, grid, (True, True, False))
    assert q1.shape == grid
    assert np.allclose(q2, 3.0 * q1)  # zero biases at initialisation
    assert po.level_shapes(grid) == [(12, 9, 5), (6, 5, 3), (3, 3, 2), (2, 2, 1)]


@pytest.mark.parametrize("grid,rigid", [((9, 7, 8), ((0, 0), (0, 0), (1, 1))), ((10, 9), ((0, 0), (1, 1)))])
def test_training_loss_gradient_matches_finite_differences(grid, rigid):
    """The whole training loss, the pressure solve's gradient with its rigid-wall
    rows included: the gradient-norm energy loss and its parameter gradient
    (through the transpose of the gradient operator) against central differences."""
    nd = len(grid)
    ch = (2, 3, 4, 5)
    dx = (10.0, 10.0, 10.0)[:nd]
    wrap3 = tuple(not r[0] for r in rigid) + (False,) * (3 - nd)
    P = po.init_params(nd, ch, seed=3)
    rng = np.random.default_rng(4)
    r = rng.normal(size=grid)
    t = rng.normal(size=grid)
    c = 0.7
    E, G = po.energy_loss(P, r, t, c, grid, wrap3, rigid, dx, ch)
    eps = 1e-6
    for name in ["W_e0", "W_m3", "W_d1", "W_q"]:
        flat = P[name].reshape(-1)
        for idx in rng.choice(flat.size, size=3, replace=False):
            Pp = {k: v.copy() for k, v in P.items()}
            Pm = {k: v.copy() for k, v in P.items()}
            Pp[name].reshape(-1)[idx] += eps
            Pm[name].reshape(-1)[idx] -= eps
            fd = (po.energy_loss(Pp, r, t, c, grid, wrap3, rigid, dx, ch)[0]
                  - po.energy_loss(Pm, r, t, c, grid, wrap3, rigid, dx, ch)[0]) / (2 * eps)
            assert abs(fd - G[name].reshape(-1)[idx]) <= 1e-6 * max(1.0, abs(fd)), (name, idx, fd, G[name].reshape(-1)[idx])


def test_pressure_operator_rigid_rows_are_not_symmetric():
    """With a rigid wall the one-dimensional operator differs from its transpose
    in the rows next to the wall (the reason the training loss measures the error
    through the gradient, whose squared norm cannot be negative)."""
    M = po.lap1d_matrix(12, True, True, 1.0)
    assert not np.allclose(M, M.T)
    assert np.allclose(M[4:-4, 4:-4], M.T[4:-4, 4:-4])
    C = po.lap1d_matrix(12, False, False, 1.0)
    assert np.allclose((C @ np.ones(12)), 0.0)  # constants are in the kernel on a cyclic line


@pytest.mark.parametrize("n,rigid", [(9, False), (12, False), (8, True), (7, True)])
def test_gradient_energy_is_the_operator_energy_where_symmetric(n, rigid):
    """The loss's gradient-norm energy |G x|^2 equals x^T (-A) x of the pressure
    operator on a cyclic line, summed over the distinct points (the last point
    duplicates the first), and is never negative."""
    G = po.grad1d_matrix(n, rigid, rigid, 2.0)
    A = po.lap1d_matrix(n, rigid, rigid, 2.0)
    rng = np.random.default_rng(n)
    x = rng.normal(size=n)
    if not rigid:
        x[-1] = x[0]  # the cyclic duplicate point
        g, a = G @ x, A @ x
        assert np.isclose(float(g[:-1] @ g[:-1]), -float(x[:-1] @ a[:-1]))
    assert float((G @ x) @ (G @ x)) >= 0.0
