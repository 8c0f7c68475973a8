"""The preconditioner network's CUDA kernels (BF16 tensor-core convolutions,
pooling, up-sampling, backward, Adam) against the float64 CPU oracle."""
import numpy as np
import pytest

import precond_oracle as po
from libmpdataxx_b200.precond import PCNet, pack, unpack

pytestmark = pytest.mark.gpu

CASES = [((12, 10, 9), (1, 1, 0), (8, 16, 32, 64)), ((20, 17, 6), (1, 0, 1), (8, 8, 16, 16)),
         ((33, 30), (1, 0), (8, 16, 32, 64)), ((40, 35, 18), (1, 1, 0), (16, 16, 32, 32))]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("grid,wrap,ch", CASES)
def test_forward_and_gradients_match_oracle(grid, wrap, ch):
    nd = len(grid)
    net = PCNet(grid, wrap, ch, seed=3)
    p = net.params()
    P = unpack(p, nd, ch)
    rng = np.random.default_rng(4)
    for k in P:  # non-zero biases exercise the bias paths; the output layer starts at zero
        if k.startswith("b_"):
            P[k] = rng.normal(size=P[k].shape) * 0.05
    P["W_q"] = rng.normal(size=P["W_q"].shape) / np.sqrt(P["W_q"].shape[1] * P["W_q"].shape[2])
    net.set_params(pack(P, nd, ch))
    P = unpack(net.params(), nd, ch)
    r = rng.normal(size=grid).astype(np.float32)
    wrap3 = tuple(bool(x) for x in wrap) + (False,) * (3 - nd)
    q_ref, cache = po.forward(r.astype(np.float64), P, grid, wrap3, ch)
    q = net.forward(r)
    print("forward rel err", rel(q, q_ref))
    assert rel(q, q_ref) <= 3e-2  # BF16 activations and weights
    dq = rng.normal(size=grid).astype(np.float32)
    g = net.backward(r, dq)
    G = po.backward(dq.astype(np.float64), cache, P, grid, wrap3)
    Gv = pack(G, nd, ch)
    for name in ["W_e0", "W_e1", "W_e3", "W_m3", "W_d2", "W_d0", "W_q", "b_e0", "b_m3", "b_q"]:
        a, b = unpack(g, nd, ch)[name], G[name]
        print(name, "grad rel err", rel(a, b))
        assert rel(a, b) <= 5e-2, name
    assert rel(g, Gv.astype(np.float32)) <= 5e-2


def test_training_reduces_loss_and_keeps_biases():
    grid, wrap, ch = (24, 20, 12), (1, 1, 0), (8, 16, 32, 64)
    net = PCNet(grid, wrap, ch, seed=1)
    rng = np.random.default_rng(0)
    # a fixed smoothing target map: learn q = blurred r
    r = rng.normal(size=grid).astype(np.float32)
    t = (r + np.roll(r, 1, 0) + np.roll(r, -1, 0) + np.roll(r, 1, 1) + np.roll(r, -1, 1)) / 5.0
    losses = [net.train_step(r, t, lr=2e-3) for _ in range(60)]
    print(losses[0], losses[-1])
    assert losses[-1] < 0.5 * losses[0]
    P = unpack(net.params(), 3, ch)
    assert all(np.all(P[k] == 0) for k in P if k.startswith("b_"))
