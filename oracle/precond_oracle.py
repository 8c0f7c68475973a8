"""ORACLE -- test infrastructure only.

float64 numpy restatement of the learned GCR preconditioner network that the
CUDA library implements (libmpdataxx_b200/csrc/precond.cu), used to check the
GPU forward pass and gradients.  Nothing in the shipped library calls it.

The network maps a residual field r (one channel) to a search direction q on
the same grid.  It is a linear 4-level U-net: 3^d-point convolutions with
bias, 2^d average pooling between levels, nearest-neighbour up-sampling with
additive skip connections:

    e0 = conv(r, 1 -> C0)                      level 0
    e1 = conv(pool(e0), C0 -> C1)              level 1
    e2 = conv(pool(e1), C1 -> C2)              level 2
    e3 = conv(pool(e2), C2 -> C3)              level 3
    m3 = conv(e3, C3 -> C3)                    level 3
    d2 = conv(up(m3), C3 -> C2) + e2           level 2
    d1 = conv(up(d2), C2 -> C1) + e1           level 1
    d0 = conv(up(d1), C1 -> C0) + e0           level 0
    q  = conv(d0, C0 -> 1)                     level 0

Level l+1 has ceil(n/2) points along every axis of level l with more than one
point.  Convolutions pad cyclic axes by wrapping (modulo the level's size)
and rigid axes with zeros; pooling averages the fine points that exist;
up-sampling copies coarse point floor(p/2).  Arrays are (C, n0, n1, n2).
"""
import numpy as np

LAYERS = ["e0", "e1", "e2", "e3", "m3", "d2", "d1", "d0", "q"]


def level_shapes(grid, n_levels=4):
    g = list(grid) + [1] * (3 - len(grid))
    shapes = [tuple(g)]
    for _ in range(n_levels - 1):
        g = [(x + 1) // 2 if x > 1 else 1 for x in g]
        shapes.append(tuple(g))
    return shapes


def taps(nd):
    """Tap offsets in the order the CUDA kernels use: i slowest, k fastest."""
    r2 = (-1, 0, 1) if nd == 3 else (0,)
    return [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in r2]


def layer_dims(ch):
    c0, c1, c2, c3 = ch
    return {"e0": (1, c0, 0), "e1": (c0, c1, 1), "e2": (c1, c2, 2), "e3": (c2, c3, 3), "m3": (c3, c3, 3),
            "d2": (c3, c2, 2), "d1": (c2, c1, 1), "d0": (c1, c0, 0), "q": (c0, 1, 0)}


def init_params(nd, ch=(8, 16, 32, 64), seed=0):
    """W[name]: (cout, ntaps, cin), b[name]: (cout,); variance 1 / fan-in."""
    rng = np.random.default_rng(seed)
    nt = len(taps(nd))
    P = {}
    for name, (ci, co, _) in layer_dims(ch).items():
        P["W_" + name] = rng.normal(0.0, 1.0 / np.sqrt(nt * ci), size=(co, nt, ci))
        P["b_" + name] = np.zeros(co)
    return P


def _shift(x, off, wrap):
    """y[..., p] = x[..., p + off] along the three grid axes (zero or wrapped outside)."""
    y = x
    for ax, (o, w) in enumerate(zip(off, wrap)):
        if o == 0:
            continue
        a = ax + 1
        n = x.shape[a]
        if w:
            y = np.roll(y, -o, axis=a)
        else:
            z = np.zeros_like(y)
            src = [slice(None)] * y.ndim
            dst = [slice(None)] * y.ndim
            if o > 0:
                src[a], dst[a] = slice(o, n), slice(0, n - o)
            else:
                src[a], dst[a] = slice(0, n + o), slice(-o, n)
            z[tuple(dst)] = y[tuple(src)]
            y = z
    return y


def conv(x, W, b, wrap, nd):
    """y[co, p] = b[co] + sum_t sum_ci W[co, t, ci] x[ci, p + tap_t]."""
    y = np.zeros((W.shape[0],) + x.shape[1:])
    for t, off in enumerate(taps(nd)):
        y += np.einsum("oc,c...->o...", W[:, t, :], _shift(x, off, wrap))
    return y + b[:, None, None, None]


def conv_adj(dy, W, wrap, nd):
    """Adjoint of conv with respect to its input."""
    dx = np.zeros((W.shape[2],) + dy.shape[1:])
    for t, off in enumerate(taps(nd)):
        dx += _shift(np.einsum("oc,o...->c...", W[:, t, :], dy), tuple(-o for o in off), wrap)
    return dx


def conv_dw(dy, x, wrap, nd):
    return np.stack([np.tensordot(dy, _shift(x, off, wrap), axes=([1, 2, 3], [1, 2, 3])) for off in taps(nd)], axis=1)


def _coarse_index(fine, coarse):
    """Coarse point floor(p / 2) of every fine point p (index grids)."""
    idx = [np.minimum(np.arange(n) // 2, coarse[a] - 1) for a, n in enumerate(fine)]
    return tuple(np.meshgrid(*idx, indexing="ij"))


def pool(x, coarse):
    """Average of the fine points of every coarse point."""
    I = _coarse_index(x.shape[1:], coarse)
    s = np.zeros((x.shape[0],) + tuple(coarse))
    cnt = np.zeros(coarse)
    np.add.at(cnt, I, 1.0)
    for ch in range(x.shape[0]):
        np.add.at(s[ch], I, x[ch])
    return s / cnt


def pool_adj(dc, fine):
    coarse = dc.shape[1:]
    cnt = np.zeros(coarse)
    np.add.at(cnt, _coarse_index(fine, coarse), 1.0)
    return up(dc / cnt, fine)


def up(x, fine):
    I = _coarse_index(fine, x.shape[1:])
    return x[(slice(None),) + I]


def up_adj(df, coarse):
    I = _coarse_index(df.shape[1:], coarse)
    out = np.zeros((df.shape[0],) + tuple(coarse))
    for ch in range(df.shape[0]):
        np.add.at(out[ch], I, df[ch])
    return out


def forward(r, P, grid, wrap, ch=(8, 16, 32, 64)):
    """r: array of the grid's shape; returns (q, cache)."""
    nd = len(grid)
    sh = level_shapes(grid)
    x = np.asarray(r, dtype=np.float64).reshape((1,) + sh[0])
    c = {"r": x}
    c["e0"] = conv(x, P["W_e0"], P["b_e0"], wrap, nd)
    c["p1"] = pool(c["e0"], sh[1]); c["e1"] = conv(c["p1"], P["W_e1"], P["b_e1"], wrap, nd)
    c["p2"] = pool(c["e1"], sh[2]); c["e2"] = conv(c["p2"], P["W_e2"], P["b_e2"], wrap, nd)
    c["p3"] = pool(c["e2"], sh[3]); c["e3"] = conv(c["p3"], P["W_e3"], P["b_e3"], wrap, nd)
    c["m3"] = conv(c["e3"], P["W_m3"], P["b_m3"], wrap, nd)
    c["u2"] = up(c["m3"], sh[2]); c["d2"] = conv(c["u2"], P["W_d2"], P["b_d2"], wrap, nd) + c["e2"]
    c["u1"] = up(c["d2"], sh[1]); c["d1"] = conv(c["u1"], P["W_d1"], P["b_d1"], wrap, nd) + c["e1"]
    c["u0"] = up(c["d1"], sh[0]); c["d0"] = conv(c["u0"], P["W_d0"], P["b_d0"], wrap, nd) + c["e0"]
    c["q"] = conv(c["d0"], P["W_q"], P["b_q"], wrap, nd)
    return c["q"][0].reshape(np.shape(r)), c


def backward(dq, c, P, grid, wrap):
    """Gradients of sum(dq * q) with respect to every parameter and to r."""
    nd = len(grid)
    sh = level_shapes(grid)
    G = {}
    dq = np.asarray(dq, dtype=np.float64).reshape((1,) + sh[0])

    def lin(name, dy, x):
        G["W_" + name] = conv_dw(dy, x, wrap, nd)
        G["b_" + name] = dy.sum(axis=(1, 2, 3))
        return conv_adj(dy, P["W_" + name], wrap, nd)

    dd0 = lin("q", dq, c["d0"])
    de0 = dd0.copy()
    du0 = lin("d0", dd0, c["u0"])
    dd1 = up_adj(du0, sh[1])
    de1 = dd1.copy()
    du1 = lin("d1", dd1, c["u1"])
    dd2 = up_adj(du1, sh[2])
    de2 = dd2.copy()
    du2 = lin("d2", dd2, c["u2"])
    dm3 = up_adj(du2, sh[3])
    de3 = lin("m3", dm3, c["e3"])
    dp3 = lin("e3", de3, c["p3"])
    de2 += pool_adj(dp3, sh[2])
    dp2 = lin("e2", de2, c["p2"])
    de1 += pool_adj(dp2, sh[1])
    dp1 = lin("e1", de1, c["p1"])
    de0 += pool_adj(dp1, sh[0])
    G["r"] = lin("e0", de0, c["r"])[0]
    return G


# ---- the training loss, operator included ----
# The pressure operator A = lap() of the GCR solve (mpdata_rhs_vip_prs_common.hpp:
# 49-84, no normalisation): along every axis d, lap_tmp = grad (centred, 2 dx) with
# the pressure halo rule (cyclic: period n - 1; rigid: 2 x(edge) - x(mirror)),
# zero at a rigid wall point (set_edges), its own pressure halo rule, then the
# centred divergence.  It is a sum of one-dimensional operators, each acting along
# the lines of its axis; with rigid walls it is not symmetric, so its adjoint is
# built from the transposed one-dimensional matrices.

def _pres_src(q, n, rigid_lo, rigid_hi):
    """(qa, qb): the point q takes x[qa] (qb < 0) or 2 x[qa] - x[qb]."""
    if 0 <= q < n:
        return q, -1
    if q < 0:
        return (0, -q) if rigid_lo else (q + n - 1, -1)
    return (n - 1, 2 * (n - 1) - q) if rigid_hi else (q - (n - 1), -1)


def lap1d_matrix(n, rigid_lo, rigid_hi, dx):
    """Matrix of the one-dimensional part of lap() on a line of n points."""
    M = np.zeros((n, n))

    def aval(x, q):
        a, b = _pres_src(q, n, rigid_lo, rigid_hi)
        return x[a] if b < 0 else 2 * x[a] - x[b]

    def lt(x, q):
        if (q == 0 and rigid_lo) or (q == n - 1 and rigid_hi):
            return 0.0
        return (aval(x, q + 1) - aval(x, q - 1)) / dx / 2

    def LT(x, q):
        a, b = _pres_src(q, n, rigid_lo, rigid_hi)
        return lt(x, a) if b < 0 else 2 * lt(x, a) - lt(x, b)

    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        M[:, j] = [(LT(e, i + 1) - LT(e, i - 1)) / dx / 2 for i in range(n)]
    return M


def _apply_axes(x, mats):
    out = np.zeros_like(x)
    for ax, M in enumerate(mats):
        out += np.moveaxis(np.tensordot(M, np.moveaxis(x, ax, 0), axes=(1, 0)), 0, ax)
    return out


def pressure_lap(x, bcs, dx):
    """lap(x) of the pressure solve; bcs[d] = (rigid_lo, rigid_hi), dx[d] spacings."""
    return _apply_axes(x, [lap1d_matrix(n, lo, hi, h) for n, (lo, hi), h in zip(x.shape, bcs, dx)])


def pressure_lap_adj(x, bcs, dx):
    """The adjoint (transpose) of pressure_lap."""
    return _apply_axes(x, [lap1d_matrix(n, lo, hi, h).T for n, (lo, hi), h in zip(x.shape, bcs, dx)])


def grad1d_matrix(n, rigid_lo, rigid_hi, dx):
    """Matrix of the centred gradient of the pressure solve along a line of n points
    (lap_tmp of mpdata_rhs_vip_prs_common.hpp:49-84 before the divergence: pressure
    halo rule for the neighbours, zero on a rigid wall point)."""
    M = np.zeros((n, n))

    def aval(x, q):
        a, b = _pres_src(q, n, rigid_lo, rigid_hi)
        return x[a] if b < 0 else 2 * x[a] - x[b]

    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        for i in range(n):
            if (i == 0 and rigid_lo) or (i == n - 1 and rigid_hi):
                continue
            M[i, j] = (aval(e, i + 1) - aval(e, i - 1)) / dx / 2
    return M


def _along(M, x, ax):
    return np.moveaxis(np.tensordot(M, np.moveaxis(x, ax, 0), axes=(1, 0)), 0, ax)


def energy_loss(P, r, t, c, grid, wrap, bcs, dx, ch=(8, 16, 32, 64)):
    """Training loss of the preconditioner for a pair (residual r, correction t,
    A t = -r): the energy of the error e = c net(r) - t relative to that of t,
    measured as the squared centred gradient summed over the axes,
    E = sum_d |G_d e|^2 / sum_d |G_d t|^2 (1 for a zero output).  With cyclic
    axes this is e^T (-A) e / t^T (-A) t; with rigid walls -A is not symmetric and
    its quadratic form can be negative, while this one never is.  Returns
    (E, gradient dict of the parameters)."""
    q, cache = forward(r, P, grid, wrap, ch)
    e = c * q - t
    Gs = [grad1d_matrix(n, lo, hi, h) for n, (lo, hi), h in zip(e.shape, bcs, dx)]
    ge = [_along(G, e, ax) for ax, G in enumerate(Gs)]
    den = float(sum((_along(G, t, ax) ** 2).sum() for ax, G in enumerate(Gs)))
    E = float(sum((g ** 2).sum() for g in ge)) / den
    dq = 2 * c * sum(_along(G.T, g, ax) for ax, (G, g) in enumerate(zip(Gs, ge))) / den
    return E, backward(dq, cache, P, grid, wrap)
