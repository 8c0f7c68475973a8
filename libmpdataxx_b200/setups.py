"""Initial conditions and advector fields of the reference's test problems and
of the synthetic benchmark workloads.

Arrays are returned in the reference's accessor conventions:
  advectee(e)  -> shape grid, index (i, j, k) = cell
  advector(d)  -> view with lower bound (-1, 0, 0): shape grid for d = 0 and
                  (n0 + 1, n1, n2) for d >= 1; view element (a, b, c) holds the
                  value the reference computes at view index (a - 1, b, c)
                  (libmpdata++/concurr/detail/sharedmem.hpp:431-456, 543-577)
Expressions follow the reference's operand order so that FP64 inputs are
bit-identical to what its Blitz++ expressions produce.
"""
import math

import numpy as np

from . import opts as o


def _view_idx(shape):
    """Index grids of an advector view: first axis starts at -1."""
    g = list(np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij"))
    g[0] = g[0] - 1.0
    return g


# --- tests/paper_2015_GMD/1_advscheme_opts/advscheme_opts.cpp:24-56 -----------
def advscheme_opts(nx=601):
    i = np.arange(nx)
    box = (i <= 75) | (i >= 125)
    psi0 = np.where(box, 2.0, 4.0)
    psi1 = np.where(box, -1.0, 1.0)
    return {"grid": (nx,), "bcs": ["cyclic"] * 2, "advectee": [psi0, psi1],
            "advector": [np.full((nx,), -0.75)], "nt": 1200, "n_iters": 2}


ADVSCHEME_CASES = {"abs": o.abs, "iga": o.iga, "iga_tot": o.iga | o.tot, "iga_fct": o.iga | o.fct,
                   "iga_tot_fct": o.iga | o.tot | o.fct}


# --- plain 1D MPDATA on a periodic box (the CPU-runnable benchmark case) ------
def box_1d(nx=2000, seed=1, courant=0.5):
    """nx points cyclic (period nx - 1), constant Courant number 0.5, advectee
    0.1 + U[0, 0.01) (seed) with 1 on cells 200..400, point nx - 1 = point 0;
    run with opts 0, n_iters 2 for 1000 steps."""
    rng = np.random.default_rng(seed)
    psi = 0.1 + rng.uniform(0.0, 0.01, nx - 1)
    psi[200:401] = 1.0
    return {"grid": (nx,), "bcs": ["cyclic"] * 2, "advectee": [wrap_periodic(psi)],
            "advector": [np.full((nx,), courant)], "nt": 1000, "opts": 0, "n_iters": 2}


# --- tests/paper_2015_GMD/2_convergence_1d/convergence_1d.cpp:59-160 ----------
CONVERGENCE_SOLVERS = {"iters=1": (0, 1), "iters=2": (0, 2), "iters=3": (0, 3), "iters=3_tot": (o.tot, 3),
                       "iters=i": (o.iga, 2), "iters=2_fct": (o.fct, 2), "iters=i_fct": (o.fct | o.iga, 2),
                       "iters=i_fct_tot": (o.fct | o.iga | o.tot, 2)}
CONVERGENCE_COURANTS = [.05, .1, .15, .2, .25, .3, .35, .4, .45, .5, .55, .6, .65, .7, .75, .8, .85, .9, .95]
CONVERGENCE_DXS = [1.0 / 2 ** q for q in range(8)]


def convergence_1d(dx, courant):
    """A Gaussian (sigma 1.5) averaged over each cell, advected by one unit
    (t_max 1, velocity 1) across a 440-unit domain with open boundaries;
    returns the set-up and the cell-averaged exact solution at the end."""
    t_max, x_max, sgma, velocity, A0 = 1.0, 440.0, 1.5, 1.0, 0.0
    x0 = 0.5 * x_max
    A = 1.0 / sgma / math.sqrt(2 * math.pi)

    def gauss_int(a):
        return A0 * dx + A * sgma * math.sqrt(math.pi / 2) * (
            math.erf((a + dx / 2 - x0) / math.sqrt(2) / sgma) - math.erf((a - dx / 2 - x0) / math.sqrt(2) / sgma))

    dt = courant * dx / velocity
    cround = lambda v: int(math.floor(v + 0.5))  # C's round(): halves away from zero (v > 0)
    nx = cround(x_max / dx)
    nt = cround(t_max / dt)
    psi = np.array([gauss_int(i * dx) / dx for i in range(nx)])
    exact = np.array([gauss_int(i * dx - velocity * dt * nt) / dx for i in range(nx)])
    return {"grid": (nx,), "bcs": ["open"] * 2, "advectee": [psi], "advector": [np.full((nx,), courant)],
            "nt": nt, "dt": dt, "exact": exact}


def convergence_error(psi, exact, nt, dt):
    """sqrt(sum((psi - exact)^2) / nx) / (nt dt) (convergence_1d.cpp:152-153)"""
    return math.sqrt(float(((psi - exact) ** 2).sum()) / psi.size) / (nt * dt)


# --- tests/paper_2015_GMD/0_basic_example/basic_example.cpp:10-50 -------------
def basic_example(nx=101, dx=0.1):
    i = np.arange(nx, dtype=np.float64)
    psi = -.5 + 1 / ((dx * (i - (nx - 1) / 2.)) ** 2 + 1)
    return {"grid": (nx,), "bcs": ["open"] * 2, "advectee": [psi], "advector": [np.full((nx,), .5)],
            "nt": 100, "outfreq": 20, "opts": o.iga | o.fct, "n_iters": 2}


# --- tests/paper_2015_GMD/3_rotating_cone_2d/rotating_cone_2d.cpp:32-138 ------
def rotating_cone(nx=101, ny=101):
    dt, dx, dy, omega, h, h0 = .1, 1., 1., .1, 4., 1.
    r, x0, y0 = 15. * dx, 50 * dx, 75 * dy
    xc, yc = .5 * (nx - 1) * dx, .5 * (ny - 1) * dy
    i, j = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64), indexing="ij")
    tmp = (i * dx - x0) ** 2 + (j * dy - y0) ** 2
    psi = h0 + np.where(tmp - r ** 2 <= 0, h - np.sqrt(tmp / (r / h) ** 2), 0.)
    vi, vj = _view_idx((nx, ny))
    gx = omega * (vj * dy - yc) * dt / dx
    vi, vj = _view_idx((nx + 1, ny))
    gy = -omega * (vi * dx - xc) * dt / dy
    return {"grid": (nx, ny), "bcs": ["open"] * 4, "advectee": [psi], "advector": [gx, gy], "nt": 628 * 6,
            "dt": dt}


CONE_CASES = {"basic": (0, 2), "fct": (o.fct, 2), "iga_fct": (o.iga | o.fct, 2),
              "iga_tot_fct": (o.iga | o.tot | o.fct, 2), "iters3_tot_fct": (o.tot | o.fct, 3)}


def cone_stats(psi_init, psi_final, nt, dt):
    """rotating_cone_stats.hpp:52-67"""
    err2 = (psi_init - psi_final) ** 2
    rms = math.sqrt(err2.sum() / psi_init.shape[0] / psi_init.shape[1]) / nt / dt
    return {"min(psi)": float(psi_final.min()), "max(psi)": float(psi_final.max()), "rms error": rms}


# --- tests/paper_2015_GMD/4_revolving_sphere_3d/revolving_sphere_3d.cpp:29-100 -
def revolving_sphere(nx=59):
    dt = 0.018 * 2 * math.pi
    L = 100.
    dx = L / (nx - 1)
    dy = dz = dx
    h, r = 4., 15.
    d = 25 / math.sqrt(3)
    x0, y0, z0 = 50 - d, 50 + d, 50 + d
    i, j, k = np.meshgrid(*[np.arange(nx, dtype=np.float64)] * 3, indexing="ij")
    tmp = (i * dx - x0) ** 2 + (j * dx - y0) ** 2 + (k * dx - z0) ** 2
    psi = np.where(tmp - r ** 2 <= 0, h, 0.)
    omega, xc, yc, zc = 0.1, 50., 50., 50.
    w = omega / math.sqrt(3)
    vi, vj, vk = _view_idx((nx, nx, nx))
    gx = w * (-(vj * dy - yc) + (vk * dz - zc)) * dt / dx
    vi, vj, vk = _view_idx((nx + 1, nx, nx))
    gy = w * ((vi * dx - xc) - (vk * dz - zc)) * dt / dy
    gz = w * (-(vi * dx - xc) + (vj * dy - yc)) * dt / dz
    return {"grid": (nx, nx, nx), "bcs": ["open"] * 6, "advectee": [psi], "advector": [gx, gy, gz],
            "nt": 556, "dt": dt}


SPHERE_CASES = {"upwind": (0, 1), "basic": (0, 2), "iga": (o.iga, 2), "fct": (o.fct, 2),
                "iga_fct": (o.iga | o.fct, 2)}


def sphere_stats(ic, fc, nt, dt):
    """revolving_sphere_stats.hpp:46-64"""
    n3 = float(ic.shape[0]) ** 3
    dif = fc - ic
    return {"max(solution)": float(fc.max()), "min(solution)": float(fc.min()),
            "Linf": float(np.abs(dif).max()),
            "L2": 1.0 / (nt * dt) * math.sqrt(1.0 / n3 * float((dif ** 2).sum())),
            "L1": 1.0 / (nt * dt) * (1.0 / n3 * float(np.abs(dif).sum()))}


# --- tests/unit/cone_bugs/test_issue.cpp: FP32 fct, exact background ----------
def cone_bugs():
    nx, ny = 15, 14
    dx = dy = 1.
    h, h0, r, x0, y0 = 4., 1., 12. * dx, 1., 0.
    i, j = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64), indexing="ij")
    a = ((i * dx - x0) ** 2 + (j * dy - y0) ** 2).astype(np.float32).astype(np.float64)
    psi = h0 + np.where(a - r ** 2 <= 0, h * (1 - a / r ** 2) ** 2, 0.)
    return {"grid": (nx, ny), "bcs": ["cyclic"] * 4, "advectee": [psi.astype(np.float32).astype(np.float64)],
            "advector": [np.full((nx, ny), .3), np.full((nx + 1, ny), .3)], "nt": 2, "opts": o.fct,
            "n_iters": 2}


# --- synthetic periodic workloads (duplicated-endpoint convention: x[n-1] == x[0]) ---

def periodic_curl_2d(nx, ny, seed, n_modes=8, cmax=0.5, dtype=np.float64):
    """Divergence-free 2D Courant field from a streamfunction of random Fourier
    modes on the (nx-1) x (ny-1) periodic torus: GC_x = dPsi/dy, GC_y = -dPsi/dx
    taken as differences of Psi at cell corners, so the discrete divergence of
    the returned faces vanishes up to rounding.  Returns (gx, gy) in advector
    view layout."""
    rng = np.random.default_rng(seed)
    Px, Py = nx - 1, ny - 1
    # corner values Psi(I, J) at corner (I - 1/2, J - 1/2), periodic in (Px, Py)
    I, J = np.meshgrid(np.arange(Px, dtype=np.float64), np.arange(Py, dtype=np.float64), indexing="ij")
    psi = np.zeros((Px, Py))
    for _ in range(n_modes):
        kx, ky = rng.integers(1, 5, size=2)
        amp = rng.normal()
        ph = rng.uniform(0, 2 * math.pi)
        psi += amp * np.cos(2 * math.pi * (kx * I / Px + ky * J / Py) + ph)
    # face (i+1/2, j) between corners (i+1/2, j-1/2) and (i+1/2, j+1/2): GC_x = Psi(i+1, j+1) - Psi(i+1, j)
    gxu = np.roll(np.roll(psi, -1, 0), -1, 1) - np.roll(psi, -1, 0)     # (Px, Py), index (i, j) -> face i+1/2
    # face (i, j+1/2): GC_y = -(Psi(i+1, j+1) - Psi(i, j+1))
    gyu = -(np.roll(np.roll(psi, -1, 0), -1, 1) - np.roll(psi, -1, 1))  # (Px, Py), index (i, j) -> face j+1/2
    s = cmax / max(np.abs(gxu).max(), np.abs(gyu).max())
    gxu *= s
    gyu *= s
    gxu = gxu.astype(dtype).astype(np.float64)
    gyu = gyu.astype(dtype).astype(np.float64)
    # x view: element (a, b) = face (a - 1 + 1/2, b) over a in [0, nx-1], b in [0, ny-1]
    a = (np.arange(nx) - 1) % Px
    b = np.arange(ny) % Py
    gx = gxu[np.ix_(a, b)]
    # y view: element (a, b) = GC_y at x = a - 1, face b - 1 + 1/2 (view index b <-> face b - 1/2)
    a = (np.arange(nx + 1) - 1) % Px
    b = (np.arange(ny) - 1) % Py
    gy = gyu[np.ix_(a, b)]
    return gx, gy


def periodic_curl_3d(n, seed, n_modes=8, cmax=0.4, dtype=np.float32):
    """Divergence-free 3D Courant field: discrete curl of a vector potential A
    (3 components of random Fourier modes periodic on the (n-1)-cell torus,
    integer wave-vectors in [1, 4]^3, N(0,1) amplitudes, U[0, 2pi) phases),
    computed in FP64 on cell edges so that the face fluxes have zero discrete
    divergence.  n is an int (cube) or a 3-tuple.  Returns (gx, gy, gz) in
    advector view layout."""
    n0, n1, n2 = (n, n, n) if np.isscalar(n) else tuple(n)
    rng = np.random.default_rng(seed)
    P = (n0 - 1, n1 - 1, n2 - 1)
    I, J, K = np.meshgrid(*[np.arange(p, dtype=np.float64) for p in P], indexing="ij")
    A = []
    for _c in range(3):
        a = np.zeros(P)
        for _ in range(n_modes):
            kv = rng.integers(1, 5, size=3)
            amp = rng.normal()
            ph = rng.uniform(0, 2 * math.pi)
            a += amp * np.cos(2 * math.pi * (kv[0] * I / P[0] + kv[1] * J / P[1] + kv[2] * K / P[2]) + ph)
        A.append(a)
    Ax, Ay, Az = A
    # A on cell edges: Ax[i,j,k] at (i, j+1/2, k+1/2), Ay at (i+1/2, j, k+1/2), Az at (i+1/2, j+1/2, k);
    # the flux through each face is the circulation of A around it, so the
    # discrete divergence of every cell vanishes identically
    b = lambda x, ax: np.roll(x, 1, ax)   # x[i-1]
    fx = (Az - b(Az, 1)) - (Ay - b(Ay, 2))   # face (i+1/2, j, k)
    fy = (Ax - b(Ax, 2)) - (Az - b(Az, 0))   # face (i, j+1/2, k)
    fz = (Ay - b(Ay, 0)) - (Ax - b(Ax, 1))   # face (i, j, k+1/2)
    s = cmax / max(np.abs(fx).max(), np.abs(fy).max(), np.abs(fz).max())
    fx, fy, fz = [(f * s).astype(dtype).astype(np.float64) for f in (fx, fy, fz)]
    a0 = (np.arange(n0) - 1) % P[0]
    a1 = (np.arange(n0 + 1) - 1) % P[0]
    j_ = np.arange(n1) % P[1]
    jm = (np.arange(n1) - 1) % P[1]
    k_ = np.arange(n2) % P[2]
    km = (np.arange(n2) - 1) % P[2]
    gx = fx[np.ix_(a0, j_, k_)]
    gy = fy[np.ix_(a1, jm, k_)]
    gz = fz[np.ix_(a1, j_, km)]
    return gx, gy, gz


def wrap_periodic(u):
    """Apply the duplicated-endpoint convention to a field defined on the
    (n-1)^d unique cells: returns the n^d array with x[n-1] = x[0] per axis."""
    for ax in range(u.ndim):
        u = np.concatenate([u, np.take(u, [0], axis=ax)], axis=ax)
    return u


# --- tests/paper_2015_GMD/8_boussinesq_2d/boussinesq_2d.cpp:17-117 ------------
def boussinesq_2d(nx=201, ny=201, r0=250.0):
    """Buoyant thermal (Smolarkiewicz & Pudykiewicz 1992, fig. 3): equations
    (u, w, tht), cyclic in x and y, cr pressure solver, 800 steps."""
    dx = 10.0
    tht_ref = 300.0
    i, j = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64), indexing="ij")
    tht = tht_ref + np.where((i * dx - 4 * r0) ** 2 + (j * dx - 1.04 * r0) ** 2 <= r0 ** 2, 0.5, 0.0)
    return {"grid": (nx, ny), "bcs": ["cyclic"] * 4, "advectee": [np.zeros((nx, ny)), np.zeros((nx, ny)), tht],
            "tht_e": np.full((nx, ny), tht_ref), "dt": 0.75, "dx": (dx, dx, 1.0), "tht_ref": tht_ref, "g": 9.81,
            "prs_tol": 1e-7, "nt": 800, "prs_k": 1}


def boussinesq_stats(tht, u, w, tht_ref, init):
    """The statistics printed by tests/paper_2015_GMD/8_boussinesq_2d/boussinesq_stats.hpp:58-118:
    sums leave out the first row and column (duplicated cyclic edge)."""
    pert = (tht - tht_ref)[1:, 1:]
    s2 = float((((init - tht_ref)[1:, 1:]) ** 2).sum())
    return {"min(tht)": float(tht.min()), "max(tht)": float(tht.max()),
            "max(velocity)": float(np.sqrt(u ** 2 + w ** 2).max()),
            "error_2": (float((pert ** 2).sum()) - s2) / s2 * 100}


def boussinesq_bubble_3d(nx=256, ny=256, nz=128, seed=6, dx=10.0, n_bv=0.01, dtype=np.float64):
    """Stably stratified 3D thermal: tht_e(z) = 300 exp(N^2 z / g), zero wind,
    a +0.5 K sphere of radius 0.1 nx dx centred at (Lx/2, Ly/2, Lz/4) plus
    seeded uniform noise of +-0.01 K; x and y cyclic, z rigid.  Equations
    (u, v, w, tht)."""
    g, tref = 9.81, 300.0
    rng = np.random.default_rng(seed)
    i, j, k = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64),
                          np.arange(nz, dtype=np.float64), indexing="ij")
    z = k * dx
    tht_e = tref * np.exp(n_bv ** 2 * z / g)
    r = 0.1 * nx * dx
    inside = (i * dx - 0.5 * (nx - 1) * dx) ** 2 + (j * dx - 0.5 * (ny - 1) * dx) ** 2 + (z - 0.25 * (nz - 1) * dx) ** 2 <= r * r
    tht = tht_e + np.where(inside, 0.5, 0.0) + rng.uniform(-0.01, 0.01, size=(nx, ny, nz))
    # duplicated-endpoint convention of the cyclic axes
    tht[-1, :, :] = tht[0, :, :]
    tht[:, -1, :] = tht[:, 0, :]
    zero = np.zeros((nx, ny, nz))
    return {"grid": (nx, ny, nz), "bcs": ["cyclic", "cyclic", "cyclic", "cyclic", "rigid", "rigid"],
            "advectee": [zero, zero.copy(), zero.copy(), tht.astype(dtype)], "tht_e": tht_e.astype(dtype),
            "dt": 0.75, "dx": (dx, dx, dx), "tht_ref": tref, "g": g, "prs_tol": 1e-7, "prs_k": 1}


def batched_problems(n=256, seed=5, lo=64, hi=1024, dtype=np.float32, cmax=0.5):
    """Independent 2D cyclic problems of uneven sizes: side lengths drawn
    uniformly from [lo, hi] per axis (seed), each with its own divergence-free
    random-Fourier Courant field (seed 1000 + p, max |C| = cmax) and an
    i.i.d. log-normal(0, 1) advectee (seed 2000 + p).  Returns a list of
    set-ups in the reference's accessor conventions."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, size=(n, 2))
    out = []
    for p, (nx, ny) in enumerate(sizes):
        nx, ny = int(nx), int(ny)
        gx, gy = periodic_curl_2d(nx, ny, 1000 + p, cmax=cmax, dtype=dtype)
        psi = np.random.default_rng(2000 + p).lognormal(0.0, 1.0, size=(nx - 1, ny - 1))
        out.append({"grid": (nx, ny), "bcs": ["cyclic"] * 4, "advectee": [wrap_periodic(psi).astype(dtype)],
                    "advector": [gx.astype(dtype), gy.astype(dtype)]})
    return out


def boussinesq_run(setup, opts=None, n_iters=2, dtype=np.float64, prs_scheme=None, prs_fp64=False):
    """concurr::cuda<solvers::boussinesq<...>> loaded with a Boussinesq set-up
    (equations (u, [v,] w, tht) as in the reference's tests, boussinesq_2d.cpp:27-30).
    Optional set-up keys: "impl_tht" (bool), "vip_vab" (solvers.noab/expl/impl), and
    the arrays "tht_abs", "hflux_frc", "vab_coeff", "vab_relax" (list per dimension)."""
    from . import bcond, concurr, solvers
    nd = len(setup["grid"])

    class ct(solvers.ct_params_default_t):
        pass

    ct.real_t = dtype
    ct.n_dims = nd
    ct.n_eqns = nd + 1
    ct.opts = o.iga | o.fct if opts is None else opts
    ct.rhs_scheme = solvers.trapez
    k = setup.get("prs_k", 1)
    ct.prs_scheme = prs_scheme if prs_scheme is not None else (solvers.cr if k == 1 else solvers.gcrk)
    ct.prs_k_iters = k
    ct.impl_tht = bool(setup.get("impl_tht", False))
    ct.vip_vab = int(setup.get("vip_vab", solvers.noab))

    class ix:
        pass

    ix.vip_i, ix.vip_j = 0, 1
    if nd == 3:
        ix.vip_k = 2
    ix.tht = nd
    ct.ix = ix
    p = solvers.boussinesq.rt_params_t(grid_size=list(setup["grid"]), n_iters=n_iters, dt=setup["dt"],
                                       di=setup["dx"][0], dj=setup["dx"][1], dk=setup["dx"][2],
                                       prs_tol=setup["prs_tol"], g=setup["g"], Tht_ref=setup["tht_ref"],
                                       prs_fp64=prs_fp64)
    run = concurr.cuda(solvers.boussinesq(ct), *[getattr(bcond, b) for b in setup["bcs"]], p=p)
    run.sclr_array("tht_e")[...] = setup["tht_e"]
    for name in ("tht_abs", "hflux_frc"):
        if name in setup:
            run.sclr_array(name)[...] = setup[name]
    if "vab_coeff" in setup:
        run.vab_coefficient()[...] = setup["vab_coeff"]
        for d, a in enumerate(setup["vab_relax"]):
            run.vab_relaxed_state(d)[...] = a
    for e, a in enumerate(setup["advectee"]):
        run.advectee(e)[...] = a
    return run
