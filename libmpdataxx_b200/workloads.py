"""Synthetic benchmark workloads, generated on the GPU with torch (seeded).

Each builder returns device tensors laid out as the run API expects (advectee
n0 x n1 x n2, advector views with lower bound (-1, 0, 0)), and a description.
All periodic fields follow the duplicated-endpoint convention of libmpdata++'s
cyclic boundaries: point n-1 equals point 0 along every axis.

  advection_3d   3D MPDATA, 512^3 FP32, opts fct|iga, n_iters = 2: divergence-free
                 deformational flow (discrete curl of a 3-component vector
                 potential of 8 random Fourier modes each; wave-vectors in
                 [1, 4]^3, N(0, 1) amplitudes, U[0, 2pi) phases; seed 3) scaled to
                 max |C| = 0.4; advectee = 5 Gaussian blobs (centres U[0, n-1)^3,
                 width 0.05 (n-1), amplitude 1; seed 4).
  rotation_2d    2D MPDATA+FCT, 1024^2, n_iters = 3: solid-body rotation about the
                 domain centre (one revolution in 6283 steps), cone of radius
                 0.15 nx and height 4 on a zero background; the rotation is
                 exact within 0.48 (nx-1) of the centre along each axis and
                 clipped beyond (max face Courant number 0.49).
"""
import math

import numpy as np


def _torch():
    import torch
    return torch


def _view_index(n, first_axis_extra, shift, device):
    """Index vector of one advector-view axis into the unique-face array."""
    torch = _torch()
    length = n + (1 if first_axis_extra else 0)
    return (torch.arange(length, device=device) - shift) % (n - 1)


def advection_3d(n=512, seed_flow=3, seed_blobs=4, cmax=0.4, n_modes=8, dtype="float32", device="cuda"):
    torch = _torch()
    dt = getattr(torch, dtype)
    P = n - 1
    rng = np.random.default_rng(seed_flow)
    idx = torch.arange(P, dtype=torch.float64, device=device)
    A = []
    for _c in range(3):
        a = torch.zeros((P, P, P), dtype=torch.float64, device=device)
        for _ in range(n_modes):
            kv = rng.integers(1, 5, size=3)
            amp = float(rng.normal())
            ph = float(rng.uniform(0, 2 * math.pi))
            w = 2 * math.pi / P
            a += amp * torch.cos((kv[0] * w) * idx[:, None, None] + (kv[1] * w) * idx[None, :, None]
                                 + (kv[2] * w) * idx[None, None, :] + ph)
        A.append(a)
    Ax, Ay, Az = A
    b = lambda x, ax: torch.roll(x, 1, ax)  # x[i-1]
    # circulation of A (on cell edges) around each face: zero discrete divergence
    fx = (Az - b(Az, 1)) - (Ay - b(Ay, 2))
    fy = (Ax - b(Ax, 2)) - (Az - b(Az, 0))
    fz = (Ay - b(Ay, 0)) - (Ax - b(Ax, 1))
    del A, Ax, Ay, Az
    s = cmax / max(float(fx.abs().max()), float(fy.abs().max()), float(fz.abs().max()))
    fx, fy, fz = [(f * s).to(dt) for f in (fx, fy, fz)]
    i0 = _view_index(n, False, 1, device)
    i1 = _view_index(n, True, 1, device)
    j0 = _view_index(n, False, 0, device)
    jm = _view_index(n, False, 1, device)
    gx = fx[i0][:, j0][:, :, j0].contiguous()
    gy = fy[i1][:, jm][:, :, j0].contiguous()
    gz = fz[i1][:, j0][:, :, jm].contiguous()
    del fx, fy, fz
    # advectee: 5 Gaussian blobs with periodic (minimum-image) distance
    rng = np.random.default_rng(seed_blobs)
    sig = 0.05 * P
    psi = torch.zeros((P, P, P), dtype=torch.float64, device=device)
    for _ in range(5):
        c = rng.uniform(0, P, size=3)
        d2 = 0
        for ax, cc in enumerate(c):
            dd = (idx - cc).abs()
            dd = torch.minimum(dd, P - dd) ** 2
            shape = [1, 1, 1]
            shape[ax] = P
            d2 = d2 + dd.reshape(shape)
        psi += torch.exp(-d2 / (2 * sig * sig))
    psi = psi.to(dt)
    full = torch.arange(n, device=device) % P
    psi = psi[full][:, full][:, :, full].contiguous()
    if device != "cpu":
        torch.cuda.synchronize()  # the fields are complete when handed to another stream
    return {"grid": (n, n, n), "advectee": [psi], "advector": [gx, gy, gz],
            "desc": f"3D {n}^3 cyclic, fct|iga, n_iters=2, {dtype}; curl flow max|C|={cmax} (seed {seed_flow}), "
                    f"5 Gaussian blobs (seed {seed_blobs})"}


def rotation_2d(n=1024, dtype="float64", device="cuda"):
    """Solid-body rotation about the centre of the periodic domain: GC_x(face
    i+1/2, j) = w (j - yc), GC_y(i, face j+1/2) = -w (i - xc) with w = 2 pi / 6283
    (rotating_cone_2d.cpp:131-132 with omega dt / dx replaced by w); cone of
    radius 0.15 nx and height 4 at (0.5 nx, 0.75 nx) on a zero background.

    The offsets j - yc and i - xc are clipped to +-0.48 (nx - 1).  Unclipped, the
    corner cells of the domain have |C_x| + |C_y| = 1.02 (face Courant numbers
    0.51 on both axes), beyond the donor-cell limit of 1: over a full revolution
    the tiny values that diffuse there grow by ~17 % per step until they overflow
    (FP32 after ~1000 steps, FP64 after ~6000), in the reference-structured
    kernels as in the fused ones.  Clipped, every cell has |C_x| + |C_y| <= 0.98
    and the cone's path (within 0.41 nx of the centre) still sees the exact
    rotation; GC_x still depends on j alone and GC_y on i alone, so the field
    stays divergence-free."""
    torch = _torch()
    dt = getattr(torch, dtype)
    P = n - 1
    w = 2 * math.pi / 6283
    xc = yc = 0.5 * (P - 1)
    i = torch.arange(n, dtype=torch.float64, device=device)
    # faces follow the periodic convention: view index a <-> face (a-1)+1/2 (x), b <-> face (b-1)+1/2 (y view)
    jx = (torch.arange(n, device=device) % P).to(torch.float64)
    lim = 0.48 * P
    gx = (w * torch.clamp(jx - yc, -lim, lim))[None, :].expand(n, n).contiguous()
    ix = ((torch.arange(n + 1, device=device) - 1) % P).to(torch.float64)
    gy = (-w * torch.clamp(ix - xc, -lim, lim))[:, None].expand(n + 1, n).contiguous()
    r = 0.15 * n
    x0, y0 = 0.5 * n, 0.75 * n
    I, J = torch.meshgrid(i % P, i % P, indexing="ij")
    d = torch.sqrt((I - x0) ** 2 + (J - y0) ** 2)
    psi = torch.clamp(4 * (1 - d / r), min=0)
    out = [psi.to(dt).contiguous(), gx.to(dt), gy.to(dt)]
    if device != "cpu":
        torch.cuda.synchronize()
    return {"grid": (n, n), "advectee": [out[0]], "advector": out[1:],
            "desc": f"2D {n}^2 cyclic rotation, cone r=0.15 nx h=4, {dtype}"}
