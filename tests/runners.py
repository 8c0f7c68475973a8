"""Helpers shared by the tests: run one of the reference's set-ups through the
oracle or through the CUDA library and return the advectees."""
import os

import numpy as np

from oracle import Oracle


def load(obj, setup):
    for e, a in enumerate(setup["advectee"]):
        obj.set_advectee(a, e)
    for d, a in enumerate(setup["advector"]):
        obj.set_advector(a, d)


def run_oracle(setup, opts, n_iters=2, dtype=np.float64, nt=None, fast=False, max_abs_div_eps=None):
    orc = Oracle(setup["grid"], opts, n_iters=n_iters, n_eqns=len(setup["advectee"]), bcs=setup["bcs"],
                 dtype=dtype, fast=fast, max_abs_div_eps=max_abs_div_eps)
    load(orc, setup)
    orc.advance(setup["nt"] if nt is None else nt)
    return [orc.advectee(e) for e in range(len(setup["advectee"]))]


def bq_params(setup):
    dx = setup["dx"]
    return {"prm": [setup["dt"], dx[0], dx[1], dx[2], setup["prs_tol"], setup["g"], setup["tht_ref"], -1.0],
            "prs_k": setup.get("prs_k", 1)}


def bq_oracle(setup, opts=None, n_iters=2, dtype=np.float64, fast=False):
    """The CPU oracle of solvers::boussinesq loaded with a Boussinesq set-up."""
    from libmpdataxx_b200 import opts as o
    bcs = ["rigid" if b == "gndsky" else b for b in setup["bcs"]]  # gndsky_3d.hpp: rigid for these fields
    orc = Oracle(setup["grid"], o.iga | o.fct if opts is None else opts, n_iters=n_iters, bcs=bcs,
                 dtype=dtype, fast=fast, boussinesq=bq_params(setup))
    orc.set_sclr_array("tht_e", setup["tht_e"])
    if setup.get("impl_tht"):
        orc.set_param("impl_tht", 1)
    if setup.get("vip_vab"):
        orc.set_param("vip_vab", int(setup["vip_vab"]))
    for name in ("tht_abs", "hflux_frc", "vab_coeff"):
        if name in setup:
            orc.set_sclr_array(name, setup[name])
    for d, a in enumerate(setup.get("vab_relax", [])):
        orc.set_sclr_array("vab_relax%d" % d, a)
    for e, a in enumerate(setup["advectee"]):
        orc.set_advectee(a, e)
    return orc


def bq_run(setup, opts=None, n_iters=2, dtype=np.float64, prs_scheme=None, prs_fp64=False):
    """concurr::cuda<solvers::boussinesq<...>> loaded with a Boussinesq set-up."""
    from libmpdataxx_b200 import setups
    return setups.boussinesq_run(setup, opts=opts, n_iters=n_iters, dtype=dtype, prs_scheme=prs_scheme,
                                 prs_fp64=prs_fp64)


# ---- 4_revolving_sphere_3d output fields (tests/golden/revolving_sphere_fields.npz) ----
def _block_sums(f, b):
    idx = [np.arange(0, n, b) for n in f.shape]
    r = lambda x: np.add.reduceat(np.add.reduceat(np.add.reduceat(x, idx[0], 0), idx[1], 1), idx[2], 2)
    return r(f)


def check_sphere_fields(case, psi):
    """Compare a 59^3 result with the reference's float32 HDF5 output after 556 steps.

    The reference stores float32 (output/hdf5.hpp: flttype_output); the result is
    rounded to float32 the same way and compared cell by cell on three full planes
    through the sphere's centre, and by sums over 6^3-cell blocks on the whole
    field.  A cell may differ by one float32 ulp, or by 1e-15 in absolute terms:
    the reference evaluated the set-up's rotation (revolving_sphere_3d.cpp:84-86)
    in an -Ofast build, which leaves Courant numbers of order 1e-16 on the faces of
    the cells on the rotation axis where the exact value (and the set-up's here) is
    zero, so those cells hold values below 3e-16 in the reference's output and
    exact zeros here."""
    ref = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "revolving_sphere_fields.npz"))
    c = ref["centre"]
    f = np.asarray(psi).astype(np.float32).astype(np.float64)
    planes = {"plane0": f[c[0], :, :], "plane1": f[:, c[1], :], "plane2": f[:, :, c[2]]}
    exact = total = 0
    for name, got in planes.items():
        g = ref[case + "/" + name].astype(np.float64)
        tol = np.maximum(np.spacing(np.abs(ref[case + "/" + name])).astype(np.float64), 1e-15)
        bad = np.abs(got - g) > tol
        assert not bad.any(), (name, np.argwhere(bad)[:5], got[bad][:5], g[bad][:5])
        exact += int((got == g).sum())
        total += g.size
    assert exact >= 0.99 * total, (exact, total)
    b = int(ref["block"])
    s = _block_sums(f, b)
    tol = 2.0 ** -23 * ref[case + "/block_abs"] + b ** 3 * 1e-15
    err = np.abs(s - ref[case + "/block_sum"])
    assert (err <= tol).all(), (float(err.max()), np.argwhere(err > tol)[:5])
    return exact, total
