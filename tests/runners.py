"""Helpers shared by the tests: run one of the reference's set-ups through the
oracle or through the CUDA library and return the advectees."""
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
    orc = Oracle(setup["grid"], o.iga | o.fct if opts is None else opts, n_iters=n_iters, bcs=setup["bcs"],
                 dtype=dtype, fast=fast, boussinesq=bq_params(setup))
    orc.set_sclr_array("tht_e", setup["tht_e"])
    for e, a in enumerate(setup["advectee"]):
        orc.set_advectee(a, e)
    return orc


def bq_run(setup, opts=None, n_iters=2, dtype=np.float64, prs_scheme=None, prs_fp64=False):
    """concurr::cuda<solvers::boussinesq<...>> loaded with a Boussinesq set-up
    (equations (u, [v,] w, tht) as in the reference's tests)."""
    from libmpdataxx_b200 import bcond, concurr, opts as o, solvers
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
    for e, a in enumerate(setup["advectee"]):
        run.advectee(e)[...] = a
    return run
