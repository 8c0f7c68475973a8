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
    """concurr::cuda<solvers::boussinesq<...>> loaded with a Boussinesq set-up."""
    from libmpdataxx_b200 import setups
    return setups.boussinesq_run(setup, opts=opts, n_iters=n_iters, dtype=dtype, prs_scheme=prs_scheme,
                                 prs_fp64=prs_fp64)
