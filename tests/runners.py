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
