"""The debug build (libmpdx_debug.so, MPDX_LIBRARY=debug): every field access of the
general path, the Boussinesq solver and the field views is bounds-checked (an access
outside a field's allocation fails the call), and new fields are filled with NaN, so
that a value read before anything wrote it shows in the results.  Runs a set of
configurations through it in a separate process and requires them to finish without
an out-of-range access, without NaN, and equal to the oracle."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + "/tests"); sys.path.insert(0, ROOT + "/oracle")
import numpy as np
from libmpdataxx_b200 import _lib, setups
from libmpdataxx_b200 import opts as o
from oracle import Oracle
from runners import load, bq_run, bq_oracle
from test_gpu_parity import make_run, random_setup

assert _lib.SO_PATH.endswith("libmpdx_debug.so"), _lib.SO_PATH
out = {}
def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
cases = [((23, 19), ["cyclic"] * 4, o.iga | o.fct, 2, "auto"),       # fused 2D
         ((23, 19), ["open"] * 4, o.fct, 2, "general"),
         ((11, 11, 11), ["rigid"] * 6, o.tot, 2, "general"),
         ((13, 13, 13), ["cyclic"] * 6, o.iga | o.fct, 2, "auto"),  # fused 3D
         ((17, 19), ["cyclic"] * 4, o.iga | o.tot | o.fot, 2, "general"),
         ((40,), ["cyclic"] * 2, 0, 2, "auto")]                      # one-block 1D
for k, (grid, bcs, opts, iters, path) in enumerate(cases):
    s = random_setup(grid, bcs, seed=k + 3, signed=bool(opts & o.iga))
    eps = 1e30 if "rigid" in bcs else 1e-10
    run = make_run(grid, opts, n_iters=iters, bcs=bcs, max_abs_div_eps=eps, path=path)
    run.set_advectee(s["advectee"][0])
    for d, a in enumerate(s["advector"]):
        run.set_advector(a, d)
    run.advance(3)
    orc = Oracle(grid, opts, n_iters=iters, bcs=bcs, max_abs_div_eps=eps)
    load(orc, s)
    orc.advance(3)
    got = run.advectee()
    out[f"case{k}"] = {"finite": bool(np.isfinite(got).all()), "rel": rel(got, orc.advectee())}
# the Boussinesq solver with its GCR pressure solve
s = setups.boussinesq_bubble_3d(16, 16, 12)
run = bq_run(s, dtype=np.float64)
run.advance(2)
orc = bq_oracle(s)
orc.advance(2)
errs = [rel(run.advectee(e), orc.advectee(e)) for e in range(4)]
out["boussinesq"] = {"finite": all(bool(np.isfinite(run.advectee(e)).all()) for e in range(4)), "rel": max(errs)}
print(json.dumps(out))
"""


def test_debug_build_runs_clean():
    so = os.path.join(ROOT, "libmpdataxx_b200", "libmpdx_debug.so")
    assert os.path.exists(so), "the debug library is built with the rest (make -C libmpdataxx_b200/csrc)"
    env = dict(os.environ, MPDX_LIBRARY="debug")
    p = subprocess.run([sys.executable, "-c", "ROOT = " + repr(ROOT) + "\n" + SCRIPT], env=env, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    res = json.loads(p.stdout.strip().splitlines()[-1])
    for name, r in res.items():
        assert r["finite"], name
        assert r["rel"] <= 1e-12, (name, r["rel"])
