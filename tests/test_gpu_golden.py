"""The reference's own golden results, reproduced by the CUDA path.

Same set-ups and tolerances as tests/test_oracle_golden.py (which pins the
oracle), but the numbers come from the GPU through the C ABI."""
import json
import os

import numpy as np
import pytest

from libmpdataxx_b200 import opts as o, setups
from runners import check_sphere_fields
from test_gpu_parity import make_run

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def golden():
    with open(os.path.join(GOLD, "golden_stats.json")) as f:
        return json.load(f)


def run_setup(s, opts, n_iters, dtype=np.float64, path="general"):
    run = make_run(s["grid"], opts, n_iters=n_iters, n_eqns=len(s["advectee"]), bcs=s["bcs"], dtype=dtype, path=path)
    for e, a in enumerate(s["advectee"]):
        run.set_advectee(a, e)
    for d, a in enumerate(s["advector"]):
        run.set_advector(a, d)
    return run


@pytest.mark.parametrize("case", list(setups.ADVSCHEME_CASES))
def test_advscheme_opts_1d(case):
    ref = np.load(os.path.join(GOLD, "advscheme_opts.npz"))[case]
    s = setups.advscheme_opts()
    run = run_setup(s, setups.ADVSCHEME_CASES[case], 2)
    run.advance(s["nt"])
    np.testing.assert_allclose(run.advectee(0), ref[2], rtol=0, atol=6e-6)
    np.testing.assert_allclose(run.advectee(1), ref[3], rtol=0, atol=6e-6)


def test_basic_example_1d():
    ref = np.load(os.path.join(GOLD, "basic_example.npz"))
    s = setups.basic_example()
    run = run_setup(s, s["opts"], 2)
    for rec in ref["records"][1:]:
        run.advance(20)
        np.testing.assert_allclose(run.advectee(), rec, rtol=0, atol=6e-6)


@pytest.mark.parametrize("case", list(setups.CONE_CASES))
def test_rotating_cone_2d(case):
    s = setups.rotating_cone()
    opts, iters = setups.CONE_CASES[case]
    run = run_setup(s, opts, iters)
    run.advance(s["nt"])
    st = setups.cone_stats(s["advectee"][0], run.advectee(), s["nt"], s["dt"])
    want = golden()["rotating_cone_2d"][case]
    for k in ["min(psi)", "max(psi)", "rms error"]:
        assert abs(st[k] - want["tN:" + k]) <= 6e-9, (k, st[k], want["tN:" + k])


@pytest.mark.parametrize("case", list(setups.SPHERE_CASES))
def test_revolving_sphere_3d(case):
    s = setups.revolving_sphere()
    opts, iters = setups.SPHERE_CASES[case]
    run = run_setup(s, opts, iters)
    run.advance(s["nt"])
    out = run.advectee()
    st = setups.sphere_stats(s["advectee"][0], out, s["nt"], s["dt"])
    want = golden()["revolving_sphere_3d"][case]
    for k in ["max(solution)", "min(solution)", "Linf", "L2", "L1"]:
        assert abs(st[k] - want["tN:" + k]) <= 6e-9, (k, st[k], want["tN:" + k])
    check_sphere_fields(case, out)


# 2_convergence_1d: all 8 grid steps x 19 Courant numbers x 8 solvers, 4 significant digits
def test_convergence_1d_all():
    import math
    conv = golden()["convergence_1d"]
    want = {(k, dx, c): e for k, rows in conv.items() for dx, c, e in rows}
    checked = 0
    for dx in setups.CONVERGENCE_DXS:
        for cour in setups.CONVERGENCE_COURANTS:
            s = setups.convergence_1d(dx, cour)
            for key, (opts, iters) in setups.CONVERGENCE_SOLVERS.items():
                run = make_run(s["grid"], opts, n_iters=iters, bcs=s["bcs"])
                run.set_advectee(s["advectee"][0])
                run.set_advector(s["advector"][0], 0)
                run.advance(s["nt"])
                got = setups.convergence_error(run.advectee(), s["exact"], s["nt"], s["dt"])
                w = want[(key, dx, cour)]
                assert abs(got - w) <= 0.5e-4 * 10 ** math.floor(math.log10(abs(w))) * 1.01, (key, dx, cour, got, w)
                run.close()
                checked += 1
    assert checked == 8 * 19 * 8


# the output path on the same run: fields leave the GPU only at the output steps
# (0 and 556) and are written in the reference's layout; the written psi passes
# the field check and the XDMF files equal the reference's
def test_revolving_sphere_output(tmp_path):
    import sys
    from libmpdataxx_b200 import output
    sys.path.insert(0, GOLD)
    import hdf5_read
    with open(os.path.join(GOLD, "output_layout.json")) as f:
        layout = json.load(f)
    s = setups.revolving_sphere()
    opts, iters = setups.SPHERE_CASES["fct"]
    run = run_setup(s, opts, iters)
    dx = 100.0 / (59 - 1)
    w = output.hdf5_xdmf(str(tmp_path), s["grid"], s["dt"], (dx, dx, dx), {0: "psi"}, opts_str="fct", n_iters=iters)
    w.run(run, s["nt"], s["nt"])
    psi = hdf5_read.read_dataset(str(tmp_path / "timestep0000000556.h5"), "psi")
    check_sphere_fields("fct", psi.astype(np.float64))
    for name in ["timestep0000000000.xmf", "timestep0000000556.xmf", "temp.xmf"]:
        with open(str(tmp_path / name)) as fh:
            assert fh.read() == layout[name], name
