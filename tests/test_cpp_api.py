"""The header-only C++ API (concurr::cuda): programs written like the
reference's own tests compile against it here (no GPU needed) and, on a GPU,
reproduce the reference's golden results."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
BUILD = os.path.join(ROOT, "tests", "cpp", "_build")
LIBDIR = os.path.join(ROOT, "libmpdataxx_b200")


def _newest_input(src):
    """mtime of the program's source or of any header it can include (mpdx.h, the C++ API)."""
    t = os.path.getmtime(src)
    for top in (os.path.join(LIBDIR, "include"), os.path.join(ROOT, "include")):
        for d, _, files in os.walk(top):
            for f in files:
                t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def build(name):
    os.makedirs(BUILD, exist_ok=True)
    exe = os.path.join(BUILD, name)
    src = os.path.join(CPP, name + ".cpp")
    if not os.path.exists(exe) or os.path.getmtime(exe) < _newest_input(src):
        subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(LIBDIR, "include"), "-I",
                        os.path.join(ROOT, "include"), src, "-o", exe, "-L", LIBDIR, "-lmpdx",
                        f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


@pytest.mark.parametrize("name", ["advscheme_opts", "revolving_sphere"])
def test_cpp_programs_compile(name):
    assert os.path.exists(build(name))


@pytest.mark.gpu
def test_cpp_advscheme_opts_matches_golden():
    out = subprocess.run([build("advscheme_opts")], capture_output=True, text=True, check=True).stdout.split()
    vals = np.array([float(x) for x in out]).reshape(5, 2, 601)
    gold = np.load(os.path.join(ROOT, "tests", "golden", "advscheme_opts.npz"))
    for c, case in enumerate(["abs", "iga", "iga_tot", "iga_fct", "iga_tot_fct"]):
        np.testing.assert_allclose(vals[c, 0], gold[case][2], rtol=0, atol=6e-6)
        np.testing.assert_allclose(vals[c, 1], gold[case][3], rtol=0, atol=6e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("case,opts,iters", [("iga_fct", 33, 2), ("basic", 0, 2)])
def test_cpp_revolving_sphere_matches_golden(case, opts, iters):
    out = subprocess.run([build("revolving_sphere"), str(opts), str(iters)], capture_output=True, text=True,
                         check=True).stdout.split()
    got = [float(x) for x in out]
    with open(os.path.join(ROOT, "tests", "golden", "golden_stats.json")) as f:
        want = json.load(f)["revolving_sphere_3d"][case]
    for v, k in zip(got, ["max(solution)", "min(solution)", "Linf", "L2", "L1"]):
        assert abs(v - want["tN:" + k]) <= 6e-9, (k, v, want["tN:" + k])
