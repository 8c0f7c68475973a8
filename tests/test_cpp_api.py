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


@pytest.mark.parametrize("name", ["advscheme_opts", "revolving_sphere", "output_layout", "revolving_sphere_output",
                                  "output_outstart"])
def test_cpp_programs_compile(name):
    assert os.path.exists(build(name))


def _output_layout():
    with open(os.path.join(ROOT, "tests", "golden", "output_layout.json")) as f:
        return json.load(f)


def test_cpp_output_writer_matches_reference_layout(tmp_path):
    """The C++ writer's const.h5 messages, coordinates, times and XDMF files are the
    reference's (the same checks as tests/test_output.py for the Python writer)."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import hdf5_read
    subprocess.run([build("output_layout"), str(tmp_path)], check=True)
    r = _output_layout()
    f = hdf5_read.File(str(tmp_path / "const.h5"))
    for key, hexbytes in r["messages"].items():
        name, t = key.split("/")
        if name != "psi":
            assert f.message_bytes(name, int(t)).hex() == hexbytes, key
    mine = f.attribute_messages("advection")
    assert {k: v.hex() for k, v in mine.items()} == r["advection"]
    np.testing.assert_array_equal(f.dataset("X")[:, 0, 0], np.float32(r["coords"]["X"]))
    np.testing.assert_array_equal(f.dataset("Z")[0, 0, :], np.float32(r["coords"]["Z"]))
    np.testing.assert_array_equal(f.dataset("T"), np.float32(r["coords"]["T"]))
    for name in ["timestep0000000000.xmf", "timestep0000000556.xmf", "temp.xmf"]:
        assert (tmp_path / name).read_text() == r[name], name
    g = hdf5_read.File(str(tmp_path / "timestep0000000556.h5"))
    assert g.message_bytes("psi", 3).hex() == r["messages"]["psi/3"]


@pytest.mark.gpu
def test_cpp_revolving_sphere_output_matches_golden(tmp_path):
    """output::hdf5_xdmf<slv_t> on concurr::cuda: the written field passes the 3D
    golden field check and the XDMF files are the reference's."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import hdf5_read
    from runners import check_sphere_fields
    subprocess.run([build("revolving_sphere_output"), str(tmp_path)], check=True)
    psi = hdf5_read.read_dataset(str(tmp_path / "timestep0000000556.h5"), "psi")
    check_sphere_fields("fct", psi.astype(np.float64))
    r = _output_layout()
    for name in ["timestep0000000000.xmf", "timestep0000000556.xmf", "temp.xmf"]:
        assert (tmp_path / name).read_text() == r[name], name


@pytest.mark.gpu
def test_cpp_output_outstart_records_start_state_and_t0(tmp_path):
    """outstart > 0: the state at the start of every advance() call is recorded
    (output_common.hpp hook_ante_loop) and T holds t = 0 before the output
    times outstart, outstart + outfreq, ... (output/hdf5.hpp T axis)."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import hdf5_read
    one, two = tmp_path / "one", tmp_path / "two"
    subprocess.run([build("output_outstart"), str(one), "1"], check=True)
    names = sorted(p.name for p in one.glob("timestep*.h5"))
    assert names == ["timestep%010d.h5" % t for t in (0, 4, 6, 8, 10)], names
    np.testing.assert_array_equal(hdf5_read.File(str(one / "const.h5")).dataset("T"),
                                  np.float32([0.0, 2.0, 3.0, 4.0, 5.0]))
    psi0 = hdf5_read.read_dataset(str(one / "timestep0000000000.h5"), "psi")
    assert psi0.shape == (16, 12) and psi0.min() == 1.0 and psi0.max() == 2.0
    subprocess.run([build("output_outstart"), str(two), "2"], check=True)
    names = sorted(p.name for p in two.glob("timestep*.h5"))
    assert names == ["timestep%010d.h5" % t for t in (0, 4, 6, 8, 10, 12)], names
    # the second call's const.h5 is rewritten for its nt = 3: (3 - 4) / 2 truncates to 0,
    # so T = [0, outstart dt] as the reference computes it
    np.testing.assert_array_equal(hdf5_read.File(str(two / "const.h5")).dataset("T"), np.float32([0.0, 2.0]))
    assert (two / "temp.xmf").read_text().count("timestep0000000010.xmf") == 2


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
