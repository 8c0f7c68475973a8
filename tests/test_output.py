"""The output path (libmpdataxx_b200/output.py) against the reference's own output
files of the revolving-sphere fct run (tests/golden/output_layout.json, made by
make_golden.py from tests/paper_2015_GMD/4_revolving_sphere_3d/refdata/fct):

  * XDMF files byte for byte;
  * const.h5: the raw HDF5 dataspace, datatype and fill-value messages of T, X, Y,
    Z and every attribute message of the "advection" group byte for byte, the
    coordinate values and the output times exactly;
  * the psi dataset's datatype message byte for byte, its shape;
  * a write-read round trip through tests/golden/hdf5_read.py."""
import json
import math
import os
import sys

import numpy as np
import pytest

from libmpdataxx_b200 import output, setups

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLD)
import hdf5_read  # noqa: E402


def ref():
    with open(os.path.join(GOLD, "output_layout.json")) as f:
        return json.load(f)


def sphere_writer(outdir):
    s = setups.revolving_sphere()
    dx = 100.0 / (59 - 1)
    return output.hdf5_xdmf(outdir, s["grid"], s["dt"], (dx, dx, dx), {0: "psi"}, opts_str="fct", n_iters=2), s


def test_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    a = rng.normal(size=(5, 6, 7)).astype(np.float32)
    b = rng.normal(size=11)
    c = np.arange(12, dtype=np.int32).reshape(3, 4)
    p = str(tmp_path / "x.h5")
    output.write_h5(p, {"psi": a, "T": b, "ints": c}, {"grp": {"s": "abc", "f": 1.5, "i": 7, "b": True}})
    f = hdf5_read.File(p)
    assert hdf5_read.list_root(p) == ["T", "grp", "ints", "psi"]
    np.testing.assert_array_equal(f.dataset("psi"), a)
    np.testing.assert_array_equal(f.dataset("T"), b)
    np.testing.assert_array_equal(f.dataset("ints"), c)
    at = f.attributes("grp")
    assert at["s"] == "abc" and at["f"] == np.float32(1.5) and at["i"] == 7 and at["b"] == 1


def test_const_h5_matches_reference(tmp_path):
    r = ref()
    w, s = sphere_writer(str(tmp_path))
    w.start([0.0, 556 * s["dt"]])
    f = hdf5_read.File(str(tmp_path / "const.h5"))
    for key, hexbytes in r["messages"].items():
        name, t = key.split("/")
        if name == "psi":
            continue
        assert f.message_bytes(name, int(t)).hex() == hexbytes, key
    mine = f.attribute_messages("advection")
    assert sorted(mine) == sorted(r["advection"])
    for k, hexbytes in r["advection"].items():
        assert mine[k].hex() == hexbytes, k
    X, Y, Z = (f.dataset(a) for a in "XYZ")
    assert list(X.shape) == r["coords"]["shape"]
    np.testing.assert_array_equal(X[:, 0, 0], np.float32(r["coords"]["X"]))
    np.testing.assert_array_equal(Y[0, :, 0], np.float32(r["coords"]["Y"]))
    np.testing.assert_array_equal(Z[0, 0, :], np.float32(r["coords"]["Z"]))
    np.testing.assert_array_equal(f.dataset("T"), np.float32(r["coords"]["T"]))


def test_records_and_xdmf_match_reference(tmp_path):
    r = ref()
    w, s = sphere_writer(str(tmp_path))
    w.start([0.0, 556 * s["dt"]])
    psi = s["advectee"][0]
    w.record(0, {"psi": psi})
    w.record(556, {"psi": psi})
    for name in ["timestep0000000000.xmf", "timestep0000000556.xmf", "temp.xmf"]:
        with open(str(tmp_path / name)) as fh:
            assert fh.read() == r[name], name
    f = hdf5_read.File(str(tmp_path / "timestep0000000556.h5"))
    assert f.message_bytes("psi", 3).hex() == r["messages"]["psi/3"]
    assert f.dataset("psi").shape == (59, 59, 59)
    np.testing.assert_array_equal(f.dataset("psi"), psi.astype(np.float32))


def test_1d_output_rejected(tmp_path):
    with pytest.raises(ValueError, match="2D and 3D"):
        output.hdf5_xdmf(str(tmp_path), (10,), 1.0, (1.0,), {0: "psi"})


def test_run_records_on_output_steps_and_advances_all_steps(tmp_path):
    """run(): records at 0 and every outfreq steps, reads fields back only there, and
    advances the steps after the last output step too."""
    class FakeRun:
        def __init__(self):
            self.t, self.reads = 0, []

        def advance(self, n):
            self.t += n

        def advectee(self, e):
            self.reads.append(self.t)
            return np.full((4, 5), float(self.t))

    w = output.hdf5_xdmf(str(tmp_path), (4, 5), 0.5, (1.0, 2.0), {0: "psi"})
    r = FakeRun()
    w.run(r, 10, 3)
    assert r.t == 10 and r.reads == [0, 3, 6, 9]
    assert w.timesteps == ["timestep%010d.xmf" % t for t in (0, 3, 6, 9)]
    f = hdf5_read.File(str(tmp_path / "timestep0000000006.h5"))
    np.testing.assert_array_equal(f.dataset("psi"), np.full((4, 5), 6.0, np.float32))
    c = hdf5_read.File(str(tmp_path / "const.h5"))
    np.testing.assert_array_equal(c.dataset("T"), np.float32([0.0, 1.5, 3.0, 4.5]))
    np.testing.assert_array_equal(c.dataset("Y")[0, :], np.float32(2.0 * np.arange(6)))
