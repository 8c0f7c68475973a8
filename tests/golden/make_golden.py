"""Extract the reference's own golden data into small committed fixtures.

Runs only where the libmpdata++ source tree is available (it reads the
gzip'd refdata files of its test suite as text); the GPU host never runs it.
Outputs, next to this script:

  golden_stats.json   rotating-cone (2D) and revolving-sphere (3D) error stats,
                      2D Boussinesq per-10-step stats (min/max theta, max |u|),
                      1D convergence errors (8 solvers x 8 grid steps x 19 Courant numbers)
  advscheme_opts.npz  1D field dumps of tests/paper_2015_GMD/1_advscheme_opts
                      (601 cells, 5 option sets, t=0 and t=1200, 2 equations)
  basic_example.npz   1D field dumps of tests/paper_2015_GMD/0_basic_example
                      (101 cells, every 20 steps up to t=100)
  output_layout.json  the reference's output of the revolving-sphere fct run: its
                      XDMF files, the raw HDF5 messages of const.h5 (datasets and
                      attributes) and its coordinate samples
  revolving_sphere_fields.npz
                      the 3D psi fields of tests/paper_2015_GMD/4_revolving_sphere_3d
                      after 556 steps (HDF5, float32, read by hdf5_read.py): three
                      full planes through the sphere's centre and sums over 6^3-cell
                      blocks of the whole 59^3 field (the full fields would be 4 MB)

Usage:  python tests/golden/make_golden.py [path-to-libmpdataxx-checkout]
"""
import gzip
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_gz(path):
    with gzip.open(path, "rt") as f:
        return f.read()


def parse_gnuplot_log(text):
    """Split a gnuplot command stream into plots; each plot is a list of
    inline datasets (lists of floats) terminated by 'e' lines."""
    plots, cur, ds, name = [], None, None, None
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("set output"):
            name = s.split("'")[1]
        elif s.startswith("plot") or s.startswith("splot"):
            cur = {"name": name, "data": []}
            plots.append(cur)
            ds = []
        elif s == "e":
            cur["data"].append(ds)
            ds = []
        elif cur is not None and s and re.match(r"^[-+0-9.eE ]+$", s):
            ds.append([float(x) for x in s.split()])
    return plots


def stats_file(path):
    out = {}
    for line in read_gz(path).splitlines():
        if "=" in line:
            k, v = line.split("=", 1)
            k = k.strip()
            if k == "timestep":
                ts = int(v)
                out.setdefault("timesteps", []).append(ts)
                continue
            key = k if len(out.get("timesteps", [])) <= 1 else k
            try:
                val = float(v)
            except ValueError:
                continue
            prefix = "t0" if len(out["timesteps"]) == 1 else "tN"
            out[prefix + ":" + key] = val
    return out


def boussinesq_stats(path):
    rows, cur = [], None
    head = {}
    for line in read_gz(path).splitlines():
        if "=" not in line:
            continue
        k, v = [x.strip() for x in line.split("=", 1)]
        if k == "timestep":
            cur = {"timestep": int(v)}
            rows.append(cur)
        elif k.startswith("sum of initial perturbation squared"):
            head["sum_init_pert_2"] = float(v)
        elif k.startswith("sum of initial perturbation"):
            head["sum_init_pert"] = float(v)
        elif cur is not None:
            try:
                cur[k] = float(v)
            except ValueError:
                pass
    rows = [r for r in rows if r["timestep"] > 0]
    return {"header": head, "rows": rows}


SPHERE_BLOCK = 6


def sphere_fields(gmd):
    """Planes and block sums of the reference's 59^3 float32 output fields."""
    sys.path.insert(0, HERE)
    import hdf5_read
    d = os.path.join(gmd, "4_revolving_sphere_3d", "refdata")
    out = {}
    g0 = hdf5_read.read_dataset(os.path.join(d, "common", "timestep0000000000.h5"), "psi").astype(np.float64)
    # planes through the centre of the initial sphere (one revolution brings it back)
    w = g0 / g0.sum()
    idx = np.indices(g0.shape)
    centre = [int(round(float((w * idx[a]).sum()))) for a in range(3)]
    out["centre"] = np.array(centre)
    out["block"] = np.array(SPHERE_BLOCK)
    for case in ["upwind", "basic", "iga", "fct", "iga_fct"]:
        g = hdf5_read.read_dataset(os.path.join(d, case, "timestep0000000556.h5"), "psi")
        assert g.dtype == np.float32 and g.shape == (59, 59, 59)
        out[case + "/plane0"] = g[centre[0], :, :]
        out[case + "/plane1"] = g[:, centre[1], :]
        out[case + "/plane2"] = g[:, :, centre[2]]
        s, a = block_sums(g)
        out[case + "/block_sum"] = s
        out[case + "/block_abs"] = a
    return out


def output_layout(gmd):
    """The reference's output files of the revolving-sphere fct run: XDMF texts,
    the raw HDF5 messages of const.h5's datasets and attributes, coordinate samples."""
    sys.path.insert(0, HERE)
    import hdf5_read
    d = os.path.join(gmd, "4_revolving_sphere_3d", "refdata", "fct")
    out = {}
    for name in ["timestep0000000000.xmf", "timestep0000000556.xmf", "temp.xmf"]:
        with open(os.path.join(d, name)) as f:
            out[name] = f.read()
    c = hdf5_read.File(os.path.join(d, "const.h5"))
    msgs = {}
    for ds in ["T", "X", "Y", "Z"]:
        for t in (0x0001, 0x0003, 0x0005):
            msgs["%s/%d" % (ds, t)] = c.message_bytes(ds, t).hex()
    psi = hdf5_read.File(os.path.join(d, "timestep0000000556.h5"))
    msgs["psi/3"] = psi.message_bytes("psi", 0x0003).hex()
    msgs["psi/1"] = psi.message_bytes("psi", 0x0001).hex()
    out["messages"] = msgs
    out["advection"] = {k: v.hex() for k, v in c.attribute_messages("advection").items()}
    X, Y, Z = (c.dataset(a) for a in "XYZ")
    out["coords"] = {"X": X[:, 0, 0].tolist(), "Y": Y[0, :, 0].tolist(), "Z": Z[0, 0, :].tolist(),
                     "shape": list(X.shape), "T": c.dataset("T").tolist()}
    return out


def block_sums(f):
    """FP64 sums of f and |f| over blocks of SPHERE_BLOCK^3 cells (edge blocks smaller)."""
    f = np.asarray(f, dtype=np.float64)
    b = SPHERE_BLOCK
    s = np.add.reduceat(np.add.reduceat(np.add.reduceat(f, np.arange(0, f.shape[0], b), 0),
                                        np.arange(0, f.shape[1], b), 1), np.arange(0, f.shape[2], b), 2)
    a = np.add.reduceat(np.add.reduceat(np.add.reduceat(np.abs(f), np.arange(0, f.shape[0], b), 0),
                                        np.arange(0, f.shape[1], b), 1), np.arange(0, f.shape[2], b), 2)
    return s, a


def main(ref):
    gmd = os.path.join(ref, "tests", "paper_2015_GMD")
    golden = {"source": "libmpdata++ tests/paper_2015_GMD refdata"}

    cone = {}
    for case in ["basic", "fct", "iters3_tot_fct", "iga_fct", "iga_tot_fct"]:
        cone[case] = stats_file(os.path.join(gmd, "3_rotating_cone_2d", "refdata", f"stats_{case}_.txt.gz"))
    golden["rotating_cone_2d"] = cone

    sphere = {}
    for case in ["upwind", "basic", "iga", "fct", "iga_fct"]:
        sphere[case] = stats_file(os.path.join(gmd, "4_revolving_sphere_3d", "refdata", f"stats_{case}.txt.gz"))
    golden["revolving_sphere_3d"] = sphere

    golden["boussinesq_2d"] = boussinesq_stats(os.path.join(gmd, "8_boussinesq_2d", "refdata", "stats.txt.gz"))

    # 2_convergence_1d: rows "dx  courant  error" (4 significant digits) per solver key
    conv = {}
    for key in ["iters=1", "iters=2", "iters=3", "iters=3_tot", "iters=i", "iters=2_fct", "iters=i_fct",
                "iters=i_fct_tot"]:
        rows = []
        for line in read_gz(os.path.join(gmd, "2_convergence_1d", "refdata", f"err_mpdata_{key}.txt.gz")).splitlines():
            if line.strip():
                rows.append([float(x) for x in line.split()])
        conv[key] = rows
    golden["convergence_1d"] = conv

    with open(os.path.join(HERE, "golden_stats.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)

    plots = parse_gnuplot_log(read_gz(os.path.join(gmd, "1_advscheme_opts", "refdata", "log-orig.gz")))
    arrs = {}
    for p in plots:
        tag = p["name"].replace("out_", "").replace(".svg", "")
        data = np.array([[v[0] for v in ds] for ds in p["data"]], dtype=np.float64)
        arrs[tag] = data  # 4 datasets x 601 values
    np.savez_compressed(os.path.join(HERE, "advscheme_opts.npz"), **arrs)

    plots = parse_gnuplot_log(read_gz(os.path.join(gmd, "0_basic_example", "refdata", "log-orig.gz")))
    # 1D splot output repeats every value twice to emulate histeps
    # (libmpdata++/output/gnuplot.hpp:167-175); keep one copy per cell
    recs = [np.array([v[0] for v in ds])[::2] for p in plots for ds in p["data"]]
    np.savez_compressed(os.path.join(HERE, "basic_example.npz"), records=np.array(recs),
                        timesteps=np.arange(0, 101, 20))
    np.savez_compressed(os.path.join(HERE, "revolving_sphere_fields.npz"), **sphere_fields(gmd))
    with open(os.path.join(HERE, "output_layout.json"), "w") as f:
        json.dump(output_layout(gmd), f, indent=1, sort_keys=True)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the libmpdata++ source tree>")
    main(sys.argv[1])
