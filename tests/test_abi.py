"""CPU-side checks of the C ABI: the library loads, exports every entry point
that include/mpdx.h declares, its structs match the header's layout, and
argument validation (which runs before any CUDA call) reports the reference's
errors.  No kernel is launched here."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from libmpdataxx_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mpdx.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(mpdx_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_python_binding_exports():
    assert declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.SO_PATH], capture_output=True, text=True, check=True).stdout
    syms = set(re.findall(r" T (mpdx_\w+)", out))
    for name in declared():
        assert name in syms, name
        assert hasattr(L, name)


def test_struct_layout_matches_header():
    src = f"""
    #include <stdio.h>
    #include <stddef.h>
    #include "{HEADER}"
    int main() {{
      printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(mpdx_config), offsetof(mpdx_config, prs_fp64),
             sizeof(mpdx_step_stats), offsetof(mpdx_step_stats, path), sizeof(mpdx_tuning3d),
             offsetof(mpdx_tuning3d, ms));
      return 0;
    }}"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-std=c99", "-o", exe, c], check=True)
        vals = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert vals == [ctypes.sizeof(_lib.Config), _lib.Config.prs_fp64.offset,
                    ctypes.sizeof(_lib.StepStats), _lib.StepStats.path.offset,
                    ctypes.sizeof(_lib.Tuning3D), _lib.Tuning3D.ms.offset]


def _cfg(**kw):
    L = _lib.lib()
    c = _lib.Config()
    L.mpdx_config_default(ctypes.byref(c))
    for k, v in kw.items():
        if k == "grid":
            for q, g in enumerate(v):
                c.grid[q] = g
        else:
            setattr(c, k, v)
    return c


def _create(c):
    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.mpdx_create(ctypes.byref(c), ctypes.byref(h))
    msg = L.mpdx_create_error().decode()
    if h:
        L.mpdx_destroy(h)
    return rc, msg


def test_defaults_follow_reference():
    c = _cfg()
    from libmpdataxx_b200 import opts as o
    assert c.opts == o.iga | o.fct and c.n_iters == 2 and c.prs_k_iters == 4 and c.g == 9.81


def test_bogus_grid_size():
    rc, msg = _create(_cfg(n_dims=2, grid=(0, 5, 1)))
    assert rc == _lib.MPDX_E_GRID and msg == "libmpdata++: bogus grid size"


def test_unsupported_option_rejected():
    from libmpdataxx_b200 import opts as o
    rc, msg = _create(_cfg(n_dims=2, grid=(8, 8, 1), opts=1 << 13))  # no such option
    assert rc == _lib.MPDX_E_UNSUPPORTED and "not built" in msg
    # fot: the 2D FOT's static_asserts (formulae_mpdata_hot_2d.hpp:147-149)
    for bad in (o.fot, o.fot | o.tot, o.fot | o.iga, o.fot | o.iga | o.div_2nd):
        rc, msg = _create(_cfg(n_dims=2, grid=(8, 8, 1), opts=bad))
        assert rc == _lib.MPDX_E_ARG and "fot" in msg, bad
    # the divergence form's own rules (formulae_mpdata_{1,2,3}d.hpp enable_ifs / static_asserts)
    for bad in (o.div_3rd, o.div_2nd | o.div_3rd | o.div_3rd_dt, o.div_2nd | o.tot, o.div_2nd | o.dfl):
        rc, _ = _create(_cfg(n_dims=2, grid=(8, 8, 1), opts=bad))
        assert rc == _lib.MPDX_E_ARG, bad
    rc, _ = _create(_cfg(n_dims=2, grid=(8, 8, 1), opts=o.iga | o.abs))
    assert rc == _lib.MPDX_E_ARG


def test_null_arguments():
    L = _lib.lib()
    assert L.mpdx_create(None, None) == _lib.MPDX_E_ARG
    assert L.mpdx_advance(None, 1) == _lib.MPDX_E_ARG
    assert L.mpdx_last_error(None) == b"invalid handle"


def test_option_and_parameter_validation():
    from libmpdataxx_b200 import opts as o
    # nug is built for solvers::mpdata only
    rc, msg = _create(_cfg(solver=_lib.SOLVER_BOUSSINESQ, n_dims=2, n_eqns=3, grid=(8, 8, 1), opts=o.nug | o.fct,
                           dt=0.1, tht_ref=300.0))
    assert rc == _lib.MPDX_E_UNSUPPORTED and "nug" in msg
    rc, msg = _create(_cfg(n_dims=2, grid=(8, 8, 1), upwind_filter_freq=-1))
    assert rc == _lib.MPDX_E_ARG and "upwind_filter_freq" in msg
    # fot with iga and tot (or div_3rd) in 2D; in 1D and 3D the reference's formulae never
    # add fourth-order terms, so there the option is accepted and changes nothing
    for nd, grid, opts in ((2, (8, 8, 1), o.iga | o.tot | o.fot), (2, (8, 8, 1), o.iga | o.div_2nd | o.div_3rd | o.fot),
                           (3, (8, 8, 8), o.iga | o.fot), (1, (8, 1, 1), o.fot)):
        rc, msg = _create(_cfg(n_dims=nd, grid=grid, opts=opts))
        assert rc in (_lib.MPDX_OK, _lib.MPDX_E_CUDA), (nd, opts, msg)  # validation passed (no GPU: CUDA error)
    # the divergence form is built for solvers::mpdata (its advector is constant in time)
    rc, msg = _create(_cfg(solver=_lib.SOLVER_BOUSSINESQ, n_dims=2, n_eqns=3, grid=(8, 8, 1), opts=o.div_2nd,
                           dt=0.1, tht_ref=300.0))
    assert rc == _lib.MPDX_E_UNSUPPORTED and "solvers::mpdata" in msg
    # ... and for at most two passes (a third reads halo faces the reference never fills)
    rc, msg = _create(_cfg(n_dims=2, grid=(8, 8, 1), opts=o.div_2nd | o.div_3rd, n_iters=3))
    assert rc == _lib.MPDX_E_UNSUPPORTED and "n_iters" in msg


def test_async_transfer_arguments():
    L = _lib.lib()
    assert L.mpdx_set_field_async(None, 0, 0, None) == _lib.MPDX_E_ARG
    assert L.mpdx_get_field_async(None, 0, 0, None) == _lib.MPDX_E_ARG


def test_fused3d_bulk_copy_mode():
    """The process-wide plane-copy mode of the fused FP32 3D kernel: bulk copies by
    default, a negative mode only queries, any nonzero mode means on."""
    L = _lib.lib()
    assert L.mpdx_fused3d_bulk_copies(-1) == 1
    assert L.mpdx_fused3d_bulk_copies(0) == 1
    assert L.mpdx_fused3d_bulk_copies(-1) == 0
    assert L.mpdx_fused3d_bulk_copies(5) == 0
    assert L.mpdx_fused3d_bulk_copies(-1) == 1


def test_fused3d_planes_per_cta_setting():
    """The process-wide planes per CTA of the fused 3D kernel: tuned (0) by default,
    a negative value only queries, invalid values change nothing and return -1."""
    L = _lib.lib()
    assert L.mpdx_fused3d_planes_per_cta(-1) == 0
    for bad in (4, 6, 514, 1000, 33):
        assert L.mpdx_fused3d_planes_per_cta(bad) == -1
    assert L.mpdx_fused3d_planes_per_cta(-1) == 0
    assert L.mpdx_fused3d_planes_per_cta(96) == 0
    assert L.mpdx_fused3d_planes_per_cta(-1) == 96
    assert L.mpdx_fused3d_planes_per_cta(0) == 96
    assert L.mpdx_fused3d_planes_per_cta(-1) == 0
    out = _lib.Tuning3D()
    assert L.mpdx_fused3d_tuning(None, ctypes.byref(out)) == _lib.MPDX_E_ARG
