"""ORACLE -- test infrastructure only.

ctypes binding of the CPU restatement in oracle/ (liboracle.so: IEEE parity
build; liboracle_omp.so: -Ofast + OpenMP build timed as the CPU baseline).
Imported only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
leg.  The object mirrors the reference's run object: advectee(e) / advector(d)
arrays in the reference's view index conventions, advance(nt).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

_libs = {}


def build():
    """Compile both oracle builds (make is incremental)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(fast=False):
    name = "liboracle_omp.so" if fast else "liboracle.so"
    if name in _libs:
        return _libs[name]
    path = os.path.join(BUILD, name)
    if not os.path.exists(path):
        build()
    L = ctypes.CDLL(path)
    vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    L.orc_mpdata_create.restype = vp
    L.orc_mpdata_create.argtypes = [ctypes.c_int, ctypes.c_int, ip, ctypes.c_int, ctypes.c_uint, ctypes.c_int,
                                    ip, ctypes.c_double, ctypes.c_char_p, ctypes.c_int]
    L.orc_boussinesq_create.restype = vp
    L.orc_boussinesq_create.argtypes = [ctypes.c_int, ctypes.c_int, ip, ctypes.c_uint, ctypes.c_int, ip, dp,
                                        ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    L.orc_destroy.argtypes = [vp]
    for f in ("orc_set_advectee", "orc_get_advectee", "orc_set_advector", "orc_get_advector"):
        getattr(L, f).argtypes = [vp, ctypes.c_int, dp]
        getattr(L, f).restype = ctypes.c_int
    L.orc_set_sclr_array.argtypes = [vp, ctypes.c_char_p, dp]
    L.orc_set_sclr_array.restype = ctypes.c_int
    L.orc_set_param.argtypes = [vp, ctypes.c_char_p, ctypes.c_double]
    L.orc_set_param.restype = ctypes.c_int
    L.orc_advance.argtypes = [vp, ctypes.c_longlong]
    L.orc_advance.restype = ctypes.c_int
    L.orc_timestep.argtypes = [vp]
    L.orc_timestep.restype = ctypes.c_longlong
    L.orc_last_iters.argtypes = [vp]
    L.orc_last_iters.restype = ctypes.c_longlong
    L.orc_last_error.argtypes = [vp]
    L.orc_last_error.restype = ctypes.c_char_p
    L.orc_set_threads.argtypes = [ctypes.c_int]
    L.orc_max_threads.restype = ctypes.c_int
    _libs[name] = L
    return L


def set_threads(n, fast=True):
    """OpenMP threads of the oracle's parallel loops from now on."""
    lib(fast).orc_set_threads(int(n))


def max_threads(fast=True):
    return lib(fast).orc_max_threads()


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ints(v):
    return (ctypes.c_int * len(v))(*v)


class Oracle:
    """CPU restatement of one concurr run (solvers::mpdata or boussinesq)."""

    def __init__(self, grid, opts, n_iters=2, n_eqns=1, bcs=None, dtype=np.float64,
                 max_abs_div_eps=None, fast=False, boussinesq=None, upwind_filter_freq=0):
        self.L = lib(fast)
        self.grid = tuple(int(g) for g in grid)
        self.nd = len(self.grid)
        self.n_eqns = n_eqns
        bcs = bcs or ["cyclic"] * (2 * self.nd)
        kinds = {"cyclic": 0, "open": 1, "rigid": 2}
        bc = [kinds[b] for b in bcs]
        dt = 8 if np.dtype(dtype) == np.float64 else 4
        err = ctypes.create_string_buffer(512)
        if boussinesq is None:
            self.h = self.L.orc_mpdata_create(dt, self.nd, _ints(self.grid), n_eqns, int(opts), int(n_iters),
                                              _ints(bc), -1.0 if max_abs_div_eps is None else float(max_abs_div_eps),
                                              err, 512)
        else:
            prm = np.array(boussinesq["prm"], dtype=np.float64)
            self.h = self.L.orc_boussinesq_create(dt, self.nd, _ints(self.grid), int(opts), int(n_iters), _ints(bc),
                                                  _dptr(prm), int(boussinesq.get("prs_k", 1)), err, 512)
        if not self.h:
            raise RuntimeError(err.value.decode())
        if upwind_filter_freq:
            self._check(self.L.orc_set_param(self.h, b"upwind_filter_freq", float(upwind_filter_freq)))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.L.orc_last_error(self.h).decode())

    def advector_shape(self, d):
        s = list(self.grid)
        if d > 0:
            s[0] += 1
        return tuple(s)

    def set_advectee(self, a, e=0):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.grid)
        self._check(self.L.orc_set_advectee(self.h, e, _dptr(a)))

    def advectee(self, e=0):
        out = np.empty(self.grid)
        self._check(self.L.orc_get_advectee(self.h, e, _dptr(out)))
        return out

    def set_advector(self, a, d=0):
        a = np.ascontiguousarray(np.broadcast_to(a, self.advector_shape(d)), dtype=np.float64)
        self._check(self.L.orc_set_advector(self.h, d, _dptr(a)))

    def advector(self, d=0):
        out = np.empty(self.advector_shape(d))
        self._check(self.L.orc_get_advector(self.h, d, _dptr(out)))
        return out

    def set_sclr_array(self, name, a):
        a = np.ascontiguousarray(np.broadcast_to(a, self.grid), dtype=np.float64)
        self._check(self.L.orc_set_sclr_array(self.h, name.encode(), _dptr(a)))

    def set_param(self, name, value):
        """A parameter the reference fixes at compile time or in rt_params (upwind_filter_freq;
        impl_tht and vip_vab of the Boussinesq solver), set before the first advance."""
        self._check(self.L.orc_set_param(self.h, name.encode(), float(value)))

    def set_g_factor(self, a):
        """g_factor() = a (nug option): G at the interior points."""
        self.set_sclr_array("G", a)

    def advance(self, nt):
        self._check(self.L.orc_advance(self.h, int(nt)))

    @property
    def timestep(self):
        return self.L.orc_timestep(self.h)

    @property
    def last_iters(self):
        return self.L.orc_last_iters(self.h)
