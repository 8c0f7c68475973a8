"""concurr::cuda -- the run object of the reference's API on top of the CUDA library.

Mirrors libmpdata++'s concurr::{serial,openmp,threads}<solver_t, bc...>
(concurr/detail/concurr_common.hpp:122-454, concurr/any.hpp:15-74):

    run = cuda(solvers.mpdata(ct_params), bcond.cyclic, bcond.cyclic, ..., p=rt)
    run.advectee(e)[...] = ...      # writable host mirror of the device field
    run.advector(d)[...] = ...      # view with lower bound (-1, 0, 0): element a <-> index a - 1
    run.advance(nt)
    run.advectee(e)                  # state after nt steps (downloaded on access)

Host mirrors handed out by advectee()/advector()/sclr_array() since the last
advance() are uploaded before the next one (the reference's views alias solver
memory, so a write through a view is seen by the next step); a mirror that was
not handed out again is not uploaded again, so write through a view obtained
after the last advance().  After advance() the advectee mirrors are refreshed
on the next access.  Fields otherwise stay on the device.
"""
import ctypes

import numpy as np

from . import _lib
from .solvers import boussinesq as _bq


def _check(L, h, rc):
    if rc != _lib.MPDX_OK:
        msg = L.mpdx_last_error(h).decode() if h else L.mpdx_create_error().decode()
        raise _lib.MpdxError(rc, _lib.MESSAGES.get(rc, msg) if rc in _lib.MESSAGES else msg)


class cuda:
    def __init__(self, solver, *bcs, p=None, path="auto"):
        self.solver = solver
        ct = solver.ct
        self.nd = int(ct.n_dims)
        if len(bcs) != 2 * self.nd:
            raise TypeError(f"expected {2 * self.nd} boundary conditions, got {len(bcs)}")
        if p is None:
            raise TypeError("rt_params p is required")
        self.p = p
        self.real_t = np.dtype(ct.real_t)
        self.n_eqns = int(ct.n_eqns)
        self.grid = tuple(int(g) for g in p.grid_size)[: self.nd]
        L = _lib.lib()
        self.L = L
        cfg = _lib.Config()
        L.mpdx_config_default(ctypes.byref(cfg))
        cfg.solver = _lib.SOLVER_BOUSSINESQ if isinstance(solver, _bq) else _lib.SOLVER_MPDATA
        cfg.n_dims = self.nd
        cfg.n_eqns = self.n_eqns
        for d in range(3):
            cfg.grid[d] = self.grid[d] if d < self.nd else 1
        cfg.opts = int(ct.opts)
        cfg.n_iters = int(getattr(p, "n_iters", 2))
        cfg.dtype = self.real_t.itemsize
        for q, b in enumerate(bcs):
            cfg.bcs[q] = _lib.BC[b if isinstance(b, str) else b.name]
        cfg.dt = float(getattr(p, "dt", 0.0))
        cfg.di = float(getattr(p, "di", 1.0) or 1.0)
        cfg.dj = float(getattr(p, "dj", 1.0) or 1.0)
        cfg.dk = float(getattr(p, "dk", 1.0) or 1.0)
        eps = getattr(p, "max_abs_div_eps", None)
        cfg.max_abs_div_eps = -1.0 if eps is None else float(eps)
        cfg.upwind_filter_freq = int(getattr(p, "upwind_filter_freq", 0) or 0)
        cfg.sptl_intrp = int(getattr(ct, "sptl_intrp", 0))
        cfg.path = {"auto": _lib.PATH_AUTO, "general": _lib.PATH_GENERAL, "fused": _lib.PATH_FUSED}[path]
        if isinstance(solver, _bq):
            solver.fill_config(cfg, p)
        h = ctypes.c_void_p()
        rc = L.mpdx_create(ctypes.byref(cfg), ctypes.byref(h))
        _check(L, None, rc)
        self.h = h
        self._mirrors = {}   # (kind, idx) -> ndarray
        self._fresh = set()  # mirrors known to equal the device copy
        self._dirty = set()  # mirrors handed out since the last upload

    # -- lifetime --------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.mpdx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # -- views ------------------------------------------------------------
    def _shape(self, kind, idx):
        if kind == _lib.FIELD_ADVECTOR:
            s = list(self.grid)
            if idx > 0:
                s[0] += 1
            return tuple(s)
        return self.grid

    def _mirror(self, kind, idx):
        key = (kind, idx)
        a = self._mirrors.get(key)
        if a is None:
            a = np.empty(self._shape(kind, idx), dtype=self.real_t)
            self._mirrors[key] = a
        if key not in self._fresh:
            _check(self.L, self.h, self.L.mpdx_get_field(self.h, kind, idx, a.ctypes.data, None))
            self._fresh.add(key)
        self._dirty.add(key)
        return a

    def advectee(self, e=0):
        return self._mirror(_lib.FIELD_ADVECTEE, e)

    def advector(self, d=0):
        return self._mirror(_lib.FIELD_ADVECTOR, d)

    _SCLR = {"tht_e": _lib.SCLR_THT_E, "tht_abs": _lib.SCLR_THT_ABS, "hflux_frc": _lib.SCLR_HFLUX_FRC}

    def sclr_array(self, name, n=0):
        """Named scalar arrays of the Boussinesq solver (boussinesq_common.hpp:20-60)."""
        if name not in self._SCLR:
            raise KeyError(name)
        return self._mirror(_lib.FIELD_SCLR_ARRAY, self._SCLR[name])

    def vab_coefficient(self):
        """vab_coefficient() (concurr_common.hpp:420-423): the velocity absorber's coefficient."""
        return self._mirror(_lib.FIELD_SCLR_ARRAY, _lib.SCLR_VAB_COEFF)

    def vab_relaxed_state(self, d=0):
        """vab_relaxed_state(d) (concurr_common.hpp:425-428): the velocity the absorber relaxes to."""
        return self._mirror(_lib.FIELD_SCLR_ARRAY, _lib.SCLR_VAB_RELAX + d)

    def g_factor(self):
        """G of the nug option (sharedmem.hpp:373-380): a writable mirror, uploaded before the next advance."""
        return self._mirror(_lib.FIELD_G, 0)

    def set_g_factor(self, a):
        self.set_field(_lib.FIELD_G, 0, a)

    def advectee_global(self, e=0):
        return self.advectee(e)

    def _flush(self):
        for (kind, idx), a in self._mirrors.items():
            if (kind, idx) in self._fresh and (kind, idx) in self._dirty:
                _check(self.L, self.h, self.L.mpdx_set_field(self.h, kind, idx, np.ascontiguousarray(a).ctypes.data, None))
        self._dirty = set()
        # state fields change on the device; advectors, scalar arrays and G do not
        self._fresh = {k for k in self._fresh if k[0] in (_lib.FIELD_ADVECTOR, _lib.FIELD_SCLR_ARRAY, _lib.FIELD_G)}

    # -- explicit transfers ---------------------------------------------------
    def set_field(self, kind, idx, a):
        a = np.ascontiguousarray(np.broadcast_to(a, self._shape(kind, idx)), dtype=self.real_t)
        _check(self.L, self.h, self.L.mpdx_set_field(self.h, kind, idx, a.ctypes.data, None))
        self._mirrors.pop((kind, idx), None)
        self._fresh.discard((kind, idx))
        self._dirty.discard((kind, idx))

    def set_advectee(self, a, e=0):
        self.set_field(_lib.FIELD_ADVECTEE, e, a)

    def set_advector(self, a, d=0):
        self.set_field(_lib.FIELD_ADVECTOR, d, a)

    def set_field_device(self, kind, idx, ptr):
        _check(self.L, self.h, self.L.mpdx_set_field_device(self.h, kind, idx, ctypes.c_void_p(ptr)))
        self._mirrors.pop((kind, idx), None)
        self._fresh.discard((kind, idx))
        self._dirty.discard((kind, idx))

    def get_field_device(self, kind, idx, ptr):
        _check(self.L, self.h, self.L.mpdx_get_field_device(self.h, kind, idx, ctypes.c_void_p(ptr)))

    def set_field_async(self, kind, idx, ptr):
        """Upload from page-locked host memory at ptr (C order) without waiting;
        the buffer must stay untouched until sync()."""
        _check(self.L, self.h, self.L.mpdx_set_field_async(self.h, kind, idx, ctypes.c_void_p(ptr)))
        self._mirrors.pop((kind, idx), None)
        self._fresh.discard((kind, idx))
        self._dirty.discard((kind, idx))

    def get_field_async(self, kind, idx, ptr):
        """Download into page-locked host memory at ptr (C order), complete after sync()."""
        _check(self.L, self.h, self.L.mpdx_get_field_async(self.h, kind, idx, ctypes.c_void_p(ptr)))

    # -- time stepping ----------------------------------------------------------
    def advance(self, nt):
        self._flush()
        _check(self.L, self.h, self.L.mpdx_advance(self.h, int(nt)))

    def sync(self):
        _check(self.L, self.h, self.L.mpdx_sync(self.h))

    @property
    def stream(self):
        return self.L.mpdx_stream(self.h)

    def stats(self):
        s = _lib.StepStats()
        _check(self.L, self.h, self.L.mpdx_stats(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in _lib.StepStats._fields_}

    def tuning3d(self):
        """The fused 3D kernel's planes-per-CTA tuner on this handle (no counterpart in the
        reference): {"chosen": planes per CTA (0 while tuning), "candidates": [(planes, ms per step)]}."""
        t = _lib.Tuning3D()
        _check(self.L, self.h, self.L.mpdx_fused3d_tuning(self.h, ctypes.byref(t)))
        return {"chosen": t.chosen, "candidates": [(t.lx[q], t.ms[q]) for q in range(t.n_candidates)]}

    # -- learned GCR preconditioner (Boussinesq solvers; no counterpart in the reference) --
    def precond_record(self, max_pairs):
        """Keep the (initial residual, correction) pair of each of the next max_pairs pressure solves."""
        _check(self.L, self.h, self.L.mpdx_precond_record(self.h, int(max_pairs)))

    def precond_set_directions(self, nl):
        """Learned corrections at the start of every learned solve: 0..64 (1 by default), or -1 to tune them by solve time."""
        _check(self.L, self.h, self.L.mpdx_precond_set_directions(self.h, int(nl)))

    def precond_directions(self):
        """Learned search directions at the start of the last learned solve (-1: none yet)."""
        return int(self.L.mpdx_precond_directions(self.h))

    def precond_pairs(self):
        return int(self.L.mpdx_precond_pairs(self.h))

    def precond_train(self, steps, lr=1e-3, seed=0):
        """Adam steps of the network on the recorded pairs; returns the mean loss of the last tenth."""
        loss = ctypes.c_double()
        _check(self.L, self.h, self.L.mpdx_precond_train(self.h, int(steps), float(lr), int(seed), ctypes.byref(loss)))
        return loss.value

    def precond_enable(self, on=True):
        """GCR search directions from the network's output (flexible GCR) instead of the residual."""
        _check(self.L, self.h, self.L.mpdx_precond_enable(self.h, 1 if on else 0))

    def precond_params(self):
        n = int(self.L.mpdx_precond_num_params(self.h))
        if n < 0:
            raise _lib.MpdxError(_lib.MPDX_E_UNSUPPORTED, self.L.mpdx_last_error(self.h).decode())
        out = np.empty(n, dtype=np.float32)
        _check(self.L, self.h, self.L.mpdx_precond_get_params(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def precond_loss_grad(self, r, t, c, grad=True):
        """Energy-norm training loss of the learned preconditioner for one pair
        (residual r, correction t with A t = -r, interior arrays) at output scale
        c, and its gradient with respect to the network parameters."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64)
        loss = ctypes.c_double()
        g = np.zeros(self.L.mpdx_precond_num_params(self.h), dtype=np.float32) if grad else None
        dp = ctypes.POINTER(ctypes.c_double)
        _check(self.L, self.h, self.L.mpdx_precond_loss_grad(
            self.h, r.ctypes.data_as(dp), t.ctypes.data_as(dp), float(c), ctypes.byref(loss),
            g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if grad else None))
        return loss.value, g

    def set_precond_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(self.L, self.h, self.L.mpdx_precond_set_params(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def min(self, e=0):
        """run.min(e): equation 0 from the device-side statistics (no field download)."""
        if e == 0:
            self._flush()
            return float(self.stats()["min"])
        return float(self.advectee(e).min())

    def max(self, e=0):
        if e == 0:
            self._flush()
            return float(self.stats()["max"])
        return float(self.advectee(e).max())

    def time(self):
        st = self.stats()
        return st["timestep"] * float(getattr(self.p, "dt", 0.0))


class batch:
    """Advance many independent 2D run objects together (no counterpart in the
    reference): one persistent fused launch per step over all problems, tile
    shape chosen by timing the first steps, or one launch per problem
    (mode="per_problem").  Results equal those of advancing each run alone.

        runs = [cuda(solvers.mpdata(ct), bcond.cyclic, ..., p=p_k) for p_k in params]
        b = batch(runs)
        b.advance(500)
        runs[3].advectee()
    """

    def __init__(self, runs, mode="persistent"):
        self.runs = list(runs)
        L = _lib.lib()
        self.L = L
        hs = (ctypes.c_void_p * len(self.runs))(*[r.h.value for r in self.runs])
        h = ctypes.c_void_p()
        m = {"persistent": _lib.BATCH_PERSISTENT, "per_problem": _lib.BATCH_PER_PROBLEM}[mode]
        rc = L.mpdx_batch_create(hs, len(self.runs), m, ctypes.byref(h))
        if rc != _lib.MPDX_OK:
            raise _lib.MpdxError(rc, L.mpdx_create_error().decode())
        self.h = h

    def _check(self, rc):
        if rc != _lib.MPDX_OK:
            raise _lib.MpdxError(rc, self.L.mpdx_batch_last_error(self.h).decode())

    def advance(self, nt):
        for r in self.runs:
            r._flush()
        self._check(self.L.mpdx_batch_advance(self.h, int(nt)))

    def sync(self):
        self._check(self.L.mpdx_batch_sync(self.h))

    def info(self):
        i = _lib.BatchInfo()
        self._check(self.L.mpdx_batch_get_info(self.h, ctypes.byref(i)))
        d = {k: getattr(i, k) for k, _ in _lib.BatchInfo._fields_ if k != "tune_ms"}
        d["tune_ms"] = list(i.tune_ms)[: i.n_candidates]
        d["mode"] = "persistent" if i.mode == _lib.BATCH_PERSISTENT else "per_problem"
        return d

    def close(self):
        if getattr(self, "h", None):
            self.L.mpdx_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
