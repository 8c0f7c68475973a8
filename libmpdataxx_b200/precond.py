"""The learned GCR preconditioner network on its own (C ABI mpdx_pcnet_*).

    net = PCNet(grid=(64, 64, 32), wrap=(1, 1, 0), channels=(8, 16, 32, 64))
    q = net.forward(r)                 # r, q: float32 arrays of the grid's shape
    g = net.backward(r, dq)            # gradient of sum(dq * net(r)) over the parameters
    loss = net.train_step(r, target, lr=1e-3)

Parameters are one float32 vector: for each layer e0 e1 e2 e3 m3 d2 d1 d0 q the
weights (cout, taps, cin) then the biases (cout)."""
import ctypes

import numpy as np

from . import _lib

LAYERS = ["e0", "e1", "e2", "e3", "m3", "d2", "d1", "d0", "q"]


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class PCNet:
    def __init__(self, grid, wrap, channels=(8, 16, 32, 64), seed=0):
        self.L = _lib.lib()
        self.grid = tuple(int(g) for g in grid)
        self.nd = len(self.grid)
        self.channels = tuple(int(c) for c in channels)
        g = (ctypes.c_int * 3)(*(list(self.grid) + [1] * (3 - self.nd)))
        w = (ctypes.c_int * 3)(*(list(int(x) for x in wrap) + [1] * (3 - len(wrap))))
        c = (ctypes.c_int * 4)(*self.channels)
        h = ctypes.c_void_p()
        rc = self.L.mpdx_pcnet_create(self.nd, g, w, c, int(seed), ctypes.byref(h))
        if rc != _lib.MPDX_OK:
            raise _lib.MpdxError(rc, self.L.mpdx_pcnet_create_error().decode())
        self.h = h
        self.n_params = int(self.L.mpdx_pcnet_num_params(h))

    def _check(self, rc):
        if rc != _lib.MPDX_OK:
            raise _lib.MpdxError(rc, self.L.mpdx_pcnet_last_error(self.h).decode())

    def params(self):
        out = np.empty(self.n_params, dtype=np.float32)
        self._check(self.L.mpdx_pcnet_get_params(self.h, _fptr(out)))
        return out

    def set_params(self, p):
        p = _f32(p).reshape(-1)
        assert p.size == self.n_params
        self._check(self.L.mpdx_pcnet_set_params(self.h, _fptr(p)))

    def forward(self, r):
        r = _f32(r).reshape(self.grid)
        q = np.empty(self.grid, dtype=np.float32)
        self._check(self.L.mpdx_pcnet_forward(self.h, _fptr(r), _fptr(q)))
        return q

    def backward(self, r, dq):
        r = _f32(r).reshape(self.grid)
        dq = _f32(dq).reshape(self.grid)
        g = np.empty(self.n_params, dtype=np.float32)
        self._check(self.L.mpdx_pcnet_backward(self.h, _fptr(r), _fptr(dq), _fptr(g)))
        return g

    def train_step(self, r, target, lr=1e-3):
        r = _f32(r).reshape(self.grid)
        t = _f32(target).reshape(self.grid)
        loss = ctypes.c_double()
        self._check(self.L.mpdx_pcnet_train_step(self.h, _fptr(r), _fptr(t), float(lr), ctypes.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            self.L.mpdx_pcnet_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def unpack(vec, nd, channels=(8, 16, 32, 64)):
    """Split a parameter vector into the oracle's {W_name: (cout, taps, cin), b_name: (cout,)} dict."""
    nt = 27 if nd == 3 else 9
    c0, c1, c2, c3 = channels
    dims = {"e0": (1, c0), "e1": (c0, c1), "e2": (c1, c2), "e3": (c2, c3), "m3": (c3, c3),
            "d2": (c3, c2), "d1": (c2, c1), "d0": (c1, c0), "q": (c0, 1)}
    out, off = {}, 0
    for name in LAYERS:
        ci, co = dims[name]
        n = co * nt * ci
        out["W_" + name] = np.asarray(vec[off:off + n], dtype=np.float64).reshape(co, nt, ci)
        off += n
        out["b_" + name] = np.asarray(vec[off:off + co], dtype=np.float64)
        off += co
    return out


def pack(P, nd, channels=(8, 16, 32, 64)):
    parts = []
    for name in LAYERS:
        parts.append(np.asarray(P["W_" + name], dtype=np.float32).reshape(-1))
        parts.append(np.asarray(P["b_" + name], dtype=np.float32).reshape(-1))
    return np.concatenate(parts)
