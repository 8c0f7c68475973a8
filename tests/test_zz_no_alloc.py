"""mpdx_field_stats_noalloc: field statistics with no device allocation.

Some callers cannot allocate device memory where they need the numbers (for
example code whose free device memory is owned by a caching or pooled
allocator, or a loop whose memory budget is fixed when it starts).  This entry
point serves them: it keeps its scratch in a fixed-size file-scope device
array instead of allocating.  The test calls it through the C ABI on a field
and checks it against mpdx_stats() of a solver holding the same field, on two
calls in a row (the second call reuses the scratch the first one left
behind).  This file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from libmpdataxx_b200 import _lib

pytestmark = pytest.mark.gpu


def _entry():
    L = _lib.lib()
    f = L.mpdx_field_stats_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                  ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
    f.restype = ctypes.c_int
    return f


def _i64(v):
    return (ctypes.c_int64 * 3)(*v)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_stats_match_solver_stats(dtype):
    import torch
    from test_gpu_parity import make_run

    grid = (37, 29, 45)
    rng = np.random.default_rng(123)
    psi = rng.uniform(-2.0, 5.0, size=grid).astype(dtype)
    run = make_run(grid, 0, n_iters=1, dtype=dtype, max_abs_div_eps=1.0)
    run.set_advectee(psi)
    ref = run.stats()  # mass over the unique cells (point n-1 of each cyclic axis excluded)

    dev = torch.from_numpy(psi).cuda()
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    f = _entry()
    n = _i64(grid)
    strides = _i64(dev.stride())
    m = _i64([g - 1 for g in grid])
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out.zero_()
        rc = f(dev.data_ptr(), np.dtype(dtype).itemsize, n, strides, m, out.data_ptr(), stream, err, 256)
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        mass, mn, mx = out.tolist()
        assert abs(mass - ref["mass"]) <= 1e-12 * max(1.0, abs(ref["mass"])), (call, mass, ref["mass"])
        assert mn == ref["min"] and mx == ref["max"], (call, mn, mx, ref)
    run.close()


def test_noalloc_rejects_oversized_fields():
    import torch
    dev = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    rc = _entry()(dev.data_ptr(), 8, _i64([8193, 1, 1]), _i64([1, 1, 1]), _i64([8193, 1, 1]), out.data_ptr(),
                  None, err, 256)
    assert rc == _lib.MPDX_E_ARG and "8192" in err.value.decode()
    # slice extents that the int-indexed kernels cannot address: each one alone,
    # and a product at 2^31 or beyond (no launch happens, nothing is read)
    for n in ([1, 2 ** 31, 1], [1, 1, 2 ** 31], [1, 2 ** 16, 2 ** 15], [1, 2 ** 62, 2 ** 62]):
        rc = _entry()(dev.data_ptr(), 8, _i64(n), _i64([1, 1, 1]), _i64([0, 0, 0]), out.data_ptr(), None, err, 256)
        assert rc == _lib.MPDX_E_ARG and "2^31" in err.value.decode(), (n, err.value)
