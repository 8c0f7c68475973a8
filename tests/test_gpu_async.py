"""Asynchronous pinned-memory transfers (mpdx_set_field_async /
mpdx_get_field_async): round trips through the pitched copies into the padded
field layout, and a pipelined host loop (advector upload overlapping the
previous step's download) that must give the synchronous loop's results bit
for bit."""
import numpy as np
import pytest
import torch

from libmpdataxx_b200 import _lib, opts as o, setups
from test_gpu_parity import make_run

pytestmark = pytest.mark.gpu


def pinned(a):
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


@pytest.mark.parametrize("grid", [(37,), (19, 23), (13, 11, 17)])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_async_round_trip(grid, dtype):
    run = make_run(grid, o.fct, dtype=dtype, max_abs_div_eps=1e30)
    rng = np.random.default_rng(len(grid))
    keep = []
    for kind, idx in [(_lib.FIELD_ADVECTEE, 0)] + [(_lib.FIELD_ADVECTOR, d) for d in range(len(grid))]:
        a = rng.normal(size=run._shape(kind, idx)).astype(dtype)
        t, h = pinned(a)
        keep.append(t)
        run.set_field_async(kind, idx, t.data_ptr())
        out_t = torch.empty(a.shape, dtype=t.dtype).pin_memory()
        keep.append(out_t)
        run.get_field_async(kind, idx, out_t.data_ptr())   # ordered after the upload of the same field
        run.sync()
        np.testing.assert_array_equal(out_t.numpy(), a)
        back = np.empty_like(a)
        run.L.mpdx_get_field(run.h, kind, idx, back.ctypes.data, None)  # synchronous path sees it too
        np.testing.assert_array_equal(back, a)


@pytest.mark.parametrize("grid,opts", [((24, 22, 41), o.iga | o.fct), ((40, 300), o.fct)])
def test_pipelined_loop_equals_synchronous_loop(grid, opts):
    s_in = []
    rng = np.random.default_rng(5)
    for k in range(4):
        if len(grid) == 3:
            adv = list(setups.periodic_curl_3d(grid, 7 + k, cmax=0.4, dtype=np.float32))
        else:
            adv = list(setups.periodic_curl_2d(grid[0], grid[1], 7 + k, cmax=0.4, dtype=np.float32))
        psi = setups.wrap_periodic(rng.uniform(0.5, 2.0, size=tuple(g - 1 for g in grid))).astype(np.float32)
        s_in.append([psi] + [a.astype(np.float32) for a in adv])
    ref = make_run(grid, opts, dtype=np.float32, path="auto", max_abs_div_eps=1e-5)
    want = []
    for step in s_in:
        ref.set_advectee(step[0])
        for d, a in enumerate(step[1:]):
            ref.set_advector(a, d)
        ref.advance(1)
        want.append(ref.advectee().copy())
    run = make_run(grid, opts, dtype=np.float32, path="auto", max_abs_div_eps=1e-5)
    hin = [[pinned(a)[0] for a in step] for step in s_in]
    hout = [torch.empty(grid, dtype=torch.float32).pin_memory() for _ in s_in]
    for k, step in enumerate(hin):
        for d, t in enumerate(step[1:]):
            run.set_field_async(_lib.FIELD_ADVECTOR, d, t.data_ptr())
        run.set_field_async(_lib.FIELD_ADVECTEE, 0, step[0].data_ptr())
        run.advance(1)
        run.get_field_async(_lib.FIELD_ADVECTEE, 0, hout[k].data_ptr())
    run.sync()
    for k in range(len(s_in)):
        np.testing.assert_array_equal(hout[k].numpy(), want[k])
    assert run.stats()["timestep"] == len(s_in)
