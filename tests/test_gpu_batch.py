"""Batched advance of independent 2D problems in one persistent launch.

The batched results must equal (bit for bit) those of advancing every problem
alone through the fused path, in both batch modes; the FP64 batch must match
the oracle to 1e-12."""
import numpy as np
import pytest

from libmpdataxx_b200 import bcond, concurr, opts as o, setups, solvers
from oracle import Oracle
from runners import load

pytestmark = pytest.mark.gpu


def make(s, opts, n_iters, dtype):
    class ct(solvers.ct_params_default_t):
        pass

    ct.real_t = dtype
    ct.n_dims = 2
    ct.n_eqns = 1
    ct.opts = opts
    p = solvers.mpdata.rt_params_t(grid_size=list(s["grid"]), n_iters=n_iters, max_abs_div_eps=1e-6)
    run = concurr.cuda(solvers.mpdata(ct), *[getattr(bcond, b) for b in s["bcs"]], p=p, path="fused")
    run.set_advectee(s["advectee"][0])
    for d, a in enumerate(s["advector"]):
        run.set_advector(a, d)
    return run


@pytest.mark.parametrize("opts,n_iters", [(o.fct, 2), (o.iga | o.fct, 2), (o.fct, 3), (0, 2)])
@pytest.mark.parametrize("mode", ["persistent", "per_problem"])
def test_batch_equals_individual_runs_fp32(opts, n_iters, mode):
    probs = setups.batched_problems(n=9, seed=11, lo=20, hi=300)
    alone = [make(s, opts, n_iters, np.float32) for s in probs]
    for r in alone:
        r.advance(33)
    runs = [make(s, opts, n_iters, np.float32) for s in probs]
    b = concurr.batch(runs, mode=mode)
    b.advance(5)
    b.advance(8)   # tuning (8 candidates x 3 steps) spans calls; odd step counts exercise both parities
    b.advance(20)
    for r, a in zip(runs, alone):
        assert r.stats()["timestep"] == 33
        np.testing.assert_array_equal(r.advectee(), a.advectee())
    info = b.info()
    assert info["n_problems"] == 9 and info["cells"] == sum(s["grid"][0] * s["grid"][1] for s in probs)
    if mode == "persistent":
        assert info["n_candidates"] == 8 and info["tile_nt"] == 32 and info["tile_lx"] in (16, 32, 64, 128)
        assert all(t > 0 for t in info["tune_ms"][:info["n_candidates"]])
        assert info["grid"] > 0
    b.close()


def test_batch_fp64_matches_oracle():
    probs = setups.batched_problems(n=4, seed=3, lo=17, hi=90, dtype=np.float64)
    runs = [make(s, o.iga | o.fct, 2, np.float64) for s in probs]
    b = concurr.batch(runs)
    b.advance(7)
    for s, r in zip(probs, runs):
        orc = Oracle(s["grid"], o.iga | o.fct, n_iters=2, bcs=s["bcs"], max_abs_div_eps=1e-6)
        load(orc, s)
        orc.advance(7)
        ref = orc.advectee()
        assert np.abs(r.advectee() - ref).max() <= 1e-12 * np.abs(ref).max()


def test_batch_then_single_advance_continues():
    probs = setups.batched_problems(n=3, seed=4, lo=30, hi=80)
    runs = [make(s, o.fct, 2, np.float32) for s in probs]
    alone = [make(s, o.fct, 2, np.float32) for s in probs]
    b = concurr.batch(runs)
    b.advance(7)
    for r in runs:
        r.advance(2)
    b.advance(1)
    for r in alone:
        r.advance(10)
    for r, a in zip(runs, alone):
        np.testing.assert_array_equal(r.advectee(), a.advectee())


def test_batch_rejects_mixed_problems():
    probs = setups.batched_problems(n=2, seed=4, lo=30, hi=80)
    r1 = make(probs[0], o.fct, 2, np.float32)
    r2 = make(probs[1], o.iga | o.fct, 2, np.float32)
    with pytest.raises(RuntimeError, match="same opts"):
        concurr.batch([r1, r2])
    r3 = make(probs[1], o.fct, 2, np.float64)
    with pytest.raises(RuntimeError, match="same dtype"):
        concurr.batch([r1, r3])


@pytest.mark.parametrize("mode", ["persistent", "per_problem"])
def test_batch_after_async_uploads_equals_synchronous_uploads(mode):
    """Fields uploaded with the asynchronous entry points right before a batched
    advance are in place when the batch reads them (the batch waits for every
    member's pending transfers)."""
    import torch
    from libmpdataxx_b200 import _lib
    probs = setups.batched_problems(n=5, seed=17, lo=200, hi=600)
    want = [make(s, o.fct, 2, np.float32) for s in probs]
    bw = concurr.batch(want, mode=mode)
    bw.advance(3)
    runs = [make(s, o.fct, 2, np.float32) for s in probs]
    b = concurr.batch(runs, mode=mode)
    b.advance(3)
    b.sync()
    # upload a new advectee (the synchronous twin gets the same one) and advance at once
    rng = np.random.default_rng(3)
    keep = []
    for r, w, s in zip(runs, want, probs):
        a = setups.wrap_periodic(rng.uniform(0.5, 2.0, size=tuple(g - 1 for g in s["grid"]))).astype(np.float32)
        t = torch.from_numpy(a).pin_memory()
        keep.append(t)
        r.set_field_async(_lib.FIELD_ADVECTEE, 0, t.data_ptr())
        w.set_advectee(a)
    b.advance(4)
    bw.advance(4)
    for r, w in zip(runs, want):
        np.testing.assert_array_equal(r.advectee(), w.advectee())
