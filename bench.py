"""Benchmark: MPDATA step throughput (cell-updates/s) against the HBM roofline.

Workload (N = 1): 3D MPDATA, 512^3 cyclic, FP32 advection with FP64 mass sums,
opts fct|iga, n_iters = 2, a divergence-free random-Fourier flow scaled to max
Courant 0.4 and 5 Gaussian blobs (libmpdataxx_b200/workloads.py).  One step =
one MPDATA+FCT step of the whole grid (one fused kernel launch).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 (torchrun, one process per GPU) every rank advances its own replica
(the path does not shard on one GPU: "replicas only"); value = all ranks' cell
updates / the slowest rank's device time.

With N = 1 the line also carries "batched_2d" (256 uneven 2D problems in one
persistent launch vs one launch per problem) and "gcr" (3D Boussinesq pressure
solves to max|err| <= 1e-7/dt: iterations and device time per solve, plain GCR
vs GCR with the learned preconditioner trained on the first solves).

--impl reference times the reference's CPU path on this host's cores: the CPU
restatement in oracle/ (the reference itself cannot be built here: it needs
Blitz++ and Boost), compiled with the reference's release flags plus OpenMP,
on the same 512^3 configuration.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL = 20  # FP32: psi^n 4 + GC 3 x 4 + psi^{n+1} 4
TUNE_STEPS_3D = 17  # the fused 3D chunk-length tuner: 1 untimed step + 8 candidates x 2 timed steps


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        rows = [r for r in self.samples if len(r) >= 9]
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        out["sm_mhz"] = statistics.median(sm) if sm else None
        out["sm_max_mhz"] = float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        out["reasons"] = sorted(reasons)
        out["samples"] = len(rows)
        return out


def dist_init():
    """One process per GPU under torchrun (RANK/LOCAL_RANK/WORLD_SIZE from the
    environment); NCCL between GPUs, gloo where there is no GPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x, world):
    """The largest of the ranks' values of x (every rank gets it); x itself on one rank."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(world, units_per_rank, steps, seconds):
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return world * units_per_rank * steps / seconds


def dist_done(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def build_run(w, dtype, torch):
    from libmpdataxx_b200 import bcond, concurr, opts, solvers

    class ct(solvers.ct_params_default_t):
        pass

    ct.real_t = {"float32": "float32", "float64": "float64"}[dtype]
    ct.n_dims = 3
    ct.n_eqns = 1
    ct.opts = opts.fct | opts.iga
    p = solvers.mpdata.rt_params_t(grid_size=list(w["grid"]), n_iters=2, max_abs_div_eps=1e-6)
    run = concurr.cuda(solvers.mpdata(ct), *[bcond.cyclic] * 6, p=p)
    from libmpdataxx_b200 import _lib
    run.set_field_device(_lib.FIELD_ADVECTEE, 0, w["advectee"][0].data_ptr())
    for d, a in enumerate(w["advector"]):
        run.set_field_device(_lib.FIELD_ADVECTOR, d, a.data_ptr())
    return run


def bulk_copy_tiles(n, rows=32, ty=26, tz=56):
    """(tiles whose planes come in as bulk-tensor copies, tiles) of one plane chunk
    of the fused 3D kernel on an n^3 grid: the tiles inside the periods along j and k."""
    P = n - 1
    nz, ny = -(-P // tz), -(-P // ty)
    inner = 0
    if P >= 64 and P >= rows:
        for t in range(ny * nz):
            j0, k0 = (t // nz) * ty, (t % nz) * tz
            inner += k0 >= 4 and k0 + 60 <= P and j0 >= 3 and j0 + rows - 3 <= P
    return inner, ny * nz


def plane_copy_ab(run, stream, torch, n, steps=10):
    """Device time per step of the headline kernel with its bulk-tensor plane copies
    (the default) and with per-thread copies in every tile, alternated twice,
    outside the timed region; both modes give bitwise-identical fields."""
    from libmpdataxx_b200 import _lib
    L = _lib.lib()
    res = {1: [], 0: []}
    try:
        for _ in range(2):
            for mode in (1, 0):
                L.mpdx_fused3d_bulk_copies(mode)
                run.advance(1)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(stream):
                    e0.record(stream)
                    run.advance(steps)
                    e1.record(stream)
                torch.cuda.synchronize()
                res[mode].append(e0.elapsed_time(e1) / steps)
    finally:
        L.mpdx_fused3d_bulk_copies(1)
    inner, tiles = bulk_copy_tiles(n)
    return {"bulk_tensor_ms": min(res[1]), "per_thread_ms": min(res[0]), "tiles_with_bulk_copies": inner,
            "tiles_per_plane_chunk": tiles}


def cpu_port_time(host, steps, warmup):
    """The oracle's -Ofast + OpenMP build (the CPU restatement of the reference's
    path) on the whole 3D workload `host` (numpy advectee and advector views):
    `warmup` untimed steps, then `steps` timed ones; returns (seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    from libmpdataxx_b200 import opts
    from oracle import Oracle
    psi, gx, gy, gz = host
    orc = Oracle(psi.shape, opts.fct | opts.iga, n_iters=2, dtype=psi.dtype.type, fast=True, max_abs_div_eps=1e-6)
    orc.set_advectee(psi)
    for d, a in enumerate((gx, gy, gz)):
        orc.set_advector(a, d)
    orc.advance(max(1, warmup))  # ante-loop checks and first touch of every field
    t0 = time.perf_counter()
    orc.advance(steps)
    dt = time.perf_counter() - t0
    del orc
    import oracle as orc_mod
    return dt, orc_mod.max_threads()


def cpu_baseline(host, n, steps=5):
    """Oracle (CPU restatement, -Ofast + OpenMP on all host threads) on the bench's
    own n^3 workload (same flow and blobs), `steps` steps."""
    dt, threads = cpu_port_time(host, steps, 1)
    return {"value": n ** 3 * steps / dt, "unit": "cell-updates/s", "cores": threads, "kind": "port",
            "sample": f"the full {n}^3 fct|iga n_iters=2 FP32 workload of this line (same flow and blobs), "
                      f"{steps} steps after 1 untimed, {dt:.1f} s; oracle -Ofast + OpenMP"}


def fp64_error(w, fp32_state, steps, torch):
    """Error of the FP32 headline run against an FP64 run of the same inputs: the
    FP32 advectee and advector promoted to FP64, advanced `steps` steps by the
    FP64 fused kernel (the FP64 path equals the FP64 CPU restatement of the
    reference to <= 1e-12), compared with the FP32 state after as many steps."""
    from libmpdataxx_b200 import _lib
    w64 = {"grid": w["grid"], "advectee": [w["advectee"][0].double()], "advector": [a.double() for a in w["advector"]]}
    run = build_run(w64, "float64", torch)
    run.advance(steps)
    out = torch.empty_like(w64["advectee"][0])
    run.get_field_device(_lib.FIELD_ADVECTEE, 0, out.data_ptr())
    run.sync()
    run.close()
    d = fp32_state.double() - out
    n = w["grid"][0]
    return {"vs": "FP64 run of the same (FP32-rounded) inputs through the FP64 fused kernel", "after_steps": steps,
            "max_abs": float(d.abs().max()), "l2": float(d.square().mean().sqrt()),
            "field_max": float(out.abs().max()), "cells": n ** 3}


def batched_extra(n_problems=256, steps=50):
    """C4: independent 2D fct problems of uneven sizes, one persistent launch per
    step in a CUDA graph (autotuned tile) vs one launch per problem per step."""
    import numpy as np
    from libmpdataxx_b200 import bcond, concurr, opts, setups, solvers
    probs = setups.batched_problems(n=n_problems)
    cells = sum(s["grid"][0] * s["grid"][1] for s in probs)

    class ct(solvers.ct_params_default_t):
        pass

    ct.real_t = np.float32
    ct.n_dims = 2
    ct.n_eqns = 1
    ct.opts = opts.fct
    out = {"workload": f"{n_problems} cyclic 2D fct problems, sides 64..1024, FP32", "cells_per_step": cells}
    for mode, k in (("persistent", steps), ("per_problem", max(5, steps // 5))):
        runs = []
        for s in probs:
            p = solvers.mpdata.rt_params_t(grid_size=list(s["grid"]), n_iters=2, max_abs_div_eps=1e-6)
            r = concurr.cuda(solvers.mpdata(ct), *[bcond.cyclic] * 4, p=p, path="fused")
            r.set_advectee(s["advectee"][0])
            for d, a in enumerate(s["advector"]):
                r.set_advector(a, d)
            runs.append(r)
        b = concurr.batch(runs, mode=mode)
        b.advance(30)  # the first 24 steps are the autotuner's (8 candidates x 3 steps)
        b.sync()
        t0 = time.perf_counter()
        b.advance(k)
        b.sync()
        dt = (time.perf_counter() - t0) / k
        out[mode] = {"ms_per_step": dt * 1e3, "cell_updates_per_s": cells / dt}
        if mode == "persistent":
            i = b.info()
            out["tile"] = {"nt": i["tile_nt"], "lx": i["tile_lx"], "grid": i["grid"], "tune_ms": i["tune_ms"],
                           "candidates": "rows per item 16/32/64/128 x all or half of the resident CTAs, 3 timed steps each"}
        b.close()
        for r in runs:
            r.close()
    out["speedup_vs_per_problem"] = out["persistent"]["cell_updates_per_s"] / out["per_problem"]["cell_updates_per_s"]
    return out


def box_1d_extra(steps=1000):
    """C1: 1D plain MPDATA (opts 0, n_iters 2), 2000 cyclic points, FP64, 1000 steps:
    device time on the solver's stream (the general path: one kernel per formula
    and halo fill, launch-bound at this size), mass and minimum after the run, and
    the CPU restatement on the same set-up (one thread and all threads)."""
    import numpy as np
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from libmpdataxx_b200 import bcond, concurr, setups, solvers
    from oracle import Oracle
    s = setups.box_1d()
    nx = s["grid"][0]

    class ct(solvers.ct_params_default_t):
        pass

    ct.real_t = np.float64
    ct.n_dims = 1
    ct.n_eqns = 1
    ct.opts = s["opts"]
    p = solvers.mpdata.rt_params_t(grid_size=[nx], n_iters=s["n_iters"])
    run = concurr.cuda(solvers.mpdata(ct), *[bcond.cyclic] * 2, p=p)
    run.set_advectee(s["advectee"][0])
    run.set_advector(s["advector"][0], 0)
    m0 = run.stats()["mass"]
    run.advance(5)
    run.sync()
    stream = torch.cuda.ExternalStream(run.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        run.advance(steps - 5)
        e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / (steps - 5)
    st = run.stats()
    run.close()
    out = {"workload": f"1D {nx} cyclic, opts 0, n_iters 2, FP64, box on 0.1 + noise, C = 0.5, {steps} steps",
           "ms_per_step": ms, "cell_updates_per_s": nx / (ms * 1e-3), "after_steps": steps,
           "mass_rel_drift": (st["mass"] - m0) / m0, "min": st["min"]}
    import oracle as orc_mod
    threads = orc_mod.max_threads()
    for label, nthr in (("cpu_port_1_thread", 1), ("cpu_port_all_threads", threads)):
        orc_mod.set_threads(nthr)
        orc = Oracle(s["grid"], s["opts"], n_iters=s["n_iters"], bcs=s["bcs"], fast=True)
        orc.set_advectee(s["advectee"][0])
        orc.set_advector(s["advector"][0], 0)
        orc.advance(5)
        t0 = time.perf_counter()
        orc.advance(steps - 5)
        dt = (time.perf_counter() - t0) / (steps - 5)
        out[label] = {"ms_per_step": dt * 1e3, "cell_updates_per_s": nx / dt, "threads": nthr}
    orc_mod.set_threads(threads)
    return out


def rotation_extra(n=1024, steps=200, revolution=6283):
    """C2: 2D n^2 cyclic solid-body rotation of a cone, fct, n_iters=3, in FP32 and
    FP64 (fused 2D kernel; the FP32 fields, 12 MB, fit in L2): device time per step
    on the solver's stream over `steps` steps, then on to one full revolution:
    FP32 - FP64 differences, the error against the initial cone, minimum, maximum
    and mass drift."""
    import numpy as np
    import torch
    from libmpdataxx_b200 import _lib, bcond, concurr, opts, solvers, workloads
    out = {"workload": f"2D {n}^2 cyclic solid-body rotation (offsets clipped at 0.48 (n-1)), cone h=4 r=0.15n, fct, "
                       f"n_iters=3, one revolution", "steps": steps}
    fields = {}
    for dt in ("float32", "float64"):
        w = workloads.rotation_2d(n, dtype=dt)

        class ct(solvers.ct_params_default_t):
            pass

        ct.real_t = dt
        ct.n_dims = 2
        ct.n_eqns = 1
        ct.opts = opts.fct
        p = solvers.mpdata.rt_params_t(grid_size=[n, n], n_iters=3, max_abs_div_eps=1e-6)
        run = concurr.cuda(solvers.mpdata(ct), *[bcond.cyclic] * 4, p=p)
        run.set_field_device(_lib.FIELD_ADVECTEE, 0, w["advectee"][0].data_ptr())
        for d, a in enumerate(w["advector"]):
            run.set_field_device(_lib.FIELD_ADVECTOR, d, a.data_ptr())
        m0 = run.stats()["mass"]
        run.advance(3)
        run.sync()
        stream = torch.cuda.ExternalStream(run.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            run.advance(steps)
            e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        run.advance(revolution - 3 - steps)
        st = run.stats()
        fields[dt] = np.array(run.advectee(), dtype=np.float64)
        err = fields[dt] - w["advectee"][0].double().cpu().numpy()
        out[dt] = {"ms_per_step": ms, "cell_updates_per_s": n * n / (ms * 1e-3),
                   "path": "fused" if st["path"] == _lib.PATH_FUSED else "general",
                   "after_steps": revolution, "min": st["min"], "max": st["max"],
                   "mass_rel_drift": (st["mass"] - m0) / m0,
                   "vs_initial_cone": {"max_abs": float(np.abs(err).max()), "l2": float(np.sqrt((err * err).mean()))}}
        run.close()
    d = fields["float32"] - fields["float64"]
    out["fp32_vs_fp64"] = {"after_steps": revolution, "max_abs": float(np.abs(d).max()),
                           "l2": float(np.sqrt((d * d).mean()))}
    return out


def gcr_extra(grid=(256, 256, 128), record=200, train=400, compare=1000):
    """C5: 3D Boussinesq, FP32 advection with FP64 GCR (cr; a third run with gcrk,
    k = 4, alongside) to max|err| <= 1e-7/dt.
    Two identical runs advance `record` steps; one records the (residual,
    correction) pairs of its solves (their start and iterations 16/32/64), which
    train the learned preconditioner.  Then both advance `compare` more steps, one
    with plain GCR and one with the learned preconditioner (one learned
    correction at the start of each solve, then plain GCR): iterations (the
    learned correction included) and device time per solve, averaged over the
    solves."""
    import numpy as np
    from libmpdataxx_b200 import setups
    s = setups.boussinesq_bubble_3d(*grid)
    plain = setups.boussinesq_run(s, dtype=np.float32, prs_fp64=True)
    learn = setups.boussinesq_run(s, dtype=np.float32, prs_fp64=True)
    gcrk4 = setups.boussinesq_run(dict(s, prs_k=4), dtype=np.float32, prs_fp64=True)
    learn.precond_record(4 * record)
    for r in (plain, learn, gcrk4):
        r.advance(record)
        r.sync()
    n_pairs = learn.precond_pairs()
    t0 = time.perf_counter()
    loss = learn.precond_train(train, lr=1e-3)
    t_train = time.perf_counter() - t0
    learn.precond_enable(True)
    it_p, ms_p, it_l, ms_l, it_k, ms_k, fb, nls = [], [], [], [], [], [], 0, {}
    for _ in range(compare):
        plain.advance(1)
        learn.advance(1)
        gcrk4.advance(1)
        sp, sl, sk = plain.stats(), learn.stats(), gcrk4.stats()
        it_p.append(sp["gcr_iters"]); ms_p.append(sp["gcr_ms"])
        it_l.append(sl["gcr_iters"]); ms_l.append(sl["gcr_ms"])
        it_k.append(sk["gcr_iters"]); ms_k.append(sk["gcr_ms"])
        fb += int(sl["gcr_fallback"] == 2)
        nl = learn.precond_directions()
        nls[nl] = nls.get(nl, 0) + 1
    plain.close()
    learn.close()
    gcrk4.close()
    return {"workload": f"3D Boussinesq {grid[0]}x{grid[1]}x{grid[2]}, x/y cyclic, z rigid, FP32 advection, FP64 GCR (cr), "
                        f"prs_tol 1e-7; {record} recorded plain solves, then {compare} solves each, plain and learned",
            "plain": {"iters_per_solve": statistics.mean(it_p), "ms_per_solve": statistics.mean(ms_p)},
            "plain_gcrk4": {"iters_per_solve": statistics.mean(it_k), "ms_per_solve": statistics.mean(ms_k),
                            "scheme": "gcrk, k = 4 (restarted every 4 directions), same flow, same solves"},
            "learned": {"iters_per_solve": statistics.mean(it_l), "ms_per_solve": statistics.mean(ms_l),
                        "solves_redone_with_plain_gcr": fb,
                        "learned_directions_per_solve": {str(k): v for k, v in sorted(nls.items())},
                        "last_500": {"iters_per_solve": statistics.mean(it_l[-500:]),
                                     "ms_per_solve": statistics.mean(ms_l[-500:])}},
            "time_to_tol_speedup": statistics.mean(ms_p) / statistics.mean(ms_l),
            "time_to_tol_speedup_last_500": statistics.mean(ms_p[-500:]) / statistics.mean(ms_l[-500:]),
            "training": {"pairs": n_pairs, "adam_steps": train,
                         "heldout_loss_relative_energy": loss, "seconds": t_train}}


def reference_arm(args, rank):
    """The reference's CPU path (its CPU restatement: the reference itself needs
    Blitz++ and Boost, absent here) on this host's cores, on the same workload as
    the GPU arm: the 512^3 flow and blobs of workloads.advection_3d, generated on
    the host; every step is one full-grid MPDATA step."""
    if rank != 0:
        return
    from libmpdataxx_b200 import workloads
    w = workloads.advection_3d(n=args.size, dtype=args.dtype, device="cpu")
    host = [w["advectee"][0].numpy()] + [a.numpy() for a in w["advector"]]
    del w
    dt, threads = cpu_port_time(host, args.steps, args.warmup)
    n = args.size
    value = n ** 3 * args.steps / dt
    line = {"impl": "reference", "metric": "cell-updates/s per MPDATA step", "value": value,
            "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.dtype == "float32" else "f64", "data": "synthetic",
            "config": {"workload": f"3D MPDATA {n}^3 cyclic fct|iga n_iters=2 {args.dtype} (FP64 mass sums)",
                       "grid": [n] * 3, "opts": "fct|iga", "n_iters": 2, "same_config": True},
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                             "sample": f"the full {n}^3 workload every step ({args.steps} timed steps after "
                                       f"{args.warmup}); CPU restatement of the reference (reference unbuildable "
                                       "here: Blitz++/Boost absent), -Ofast + OpenMP"},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--size", type=int, default=512, help="grid points per axis of the 3D workload")
    ap.add_argument("--dtype", default="float32")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the 2D rotation, batched-2D and Boussinesq/GCR measurements")
    ap.add_argument("--extra", choices=["box_1d", "rotation_2d", "batched_2d", "gcr"],
                    help="run only this one extra measurement on one GPU and print its JSON object")
    args = ap.parse_args()
    if args.impl == "reference":
        # CPU work on rank 0 alone: no process group (the other ranks exit at once)
        reference_arm(args, int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_init()

    import torch
    torch.cuda.set_device(local)
    if args.extra:
        fn = {"box_1d": box_1d_extra, "rotation_2d": rotation_extra, "batched_2d": batched_extra, "gcr": gcr_extra}[args.extra]
        print(json.dumps({args.extra: fn()}))
        return
    from libmpdataxx_b200 import _lib, workloads
    w = workloads.advection_3d(n=args.size, dtype=args.dtype)
    run = build_run(w, args.dtype, torch)
    n_cells = float(args.size) ** 3
    stream = torch.cuda.ExternalStream(run.stream)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # untimed set-up steps: the handle's chunk-length tuner (one untimed step, then two
    # timed steps for each of eight planes-per-CTA candidates), then the warm-up
    run.advance(TUNE_STEPS_3D)
    for _ in range(max(args.warmup, 3)):
        run.advance(1)
    run.sync()
    assert run.stats()["path"] == _lib.PATH_FUSED, "fused path not taken"
    tuning = run.tuning3d()

    # device-timed region: inputs resident in HBM, one fused launch per step
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for k in range(args.steps):
            run.advance(1)
            ev[k + 1].record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    steps_done = TUNE_STEPS_3D + max(args.warmup, 3) + args.steps
    state = torch.empty_like(w["advectee"][0])
    run.get_field_device(_lib.FIELD_ADVECTEE, 0, state.data_ptr())
    per = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    ms_total = max_over_ranks(ev[0].elapsed_time(ev[-1]), world)
    ms_step = ms_total / args.steps
    value = aggregate(world, n_cells, args.steps, ms_total / 1e3)

    # end-to-end through the public API: every step uploads its inputs from
    # pinned host memory, advances one step and reads the result back, with the
    # asynchronous transfer entry points (the upload of step k+1's advector
    # overlaps the download of step k's advectee)
    host_in = [a.cpu().pin_memory() for a in w["advectee"] + w["advector"]]
    host_out = torch.empty_like(w["advectee"][0], device="cpu").pin_memory()
    itemsize = host_out.element_size()
    h2d = sum(t.numel() for t in host_in) * itemsize
    d2h = host_out.numel() * itemsize
    e2e_steps = max(2, min(args.steps, 5))
    run.sync()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for d in range(3):
            run.set_field_async(_lib.FIELD_ADVECTOR, d, host_in[1 + d].data_ptr())
        run.set_field_async(_lib.FIELD_ADVECTEE, 0, host_in[0].data_ptr())
        run.advance(1)
        run.get_field_async(_lib.FIELD_ADVECTEE, 0, host_out.data_ptr())
    run.sync()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = aggregate(world, n_cells, e2e_steps, e2e_s)

    if rank != 0:
        run.close()
        dist_done(world)
        return
    try:
        copies = plane_copy_ab(run, stream, torch, args.size)
    except Exception as e:  # noqa: BLE001
        copies = {"error": f"{type(e).__name__}: {e}"}
    hbm, src = peaks()
    avg_launch_ms = statistics.mean(per)
    achieved = BYTES_PER_CELL * n_cells / (avg_launch_ms / 1e3) / 1e9
    traffic, traffic_src = None, None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        key = f"fused3d_{args.dtype}_{args.size}"
        if key in tj:
            traffic = tj[key]
            traffic_src = tj.get("_source", {}).get(key)
    line = {
        "metric": "cell-updates/s per MPDATA step", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.dtype == "float32" else "f64",
        "data": "synthetic",
        "config": {"workload": f"3D MPDATA {args.size}^3 cyclic fct|iga n_iters=2 {args.dtype} (FP64 mass sums)",
                   "grid": [args.size] * 3, "opts": "fct|iga", "n_iters": 2, "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2 ({BYTES_PER_CELL * n_cells / 1e9:.2f} GB per step)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "traffic_source": traffic_src, "peak_source": src,
                     "bytes_per_launch": BYTES_PER_CELL * n_cells, "avg_launch_ms": avg_launch_ms},
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "plane_copies": copies,
        "planes_per_cta": {"chosen": tuning["chosen"], "ms_per_step": {str(lx): ms for lx, ms in tuning["candidates"]},
                           "tuning_steps": TUNE_STEPS_3D},
    }
    line["error"] = fp64_error(w, state, steps_done, torch)
    del state
    if world == 1 and not args.no_cpu_baseline:
        host = [t.cpu().numpy() for t in w["advectee"] + w["advector"]]
        line["cpu_baseline"] = cpu_baseline(host, args.size)
        del host
    if world == 1 and not args.no_extras:
        # a failing extra measurement is reported in its own key; the headline stands
        for name, fn in (("box_1d", box_1d_extra), ("rotation_2d", rotation_extra),
                         ("batched_2d", batched_extra), ("gcr", gcr_extra)):
            try:
                line[name] = fn()
            except Exception as e:  # noqa: BLE001
                line[name] = {"error": f"{type(e).__name__}: {e}"}
    print(json.dumps(line), flush=True)
    run.close()
    dist_done(world)


if __name__ == "__main__":
    main()
