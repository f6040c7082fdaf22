#!/usr/bin/env python
"""Benchmark of the B200 hydro step: FP64 cell-updates/s on the 256^3 turbulent box.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 256]

One step is one full iteration of the reference's main loop (state, courant,
dt control, half-dt source, two SSP-RK2 flux stages, half-dt source) over a
256^3-interior box (260^3 cells with ghosts) with a seeded lognormal density,
uniform pressure and solenoidal Mach-1 velocity, gamma=5/3, CFL 0.4, outflow
walls (synthetic input, no dataset).  The unit of work is one interior cell
advanced one step.

ours: K steps timed with CUDA events on the library's stream after W warm-up
steps, barrier and synchronize on both sides, max over ranks.  Under torchrun
every rank advances its own replica of the box (the step has no exchange; the
reference runs on one node's shared memory), so value = ranks x cells x K / t.
The JSON line also carries the end-to-end figure through the C ABI with host
arrays (bx_step_host: cons from pinned memory in, one step, cons back, every
step; the three separate calls and the full cons/u/p arrays beside it), the
HBM roofline of the dominant stage kernel, the FP64 roofline, nvidia-smi clocks
sampled during the timed region, the oracle timed on the host cores, the GPU
path against the oracle on the same 256^3 state after a few steps (`parity`),
and the other two figures of the metric at their own configurations:
`adjoint_c4` (adjoint/forward time ratio, 128^3, 200 steps, 15 snapshots, with
finite-difference checks) and `batched_c3` (4096 Riemann boxes, 50 steps,
boxes/s against the plain path looped over the same ensemble).

reference: the reference's algorithm on the CPU (oracle/bx_oracle.c, a
line-by-line C restatement of the Fortran, OpenMP on all host cores, ghost loop
parallel like the reference's) on the same 256^3 workload (--ref-n to shrink
it), K steps after W warm-up steps; rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 cell-updates/s"
UNIT = "cell-updates/s"
FALLBACK_HBM = 6650.0


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def measured_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], [], set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), samples=len(sm),
                       reasons=sorted(reasons))
        return out


def timed_steps(step, min_steps, seconds, max_steps=200):
    """Run step() at least min_steps times and until `seconds` of host time have
    passed (at most max_steps): a bounded sample.  Returns (steps, seconds)."""
    n = 0
    t0 = time.perf_counter()
    while n < min_steps or (n < max_steps and time.perf_counter() - t0 < seconds):
        step()
        n += 1
    return n, time.perf_counter() - t0


def cpu_sample(st, steps=2, seconds=10.0, threads=None):
    """The oracle (reference algorithm, OpenMP) on at least `steps` steps and
    `seconds` of host time of the state, after one warm-up step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = threads or os.cpu_count()
    O.set_threads(threads)
    o = O.Oracle(st.params, racy_ghosts=True)
    o.set_state(st.cons, st.u, st.p, st.adindx)
    o.step()  # warm-up (first touch of every array)
    n, dt = timed_steps(o.step, steps, seconds)
    o.close()
    cells = st.params.n_active()
    return cells * n / dt, threads, dt, n


def parity_full_size(st, steps):
    """The GPU path and the oracle advanced `steps` steps from the same full-size
    state (the oracle with the sequential ghost sweep, the order the GPU
    implements); the reference's arrays after the last step and the clock after
    every step compared.  Bit-identical results give zero differences."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from boxzyhydro_b200.hydro import Hydro
    O.set_threads(os.cpu_count())
    o = O.Oracle(st.params)
    o.set_state(st.cons, st.u, st.p, st.adindx)
    g = Hydro(st.params)
    g.upload_state(st)
    clock_equal, paths = True, []
    t0 = time.perf_counter()
    for _ in range(steps):
        if not (o.step() and g.step()):
            break
        paths.append(g.status()[1])
        co, cg = o.clock(), g.clock()
        clock_equal &= all(co[k] == cg[k] for k in ("time", "dt", "dtold", "step"))
    c0, u0, p0, _ = o.get_state()
    c1, u1, p1 = g.download()
    g.close()
    o.close()
    rel = float(np.max(np.abs(c0 - c1) / np.maximum(np.abs(c0), 1e-300)))
    return {"steps": len(paths), "max_rel_diff_cons": rel,
            "max_abs_diff_u": float(np.max(np.abs(u0 - u1))),
            "max_abs_diff_p": float(np.max(np.abs(p0 - p1))),
            "bit_identical": bool(np.array_equal(c0, c1) and np.array_equal(u0, u1)
                                  and np.array_equal(p0, p1)),
            "clock_equal": bool(clock_equal),
            "gpu_path_per_step": ["fused" if x == 1 else "per-phase" for x in paths],
            "oracle": "oracle/bx_oracle.c, sequential ghost sweep, OpenMP",
            "wall_s": time.perf_counter() - t0}


def physics_arm(args, rank, world, local):
    """The rows beyond the plain step on the turbulent box: angular-momentum
    fluxing (fluxangmom, yoffset 0.75: the rotation axis a quarter box below
    the box; with the axis inside the box the near-axis pressure terms push
    velocities past vlimit within a few steps and the limiter's steps run on
    the per-phase kernels, in the oracle too), the tabulated EOS (H2STAT >= 0
    with synthetic ideal-gas tables of the eos module's layout) and the gravity
    coupling (a softened point-mass potential handed over from page-locked host
    memory before every step, its upload and calc_gforce inside the timed
    region).  All three run on the fused stage kernels (the line gives each
    variant's path and the status bits of its steps).  Device-timed steps and
    the oracle with the same physics on a bounded sample of the host cores."""
    import dataclasses

    import numpy as np
    import torch
    from boxzyhydro_b200 import grid as G
    from boxzyhydro_b200 import ic
    from tests.eos_tables import synthetic_table
    from boxzyhydro_b200.hydro import Hydro

    if rank != 0:
        return 0
    base = ic.turbulent_box(n=args.n, seed=args.seed)
    hp0 = base.params
    cells = hp0.n_active()
    x, y, z = G.cell_centres(hp0.nx, hp0.ny, hp0.nz, hp0.dx, hp0.dy, hp0.dz)
    phi = torch.empty(hp0.ngrid, dtype=torch.float64, pin_memory=True).numpy()
    phi[:] = -0.1 / np.sqrt(x * x + y * y + z * z + 0.01)
    tab = synthetic_table()
    variants = {
        "fluxang": dict(params=dataclasses.replace(hp0, fluxangmom=True, yoffset=0.75)),
        "eostable": dict(params=dataclasses.replace(hp0, h2stat=1), table=tab),
        "gravity": dict(params=hp0, phi=phi),
    }
    out = {}
    stream = torch.cuda.Stream()
    for name, v in variants.items():
        hp = v["params"]
        g = Hydro(hp)
        g.set_stream(stream.cuda_stream)
        g.upload(base.cons, base.u, base.p)
        if "table" in v:
            g.set_eos_table(v["table"])

        def one():
            if "phi" in v:
                g.set_phi(v["phi"])
            g.step()

        for _ in range(args.warmup):
            one()
        g.profile(True)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            one()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        prof = g.profile_read()
        bits, path = g.status()
        g.close()
        rec = {"value": cells * args.steps / (ms * 1e-3), "unit": UNIT,
               "ms_per_step": ms / args.steps, "steps": args.steps,
               "path": "fused stage kernels" if path == 1 else "per-phase kernels",
               "status_bits": bits, "gpu_launches": prof["launches"]}
        if not args.no_cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O
            threads = os.cpu_count()
            O.set_threads(threads)
            o = O.Oracle(hp, racy_ghosts=True)
            if "table" in v:
                o.set_eos_table(v["table"])
            o.set_state(base.cons, base.u, base.p, base.adindx)

            def cpu_one():
                if "phi" in v:
                    o.set_gforce(o.calc_gforce(v["phi"]))
                o.step()

            cpu_one()
            n, secs = timed_steps(cpu_one, args.cpu_steps, args.cpu_seconds)
            o.close()
            rec["cpu_baseline"] = {
                "value": cells * n / secs, "unit": UNIT, "cores": threads,
                "kind": "port", "sample": f"{n} steps after one warm-up step "
                                          f"({secs:.1f} s), oracle/bx_oracle.c, OpenMP"}
        out[name] = rec
    line = {"metric": METRIC, "unit": UNIT, "n_gpus": 1, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"turbulent box {args.n}^3 interior, gamma=5/3, CFL 0.4, "
                                   "outflow walls, with each physics option in turn",
                       "cells_per_step": cells},
            "variants": out}
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(ms, world, device=None):
    """The slowest rank's time (the timing rule for N > 1: every rank takes its
    device time between barriers, the job's time is the maximum)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(world, units_per_rank, steps, ms):
    """Whole-job throughput of N replicas: units of all ranks / the job's time."""
    return world * units_per_rank * steps / (ms * 1e-3)


def reference_arm(args, rank):
    if rank != 0:
        return 0
    from boxzyhydro_b200 import ic
    n = args.ref_n
    st = ic.turbulent_box(n=n, seed=args.seed)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = os.cpu_count()
    O.set_threads(threads)
    o = O.Oracle(st.params, racy_ghosts=True)
    o.set_state(st.cons, st.u, st.p, st.adindx)
    for _ in range(args.warmup):
        o.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step()
    dt = time.perf_counter() - t0
    cells = st.params.n_active()
    value = cells * args.steps / dt
    sample = (f"{n}^3-interior turbulent box ({cells} cells), "
              f"{args.steps} steps after {args.warmup} warm-up, C restatement of the "
              "reference loop (oracle/bx_oracle.c), OpenMP, parallel ghost loop")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"turbulent box {n}^3 interior ({st.params.nx}x{st.params.ny}x"
                               f"{st.params.nz} with ghosts), lognormal rho sigma_ln=0.5, "
                               "solenoidal Mach-1 v, p=1, gamma=5/3, CFL 0.4, outflow walls",
                   "cells_per_step": cells},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def batched_arm(args, rank, world, local):
    line = batched_measure(args, rank, world, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def batched_measure(args, rank, world, local, init_dist=True):
    """C3: an ensemble of independent Riemann boxes (sides drawn from
    {32,48,64,96}, interior), each with its own gamma and dt, advanced `steps`
    steps in CUDA-graph runs of the batched path; boxes/s = boxes x steps / device
    time.  Beside it, the single-grid path looped over a stratified sample of the
    same boxes (extrapolated to the ensemble by box size), and a bit-for-bit check
    of sampled boxes against single-grid runs."""
    import numpy as np
    import torch

    from boxzyhydro_b200 import ic
    from boxzyhydro_b200.batch import Batch, pool_bytes
    from boxzyhydro_b200.hydro import Hydro

    torch.cuda.set_device(local)
    if world > 1 and init_dist:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    # each rank advances an ensemble of its own (seeded by rank): replicas
    spec = ic.riemann_ensemble_spec(nbox=args.nbox, seed=args.seed + rank)
    free, _ = torch.cuda.mem_get_info()
    budget = 0.80 * free
    chunks, cur, cur_b = [], [], 0
    for s in spec:
        nb = 3 * 5 * 8 * (s["side"] + 4) ** 3
        if cur and cur_b + nb > budget:
            chunks.append(cur)
            cur, cur_b = [], 0
        cur.append(s)
        cur_b += nb
    if cur:
        chunks.append(cur)
    stream = torch.cuda.Stream()
    total_ms = 0.0
    launches = 0
    checked, maxdiff, solo = 0, 0.0, 0
    tuned = []
    check_every = max(1, args.nbox // args.check_boxes)
    t_wall0 = time.perf_counter()
    for ci, chunk in enumerate(chunks):
        params = [ic.riemann_params(s["side"], s["gamma"]) for s in chunk]
        b = Batch(params)
        b.set_stream(stream.cuda_stream)
        for i, s in enumerate(chunk):
            b.upload(i, ic.riemann_box_cons(s["side"], s["axis"], s["left"], s["right"],
                                            s["gamma"]))
        b.run(args.warmup)
        if args.persistent:
            b.set_persistent(True)
        if not args.no_autotune:
            zc, tms = b.autotune(reps=2)
            _, ttx, tty, _ = b.tile_shape
            tuned.append({"tile_depth": "whole box" if zc >= 1 << 30 else
                          ("default rule" if zc == 0 else zc), "trial_ms_per_step": tms,
                          "tile_columns": f"{ttx}x{tty}",
                          "launch_form": "persistent" if b.persistent else "4 per step"})
        b.run(args.steps)
        inf = b.info()
        total_ms += inf["last_run_ms"]
        launches += inf["launches"]
        solo += inf["solo_boxes"]
        base = sum(len(c) for c in chunks[:ci])
        for i, s in enumerate(chunk):
            if (base + i) % check_every:
                continue
            cb, ub, pb = b.download(i)
            h = Hydro(params[i])
            c0 = ic.riemann_box_cons(s["side"], s["axis"], s["left"], s["right"], s["gamma"])
            h.upload(c0, c0[:, 1:4] / c0[:, 0:1])
            h.run(nsteps=args.warmup + args.steps)
            ca, ua, pa = h.download()
            h.close()
            d = float(np.max(np.abs(ca - cb) / np.maximum(np.abs(ca), 1e-300)))
            maxdiff = max(maxdiff, d)
            checked += 1
        b.close()
    total_ms = max_over_ranks(total_ms, world, "cuda")
    value = weak_value(world, args.nbox, args.steps, total_ms)

    # single-grid path looped over the whole ensemble (--loop-sample 0) or over a
    # stratified sample, extrapolated by size
    sizes = sorted({s["side"] for s in spec})
    per_size_ms = {}
    for side in sizes:
        sample = [s for s in spec if s["side"] == side]
        if args.loop_sample > 0:
            sample = sample[: args.loop_sample]
        ms_list = []
        for s in sample:
            h = Hydro(ic.riemann_params(side, s["gamma"]))
            h.set_stream(stream.cuda_stream)
            c0 = ic.riemann_box_cons(side, s["axis"], s["left"], s["right"], s["gamma"])
            h.upload(c0, c0[:, 1:4] / c0[:, 0:1])
            h.run(nsteps=args.warmup)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h.run(nsteps=args.steps)
            e1.record(stream)
            e1.synchronize()
            ms_list.append(e0.elapsed_time(e1))
            h.close()
        per_size_ms[side] = sum(ms_list) / len(ms_list)
    # with the whole ensemble this sum is the measured loop time itself
    loop_ms = max_over_ranks(sum(per_size_ms[s["side"]] for s in spec), world, "cuda")
    loop_value = weak_value(world, args.nbox, args.steps, loop_ms)
    cells = sum(s["side"] ** 3 for s in spec)
    line = {
        "metric": "batched boxes/s", "value": value, "unit": "box-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"{args.nbox} Riemann boxes, interior sides from "
                               "{32,48,64,96} (seeded), rho,p ~ logU[0.1,10], v_n ~ U[-1,1], "
                               "random split axis, gamma in {1.4,5/3}, CFL 0.1, outflow walls, "
                               f"{args.steps} steps after {args.warmup} warm-up",
                   "interior_cells": cells, "chunks": len(chunks),
                   "cell_updates_per_s": weak_value(world, cells, args.steps, total_ms)},
        "loop_single_grid": {"value": loop_value, "unit": "box-steps/s",
                             "ms_per_box_run_by_side": per_size_ms,
                             "sample_per_side": args.loop_sample if args.loop_sample > 0
                             else "all (every box of the ensemble run alone)"},
        "speedup_vs_loop": value / loop_value,
        "autotune": tuned or None,
        "parity": {"boxes_checked": checked, "max_rel_diff_cons": maxdiff,
                   "boxes_on_own_handle": solo},
        "gpu_launches": launches,
        "wall_s": time.perf_counter() - t_wall0,
    }
    if world > 1 and init_dist:
        import torch.distributed as dist
        dist.destroy_process_group()
    return line


def adjoint_arm(args, rank, world, local):
    if rank != 0:
        return 0  # one GPU: the adjoint runs on rank 0 only
    line = adjoint_measure(args, local)
    print(json.dumps(line), flush=True)
    return 0


def io_timeline_summary(tl):
    """Summary of a bx_step_host timeline (rows: slabs; columns: ms from the
    call's start to upload start/end, stage 0 enqueued after the upload, stage 1
    end, conversion end, download start/end): when each copy direction starts
    and ends, how long its copies ran, the compute's first and last stage-1
    ends, and the longest gaps between consecutive downloads."""
    import numpy as np
    up0, up1, _, s1, cv, dn0, dn1 = (tl[:, k] for k in range(7))
    o = np.argsort(dn0)
    gaps = np.maximum(dn0[o][1:] - dn1[o][:-1], 0.0) if len(o) > 1 else np.zeros(0)
    return {"slabs": int(len(tl)), "ms_end": float(dn1.max()),
            "upload_start_end_ms": [float(up0.min()), float(up1.max())],
            "upload_busy_ms": float((up1 - up0).sum()),
            "download_start_end_ms": [float(dn0.min()), float(dn1.max())],
            "download_busy_ms": float((dn1 - dn0).sum()),
            "download_idle_ms": float(gaps.sum()),
            "download_longest_gaps_ms": [float(x) for x in np.sort(gaps)[::-1][:4]],
            "stage1_first_last_end_ms": [float(s1.min()), float(s1.max())],
            "conversion_last_end_ms": float(cv.max())}


def host_mem_available():
    """MemAvailable of /proc/meminfo in bytes (0 if unreadable)."""
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    return int(ln.split()[1]) * 1024
    except OSError:
        pass
    return 0


def auto_host_plan(steps, sets, set_bytes, entries=4):
    """Host level of the adjoint's schedule for `sets` free device plane sets:
    the stride L and the device snapshots that recompute the fewest steps,
    (L, snapshots) or (0, None) when the device pool alone does better.  The
    host keeps (steps - 1) // L states in at most 45 % of its available memory
    and at most 256 GiB (pinning takes time; the library refuses more than half);
    two device sets hold segment starts and `entries` are stage-0 cache entries,
    the rest reverse each segment (the schedule's own count, bx_adj_plan)."""
    from boxzyhydro_b200.adjoint import plan
    cap = min(0.45 * host_mem_available(), float(256 << 30))
    snaps_dev = max(1, min(steps, sets - entries))
    best_cost, best = plan(steps, snaps_dev)["recomputed_first"], (0, None)
    snaps = sets - entries
    if snaps < 3:
        return best
    for L in range(2, steps):
        if ((steps - 1) // L) * set_bytes > cap:
            continue
        cost = 0
        for a in range(0, steps, L):
            seg = min(L, steps - a)
            if seg > 1:
                cost += plan(seg, snaps - 2)["recomputed_again"]
        if cost < best_cost:
            best_cost, best = cost, (L, snaps)
    return best


def adjoint_measure(args, local):
    """Discrete adjoint of an n^3 run of `steps` steps.  Loss
    0.5*||rho(T) - rho_target||^2 over interior cells; rho_target is the run of
    the unperturbed state (x-split state) or 1.01*rho(T) (turbulent state).
    Gradient w.r.t. the initial rho, m, E.  Reports the adjoint/forward
    device-time ratio, the engine's device bytes and the peak device memory in
    use (cudaMemGetInfo), the recomputed steps and the agreement with central
    finite differences (dt sequence held fixed) along seeded random
    directions.  --snapshots 0 sizes the snapshot pool to the free HBM."""
    import numpy as np
    import torch

    from boxzyhydro_b200 import grid as G
    from boxzyhydro_b200 import ic
    from boxzyhydro_b200.adjoint import AdjointEngine

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    if args.adj_ic == "blob":
        st = ic.sod_blob_box(n=n, seed=args.seed)
        ic_name = "x-split Sod state + seeded 5% Gaussian density blob, outflow walls"
    else:
        st = ic.turbulent_box(n=n, seed=args.seed)
        ic_name = "lognormal/solenoidal turbulent state, outflow walls"
    hp = st.params
    ng = hp.ngrid
    plane = ng * 8
    m = torch.tensor(G.boundary_flags(hp.nx, hp.ny, hp.nz) == 0, device=dev)
    c0 = torch.tensor(np.ascontiguousarray(st.cons.T), device=dev)
    del st
    # the automatic host level sizes the device snapshots too
    snaps = 0 if args.host_stride < 0 else args.snapshots
    # stage-0 cache entries: 8 beside a given snapshot count; when the snapshots
    # fill HBM, about a third of the free state sets (a schedule simulation of
    # 400 steps in 17 sets: 11 snapshots + 6 entries recompute least)
    entries = args.stage0_cache if args.stage0_cache > 0 else 8
    if args.keep_stage0:
        entries = 2
    if snaps <= 0:
        # engine: 7 state sets + 14 scratch planes + cache entries + (snaps + 1)
        # state sets; this arm, beside c0, while the runs are timed: the forward's
        # output (the loss adjoint), the gradient and one density plane.  The
        # finite differences afterwards take their planes from the stage-0 cache,
        # which is cut to two entries first.
        free = torch.cuda.mem_get_info(dev)[0]
        fixed = (7 * 5 + 14 + 5 + 11) * plane + (4 << 30)
        sets = int(max(3, (free - fixed) // (5 * plane)))
        if args.stage0_cache <= 0 and not args.keep_stage0:
            entries = max(2, min(8, round(0.35 * sets)))
        snaps = int(max(1, min(args.steps, sets - entries)))
        if args.host_stride < 0:
            args.host_stride, hs = auto_host_plan(args.steps, sets, 5 * plane)
            if args.host_stride >= 2:
                snaps, entries = hs, sets - hs
        elif args.host_stride >= 2:
            # host level: stride + 1 plane sets (two hold segment starts, the
            # other stride - 1 take a segment's states), the rest cache entries
            snaps = int(max(3, min(sets - 2, args.host_stride + 1)))
            if args.stage0_cache <= 0 and not args.keep_stage0:
                entries = int(max(2, sets - snaps))
    peak = [0]

    def used():
        f, t = torch.cuda.mem_get_info(dev)
        peak[0] = max(peak[0], t - f)

    eng = AdjointEngine(hp, args.steps, snaps)
    eng.stage0_cache(entries)
    if args.keep_stage0:
        eng.keep_stage0(True)
    host = None
    if args.host_stride >= 2:
        try:
            host = {"stride": args.host_stride, "pinned_bytes": eng.host_level(args.host_stride)}
        except Exception as e:  # refused (host memory): the device-only schedule runs
            host = {"stride": args.host_stride, "refused": str(e)}
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    used()

    def run(c, frozen):
        out = torch.empty_like(c)
        torch.cuda.synchronize()
        eng.forward_ptr(c.data_ptr(), out.data_ptr(), frozen=frozen)
        torch.cuda.synchronize()
        used()
        return out

    if args.adj_ic == "blob":
        st0 = ic.sod_blob_box(n=n, seed=args.seed, blob=False)
        t0 = torch.tensor(np.ascontiguousarray(st0.cons.T), device=dev)
        del st0
        out = run(t0, False)
        target = out[0].clone()
        del out, t0
    cT = run(c0, False)
    stats_fwd = eng.stats()
    if args.adj_ic != "blob":
        target = cT[0] * 1.01
    lamT = cT
    lamT[0] = (cT[0] - target) * m
    lamT[1:] = 0.0
    del cT
    loss = 0.5 * float(torch.sum(lamT[0] ** 2))
    grad = torch.empty_like(lamT)
    torch.cuda.synchronize()
    eng.backward_ptr(lamT.data_ptr(), grad.data_ptr())
    torch.cuda.synchronize()
    used()
    stt = eng.stats()
    del lamT
    ratio = stt["ms_backward"] / stats_fwd["ms_forward"]
    grad_norm2 = float(torch.sum(grad * grad))
    if (args.fd_dirs > 0 or args.fd_frozen_dirs > 0) and entries > 2:
        eng.stage0_cache(2)  # room for the difference runs' planes
    # finite differences with the frozen dt sequence
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + 99)
    scale = torch.tensor([1.0, 0.3, 0.3, 0.3, 2.0], device=dev, dtype=torch.float64)[:, None]
    rel = []
    h = 1e-7
    for k in range(args.fd_dirs):
        v = torch.randn(c0.shape, generator=gen, device=dev, dtype=torch.float64)
        v.mul_(scale).mul_(m)
        adj = float(torch.sum(grad * v))
        vals = []
        for sgn in (1.0, -1.0):
            x = torch.add(c0, v, alpha=sgn * h)
            out = run(x, True)
            del x
            vals.append(float(torch.sum((out[0] - target) ** 2 * m)))
            del out
        fd = (vals[0] - vals[1]) * 0.5 / (2 * h)
        rel.append(abs(fd - adj) / max(abs(adj), 1e-300))
        del v
    # the same differences with every branch held where the unperturbed run takes
    # it (bx_adj_forward_branches): smooth, so they check the adjoint at the ties
    # where the step is not differentiable
    rel_fb = []
    t_fb = time.perf_counter()
    gen.manual_seed(args.seed + 99)
    ob = torch.empty_like(c0)
    for k in range(min(args.fd_dirs, args.fd_frozen_dirs)):
        v = torch.randn(c0.shape, generator=gen, device=dev, dtype=torch.float64)
        v.mul_(scale).mul_(m)
        adj = float(torch.sum(grad * v))
        vals = []
        for sgn in (1.0, -1.0):
            x = torch.add(c0, v, alpha=sgn * h)
            op = torch.empty_like(c0)
            torch.cuda.synchronize()
            eng.forward_branches_ptr(c0.data_ptr(), x.data_ptr(), ob.data_ptr(), op.data_ptr())
            torch.cuda.synchronize()
            used()
            vals.append(float(torch.sum((op[0] - target) ** 2 * m)))
            del x, op
        fd = (vals[0] - vals[1]) * 0.5 / (2 * h)
        rel_fb.append(abs(fd - adj) / max(abs(adj), 1e-300))
        del v
    t_fb = time.perf_counter() - t_fb
    del ob
    line = {
        "metric": "adjoint/forward time ratio", "value": ratio, "unit": "x",
        "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": 0,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"discrete adjoint, {n}^3 interior, gamma=5/3, {ic_name}, "
                               f"{args.steps} steps, loss 0.5||rho(T)-rho_target||^2",
                   "snapshots": snaps, "keep_stage0": bool(args.keep_stage0),
                   "stage0_cache_entries": entries, "host_level": host},
        "ms_forward": stats_fwd["ms_forward"], "ms_backward": stt["ms_backward"],
        "forward_cell_updates_per_s": hp.n_active() * args.steps / (stats_fwd["ms_forward"] * 1e-3),
        "recomputed_steps": stt["recomputed_steps"],
        "recompute_fraction": stt["recomputed_steps"] / args.steps,
        "engine_device_bytes": stt["device_bytes"],
        "peak_device_bytes_in_use": peak[0],
        "loss": loss,
        "grad_norm2": grad_norm2,
        "fd_check": {"directions": args.fd_dirs, "h": h, "max_rel_diff": max(rel) if rel else None,
                     "median_rel_diff": float(np.median(rel)) if rel else None,
                     "per_direction": rel},
        "fd_frozen_branches": {
            "directions": len(rel_fb), "h": h,
            "max_rel_diff": max(rel_fb) if rel_fb else None,
            "median_rel_diff": float(np.median(rel_fb)) if rel_fb else None,
            "per_direction": rel_fb, "wall_s": t_fb,
            "map": "bx_adj_forward_branches: the run from the perturbed state with the dt "
                   "sequence and every branch of the unperturbed run"},
    }
    eng.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--ref-n", type=int, default=0, dest="ref_n",
                    help="box of the reference arm (default: --n, the headline box)")
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--e2e-steps", type=int, default=10, dest="e2e_steps")
    ap.add_argument("--cpu-steps", type=int, default=2, dest="cpu_steps",
                    help="least steps of the CPU baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, dest="cpu_seconds",
                    help="least host seconds of the CPU baseline sample (at most 200 steps)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="turb", choices=["turb", "batched", "adjoint", "physics"])
    ap.add_argument("--snapshots", type=int, default=15)
    ap.add_argument("--fd-dirs", type=int, default=16, dest="fd_dirs")
    ap.add_argument("--fd-frozen-dirs", type=int, default=16, dest="fd_frozen_dirs",
                    help="of the finite-difference directions, those also taken with frozen branches")
    ap.add_argument("--adj-ic", default="blob", choices=["blob", "turb"], dest="adj_ic")
    ap.add_argument("--keep-stage0", action="store_true", dest="keep_stage0")
    ap.add_argument("--stage0-cache", type=int, default=0, dest="stage0_cache")
    ap.add_argument("--host-stride", type=int, default=0, dest="host_stride",
                    help="adjoint: every stride-th state in pinned host memory (0: off; "
                         "-1: the stride and the device snapshots chosen from the free "
                         "device and host memory)")
    ap.add_argument("--nbox", type=int, default=4096)
    ap.add_argument("--check-boxes", type=int, default=16, dest="check_boxes")
    ap.add_argument("--no-autotune", action="store_true", dest="no_autotune")
    ap.add_argument("--persistent", action="store_true",
                    help="batched: one persistent launch per run (the autotuner may still choose)")
    ap.add_argument("--loop-sample", type=int, default=8, dest="loop_sample",
                    help="batched: boxes per side of the looped single-grid baseline "
                         "(0: every box of the ensemble)")
    ap.add_argument("--parity-steps", type=int, default=3, dest="parity_steps",
                    help="steps of the full-size GPU-vs-oracle comparison (0: skip)")
    ap.add_argument("--no-extra", action="store_true", dest="no_extra",
                    help="skip the adjoint (C4) and batched (C3) figures of the default line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.ref_n <= 0:
        args.ref_n = args.n

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return reference_arm(args, rank)
    if args.workload == "batched":
        return batched_arm(args, rank, world, local)
    if args.workload == "adjoint":
        return adjoint_arm(args, rank, world, local)
    if args.workload == "physics":
        return physics_arm(args, rank, world, local)

    import numpy as np
    import torch
    import torch.distributed as dist

    from boxzyhydro_b200 import ic
    from boxzyhydro_b200.hydro import Hydro, fp64_peak

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    st = ic.turbulent_box(n=args.n, seed=args.seed)
    hp = st.params
    cells = hp.n_active()
    g = Hydro(hp)
    stream = torch.cuda.Stream()
    g.set_stream(stream.cuda_stream)
    g.upload_state(st)
    for _ in range(args.warmup):
        g.step()

    # ---- device-timed steps
    g.profile(True)
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        g.step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), world, "cuda")
    prof = g.profile_read()
    bits, path = g.status()
    value = weak_value(world, cells, args.steps, ms)

    # ---- roofline of the dominant stage kernel
    hbm, hbm_src = measured_hbm()
    fsteps = max(prof["fused_steps"], 1)
    t0 = prof["ms_stage0"] / fsteps
    t1 = prof["ms_stage1"] / fsteps
    dom = 1 if t1 >= t0 else 0
    tdom = max(t0, t1)
    alg_bytes = 80.0 * cells  # 5 FP64 conserved fields read once and written once per pass
    achieved = alg_bytes / (tdom * 1e-3) / 1e9 if tdom > 0 else None
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "stage_traffic.json")
    if os.path.exists(tr_path):
        try:
            tr = json.load(open(tr_path))
            traffic = tr[f"stage{dom}_bytes_per_cell"] * cells
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                "kernel": f"k_stage<{dom}> (stage {dom} of SSP-RK2)",
                "ms_per_launch": tdom, "peak_source": f"{hbm_src} hbm_gbs",
                "alg_bytes_per_launch": alg_bytes}
    fp64 = None
    try:
        peak64 = fp64_peak()
        fl_path = os.path.join(ROOT, "profiles", "stage_flops.json")
        if os.path.exists(fl_path):
            fl = json.load(open(fl_path))
            flops = fl[f"stage{dom}_fp64_flops_per_cell"] * cells
            ach = flops / (tdom * 1e-3) / 1e12
            fp64 = {"bound": "fp64", "achieved": ach, "peak": peak64, "unit": "TFLOP/s",
                    "frac": ach / peak64, "peak_source": "measured DFMA probe (bx_fp64_peak)",
                    "flops_source": "FP64 operations of the method per cell, frozen from ncu "
                                    "(every division and square root at its IEEE instruction "
                                    "cost; profiles/stage_flops.json)",
                    "executed_fp64_flops_per_cell": fl.get("executed_now", {}).get(f"stage{dom}")}
        else:
            fp64 = {"bound": "fp64", "peak": peak64, "unit": "TFLOP/s"}
    except Exception as e:  # noqa: BLE001
        fp64 = {"error": str(e)}

    # ---- end to end through the C ABI with host arrays.  Each step: the state
    # goes in from pinned host memory, one step runs, the state comes back.
    # Headline form: the conserved variables (40 B per cell each way) through
    # bx_step_host, which overlaps the copies with the step; also measured as the
    # three separate calls it stands for (bx_upload_conserved + bx_step +
    # bx_download(cons)) and with the reference's full arrays cons, u, p (72 B
    # per cell each way).
    e2e = None
    if not args.no_e2e:
        ng = hp.ngrid
        L = __import__("boxzyhydro_b200")._lib.lib()
        hc = torch.empty((ng, 5), dtype=torch.float64, pin_memory=True).numpy()
        hu = torch.empty((ng, 3), dtype=torch.float64, pin_memory=True).numpy()
        hpp = torch.empty((ng,), dtype=torch.float64, pin_memory=True).numpy()
        c, u, p = g.download()
        hc[:] = c
        hu[:] = u
        hpp[:] = p
        del c, u, p

        def timed(body, nsteps):
            barrier()
            torch.cuda.synchronize()
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(nsteps):
                body()
            a1.record(stream)
            a1.synchronize()
            return max_over_ranks(a0.elapsed_time(a1), world, "cuda")

        ran = ctypes.c_int32()

        def overlapped():
            g._c(L.bx_step_host(g._h, hc.ctypes.data, hc.ctypes.data, 1e300, ctypes.byref(ran)))

        def cons_only():
            g._c(L.bx_upload_conserved(g._h, hc.ctypes.data))
            g.step()
            g._c(L.bx_download(g._h, hc.ctypes.data, None, None))

        def full_arrays():
            g.upload(hc, hu, hpp)
            g.step()
            g._c(L.bx_download(g._h, hc.ctypes.data, hu.ctypes.data, hpp.ctypes.data))

        oms = timed(overlapped, args.e2e_steps)
        ems = timed(cons_only, args.e2e_steps)
        fms = timed(full_arrays, max(2, args.e2e_steps // 2))
        nfull = max(2, args.e2e_steps // 2)

        # one step of the same input both ways, clock put back in between: the
        # overlapped call must give the three calls' result bit for bit
        x0 = hc.copy()
        clk = g.clock()
        out_a = x0.copy()
        g.step_host(out_a, out_a)
        g.set_clock(time=clk["time"], dtold=clk["dtold"], step=clk["step"])
        g.upload_conserved(x0)
        g.step()
        out_b = g.download()[0]
        same = bool(np.array_equal(out_a, out_b))
        # where the time of the overlapped call goes: one more call (not timed
        # above) with CUDA events per slab, from the state the handle holds
        hc[:] = out_b
        g.step_host_profile(True)
        overlapped()
        g.step_host_profile(False)
        timeline = io_timeline_summary(g.step_host_timeline())
        e2e = {"value": weak_value(world, cells, args.e2e_steps, oms), "unit": UNIT,
               "h2d_bytes_per_step": ng * 5 * 8, "d2h_bytes_per_step": ng * 5 * 8,
               "steps": args.e2e_steps, "ms_per_step": oms / args.e2e_steps,
               "api": "bx_step_host(cons, cons): upload, step and download of cons in one "
                      "call, copies overlapped with the step, pinned host",
               "bit_identical_to_three_calls": same,
               "timeline": timeline,
               "three_calls": {
                   "value": weak_value(world, cells, args.e2e_steps, ems), "unit": UNIT,
                   "h2d_bytes_per_step": ng * 5 * 8, "d2h_bytes_per_step": ng * 5 * 8,
                   "steps": args.e2e_steps, "ms_per_step": ems / args.e2e_steps,
                   "api": "bx_upload_conserved(cons) + bx_step + bx_download(cons), pinned host"},
               "reference_arrays": {
                   "value": weak_value(world, cells, nfull, fms), "unit": UNIT,
                   "h2d_bytes_per_step": ng * 9 * 8, "d2h_bytes_per_step": ng * 9 * 8,
                   "steps": nfull, "ms_per_step": fms / nfull,
                   "api": "bx_upload(cons,u,p) + bx_step + bx_download(cons,u,p), pinned host"}}

    # ---- CPU baseline (rank 0, one GPU only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, thr, secs, n = cpu_sample(st, steps=args.cpu_steps, seconds=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"{n} steps of the same {args.n}^3 workload after one "
                         f"warm-up step ({secs:.1f} s), oracle/bx_oracle.c (C restatement of "
                         "the reference loop), OpenMP on all host threads"}

    g.close()
    del g

    # ---- GPU against the oracle on the full-size workload (rank 0, one GPU)
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu and args.parity_steps > 0:
        parity = parity_full_size(st, args.parity_steps)

    # ---- the other two headline figures at their configurations (one GPU):
    # the adjoint/forward time ratio (C4: 128^3, 200 steps, 15 snapshots) and
    # the batched ensemble's boxes/s against the looped plain path (C3: 4096 boxes)
    adjoint_c4 = batched_c3 = None
    if world == 1 and not args.no_extra:
        import argparse as _ap
        del st
        torch.cuda.empty_cache()
        a4 = _ap.Namespace(**vars(args))
        a4.n, a4.steps, a4.snapshots, a4.stage0_cache = 128, 200, 15, 8
        a4.keep_stage0, a4.adj_ic, a4.fd_dirs, a4.fd_frozen_dirs = False, "blob", 16, 4
        try:
            adjoint_c4 = adjoint_measure(a4, local)
        except Exception as e:  # noqa: BLE001
            adjoint_c4 = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
        a3 = _ap.Namespace(**vars(args))
        a3.nbox, a3.steps, a3.warmup, a3.check_boxes = 4096, 50, 3, 16
        a3.no_autotune, a3.loop_sample, a3.persistent = False, 8, False
        try:
            batched_c3 = batched_measure(a3, rank, world, local, init_dist=False)
        except Exception as e:  # noqa: BLE001
            batched_c3 = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"turbulent box {args.n}^3 interior "
                                   f"({hp.nx}x{hp.ny}x{hp.nz} with ghosts), lognormal rho "
                                   "sigma_ln=0.5, solenoidal Mach-1 v, p=1, gamma=5/3, "
                                   "CFL 0.4, outflow walls",
                       "cells_per_step": cells, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (3 x 5 planes x 8 B x "
                             f"{hp.ngrid} cells = {3 * 40 * hp.ngrid / 1e9:.1f} GB)"},
            "clocks": clocks,
            "roofline": roofline,
            "roofline_fp64": fp64,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "parity": parity,
            "adjoint_c4": adjoint_c4,
            "batched_c3": batched_c3,
            "gpu_launches": prof["launches"],
            "path": "fused stage kernels" if path == 1 else "per-phase kernels",
            "status_bits": bits,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
