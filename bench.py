"""Benchmark of the CDR density update (one RK2 step = one "step").

Default workload: the plain 3-D configuration, one grid of 512 x 1024 cells
with 16 theta planes, two species (electrons, positive ions, both mobility 1,
diffusion 0.1), impact-ionisation table of 256 nodes, fixed field (uniform
applied Ez = -1; no field solve in the loop), drift/diffusion on every theta
plane.  Inputs are synthetic (seeded).  One step reads and writes about
940 MB, far above the 126 MB L2, so no flush is needed between steps.

Metric: FP64 cell-species updates per second (interior cells x updated
species x RK2 steps / time), whole job.  With --gpus N every rank advances its
own replica (independent runs; the path has no exchange step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the reference's own CPU implementation of the same
step (the reference C sources with the restated Fortran kernel, built under
oracle/_ref, serial build as shipped) with one process per host core, each on
its own slab of the grid's rows.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 cell-species updates/s & %HBM roofline; batched/plain; adjoint/forward"
UNIT = "cell-species updates/s"
NR, NZ, NTHETA, NS = 512, 1024, 16, 2
SAMPLE_NZ = 64                     # CPU sample: a 512 x 64 x 16 slab of the grid


def workload_config(extra=None):
    cfg = {"workload": f"plain 3-D CDR RK2 step, {NR}x{NZ} r-z cells x {NTHETA} theta planes, "
                       f"{NS} species (both mobile), 1 reaction table (256 nodes), fixed field",
           "nr": NR, "nz": NZ, "ntheta": NTHETA, "species": NS,
           "cells_per_replica": NR * NZ * NTHETA,
           "l2": "inputs larger than L2 (about 940 MB moved per step vs 126 MB L2); no flush",
           "parallelism": "replicas (one independent grid per GPU)"}
    if extra:
        cfg.update(extra)
    return cfg


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    """SM clock and clock-event reasons of one GPU, sampled in a background
    thread while the timed region runs: through NVML every ~0.5 ms (the
    timed region of a short run lasts a few milliseconds), else through
    nvidia-smi every 50 ms.  Reads only; no setting is changed."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # nvmlClocksEventReason* bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int):
        self.lines = []          # (time, sm_mhz, max_mhz, set of reasons)
        self.proc = None
        self.stop_flag = False
        self.th = None
        try:
            import pynvml
            pynvml.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[device]) if vis and vis.split(",")[device].isdigit() else device
            self.nv, self.h = pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.th = threading.Thread(target=self._poll_nvml, daemon=True)
            self.th.start()
            t0 = time.time()                 # the polling runs before the timed region starts
            while len(self.lines) < 3 and self.th.is_alive() and time.time() - t0 < 5:
                time.sleep(0.001)
            if self.lines:
                return
            self.stop_flag = True            # NVML gave nothing: nvidia-smi instead
            self.th.join(timeout=2)
            self.th = None
            self.nv = None
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read_smi, daemon=True)
        self.th.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 10:
            time.sleep(0.02)

    def _poll_nvml(self):
        nv = self.nv
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop_flag:
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                bits = int(get_reasons(self.h))
            except Exception:
                break
            rs = {n for n, b in self.BITS.items() if bits & b}
            self.lines.append((time.time(), sm, self.mx, rs))
            time.sleep(0.0005)

    def _read_smi(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            f = [x.strip() for x in line.strip().split(",")]
            try:
                sm, mx = float(f[1]), float(f[2])
            except (ValueError, IndexError):
                continue
            rs = {n for n, v in zip(names, f[5:9]) if v.lower().startswith("active")}
            self.lines.append((time.time(), sm, mx, rs))

    def stop(self):
        self.stop_flag = True
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.th is not None:
            self.th.join(timeout=2)

    def summary(self, t0: float, t1: float):
        rows = [r for r in self.lines if t0 <= r[0] <= t1]
        if not rows and self.lines:
            rows = [min(self.lines, key=lambda x: abs(x[0] - (t0 + t1) / 2))]
        sm = [r[1] for r in rows]
        mx = rows[-1][2] if rows else None
        reasons = set()
        for r in rows:
            reasons |= r[3]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.nv else "nvidia-smi"}


# ------------------------------------------------------------ CPU baseline ----
class _CStdoutToStderr:
    """Sends what C code prints on file descriptor 1 (the reference library's
    progress lines) to stderr, so that stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        try:
            C.CDLL(None).fflush(None)
        except (OSError, AttributeError):
            pass
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def cpu_baseline_sample(omp: bool, seconds: float = 12.0, max_steps: int = 10**9):
    with _CStdoutToStderr():
        return _cpu_baseline_sample(omp, seconds, max_steps)


def _cpu_baseline_sample(omp: bool, seconds: float, max_steps: int):
    """Reference CPU implementation (oracle/_ref) on a 512 x 64 x 16 slab of
    the workload; returns (cell-species updates/s, threads, kind, steps)."""
    from arcos_b200 import workloads
    from oracle import bind
    if not bind.ref_available(omp):
        omp = False
    kind = "reference" if bind.ref_available(False) else "port"
    pb = workloads.plain(nr=NR, nz=SAMPLE_NZ, ntheta=NTHETA, ion_mass=1.0, noise=1e-6, seed=0)
    threads = (os.cpu_count() or 1) if omp else 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    if kind == "reference":
        t = bind.RefTree(pb.params, pb.model, pb.specs, field_mode=bind.FIELD_FIXED, omp=omp)
        for s in range(NS):
            t.dens(0, s)[...] = pb.dens[0][s]
        er, ez, _ = pb.fields[0]
        t.set_fixed_field(0, er, ez, pb.specs[0].zeros())
        step = lambda: t.rk2_sw(50.0, per_plane=True, zero_all=False)  # noqa: E731
    else:
        t = bind.PortTree(pb.params, pb.model, pb.specs, field_mode=bind.FIELD_FIXED)
        for s in range(NS):
            t.dens(0, s)[...] = pb.dens[0][s]
        er, ez, _ = pb.fields[0]
        t.set_fixed_field(0, er, ez, pb.specs[0].zeros())
        step = lambda: t.rk2(50.0)  # noqa: E731
        threads = 1
    step()
    n, t0 = 0, time.perf_counter()
    while n < max_steps and (time.perf_counter() - t0 < seconds or n == 0):
        step()
        n += 1
    el = time.perf_counter() - t0
    return NR * SAMPLE_NZ * NTHETA * NS * n / el, threads, kind, n, el


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    with _CStdoutToStderr():
        line = _reference_line(args)
    print(json.dumps(line), flush=True)
    return 0


def _ref_slab(nz: int, seed: int, steps: int, warmup: int, barrier=None):
    """One share of the reference arm: the reference's serial step (the
    oracle/_ref build as shipped, else the CPU restatement) on a slab of nz
    rows of the grid; W untimed steps, then (after the barrier, when several
    processes share the work) K timed steps.  Returns (cell-species updates,
    seconds, kind)."""
    from oracle import bind
    from arcos_b200 import workloads
    pb = workloads.plain(nr=NR, nz=nz, ntheta=NTHETA, ion_mass=1.0, noise=1e-6, seed=seed)
    if bind.ref_available(False):
        t = bind.RefTree(pb.params, pb.model, pb.specs, field_mode=bind.FIELD_FIXED, omp=False)
        kind = "reference"
        step = lambda: t.rk2_sw(50.0, per_plane=True, zero_all=False)  # noqa: E731
    else:
        t = bind.PortTree(pb.params, pb.model, pb.specs, field_mode=bind.FIELD_FIXED)
        kind = "port"
        step = lambda: t.rk2(50.0)  # noqa: E731
    for s in range(NS):
        t.dens(0, s)[...] = pb.dens[0][s]
    er, ez, _ = pb.fields[0]
    t.set_fixed_field(0, er, ez, pb.specs[0].zeros())
    for _ in range(warmup):
        step()
    if barrier is not None:
        barrier.wait(timeout=900)
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    return NR * nz * NTHETA * NS * steps, time.perf_counter() - t0, kind


def _ref_slab_proc(nz, seed, steps, warmup, barrier, queue):
    with _CStdoutToStderr():
        try:
            queue.put(_ref_slab(nz, seed, steps, warmup, barrier))
        except BaseException as exc:          # the parent reports it
            barrier.abort()
            queue.put(("error", f"{type(exc).__name__}: {exc}", None))


def ref_slab_plan(total_steps: int, cores: int):
    """(processes, rows per slab) of the reference arm: one process per core
    (at most one per 16 rows), slabs that together cover the grid's NZ rows,
    thinned (multiples of 16 rows) so that one process's total_steps stay
    within about two minutes at ~3 s per whole-grid step on one core."""
    procs = max(1, min(cores, NZ // 16))
    budget_rows = max(16, (NZ * 40 // max(1, total_steps)) // 16 * 16)
    return procs, max(16, min(NZ, budget_rows, -(-NZ // procs)))


def _reference_line(args):
    """The reference's own CPU step on this workload, on all host cores.

    The reference's OpenMP build is not used: the parallel region of
    react_apply (src/reaction.c:95-160) shares its per-cell temporaries
    (eabs, log_e, pos, e1, e2, rate, r_mod, ...) between threads, a data race
    that makes it both slower than the serial build and wrong.  The host
    cores are used instead by one process per core, each running the serial
    build as shipped (oracle/_ref/libarcos_ref.so: the reference's C with its
    Fortran flux kernel restated) on its own slab of the grid's rows, the
    slabs' edges taken as domain boundaries; all processes start their timed
    steps together and the arm's time is the slowest process's.  The slabs
    cover the whole 512 x 1024 x 16 grid when the run is short enough (about
    3 s per whole-grid step on one core, at most ~2 minutes per process);
    otherwise they are thinner and the arm times a sample of the grid."""
    import multiprocessing as mp
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    procs, nz = ref_slab_plan(args.steps + args.warmup, cores)
    results = []
    if procs > 1:
        ctx = mp.get_context("spawn")
        barrier = ctx.Barrier(procs)
        queue = ctx.Queue()
        ps = [ctx.Process(target=_ref_slab_proc, args=(nz, i, args.steps, args.warmup, barrier, queue))
              for i in range(procs)]
        for p in ps:
            p.start()
        import queue as _queue
        t_end = time.time() + 1800
        while len(results) < procs:
            try:
                results.append(queue.get(timeout=5))
            except _queue.Empty:
                # a process that ended without reporting (a crash in the C code)
                dead = [p.exitcode for p in ps if p.exitcode not in (None, 0)]
                if dead or time.time() > t_end:
                    for p in ps:
                        if p.is_alive():
                            p.terminate()
                    raise RuntimeError(f"reference slab processes failed (exit codes {dead})"
                                       if dead else "reference slab processes timed out")
        for p in ps:
            p.join(timeout=60)
        bad = [r for r in results if r[0] == "error"]
        if bad:
            raise RuntimeError(f"reference slab process failed: {bad[0][1]}")
    else:
        results.append(_ref_slab(nz, 0, args.steps, args.warmup))
    work = sum(r[0] for r in results)
    el = max(r[1] for r in results)
    kind = results[0][2]
    value = work / el
    rows = procs * nz
    what = ("the whole grid" if rows >= NZ else f"{rows} of the grid's {NZ} rows") + \
        f" as {procs} slab(s) of {NR}x{nz}x{NTHETA}, one process per core"
    sample = (f"each step: one RK2 step of {what} (serial build as shipped; "
              f"{'the reference C' if kind == 'reference' else 'the CPU restatement'})")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload_config({"replicas": args.gpus}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


# ---------------------------------------------------------------- device ----

# ------------------------------------------------------------ extra rows ----
def _events(stream):
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _load(tree, pb):
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            tree.upload(g, "dens", a, s)
    for f, E in enumerate(pb.family_E):
        tree.set_family_field(f, *E)
    tree.set_fixed_field(pb.fields)


def extra_amr(stream, steps: int = 10):
    """Batched AMR: 4 levels, 320 patches (sides 16..256) advanced by one
    launch per kernel kind over all patches (one CUDA graph per step), the
    lean step with its kernel shape picked by the tree autotuner (tiled
    fused kernel or k_march), against one launch per patch of the general
    step, same GPU, same steps."""
    import numpy as np
    from arcos_b200 import workloads
    from arcos_b200.autotune import autotune_tree
    from arcos_b200.cdr import CdrTree
    from arcos_b200._lib import check
    pb = workloads.amr()
    out = {"workload": f"{len(pb.specs)} patches on 4 levels (root 512x1024, sides 16..256), "
                       f"{pb.cells} cells, 2 species, fixed field", "patches": len(pb.specs),
           "cells": pb.cells}
    for mode in ("batched", "per_patch"):
        tree = CdrTree(pb.params, pb.model, pb.specs, stream=stream.cuda_stream, per_patch=(mode == "per_patch"))
        _load(tree, pb)
        if mode == "batched":
            tune = autotune_tree(tree, steps=4, stream=stream)
            out["tree_autotune_ms_per_step"] = {str(k): v for k, v in tune.items()}
            out["tree_shape"] = tree.L.arcos_get_tile(tree.h)
            _load(tree, pb)
        nf = sum(1 for sp in pb.specs if sp.parent < 0)
        dts = np.zeros(nf * steps)
        tree.run(2, 50.0)
        e0, e1 = _events(stream)
        e0.record(stream)
        check(tree.L.arcos_run(tree.h, steps, 50.0, dts.ctypes.data_as(C.POINTER(C.c_double))))
        e1.record(stream)
        e1.synchronize()
        out[f"{mode}_ms_per_step"] = e0.elapsed_time(e1) / steps
        tree.close()
    out["batched_value"] = pb.cells * 2 / (out["batched_ms_per_step"] / 1e3)
    out["batched_over_per_patch"] = out["per_patch_ms_per_step"] / out["batched_ms_per_step"]
    step_bytes = 8 * (5 * 2 + 4) * pb.cells          # 8 (5S + 4) per cell and step
    gbs = step_bytes / (out["batched_ms_per_step"] / 1e3) / 1e9
    peak, src = _peak_hbm()
    out["roofline"] = {"bound": "hbm", "achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak,
                       "peak_source": src, "algorithmic_bytes_per_step": step_bytes}
    return out


def _peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fp:
            peaks = json.load(fp)
        return float(peaks["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _time_sweep(tree, stream) -> float:
    """Device time (CUDA events) of one reverse sweep through the C ABI
    (arcos_adj_backward: the replayed sweep graph plus the reduction of the
    mobility, diffusion and table gradients).  The initial-density gradients
    stay on the device until arcos_adj_get_cotangent fetches them."""
    import numpy as np
    from arcos_b200._lib import check
    ns = tree.model.no_species
    gm, gd = np.zeros(ns), C.c_double(0.0)
    gt = np.zeros(max(tree.L.arcos_adj_table_entries(tree.h), 1))
    e0, e1 = _events(stream)
    e0.record(stream)
    check(tree.L.arcos_adj_backward(tree.h, gm.ctypes.data_as(C.POINTER(C.c_double)), C.byref(gd),
                                    gt.ctypes.data_as(C.POINTER(C.c_double))))
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def extra_adjoint(stream, K: int = 64, ck: int = 64, ndir: int = 32):
    """Discrete adjoint: 256 x 512 grid, 64 RK2 steps, every state kept by the
    forward run (one segment: no recomputation in the reverse sweep; the
    sweep with checkpoints every 8 steps is timed beside it); J = 1/2 sum
    (n_e(T) - n_target)^2 cell_volume; reverse sweep time over the forward
    run's time, and central finite differences (step 1e-6 relative, 32 seeded
    smooth directions over densities, mobility, diffusion and the 256 table
    values) of the frozen-step forward."""
    import numpy as np
    from arcos_b200 import workloads
    from arcos_b200.adjoint import Adjoint, cell_volume, fd_objective_difference, smooth_direction
    from arcos_b200.cdr import CdrTree
    from arcos_b200._lib import check
    pb = workloads.plain(nr=256, nz=512, ion_mass=0.0, noise=1e-6, seed=3)
    spec = pb.specs[0]
    tree = CdrTree(pb.params, pb.model, pb.specs, stream=stream.cuda_stream)
    _load(tree, pb)
    adj = Adjoint(tree)
    vol = cell_volume(spec, pb.params.dr(0), pb.params.dz(0))
    rng = np.random.default_rng(5)
    tgt = workloads.seed_dens(spec, pb.params, rng, amp=0.11, sigma=0.09, noise=1e-6)
    for s in range(2):
        tree.upload(0, "dens", tgt, s)
    tree.run(K, 50.0)
    target = tree.download(0, "dens", 0)
    tab = pb.model.reactions[0].table
    base_vals = np.array(tab.values, dtype=np.float64)

    def apply(d0, mu, D, vals):
        for s in range(2):
            tree.upload(0, "dens", d0[s], s)
        tree.set_species_mass(0, 1.0 / mu)
        tree.set_diffusion(D)
        tree.set_table_values(0, vals, tab.underflow, tab.overflow)

    d0 = [a.copy() for a in pb.dens[0]]
    mu0, D0 = 1.0, pb.params.diffusion_coeff
    # forward cost: the plain fused run of K steps
    apply(d0, mu0, D0, base_vals)
    dts = np.zeros(K)
    tree.run(2, 50.0)
    apply(d0, mu0, D0, base_vals)
    e0, e1 = _events(stream)
    e0.record(stream)
    check(tree.L.arcos_run(tree.h, K, 50.0, dts.ctypes.data_as(C.POINTER(C.c_double))))
    e1.record(stream)
    e1.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    apply(d0, mu0, D0, base_vals)
    adj.forward(K, ck, h=50.0)              # the first call allocates the state buffers
    apply(d0, mu0, D0, base_vals)
    e0.record(stream)
    hs = adj.forward(K, ck, h=50.0)
    e1.record(stream)
    e1.synchronize()
    fwd_ck_ms = e0.elapsed_time(e1)
    ne = tree.download(0, "dens", 0)
    adj.set_cotangent(0, 0, (ne - target) * vol)
    adj.set_cotangent(0, 1, np.zeros_like(ne))
    g = adj.backward()                      # first call captures the sweep's CUDA graph
    adj.set_cotangent(0, 0, (ne - target) * vol)
    adj.set_cotangent(0, 1, np.zeros_like(ne))
    bwd_ms = _time_sweep(tree, stream)
    adj.set_cotangent(0, 0, (ne - target) * vol)
    adj.set_cotangent(0, 1, np.zeros_like(ne))
    g = adj.backward()
    # the same sweep with checkpoints every 8 steps (segments recomputed)
    apply(d0, mu0, D0, base_vals)
    adj.forward(K, 8, h=50.0)
    for _ in range(2):                      # the first call captures the sweep's CUDA graph
        adj.set_cotangent(0, 0, (ne - target) * vol)
        adj.set_cotangent(0, 1, np.zeros_like(ne))
        bwd8_ms = _time_sweep(tree, stream)
    # finite differences
    eps, worst = 1e-6, 0.0
    for _ in range(ndir):
        dd = [np.zeros(spec.shape) for _ in range(2)]
        for s in range(2):
            dd[s][0, 2:-2, 2:-2] = smooth_direction(rng, spec.nz, spec.nr)
        dmu, dD = rng.standard_normal(), rng.standard_normal()
        dv = rng.standard_normal(base_vals.shape)
        pred = sum(float(np.sum(g.dens0[0][s] * d0[s] * dd[s])) for s in range(2))
        pred += g.mobility[0] * mu0 * dmu + g.diffusion * D0 * dD + float(np.sum(g.tables[0] * base_vals * dv))
        outs = []
        for sg in (1.0, -1.0):
            apply([d0[s] * (1 + sg * eps * dd[s]) for s in range(2)], mu0 * (1 + sg * eps * dmu),
                  D0 * (1 + sg * eps * dD), base_vals * (1 + sg * eps * dv))
            adj.forward(K, ck, h_seq=hs)
            outs.append(tree.download(0, "dens", 0))
        fd = fd_objective_difference(outs[0], outs[1], target, vol, eps)
        worst = max(worst, abs(fd - pred) / abs(fd))
    tree.close()
    return {"workload": "256x512 grid, 2 species (ions immobile), 64 RK2 steps, every state kept, "
                        "gradients wrt n_e(0), n_i(0), mobility, diffusion, 256 table values",
            "forward_ms": fwd_ms, "forward_keeping_states_ms": fwd_ck_ms, "adjoint_ms": bwd_ms,
            "adjoint_timed": "one arcos_adj_backward call, CUDA events",
            "adjoint_over_forward": bwd_ms / fwd_ms,
            "adjoint_with_forward_overhead_over_forward": (bwd_ms + fwd_ck_ms - fwd_ms) / fwd_ms,
            "adjoint_ms_checkpoints_every_8": bwd8_ms,
            "adjoint_over_forward_checkpoints_every_8": bwd8_ms / fwd_ms,
            "fd_directions": ndir, "fd_step": eps, "fd_max_rel_err": worst}


def extra_kinetic(stream, K: int = 20):
    """Kinetic batch: 32 instances of uneven sizes, 6 species, 9 reactions
    with 1000-entry tables, per-instance applied field; batched fused forward
    in one launch per stage, and the adjoint of the total electron number at
    T with respect to all rate tables."""
    import numpy as np
    from arcos_b200 import workloads
    from arcos_b200.adjoint import Adjoint, cell_volume
    from arcos_b200.cdr import CdrTree
    from arcos_b200._lib import check
    from arcos_b200.autotune import autotune_tiles
    pb = workloads.kinetic_batch(n_inst=32)
    tree = CdrTree(pb.params, pb.model, pb.specs, stream=stream.cuda_stream)
    _load(tree, pb)
    tune = autotune_tiles(tree, steps=4, stream=stream)    # the tuning steps advance the state
    _load(tree, pb)
    L, h = tree.L, tree.h
    check(L.arcos_run_prepare(h, 50.0))
    check(L.arcos_run_enqueue(h, 4))
    e0, e1 = _events(stream)
    e0.record(stream)
    check(L.arcos_run_enqueue(h, K))
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / K
    ns = pb.model.no_species
    _load(tree, pb)
    adj = Adjoint(tree)
    Ka, ck = 16, 16                         # one segment: every state kept by the forward run
    adj.forward(Ka, ck, h=50.0)             # the first call allocates the state buffers
    _load(tree, pb)
    e0.record(stream)
    adj.forward(Ka, ck, h=50.0)
    e1.record(stream)
    e1.synchronize()
    fwd_keep_ms = e0.elapsed_time(e1)
    for g, sp in enumerate(pb.specs):
        vol = cell_volume(sp, pb.params.dr(0), pb.params.dz(0))
        adj.set_cotangent(g, 0, vol)
        for s in range(1, ns):
            adj.set_cotangent(g, s, np.zeros(sp.shape))
    gr = adj.backward()                     # first call captures the sweep's CUDA graph
    for g, sp in enumerate(pb.specs):
        adj.set_cotangent(g, 0, cell_volume(sp, pb.params.dr(0), pb.params.dz(0)))
        for s in range(1, ns):
            adj.set_cotangent(g, s, np.zeros(sp.shape))
    bwd = _time_sweep(tree, stream)
    # the same sweep with checkpoints every 8 steps (segments recomputed)
    _load(tree, pb)
    adj.forward(Ka, 8, h=50.0)
    for _ in range(2):                      # the first call captures the sweep's CUDA graph
        for g, sp in enumerate(pb.specs):
            adj.set_cotangent(g, 0, cell_volume(sp, pb.params.dr(0), pb.params.dz(0)))
            for s in range(1, ns):
                adj.set_cotangent(g, s, np.zeros(sp.shape))
        bwd8 = _time_sweep(tree, stream)
    tree.close()
    return {"workload": f"{len(pb.specs)} instances, {pb.cells} cells, {ns} species, "
                        f"{len(pb.model.reactions)} reactions (1000-entry tables)",
            "cells": pb.cells, "ms_per_step": ms, "value": pb.cells * ns / (ms / 1e3),
            "tile_autotune_ms_per_step": {str(k): v for k, v in tune.items()},
            "adjoint_steps": Ka, "adjoint_states": "every state kept by the forward run (one segment)",
            "adjoint_ms": bwd, "adjoint_over_forward": bwd / (ms * Ka),
            "forward_keeping_states_ms": fwd_keep_ms,
            "adjoint_with_forward_overhead_over_forward": (bwd + fwd_keep_ms - ms * Ka) / (ms * Ka),
            "adjoint_ms_checkpoints_every_8": bwd8, "adjoint_over_forward_checkpoints_every_8": bwd8 / (ms * Ka),
            "adjoint_timed": "one arcos_adj_backward call, CUDA events",
            "table_grad_norm": float(sum(np.linalg.norm(t) for t in gr.tables))}


# the reference's default refinement parameters (src/cstream.c:165-182)
REFINE_DEFAULTS = dict(threshold_eabs=0.2, level_eabs=4, threshold_charge=0.004, threshold_dens=0.004,
                       threshold_edge=1e4, brick_dr=8, brick_dz=8, max_level=3)


def _refine_state(tree_like, pb, upload):
    """Seeded state of the refinement row: the plain workload's densities
    with the ions perturbed (so the charge has structure) and a smooth |E|
    that exceeds the default threshold (0.2) only around its peak."""
    import numpy as np
    d0, d1 = pb.dens[0]
    sp = pb.specs[0]
    z = (np.arange(sp.nz + 4) - 2 + 0.5) / sp.nz
    r = (np.arange(sp.nr + 4) - 2 + 0.5) / sp.nr
    d1 = d1 * (1.0 + 0.2 * np.sin(6.0 * z))[None, :, None]
    peak = np.exp(-(r[None, :] ** 2 + (z[:, None] - 0.6) ** 2) / (2 * 0.1 ** 2))
    eabs = np.broadcast_to((0.1 + 0.3 * peak)[None], d0.shape).copy()
    upload(d0, d1, eabs)


def extra_field(stream, K: int = 100):
    """The field solved on the device at both stages of every step (c0:
    128 x 256, immobile ions; the same with 16 theta planes, solved by theta
    modes) and photoionization (two terms, 128 x 256 and 128 x 256 x 16,
    fixed field): device time per RK2 step over K steps replayed from the
    step graph, CUDA events."""
    from arcos_b200 import workloads
    from arcos_b200.cdr import CdrTree
    out = {}

    def timed(tree, name, cells, ns):
        tree.run(3, 50.0)                       # warm-up (captures the step graph)
        e0, e1 = _events(stream)
        e0.record(stream)
        tree.run(K, 50.0)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / K
        out[name] = {"ms_per_step": ms, "cells": cells, "value": cells * ns / (ms / 1e3)}

    for nt in (1, 16):
        pb = workloads.plain(nr=128, nz=256, ntheta=nt, ion_mass=0.0, noise=0.3 if nt > 1 else 0.0, seed=0)
        tree = CdrTree(pb.params, pb.model, pb.specs, stream=stream.cuda_stream)
        for s in range(2):
            tree.upload(0, "dens", pb.dens[0][s], s)
        tree.cdr_calc_charge_r(0)
        tree.set_field_poisson(True)
        timed(tree, "field_in_loop_128x256" + ("" if nt == 1 else f"x{nt}"), 128 * 256 * nt, 2)
        tree.close()
    for nt in (1, 16):
        pb = workloads.photo(nr=128, nz=256, ntheta=nt, noise=0.3 if nt > 1 else 0.0, seed=0)
        tree = CdrTree(pb.params, pb.model, pb.specs, stream=stream.cuda_stream)
        _load(tree, pb)
        timed(tree, "photo_128x256" + ("" if nt == 1 else f"x{nt}"), 128 * 256 * nt, pb.model.no_species)
        tree.close()
    out["workload"] = ("field solve in the loop (sine transform in z, tridiagonal in r, theta modes in 3-D) "
                       "and photoionization (2 terms, 5 species), device time per RK2 step")
    return out


def extra_plain_wavy(stream, K: int = 20, W: int = 5):
    """The headline grid (512 x 1024 x 16, 2 species, per-plane mode) on the
    seeded non-uniform field (both components change sign inside a tile,
    |E| sweeps the reaction table from underflow to overflow): the same
    timing as the main line (K steps replayed from the step graph after W
    warm-up steps, CUDA events) and the stage-2 kernel's roofline, so the
    headline is not only measured on the uniform field."""
    from arcos_b200 import workloads
    from arcos_b200._lib import check
    from arcos_b200.autotune import autotune_tiles
    from arcos_b200.cdr import CdrTree
    pb = workloads.plain(nr=NR, nz=NZ, ntheta=NTHETA, ion_mass=1.0, noise=1e-6, seed=0, field="wavy")
    tree = CdrTree(pb.params, pb.model, pb.specs, stream=stream.cuda_stream)
    _load(tree, pb)
    L, h = tree.L, tree.h
    tune = autotune_tiles(tree, steps=6, stream=stream)
    check(L.arcos_run_prepare(h, 50.0))
    check(L.arcos_run_enqueue(h, W))
    e0, e1 = _events(stream)
    e0.record(stream)
    check(L.arcos_run_enqueue(h, K))
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / K
    _, hlast, err = tree.family_state(0)
    ev = _events(stream)
    s2 = 0.0
    for k in range(10):
        check(L.arcos_enqueue_stage(h, 1, k & 1))
        ev[0].record(stream)
        check(L.arcos_enqueue_stage(h, 2, k & 1))
        ev[1].record(stream)
        ev[1].synchronize()
        s2 += ev[0].elapsed_time(ev[1]) / 10
    tree.close()
    cells = NR * NZ * NTHETA
    peak, src = _peak_hbm()
    bytes_s2 = 8 * (3 * NS + 2) * cells
    return {"workload": f"{NR}x{NZ}x{NTHETA} grid, 2 species, wavy fixed field (er, ez change sign "
                        "inside a tile; |E| from 0.02 to 30)",
            "ms_per_step": ms, "value": cells * NS / (ms / 1e3), "steps": K, "warmup": W,
            "stage2_ms": s2, "stage2_frac": bytes_s2 / (s2 / 1e3) / 1e9 / peak, "peak_source": src,
            "tile_autotune_ms_per_step": {str(k): v for k, v in tune.items()},
            "dt_last": hlast, "device_error_bits": err}


def extra_refine(stream, calls: int = 5):
    """Refinement criteria (cdr_refine, src/cdr.c:1630-1682) of the
    512 x 1024 x 16 grid with the reference's default parameters: one
    arcos_cdr_refine call (per-cell masks on the device, masks to the host,
    the brick search on the host) against the reference's cdr_refine on a
    512 x 64 x 16 slab on one host core, as cells per second."""
    import numpy as np
    from arcos_b200 import workloads
    from arcos_b200.cdr import CdrTree
    from oracle import bind
    pb = workloads.plain(nr=NR, nz=NZ, ntheta=NTHETA, ion_mass=1.0, noise=1e-6, seed=0)
    tree = CdrTree(pb.params, pb.model, pb.specs, stream=stream.cuda_stream)
    tree.set_fixed_field(pb.fields)

    def up(d0, d1, eabs):
        tree.upload(0, "dens", d0, 0)
        tree.upload(0, "dens", d1, 1)
        tree.cdr_set_ext_bnd_r()
        tree.cdr_calc_charge_r()
        tree.upload(0, "eabs", eabs)
    _refine_state(tree, pb, up)
    kids = tree.cdr_refine(0, **REFINE_DEFAULTS)
    stream.synchronize()
    t0 = time.perf_counter()
    for _ in range(calls):
        tree.cdr_refine(0, **REFINE_DEFAULTS)
    dev_s = (time.perf_counter() - t0) / calls
    cells = NR * NZ * NTHETA
    tree.close()
    out = {"workload": f"{NR}x{NZ}x{NTHETA} grid, seeded blobs, reference default refinement parameters",
           "children": len(kids), "device_call_ms": dev_s * 1e3, "device_cells_per_s": cells / dev_s}
    if bind.ref_available(False):
        with _CStdoutToStderr():
            spb = workloads.plain(nr=NR, nz=SAMPLE_NZ, ntheta=NTHETA, ion_mass=1.0, noise=1e-6, seed=0)
            ref = bind.RefTree(spb.params, spb.model, spb.specs, field_mode=bind.FIELD_FIXED)

            def rup(d0, d1, eabs):
                ref.dens(0, 0)[...] = d0
                ref.dens(0, 1)[...] = d1
                ref.call("ref_set_ext_bnd_r")
                ref.call("ref_calc_charge_r")
                ref.array(0, "eabs")[...] = eabs
            _refine_state(ref, spb, rup)
            ref.cdr_refine(0, **REFINE_DEFAULTS)
            t0 = time.perf_counter()
            ref.cdr_refine(0, **REFINE_DEFAULTS)
            ref_s = time.perf_counter() - t0
        out["reference_cells_per_s"] = NR * SAMPLE_NZ * NTHETA / ref_s
        out["reference_sample"] = f"one cdr_refine of a {NR}x{SAMPLE_NZ}x{NTHETA} slab, 1 core"
    return out


def run_device(args):
    import ctypes as C

    import numpy as np
    import torch
    import torch.distributed as dist

    from arcos_b200 import workloads
    from arcos_b200._lib import check
    from arcos_b200.cdr import CdrTree

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev_id = torch.cuda.current_device()

    from arcos_b200.replicas import barrier, max_over_ranks

    def allmax(x: float) -> float:
        return max_over_ranks(x, "cuda")

    pb = workloads.plain(nr=NR, nz=NZ, ntheta=NTHETA, ion_mass=1.0, noise=1e-6, seed=rank)
    stream = torch.cuda.Stream()
    tree = CdrTree(pb.params, pb.model, pb.specs, stream=stream.cuda_stream, exact=args.exact)
    for s in range(NS):
        tree.upload(0, "dens", pb.dens[0][s], s)
    tree.set_fixed_field(pb.fields)
    L, h = tree.L, tree.h
    if args.tile is None:
        from arcos_b200.autotune import autotune_tiles
        tune = autotune_tiles(tree, steps=6, stream=stream)
    else:
        tree.set_tile(args.tile)
        tune = {}
    # the lean path takes any step count; the bit-exact path alternates storage sets
    warm, steps = args.warmup, args.steps
    if args.exact:
        warm, steps = warm + (warm & 1), steps + (steps & 1)
    check(L.arcos_run_prepare(h, 50.0))
    if warm > 0:
        check(L.arcos_run_enqueue(h, warm))
    torch.cuda.synchronize()

    clk = ClockSampler(dev_id) if rank == 0 else None
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    w0 = time.time()
    e0.record(stream)
    check(L.arcos_run_enqueue(h, steps))
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    w1 = time.time()
    barrier()
    ms = e0.elapsed_time(e1) / steps
    ms = allmax(ms)
    clocks = clk.summary(w0, w1) if clk else None
    if clk:
        clk.stop()
    st, hlast, err = tree.family_state(0)
    if err:
        raise RuntimeError(f"device error bits {err}")

    cells = NR * NZ * NTHETA
    value = world * cells * NS / (ms / 1e3)

    # per-kernel durations (same work, stage kernels launched one by one)
    nk = 20
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    s1 = s2 = 0.0
    for k in range(nk):
        src = k & 1
        ev[0].record(stream)
        check(L.arcos_enqueue_stage(h, 1, src))
        ev[1].record(stream)
        check(L.arcos_enqueue_stage(h, 2, src))
        ev[2].record(stream)
        ev[2].synchronize()
        s1 += ev[0].elapsed_time(ev[1])
        s2 += ev[1].elapsed_time(ev[2])
    s1 /= nk
    s2 /= nk
    bytes_s1 = 8 * (2 * NS + 2) * cells          # reads n0[S], er, ez; writes n*[S]
    bytes_s2 = 8 * (3 * NS + 2) * cells          # reads n0[S], n*[S], er, ez; writes n1[S]
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fp:
            peaks = json.load(fp)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dom_ms, dom_bytes, dom_name = (s2, bytes_s2, "stage-2 kernel") if s2 >= s1 else (s1, bytes_s1, "stage-1 kernel")
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "stage_kernels_plain3d.json")
    if os.path.exists(prof):
        try:
            with open(prof) as fp:
                traffic = json.load(fp).get("dram_bytes_per_launch", {}).get(
                    "stage2" if dom_name.startswith("stage-2") else "stage1")
        except Exception:
            traffic = None
    step_bytes = 8 * (5 * NS + 4) * cells
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes,
                "kernel_ms": dom_ms, "step_achieved_gbs": step_bytes / (ms / 1e3) / 1e9,
                "step_frac": step_bytes / (ms / 1e3) / 1e9 / peak}

    # end to end through the C ABI with host buffers: H2D of the densities,
    # one cdr_rk2 step (arcos_run), D2H of the densities, every step
    e2e_steps = max(3, min(10, args.steps))
    sp = pb.specs[0]
    host = [torch.empty(sp.shape, dtype=torch.float64, pin_memory=True) for _ in range(NS)]
    for s in range(NS):
        host[s].numpy()[...] = tree.download(0, "dens", s)
    DPp = C.POINTER(C.c_double)
    ptrs = [C.cast(C.c_void_p(x.data_ptr()), DPp) for x in host]
    dts = np.zeros(1)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for s in range(NS):
            check(L.arcos_upload(h, 0, 0, 0, s, ptrs[s]))
        check(L.arcos_run(h, 1, 50.0, dts.ctypes.data_as(DPp)))
        for s in range(NS):
            check(L.arcos_download(h, 0, 0, 0, s, ptrs[s]))
    torch.cuda.synchronize()
    e2e_s = allmax(time.perf_counter() - t0)
    barrier()
    arr_bytes = int(np.prod(sp.shape)) * 8
    e2e = {"value": world * cells * NS * e2e_steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": NS * arr_bytes, "d2h_bytes_per_step": NS * arr_bytes,
           "steps": e2e_steps, "api": "arcos_upload + arcos_run(1 step) + arcos_download"}

    extras = {}
    if rank == 0 and not args.no_extras:
        wanted = set(args.extras.split(","))
        for name, fn in (("amr_batched", extra_amr), ("adjoint", extra_adjoint),
                         ("kinetic_batch", extra_kinetic), ("refine", extra_refine),
                         ("field", extra_field), ("plain_wavy", extra_plain_wavy)):
            if name not in wanted:
                continue
            try:
                extras[name] = fn(stream)
            except Exception as exc:          # reported, the main line stands
                extras[name] = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            v, thr, kind, n, el = cpu_baseline_sample(omp=False)
            cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": kind,
                   "sample": f"{n} RK2 steps of a {NR}x{SAMPLE_NZ}x{NTHETA} slab of the grid "
                             f"({el:.1f} s, serial build as shipped)"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": steps, "warmup": warm, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded)",
                "config": workload_config({"replicas": world}),
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": 2 * steps, "clocks": clocks,
                "stage_kernel_ms": {"stage1": s1, "stage2": s2},
                "tile_autotune_ms_per_step": {str(k): v for k, v in tune.items()},
                "limiter": "bit-exact" if args.exact else "division-free (1e-12/step)",
                "dt_last": hlast, "extras": extras}
        print(json.dumps(line), flush=True)
    tree.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-AMR, adjoint and kinetic-batch measurements")
    ap.add_argument("--extras", default="amr_batched,adjoint,kinetic_batch,refine,field,plain_wavy",
                    help="comma-separated subset of the extra measurements")
    ap.add_argument("--exact", action="store_true", help="bit-exact flux limiter")
    ap.add_argument("--tile", type=int, default=None,
                    help="fixed tile shape (0: 32x16 cells / 4 warps, 1: 32x32 / 8 warps, "
                         "2: 32x16 / 8 warps); default: autotuned")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_device(args)


if __name__ == "__main__":
    sys.exit(main())
