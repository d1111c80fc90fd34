#!/usr/bin/env python
"""Benchmark of the 2D Laplace KIFMM evaluation path on B200.

Workload (one "step"): the clustered configuration -- 1,000,000 sources in
20 Gaussian clusters (centres U[-0.9,0.9]^2, sigma 0.01), charges N(0,1),
evaluated at the sources (self-interaction excluded) and on a 1000 x 1000
grid over [-1,1]^2; at most 64 points per leaf.  A step is what the
reference's examples time: build the FMM object (quadtree), form the
expansions, evaluate at the sources, evaluate at the grid, with the
per-width operators already cached (helper reuse).
Metric: million points per second, (N_sources + N_targets) / step time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64]
    python bench.py --impl reference ...    # the reference flexmm on the host CPU

``value`` is timed on the device with CUDA events, inputs resident in HBM,
L2 flushed between steps; ``e2e`` is the same step through the public API
from pinned host buffers, copies and the read-back of both results included.
With N > 1 (torchrun) every rank runs an independent replica of the step
(the path does not shard a single problem); value sums the ranks' points
over the slowest rank's time.
"""
import argparse
import json
import os
import gc
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "Mpts/s, 1M Laplace KIFMM on 1 B200, mixed vs FP64 at rel err 1e-6; ref CPU"
NCUT = 64
NEQ = {"fp64": 60, "mixed": 24}
C_LAPLACE = 20          # flops per Laplace kernel evaluation (9 arithmetic + log as 11)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--precision", choices=sorted(NEQ), default="mixed",
                   help="headline form (the other form is measured alongside unless --only)")
    p.add_argument("--only", action="store_true", help="measure only --precision")
    p.add_argument("--n", type=int, default=1_000_000, help="sources (default: the 1M config)")
    p.add_argument("--grid", type=int, default=1000, help="grid targets per side")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batched-stokes", action="store_true",
                   help="skip the batched-Stokes (many independent problems) measurement")
    p.add_argument("--no-adjoint", action="store_true",
                   help="skip the differentiable black-box FMM (forward + backward) measurement")
    p.add_argument("--no-multi-rhs", action="store_true",
                   help="skip the multi-RHS (64 charge columns, modified Helmholtz) measurement")
    p.add_argument("--no-helmholtz", action="store_true",
                   help="skip the modified-Helmholtz mixed vs FP64 measurement")
    p.add_argument("--cpu-sample-n", type=int, default=200_000,
                   help="sources in the bounded reference sample of our arm's cpu_baseline")
    p.add_argument("--denested-steps", type=int, default=3,
                   help="reference arm: steps of the de-nested S2M variant (0: none)")
    p.add_argument("--json-only", action="store_true", help=argparse.SUPPRESS)
    p.add_argument("--ncu", action="store_true",
                   help="profiling mode: warm-up and timed steps only (no accuracy, e2e, peaks)")
    return p.parse_args()


# ----------------------------------------------------------------- helpers --
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            backend = "nccl"
        else:
            backend = "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def dist_max(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling (200 ms) while the timed loops run."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.rows = []
        self.thread = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, bufsize=1)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up must not overlap the timed work: wait for
            # its first sample (bounded), then a little more
            t_end = time.time() + 5.0
            while not self.rows and time.time() < t_end:
                time.sleep(0.05)
            time.sleep(0.2)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def wait_for_sample(self, busy=None, timeout=1.0):
        """Return just after the next sample lands: a timed loop of a few tens of
        ms then runs between two nvidia-smi queries (a query can stall the
        GPU for milliseconds).  `busy` (untimed work) runs meanwhile, so the
        GPU does not idle, and drop its clocks, before the timed loop."""
        if self.proc is None:
            return
        n0 = len(self.rows)
        t_end = time.time() + timeout
        while len(self.rows) == n0 and time.time() < t_end:
            if busy is not None:
                busy()
            else:
                time.sleep(0.001)

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread is not None:
                self.thread.join(timeout=5)

    def summary(self):
        rows = self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        num = lambda v: v.replace(".", "", 1).isdigit()
        sm = [float(r[1]) for r in rows if num(r[1])]
        smax = [float(r[2]) for r in rows if num(r[2])]
        pw = [float(r[3]) for r in rows if num(r[3])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(pw) if pw else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def gemm_peak_tflops(torch, dtype, tf32=False):
    """Throughput of this GPU for a cuBLAS GEMM (8192^3): float64 (FP64
    pipe), float32 without TF32 (FP32 FMA pipe) or float32 with TF32."""
    torch.backends.cuda.matmul.allow_tf32 = tf32
    n = 8192
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.backends.cuda.matmul.allow_tf32 = False
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


# ------------------------------------------------------------- work counts --
def work_counts(F, tx, ty, nequiv):
    """Algorithmic work of one step from the tree (kernel evaluations, GEMM flops)."""
    t = F.tree
    counts = dict(p2p_pairs_src=0, p2p_pairs_tgt=0, m2l_flops=0, s2m_ke=0, l2t_ke=0,
                  m2m_flops=0, l2l_flops=0, c2e_flops=0, nequiv=nequiv)

    def locate(px, py):
        inds = np.zeros(px.size, np.int64)
        locs = np.zeros(px.size, np.int64)
        active = np.flatnonzero(~t.Levels[0].leaf[locs])
        ind = 0
        while active.size:
            lv = t.Levels[ind]
            loc = locs[active]
            c = lv.children_ind[loc] + 2 * (px[active] > lv.xmid[loc]) + (py[active] > lv.ymid[loc])
            ind += 1
            locs[active] = c
            inds[active] = ind
            active = active[~t.Levels[ind].leaf[c]]
        return inds, locs

    def pairs(px, py):
        inds, locs = locate(px, py)
        tot = 0
        for ind in np.unique(inds):
            lv = t.Levels[ind]
            sel = locs[inds == ind]
            col = lv.colleagues[sel]
            ok = col >= 0
            tot += int(np.where(ok, lv.ns[np.where(ok, col, 0)], 0).sum())
        return tot

    x = F._x.cpu().numpy()
    y = F._y.cpu().numpy()
    counts["p2p_pairs_src"] = pairs(x, y)
    counts["p2p_pairs_tgt"] = pairs(tx, ty)
    counts["l2t_ke"] = nequiv * (x.size + tx.size)
    n = nequiv
    for ind, lv in enumerate(t.Levels):
        if ind < 2:
            continue
        prec = F.helper.get_precomputation(lv.width)
        ranks = prec.m2l_rank
        tr = t.interaction_triples(ind)
        if tr.size:
            grid49 = np.array([(a + 3) * 7 + (b + 3) for a in range(-3, 4) for b in range(-3, 4)
                               if not (abs(a) <= 1 and abs(b) <= 1)])
            pos = {g: o for o, g in enumerate(grid49)}
            per_off = np.bincount([pos[g] for g in tr[:, 1]], minlength=40)
            fl = np.where(ranks < 0, 2 * n * n, 4 * n * np.maximum(ranks, 0))
            counts["m2l_flops"] += int((per_off * fl).sum())
        up = lv.compute_upwards
        counts["s2m_ke"] += n * int(lv.ns[up].sum())
        counts["m2m_flops"] += 2 * n * 4 * n * int(((lv.children_ind >= 0)).sum())
        real = ~lv.fake_leaf
        counts["c2e_flops"] += 2 * 4 * n * n * int(real.sum())
        if ind >= 3:
            counts["l2l_flops"] += 2 * n * n * int(real.sum())
    return counts


# ---------------------------------------------------------------- our arm --
def measure(args, world, local, d, precision, flush, counts_cache):
    """Time one precision form: device-resident steps, e2e steps, accuracy, roofline."""
    import torch
    from flexmm_b200 import (KI_FMM, KI_Helper, direct_evaluation, enable_timing, read_timing,
                             set_split_evaluation)

    dev = torch.device("cuda", local)
    neq = NEQ[precision]
    n_src, n_tgt = d["x"].size, d["tx"].size
    pts = n_src + n_tgt
    xd, yd, taud, txd, tyd = (torch.from_numpy(d[k]).to(dev) for k in ("x", "y", "tau", "tx", "ty"))
    helper = KI_Helper()

    def step(x, y, tau, tx, ty):
        F = KI_FMM(x, y, "Laplace_Eval", NCUT, neq, bbox=d["bbox"], helper=helper,
                   precision=precision)
        F.build_expansions(tau)
        us = F.source_evaluation(x, y)
        ut = F.target_evaluation(tx, ty)
        return F, us, ut

    for _ in range(max(args.warmup, 1)):
        F, us, ut = step(xd, yd, taud, txd, tyd)
    torch.cuda.synchronize()
    if args.ncu:
        for _ in range(args.steps):
            step(xd, yd, taud, txd, tyd)
        torch.cuda.synchronize()
        return None

    # accuracy of this step's results: FP64 direct sums on 2000-point samples,
    # and agreement with the reference's own outputs (committed fixture)
    rng = np.random.default_rng(12345)
    si = np.sort(rng.choice(n_src, min(2000, n_src), replace=False))
    ti = np.sort(rng.choice(n_tgt, min(2000, n_tgt), replace=False))
    us_h, ut_h = us.cpu().numpy(), ut.cpu().numpy()
    ds = direct_evaluation("Laplace_Eval", xd, yd, taud, xd[si], yd[si], check=True).cpu().numpy()
    dt = direct_evaluation("Laplace_Eval", xd, yd, taud, txd[ti], tyd[ti]).cpu().numpy()
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    accuracy = {"src_rel_l2_vs_direct": rel(us_h[si], ds), "tgt_rel_l2_vs_direct": rel(ut_h[ti], dt),
                "sample": "2000 sources + 2000 grid targets, FP64 direct sum on the GPU"}
    gold = os.path.join(REPO, "tests", "golden", f"clustered_1M_q{neq}.npz")
    if args.n == 1_000_000 and args.grid == 1000 and os.path.exists(gold):
        g = np.load(gold)
        accuracy["src_rel_l2_vs_reference"] = rel(us_h[g["src_idx"]], g["src_val"])
        accuracy["tgt_rel_l2_vs_reference"] = rel(ut_h[g["tgt_idx"]], g["tgt_val"])

    # timed region: K steps, L2 flushed between steps, CUDA events on the stream
    # (the library's per-phase event timers stay off here: they put event
    # records between its kernels)
    barrier(world)
    torch.cuda.synchronize()
    times = []
    clk = ClockSampler(local).__enter__()
    step(xd, yd, taud, txd, tyd)  # one untimed step with the sampler running
    torch.cuda.synchronize()
    gc.collect()
    gc.disable()  # a collector pause inside one timed step is host noise, not the library

    def untimed():
        step(xd, yd, taud, txd, tyd)
        torch.cuda.synchronize()
    clk.wait_for_sample(busy=untimed)
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        step(xd, yd, taud, txd, tyd)
        e1.record()
        times.append((e0, e1))
    torch.cuda.synchronize()
    gc.enable()
    barrier(world)
    step_samples = [round(a.elapsed_time(b), 3) for a, b in times]
    ms_step = dist_max(sum(a.elapsed_time(b) for a, b in times) / max(args.steps, 1), world)

    # per-phase breakdown from separate, untimed steps with the timers on and
    # the evaluation in one kernel after the passes, so that every kernel's
    # time is its own (a split near field shares the SMs with the passes)
    n_phase = args.steps  # the breakdown is normalised per timed step count
    set_split_evaluation(False)
    enable_timing(True)
    read_timing()
    for _ in range(n_phase):
        flush.fill_(1.0)
        step(xd, yd, taud, txd, tyd)
    torch.cuda.synchronize()
    phases = read_timing()
    enable_timing(False)
    set_split_evaluation(None)

    # end to end through the public API from pinned host memory
    pin = {k: torch.from_numpy(d[k]).pin_memory() for k in ("x", "y", "tau", "tx", "ty")}
    # first-use costs stay untimed; results are held across steps exactly as
    # in the timed loop, so the pinned result buffers of both are allocated here
    for _ in range(max(args.warmup, 2)):
        F2, us2, ut2 = step(pin["x"], pin["y"], pin["tau"], pin["tx"], pin["ty"])
    torch.cuda.synchronize()
    e2e_ms = []
    gc.collect()
    gc.disable()  # a collector pause inside one timed step is host noise, not the library
    barrier(world)

    def untimed_e2e():
        step(pin["x"], pin["y"], pin["tau"], pin["tx"], pin["ty"])
        torch.cuda.synchronize()
    clk.wait_for_sample(busy=untimed_e2e)
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        F2, us2, ut2 = step(pin["x"], pin["y"], pin["tau"], pin["tx"], pin["ty"])
        e1.record()
        torch.cuda.synchronize()
        assert not us2.is_cuda and not ut2.is_cuda
        e2e_ms.append(e0.elapsed_time(e1))
    gc.enable()
    clk.__exit__(None, None, None)
    e2e_step = dist_max(statistics.mean(e2e_ms), world)

    def count_launches():
        """Launches of our kernels in one step (CUPTI through torch.profiler);
        run after every form's timed loops: the profiler's teardown must not
        overlap timed steps."""
        from torch.profiler import ProfilerActivity, profile
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            step(xd, yd, taud, txd, tyd)
            torch.cuda.synchronize()
        return sum(
            1 for ev in prof.events()
            if str(getattr(ev, "device_type", "")).endswith("CUDA")
            and "memcpy" not in ev.name.lower() and "memset" not in ev.name.lower()) * args.steps

    if "counts" not in counts_cache:
        counts_cache["counts"] = work_counts(F, d["tx"], d["ty"], neq)
    c = dict(counts_cache["counts"])
    scale = neq / c["nequiv"]
    c["l2t_ke"] = int(c["l2t_ke"] * scale)
    c["s2m_ke"] = int(c["s2m_ke"] * scale)
    # source evaluation on the FMM's own (unchanged) source tensors reads the
    # tree's copy: x, y are then uploaded once per step, not twice
    src_reused = F2._own_sources(pin["x"], pin["y"])
    return dict(F=F, ms_step=ms_step, step_samples=step_samples, e2e_step=e2e_step, phases=phases,
                accuracy=accuracy, src_reused=src_reused, e2e_samples=e2e_ms,
                count_launches=count_launches, clocks=clk.summary(), neq=neq,
                counts=work_counts_gemm(F, neq, c))


def work_counts_gemm(F, neq, c):
    """GEMM flops of one step at this Nequiv (the tree is the same for every Nequiv)."""
    t = F.tree
    n = neq
    out = dict(c, m2l_flops=0, m2m_flops=0, l2l_flops=0, c2e_flops=0)
    grid49 = np.array([(a + 3) * 7 + (b + 3) for a in range(-3, 4) for b in range(-3, 4)
                       if not (abs(a) <= 1 and abs(b) <= 1)])
    pos = {g: o for o, g in enumerate(grid49)}
    for ind, lv in enumerate(t.Levels):
        if ind < 2:
            continue
        ranks = F.helper.get_precomputation(lv.width).m2l_rank
        tr = t.interaction_triples(ind)
        if tr.size:
            per_off = np.bincount([pos[g] for g in tr[:, 1]], minlength=40)
            dense = F.precision == "mixed"   # the mixed form applies every M2L densely
            fl = np.where((ranks < 0) | dense, 2 * n * n, 4 * n * np.maximum(ranks, 0))
            fl = np.where(ranks == 0, 0, fl)
            out["m2l_flops"] += int((per_off * fl).sum())
        out["m2m_flops"] += 8 * n * n * int((lv.children_ind >= 0).sum())
        real = ~lv.fake_leaf
        out["c2e_flops"] += 8 * n * n * int(real.sum())
        if ind >= 3:
            out["l2l_flops"] += 2 * n * n * int(real.sum())
    return out


# DRAM bytes per launch of the dominant kernel on the default workload (1M
# clustered sources + 1000^2 grid): ncu captures of the 200k-source /
# 450^2-grid case of the same distribution, scaled by the points each
# launch evaluates, averaged over the source and grid launches
NCU_TRAFFIC_BYTES = {("mixed", "evaluate"): 46_400_000, ("fp64", "evaluate"): 60_600_000}


def roofline_of(res, precision, peaks, steps, default_workload):
    c = res["counts"]
    ke = {"evaluate": c["p2p_pairs_src"] + c["p2p_pairs_tgt"] + c["l2t_ke"], "upward": c["s2m_ke"]}
    kernel_flops = {
        "evaluate": C_LAPLACE * ke["evaluate"],
        "m2l": c["m2l_flops"],
        "upward": C_LAPLACE * ke["upward"] + c["m2m_flops"] + c["c2e_flops"] // 2,
        "downward": c["l2l_flops"] + c["c2e_flops"] // 2,
    }
    ph = res["phases"]
    dom = max(kernel_flops, key=lambda k: ph[k][0])
    ms_k, n_launch = ph[dom]
    flops_per_launch = kernel_flops[dom] * steps / max(n_launch, 1)
    achieved = flops_per_launch / (ms_k / max(n_launch, 1) * 1e-3) / 1e12
    if precision == "fp64":
        bound, peak, src = "fp64", peaks["fp64"], "cuBLAS DGEMM 8192^3 on this GPU (FP64 pipe)"
    elif dom in ("m2l", "downward"):
        bound, peak, src = "tensor", peaks["tf32"], "cuBLAS TF32 GEMM 8192^3 on this GPU"
    else:
        bound, peak, src = "fp32", peaks["fp32"], "cuBLAS SGEMM 8192^3, TF32 off, on this GPU (FP32 pipe)"
    traffic = NCU_TRAFFIC_BYTES.get((precision, dom)) if default_workload else None
    return {"bound": bound, "kernel": dom, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": traffic, "peak_source": "measured in bench.py: " + src,
            "flops_per_launch": flops_per_launch, "ms_per_launch": ms_k / max(n_launch, 1)}


def workload_config(args, world):
    """The workload both arms run and report (the same dict in both lines)."""
    return {"workload": f"clustered Laplace KIFMM, {args.n} sources + {args.grid}^2 grid targets, "
                        f"self + target evaluation",
            "n_sources": args.n, "n_targets": args.grid * args.grid,
            "ncutoff": NCUT, "nequiv": NEQ[args.precision], "precision": args.precision,
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "flushed (256 MB write) between timed GPU steps"}


def run_ours(args, world, rank, local):
    import torch
    from flexmm_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    d = workloads.clustered(n=args.n, n_grid=args.grid)
    n_src, n_tgt = d["x"].size, d["tx"].size
    pts = n_src + n_tgt
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    forms = [args.precision] + ([] if args.only else [p for p in NEQ if p != args.precision])
    cache = {}
    res = {p: measure(args, world, local, d, p, flush, cache) for p in forms}
    if args.ncu:
        return
    for r in res.values():  # after every timed loop of every form
        r["launches"] = r.pop("count_launches")()
    peaks = {"fp64": gemm_peak_tflops(torch, torch.float64),
             "fp32": gemm_peak_tflops(torch, torch.float32),
             "tf32": gemm_peak_tflops(torch, torch.float32, tf32=True)}
    main = res[args.precision]
    default_workload = args.n == 1_000_000 and args.grid == 1000

    def summary(p, r):
        return {"value": world * pts / (r["ms_step"] * 1e-3) / 1e6, "ms_per_step": r["ms_step"],
                "nequiv": r["neq"], "accuracy": r["accuracy"],
                "phase_ms_per_step": {k: v[0] / max(args.steps, 1) for k, v in r["phases"].items() if v[1]},
                "e2e_value": world * pts / (r["e2e_step"] * 1e-3) / 1e6,
                "roofline": roofline_of(r, p, peaks, args.steps, default_workload)}

    out = {
        "metric": METRIC, "value": world * pts / (main["ms_step"] * 1e-3) / 1e6, "unit": "Mpts/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": main["ms_step"],
        "ms_samples": main["step_samples"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+tf32x3/f64" if args.precision == "mixed" else "f64",
        "precision": args.precision,
        "data": "synthetic: seeded clustered sources and grid targets (no dataset)",
        "config": workload_config(args, world),
        "tree": {"levels": main["F"]._levels, "nodes": int(sum(main["F"]._counts))},
        "accuracy": main["accuracy"],
        "phase_ms_per_step": {k: v[0] / max(args.steps, 1) for k, v in main["phases"].items() if v[1]},
        "phase_note": "per-kernel event timers on separate untimed steps, own-source evaluation "
                      "in one kernel after the passes (not split)",
        "work_per_step": main["counts"],
        "clocks": main["clocks"],
        "e2e": {"value": world * pts / (main["e2e_step"] * 1e-3) / 1e6, "unit": "Mpts/s",
                "h2d_bytes_per_step": 8 * ((3 if main["src_reused"] else 5) * n_src + 2 * n_tgt),
                "d2h_bytes_per_step": 8 * (n_src + n_tgt), "ms_per_step": main["e2e_step"],
                "ms_samples": [round(v, 3) for v in main["e2e_samples"]]},
        "gpu_launches": main["launches"],
        "roofline": roofline_of(main, args.precision, peaks, args.steps, default_workload),
        "peaks_measured_tflops": peaks,
    }
    for p in forms[1:]:
        out[p] = summary(p, res[p])
    if "fp64" in res and "mixed" in res:
        out["mixed_over_fp64"] = res["fp64"]["ms_step"] / res["mixed"]["ms_step"]
    if not args.no_batched_stokes:
        out["batched_stokes"] = measure_batched_stokes(args, world)
    if not args.no_multi_rhs:
        out["multi_rhs"] = measure_multi_rhs(args, world)
    if not args.no_adjoint:
        out["bbfmm_adjoint"] = measure_bb_adjoint(args, world)
    if not args.no_helmholtz:
        out["modified_helmholtz"] = measure_helmholtz(args, world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_subprocess(args)
    if rank == 0:
        print(json.dumps(out), flush=True)


def measure_helmholtz(args, world=1, steps=5, k=10.0, neq=32):
    """K0(k r)/(2 pi), k = 10, on the headline workload (clustered sources +
    grid targets, Ncutoff 64, Nequiv 32): the mixed form (FP32 K0, 3xTF32
    translations) against the FP64 form, each step tree + expansions +
    source and target evaluation on resident inputs, CUDA events; source
    error of each against the FP64 direct sum at 2,000 sampled sources.
    Each rank runs the same problem (replicas)."""
    import numpy as np
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, direct_evaluation, workloads
    d = workloads.clustered(n=args.n, n_grid=args.grid)
    dev = torch.device("cuda", torch.cuda.current_device())
    x, y, tau, tx, ty = (torch.from_numpy(d[c]).to(dev) for c in ("x", "y", "tau", "tx", "ty"))
    si = np.random.default_rng(0).choice(d["x"].size, 2000, replace=False)
    ds = direct_evaluation("Modified_Helmholtz_Eval", d["x"], d["y"], d["tau"], d["x"][si], d["y"][si],
                           check=True, helmholtz_k=k)
    pts = d["x"].size + d["tx"].size
    res = {"workload": f"K0({k:g} r)/(2 pi), clustered {d['x'].size} sources + {args.grid}^2 grid "
                       f"targets, Ncutoff {NCUT}, Nequiv {neq}, self + target evaluation",
           "metric": "(sources + targets) / s", "unit": "Mpts/s"}
    for prec in ("mixed", "fp64"):
        helper = KI_Helper()

        def step():
            F = KI_FMM(x, y, "Modified_Helmholtz_Eval", NCUT, neq, bbox=d["bbox"], helper=helper,
                       precision=prec, helmholtz_k=k)
            F.build_expansions(tau)
            return F.source_evaluation(x, y), F.target_evaluation(tx, ty)
        for _ in range(2):
            us, _ = step()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            us, _ = step()
        e1.record()
        torch.cuda.synchronize()
        ms = dist_max(e0.elapsed_time(e1) / steps, world)
        err = float(np.linalg.norm(us.cpu().numpy()[si] - ds) / np.linalg.norm(ds))
        res[prec] = {"value": world * pts / (ms * 1e-3) / 1e6, "ms_per_step": ms,
                     "src_rel_l2_vs_direct": err, "dtype": "f32+tf32x3/f64" if prec == "mixed" else "f64"}
    res["mixed_over_fp64"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
    return res


def measure_bb_adjoint(args, world=1, steps=3):
    """The differentiation form: Laplace black-box FMM (Chebyshev order 16,
    Ncutoff 64), 500,000 sources uniform in [-1,1]^2 with charges N(0,1),
    250,000 targets uniform in [-1,1]^2; loss 0.5 ||u - u_ref||^2, u_ref
    N(0,1).  A step: forward (tree, expansions, evaluation) and backward (the
    forward tree's expansions formed again for the target gradients, the
    adjoint FMM over the targets for the charge and source gradients).
    Metric: (sources + targets) per second of forward + backward; inputs
    resident, CUDA events.  Each rank runs the same problem (replicas)."""
    import torch
    from flexmm_b200 import workloads
    from flexmm_b200.autograd import fmm_potential
    d = workloads.bbfmm()
    T = lambda a, g=True: torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=g)
    vs = [T(d[k]) for k in ("x", "y", "tau", "tx", "ty")]
    ur = T(d["u_ref"], False)
    kw = dict(method="bb", Ncutoff=NCUT, p=16, bbox=d["bbox"])

    def fwd():
        return fmm_potential(*vs, **kw)

    def step():
        for v in vs:
            v.grad = None
        u = fwd()
        (0.5 * ((u - ur) ** 2).sum()).backward()
    step()
    torch.cuda.synchronize()

    def timed(fn):
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        barrier(world)
        return dist_max(e0.elapsed_time(e1) / steps, world)
    ms_fb = timed(step)
    with torch.no_grad():
        ms_f = timed(fwd)
    pts = d["x"].size + d["tx"].size
    return {"workload": "Laplace black-box FMM p = 16, 500000 sources + 250000 targets uniform "
                        "in [-1,1]^2, loss 0.5 ||u - u_ref||^2; forward + backward (charge, "
                        "source- and target-position gradients)",
            "metric": "(sources + targets) / s", "unit": "Mpts/s", "dtype": "f64",
            "value": world * pts / (ms_fb * 1e-3) / 1e6, "ms_per_step": ms_fb,
            "forward": {"value": world * pts / (ms_f * 1e-3) / 1e6, "ms": ms_f}, "steps": steps,
            "note": "trees built inside every step; translations on the FP64 tensor-core row "
                    "GEMM; accuracy checked by the test suite (1e-8 vs FP64 direct-sum "
                    "gradients at N = 20,000)"}


def measure_multi_rhs(args, world=1, n=1_000_000, n_rhs=64, steps=3):
    """The multi-RHS batching form: 1,000,000 sources at uniform angles on a
    circle of radius 0.5 (radial jitter U(-1e-3, 1e-3)), 64 charge columns
    N(0,1) on one tree, the modified Helmholtz kernel K0(10 r)/(2 pi), Nequiv
    40, Ncutoff 64, bbox from the points, self-evaluation of every column.
    A step: tree + expansions of all 64 columns (one launch per level for all
    columns) + source evaluation (each kernel value applied to 8 columns).
    Metric: point-RHS per second, 64 N / T.  Inputs resident; CUDA events.
    With N > 1 ranks the columns are split into blocks over the ranks
    (flexmm_b200.shard, no exchange while computing)."""
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, workloads
    from flexmm_b200.shard import column_blocks
    rank = int(os.environ.get("RANK", "0"))
    d = workloads.circle(n=n, n_rhs=n_rhs)
    lo, hi = column_blocks(n_rhs, world)[rank]
    x, y = torch.from_numpy(d["x"]).cuda(), torch.from_numpy(d["y"]).cuda()
    tau = torch.from_numpy(np.ascontiguousarray(d["tau"][lo:hi])).cuda()
    from flexmm_b200 import direct_evaluation
    rng = np.random.default_rng(5)
    si = np.sort(rng.choice(n, 1000, replace=False))
    ds = {r: direct_evaluation("Modified_Helmholtz_Eval", x, y, tau[r], x[si], y[si], check=True,
                               helmholtz_k=10.0).cpu().numpy() for r in (0, hi - lo - 1)}

    def run(prec):
        helper = KI_Helper()

        def step():
            F = KI_FMM(x, y, "Modified_Helmholtz_Eval", NCUT, 40, helper=helper, helmholtz_k=10.0,
                       precision=prec)
            F.build_expansions(tau)
            return F, F.source_evaluation(x, y)
        F, u = step()
        torch.cuda.synchronize()
        # accuracy: two columns at 1000 sampled sources against the FP64 direct sum
        errs = [float(np.linalg.norm(u[r].cpu().numpy()[si] - v) / np.linalg.norm(v))
                for r, v in ds.items()]
        del F, u
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        barrier(world)
        return dist_max(e0.elapsed_time(e1) / steps, world), max(errs)
    ms, err = run("fp64")
    ms_mx, err_mx = run("mixed")
    return {"workload": f"{n} sources on a circle (r = 0.5 +- 1e-3), {n_rhs} charge columns, "
                        f"K0(10 r)/(2 pi), Nequiv 40, Ncutoff 64, self-evaluation, FP64",
            "metric": "point-RHS / s", "unit": "M point-RHS/s", "dtype": "f64",
            "value": n * n_rhs / (ms * 1e-3) / 1e6, "ms_per_step": ms, "steps": steps,
            "rel_l2_vs_direct": err,
            "accuracy_sample": "columns 0 and last of this rank, 1000 sources, FP64 direct sum",
            "note": "one launch per level for all columns (column = blockIdx.y); evaluation "
                    "shares each kernel value across 8 columns; inputs resident"
                    + (f"; columns split over {world} ranks, slowest rank's time" if world > 1 else ""),
            "mixed": {"value": n * n_rhs / (ms_mx * 1e-3) / 1e6, "ms_per_step": ms_mx,
                      "rel_l2_vs_direct": err_mx, "dtype": "f32+tf32x3/f64",
                      "note": "same workload in the mixed form: the tree once, then each column's "
                              "expansions and source evaluation in turn"}}


def measure_batched_stokes(args, world=1, n_problems=256):
    """The batching form: 256 independent FP64 Stokes problems (sizes
    log-uniform in [2,000, 200,000], sources uniform in [-1,1]^2, forces
    N(0,1)), self-evaluation, Nequiv 32, Ncutoff 64; forward and charge
    adjoint through StokesBatch, inputs resident, timed with CUDA events on
    the caller's stream (the batch streams are joined into it).  With N > 1
    ranks the problems are partitioned by cost over the ranks
    (ShardedStokesBatch: no exchange while computing): each rank times its
    own share, the slowest rank's time counts, and one all-gather afterwards
    (untimed) hands every rank all results."""
    import torch
    from flexmm_b200.batch import StokesBatch
    from flexmm_b200.shard import partition_by_cost
    rng = np.random.default_rng(4)
    sizes = np.round(np.exp(rng.uniform(np.log(2000), np.log(200000), n_problems))).astype(int)
    probs = [(rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)) for n in sizes]
    forces = [(rng.standard_normal(n), rng.standard_normal(n)) for n in sizes]
    cots = [tuple(rng.standard_normal(n) for _ in range(3)) for n in sizes]
    rank = int(os.environ.get("RANK", "0"))
    mine = partition_by_cost(sizes, world)[rank]
    dev = lambda a: torch.from_numpy(a).cuda()
    B = StokesBatch([probs[i] for i in mine], Nequiv=32, Ncutoff=64, n_streams=8)
    f_loc = [(dev(forces[i][0]), dev(forces[i][1])) for i in mine]
    c_loc = [tuple(dev(v) for v in cots[i]) for i in mine]
    total = int(sizes.sum())

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        barrier(world)
        return dist_max(e0.elapsed_time(e1) / reps, world)

    ms_f = timed(lambda: B.forward(f_loc))
    ms_a = timed(lambda: B.adjoint(c_loc))
    # the same calls captured as one CUDA graph each (one launch per batch call)
    gf, ga = B.graph("forward"), B.graph("adjoint")
    ms_gf = timed(lambda: gf.replay(f_loc))
    ms_ga = timed(lambda: ga.replay(c_loc))
    B.status()
    # trees inside the timing: the batch built from the points (every tree,
    # operators cached from the batch above) and one forward, eagerly
    tree_probs = [probs[i] for i in mine]

    def with_trees():
        Bt = StokesBatch(tree_probs, Nequiv=32, Ncutoff=64, n_streams=8, adjoint=False,
                         precomputations=B.precomputations)
        Bt.forward(f_loc)
    ms_t = timed(with_trees, reps=1)
    res = {"workload": f"{n_problems} independent Stokes problems, N_i log-uniform in "
                       f"[2000, 200000] (sum {total}), self-evaluation, Nequiv 32, Ncutoff 64, FP64",
           "metric": "sum N_i / T", "unit": "Mpts/s", "dtype": "f64", "streams": len(B.streams),
           "forward": {"value": total / (ms_f * 1e-3) / 1e6, "ms": ms_f},
           "adjoint": {"value": total / (ms_a * 1e-3) / 1e6, "ms": ms_a},
           "forward_graph": {"value": total / (ms_gf * 1e-3) / 1e6, "ms": ms_gf},
           "adjoint_graph": {"value": total / (ms_ga * 1e-3) / 1e6, "ms": ms_ga},
           "forward_with_trees": {"value": total / (ms_t * 1e-3) / 1e6, "ms": ms_t},
           "note": "concurrent per-problem plans on CUDA streams; forward / adjoint: eager calls "
                   "on built trees; *_graph: each call captured as one CUDA graph and replayed; "
                   "forward_with_trees: all 256 trees built plus one forward"}
    if world > 1:
        from flexmm_b200.shard import ShardedStokesBatch
        S = ShardedStokesBatch(probs, Nequiv=32, Ncutoff=64, n_streams=8)
        S.forward(forces)   # the gather path, once, untimed
        res.update(scaling="strong", ranks=world,
                   note="problems partitioned by points over the ranks (no exchange while "
                        "computing); slowest rank's device time; trees built outside the timing")
    return res


# ---------------------------------------------------------- reference arm --
def reference_step_fn(n_src, n_grid, neq, denested=False):
    """Closure timing one step of the reference flexmm on the host CPU.

    denested=True pre-registers a serial kernel_apply in a fresh helper before
    the FMM is built (KI_Helper.build_s2pM_function keeps a registered one,
    flexmm/flexmm2d/kifmm.py:83-92): the S2M loop over leaves stays parallel
    but its inner per-leaf loop no longer opens a nested parallel region.
    Same arithmetic, so the same results; the as-is form is the baseline."""
    from oracle import refimport  # the reference itself (shimmed copy), checker-only
    from flexmm_b200 import workloads
    refimport.load_reference()
    import numba
    from flexmm.flexmm2d.kifmm import KI_FMM, KI_Helper

    @numba.njit(fastmath=True)
    def Laplace_Eval(sx, sy, tx, ty):
        dx = tx - sx
        dy = ty - sy
        d2 = dx**2 + dy**2
        return -np.log(d2) / (4 * np.pi)

    d = workloads.clustered(n=n_src, n_grid=n_grid)
    helper = KI_Helper()
    if denested:
        @numba.njit(fastmath=True)
        def kernel_apply_serial(sx, sy, tx, ty, tau, out):
            for j in range(tx.size):
                outj = 0.0
                for i in range(sx.size):
                    outj += Laplace_Eval(sx[i], sy[i], tx[j], ty[j]) * tau[i]
                out[j] = outj
        helper.functions["kernel_eval"] = Laplace_Eval
        helper.functions["kernel_apply"] = kernel_apply_serial

    # JIT warm-up on a 5,000-point problem (the examples' protocol), with its
    # own helper so that its box widths do not enter the timed helper's cache
    w = workloads.clustered(n=5000, n_grid=20)
    wh = KI_Helper()
    if denested:
        wh.functions.update(helper.functions)
    Fw = KI_FMM(w["x"], w["y"], Laplace_Eval, NCUT, neq, bbox=w["bbox"], helper=wh)
    Fw.build_expansions(w["tau"])
    Fw.source_evaluation(w["x"], w["y"])
    Fw.target_evaluation(w["tx"], w["ty"])
    helper.functions.update({k: v for k, v in wh.functions.items() if k not in helper.functions})

    def step():
        t0 = time.perf_counter()
        F = KI_FMM(d["x"], d["y"], Laplace_Eval, NCUT, neq, bbox=d["bbox"], helper=helper)
        F.build_expansions(d["tau"])
        F.source_evaluation(d["x"], d["y"])
        F.target_evaluation(d["tx"], d["ty"])
        return time.perf_counter() - t0

    return step, d["x"].size + d["tx"].size


def reference_available():
    from oracle import refimport
    return refimport.reference_available()


def cpu_baseline_subprocess(args):
    """Time the reference on the host in a fresh process (all cores) on a
    bounded sample of the workload (--cpu-sample-n sources, a grid of about
    as many targets): best and mean of 3 steps, as-is and de-nested."""
    cores = os.cpu_count() or 1
    env = dict(os.environ, NUMBA_NUM_THREADS=str(cores), CUDA_VISIBLE_DEVICES="")
    grid = int(round(np.sqrt(args.cpu_sample_n)))
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--steps", "3",
           "--warmup", "1", "--precision", args.precision, "--n", str(args.cpu_sample_n),
           "--grid", str(grid), "--denested-steps", "3", "--json-only"]
    try:
        r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=900)
        line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
        ref = json.loads(line)
        return ref.get("cpu_baseline", {"unavailable": ref.get("unavailable")})
    except Exception as e:  # the GPU number stands without it
        return {"unavailable": f"reference run failed: {type(e).__name__}: {e}"}


def run_reference(args, world, rank):
    """The reference arm: the reference flexmm's own KI_FMM (numba, all host
    threads) on this bench's workload -- by default the full 1M-source /
    1000^2-grid configuration, the same one the GPU line reports -- one full
    problem per step (tree + build_expansions + source_evaluation +
    target_evaluation, operators warm), W warm-up and K timed steps."""
    if rank != 0:
        return
    neq = NEQ[args.precision]
    base = {"impl": "reference", "metric": METRIC, "unit": "Mpts/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded clustered sources and grid targets (no dataset)",
            "config": workload_config(args, world)}
    if not reference_available():
        base["unavailable"] = "reference copy oracle/_ref not built (needs the reference checkout)"
        print(json.dumps(base), flush=True)
        return
    cores = int(os.environ.get("NUMBA_NUM_THREADS", os.cpu_count() or 1))
    step, pts = reference_step_fn(args.n, args.grid, neq)
    for _ in range(max(args.warmup, 1)):
        step()
    ts = [step() for _ in range(max(args.steps, 1))]
    sec = statistics.mean(ts)
    value = pts / sec / 1e6
    scope = ("a bounded sample of the 1M-source / 1000^2-grid workload" if args.json_only
             else "the full workload")
    sample = (f"{scope}: reference flexmm KI_FMM as-is (numba, {cores} threads), "
              f"clustered {args.n} sources + {args.grid}^2 grid targets, Nequiv {neq}, warm JIT "
              f"(5,000-point problem) and operators (helper reuse); per step: tree + "
              f"build_expansions + source_evaluation + target_evaluation; value = mean of "
              f"{len(ts)} steps")
    cpu = {"value": value, "unit": "Mpts/s", "cores": cores, "kind": "reference",
           "sample": sample, "best_of_steps": pts / min(ts) / 1e6,
           "s_per_step": [round(t, 3) for t in ts]}
    if args.denested_steps > 0:
        dstep, _ = reference_step_fn(args.n, args.grid, neq, denested=True)
        dstep()  # operators of this helper
        dts = [dstep() for _ in range(args.denested_steps)]
        cpu["denested_s2m"] = {"value": pts / statistics.mean(dts) / 1e6,
                               "best": pts / min(dts) / 1e6, "steps": len(dts),
                               "note": "serial kernel_apply pre-registered in the helper: S2M "
                                       "without the nested parallel region; same results"}
    base.update({"value": value, "ms_per_step": sec * 1e3, "cpu_baseline": cpu,
                 "e2e": {"value": value, "unit": "Mpts/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0}})
    print(json.dumps(base), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup(args)
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
