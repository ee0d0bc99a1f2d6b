#!/usr/bin/env python
"""Throughput of the batched dense-solve engine on one B200 (or N replicas).

One step = every system of the workload solved / inverted once, inputs already
resident in HBM (``value``), and the same through the C ABI with pinned host
buffers, host<->device copies included (``e2e``).  Default workload: the
50k-cell mixed batch (per cell 10 ion-balance solves of orders 2-27 and one
macro-atom inverse of order 20-200), the configuration the headline target is
quoted on.  ``value`` runs the engine's certified mode (SIROCCO_FAST: macro-atom
inverses that pass the M-matrix certificate by Gauss-Jordan without pivoting,
everything else GSL-exact); ``plain_fp64_value`` is the same step with every
system on the GSL-exact FP64 path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config 0|1|3|4]
    python bench.py --impl reference ...   # the reference's CPU path, all host cores

Beside the engine's numbers the line reports the reference's own CPU path
(``cpu_baseline``: source/matrix_cpu.c + GSL, every host core) and the
reference's cuSOLVER build (``cusolver_reference``: source/matrix_gpu.cu, one
call per system as its CUDA_ON build makes them), each timed on a bounded
sample of the same workload outside the timed region.

The path does not shard with an exchange step: with N > 1 (torchrun) every rank
runs an independent replica of the workload ("replicas only", weak scaling);
``value`` is the systems of all ranks over the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from python_b200 import workloads as wl  # noqa: E402

METRIC = "batched solves/s at ≤1e-10 rel err: mixed-prec vs FP64 on B200 vs GSL CPU"
UNIT = "systems/s"
POP_TOL = 1e-10
L2_BYTES = 126 * 2 ** 20
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
HBM_FALLBACK_GBS = 6650.0

# DRAM traffic of the dominant kernel: the committed ncu summaries in
# profiles/ carry a machine-readable line
#     traffic-ratio: <size class> <DRAM bytes / algorithmic bytes> <workload>
# for the capture they summarise; the bench scales it to the timed launch and
# names the file it came from.
PROFILES = ROOT / "profiles"


def traffic_ratio(size_class_name: str):
    for f in sorted(PROFILES.glob("*.md")):
        for line in f.read_text().splitlines():
            parts = line.strip().strip("`").split()
            if len(parts) >= 3 and parts[0] == "traffic-ratio:" and parts[1] == size_class_name:
                return float(parts[2]), f"profiles/{f.name}"
    return None, None


WORKLOADS = {
    0: "ion-balance solve, 4096 x n=27 (config-0 generator)",
    1: "macro-atom inverse, 8192 x n=61 (config-1 generator)",
    2: "conditioning sweep: log10 kappa_2 in {2,4,6,8,10,12} x 2048 systems, ion n=27 solves and macro n=61 inverses",
    3: "50k cells: 10 ion solves n in {2..27} + 1 macro inverse n~U[20,200] per cell, shuffled",
    4: "large macro inverse, 2048 x n~U[256,1024], 10% nonzero",
}


# --------------------------------------------------------------- workloads --
def make_batches(config: int, nsys: int | None = None):
    if config == 0:
        return [wl.config0(nsys=nsys or 4096)]
    if config == 1:
        return [wl.config1(nsys=nsys or 8192)]
    if config == 2:
        raise SystemExit("config 2 is the conditioning sweep (bench.py --config 2), not a throughput workload")
    if config == 3:
        s, i = wl.config3(ncells=nsys or 50_000)
        return [s, i]
    if config == 4:
        return [wl.config4(nsys=nsys or 2048)]
    raise SystemExit(f"unknown config {config}")


# the engine's size classes, as it compiles them in (padded orders)
def _class_orders(inc: str, macro: str) -> tuple:
    text = (ROOT / "python_b200" / "csrc" / inc).read_text()
    return tuple(int(m[1]) for m in re.finditer(rf"^{macro}\(\d+, (\d+),", text, re.M))


CGJ_P = _class_orders("cgj_classes.inc", "SS_CGJ_CLASS")
SMALL_NP = _class_orders("small_classes.inc", "SS_SMALL_CLASS")
CTA_P = _class_orders("cta_classes.inc", "SS_CTA_CLASS")


def size_class(n: int, kind: str = "solve", mode: str = "fp64") -> str:
    """Mirror of the engine's bucketing (python_b200/csrc/engine.cu)."""
    if kind == "invert" and mode == "fast" and n >= 33:
        for p in CGJ_P:
            if n <= p:
                return f"cgj{p}"
        return "cgjl"   # streamed certified inverse, orders above the last class
    for np_ in SMALL_NP:
        if n <= np_:
            return f"small{np_}"
    for p in CTA_P:
        if n <= p:
            return f"cta{p}"
    return "global"


def kernel_name(kind: str, cls: str, mode: str) -> str:
    if cls == "cgjl":
        return "cgjl_inverse_kernel"
    if cls.startswith("cgj"):
        return "cgj_inverse_kernel"
    if cls.startswith("small"):
        return ("small_mixed_solve_kernel" if (mode == "mixed" and kind == "solve") else "small_exact_kernel")
    return "cta_exact_kernel" if cls.startswith("cta") else "global_exact_kernel"


def subset(batch: wl.Batch, idx: np.ndarray) -> wl.Batch:
    mats = [batch.matrix(int(s)) for s in idx]
    if batch.kind == "solve":
        return wl.from_matrices("solve", mats, [batch.rhs(int(s)) for s in idx])
    return wl.from_matrices("invert", mats)


# -------------------------------------------------------------- distributed --
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def dist_init(world: int, use_cuda: bool):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("nccl" if use_cuda else "gloo", timeout=datetime.timedelta(seconds=120))
    return dist


def reduce_max(dist, value: float, device) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(world: int, systems_per_step: int, steps: int, t_max: float) -> float:
    """Whole-job throughput: every rank's systems over the slowest rank's time."""
    return world * systems_per_step * steps / t_max


def barrier(dist, device=None):
    if dist is not None:
        if device is not None and device.type == "cuda":
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# -------------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({nm for r in rows for nm, v in zip(names, r[5:9]) if v.lower() == "active"})
        loaded = [v for v in sm if v > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- CPU side --
def cpu_reference_run(batch: wl.Batch, threads: int, seconds: float, seed: int = 0):
    """Time the reference's CPU path (oracle/_ref when built, else the C
    restatement) on a bounded sample of the batch; returns (systems/s, info)."""
    from oracle import oracle
    which = "ref" if oracle.available("ref") else "port"
    kind = "reference" if which == "ref" else "port"
    rng = np.random.default_rng(seed)
    probe = subset(batch, rng.choice(batch.nsys, size=min(32, batch.nsys), replace=False))
    t0 = time.perf_counter()
    (oracle.solve if batch.kind == "solve" else oracle.invert)(probe, which, threads=1)
    per_sys = max((time.perf_counter() - t0) / probe.nsys, 1e-7)
    want = max(threads, seconds * threads / per_sys)
    reps = 1
    if want >= batch.nsys:                       # whole batch, repeated to fill the time budget
        reps = int(np.ceil(want / batch.nsys))
        sample = batch
    else:
        sample = subset(batch, np.sort(rng.choice(batch.nsys, size=int(want), replace=False)))
    fn = oracle.solve if batch.kind == "solve" else oracle.invert
    t0 = time.perf_counter()
    for _ in range(reps):
        fn(sample, which, threads=threads)
    dt = time.perf_counter() - t0
    what = "all" if sample is batch else f"{sample.nsys} (random, seeded) of"
    info = {"kind": kind, "cores": threads,
            "sample": f"{what} {batch.nsys} systems x {reps} pass(es), {dt:.1f} s wall, {threads} pthreads, "
                      f"one serial {'solve_matrix' if batch.kind == 'solve' else 'invert_matrix'} call per "
                      f"system on a fresh copy of A"}
    return reps * sample.nsys / dt, info


def cusolver_reference_run(batch: wl.Batch, seconds: float, seed: int = 0):
    """Time the reference's cuSOLVER build (source/matrix_gpu.cu, one
    gpu_solve_matrix / gpu_invert_matrix call per system, each allocating,
    copying and freeing) on a bounded sample; returns (systems/s, info) or
    (None, reason)."""
    from oracle import oracle
    if not oracle.cusolver_available():
        return None, "reference cuSOLVER build not present (oracle/_ref/libref_cusolver.so)"
    rng = np.random.default_rng(seed)
    fn = oracle.cusolver_solve if batch.kind == "solve" else oracle.cusolver_invert
    probe = subset(batch, rng.choice(batch.nsys, size=min(8, batch.nsys), replace=False))
    fn(probe)                                    # handle creation, first-call costs
    t0 = time.perf_counter()
    fn(probe)
    per_sys = max((time.perf_counter() - t0) / probe.nsys, 1e-6)
    size = int(min(batch.nsys, max(16, seconds / per_sys)))
    idx = np.sort(rng.choice(batch.nsys, size=size, replace=False))
    sample = subset(batch, idx)
    t0 = time.perf_counter()
    out, st = fn(sample)
    dt = time.perf_counter() - t0
    # agreement with the GSL path on the same sample, for information
    from oracle import oracle as orc
    if batch.kind == "solve":
        ref, sr = orc.solve(sample, "port", threads=orc.host_threads())
        ok = sr != 4
        worst = 0.0
        for j in np.nonzero(ok)[0]:
            a, b = int(sample.offv[j]), int(sample.offv[j]) + int(sample.n[j])
            r, v = ref[a:b], out[a:b]
            sig = np.abs(r) > 1e-20 * np.abs(r).sum()
            if sig.any():
                worst = max(worst, float(np.max(np.abs(v[sig] - r[sig]) / np.abs(r[sig]))))
    else:
        ref, sr = orc.invert(sample, "port", threads=orc.host_threads())
        worst = 0.0
        for j in np.nonzero(sr == 0)[0]:
            a, b = int(sample.offA[j]), int(sample.offA[j]) + int(sample.n[j]) ** 2
            worst = max(worst, float(np.max(np.abs(out[a:b] - ref[a:b])) / np.max(np.abs(ref[a:b]))))
    info = {"value": size / dt, "unit": UNIT,
            "sample": f"{size} (random, seeded) of {batch.nsys} systems, {dt:.2f} s wall, one "
                      f"{'gpu_solve_matrix' if batch.kind == 'solve' else 'gpu_invert_matrix'} call per system "
                      f"from host memory (the reference's CUDA_ON build, cusolverDnDgetrf/getrs)",
            "max_rel_err_vs_gsl": worst}
    return size / dt, info


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle
    batches = make_batches(args.config, args.nsys)
    threads = oracle.host_threads()
    per_step = max(1.0, args.ref_seconds / (args.steps + args.warmup) / len(batches))
    for _ in range(args.warmup):
        for b in batches:
            cpu_reference_run(b, threads, per_step * 0.25)
    rates, infos = [], []
    for k in range(args.steps):
        t_sys = 0.0
        for j, b in enumerate(batches):
            r, info = cpu_reference_run(b, threads, per_step, seed=k * 7 + j)
            t_sys += b.nsys / r
            infos.append(info)
        rates.append(sum(b.nsys for b in batches) / t_sys)
    value = statistics.median(rates)
    info = dict(infos[-1])
    info["value"] = value
    info["unit"] = UNIT
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(b.nsys for b in batches) / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generators with the reference's structure)",
            "config": {"workload": WORKLOADS[args.config], "config_index": args.config},
            "cpu_baseline": info,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU side --
def measured_peaks():
    if PEAKS_FILE.exists():
        d = json.loads(PEAKS_FILE.read_text())
        return float(d.get("hbm_gbs", HBM_FALLBACK_GBS)), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def fp64_peak_tflops(device) -> float:
    """cuBLAS DGEMM throughput on this GPU (8192^3), the FP64 denominator."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def accuracy(batch, out_np, status_np, mode, sample=512, seed=1):
    """Error of the timed outputs against the reference's GSL build (oracle/_ref,
    else the restatement) on a sample."""
    from oracle import oracle
    which = "ref" if oracle.available("ref") else "port"
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(batch.nsys, size=min(sample, batch.nsys), replace=False))
    sub = subset(batch, idx)
    if batch.kind == "solve":
        xr, sr = oracle.solve(sub, which, threads=oracle.host_threads())
        worst, codes = 0.0, True
        for j, s in enumerate(idx):
            codes &= int(status_np[s]) == int(sr[j])
            if sr[j] == 4:
                continue
            n, o = int(batch.n[s]), int(batch.offv[s])
            r = xr[sub.offv[j]:sub.offv[j] + n]
            v = out_np[o:o + n]
            sig = np.abs(r) > 1e-20 * np.abs(r).sum()
            if sig.any():
                worst = max(worst, float(np.max(np.abs(v[sig] - r[sig]) / np.abs(r[sig]))))
        return worst, bool(codes), "populations above 1e-20 of each system's total, max relative error"
    ir, sr = oracle.invert(sub, which, threads=oracle.host_threads())
    worst, codes = 0.0, True
    for j, s in enumerate(idx):
        codes &= int(status_np[s]) == int(sr[j])
        if sr[j] != 0:
            continue
        n, o = int(batch.n[s]), int(batch.offA[s])
        r = ir[sub.offA[j]:sub.offA[j] + n * n]
        v = out_np[o:o + n * n]
        worst = max(worst, float(np.max(np.abs(v - r)) / np.max(np.abs(r))))
    return worst, bool(codes), "inverse, max |X - X_ref| / max |X_ref| per matrix"


def run_ours(args):
    import torch

    from python_b200 import engine
    rank, world, local = dist_env()
    dist = dist_init(world, True)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    lib = engine.load()
    assert lib.cusolver_create() == 0, engine.last_error()

    batches = make_batches(args.config, args.nsys)
    modes = []
    for b in batches:
        if args.mode == "auto":
            # ion-balance solves: only the GSL-exact FP64 path meets the 1e-10 bar
            # against the reference (its own answers are that far from exact);
            # macro-atom inverses: the certified path
            modes.append("fp64" if b.kind == "solve" else "fast")
        else:
            modes.append(args.mode)
    code = {"fp64": engine.FP64, "mixed": engine.MIXED, "fast": engine.FAST}
    if args.only_dominant:
        return run_dominant(args, engine, batches, modes, code, device)
    plans, bufs = [], []
    for b, m in zip(batches, modes):
        plans.append(engine.Plan(b, code[m]))
        A = torch.from_numpy(b.A).to(device)
        out = torch.empty(b.b.size if b.kind == "solve" else b.A.size, dtype=torch.float64, device=device)
        st = torch.full((b.nsys,), -1, dtype=torch.int32, device=device)
        diag = torch.zeros((b.nsys,), dtype=torch.int32, device=device)
        bb = torch.from_numpy(b.b).to(device) if b.kind == "solve" else None
        bufs.append((A, bb, out, st, diag))
    stream = torch.cuda.current_stream(device)
    in_bytes = sum(b.A.nbytes + (b.b.nbytes if b.kind == "solve" else 0) for b in batches)

    def step():
        for p, (A, bb, out, st, diag) in zip(plans, bufs):
            p.execute(A, out, st, b=bb, diag=diag, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(device)
    barrier(dist, device)
    clocks = ClockSampler(local).start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(device)
    barrier(dist, device)
    clock_info = clocks.stop()
    t_local = e0.elapsed_time(e1) / 1e3
    t = reduce_max(dist, t_local, device)
    nsys_step = sum(b.nsys for b in batches)
    value = aggregate(world, nsys_step, args.steps, t)
    launches = sum(p.launches for p in plans) * args.steps

    # ---- mixed sizes: the same step as one graph launch, and as one launch per size
    launch_modes = None
    if world == 1 and any(len(np.unique(b.n)) > 1 for b in batches):
        side = torch.cuda.Stream(device)
        graph = torch.cuda.CUDAGraph()
        side.wait_stream(stream)
        with torch.cuda.graph(graph, stream=side):
            for p, (A, bb, out, st, diag) in zip(plans, bufs):
                p.execute(A, out, st, b=bb, diag=diag, stream=side)
        torch.cuda.synchronize(device)
        for _ in range(2):
            graph.replay()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(args.steps):
            graph.replay()
        g1.record(stream)
        torch.cuda.synchronize(device)
        t_graph = g0.elapsed_time(g1) / 1e3 / args.steps
        # one plan (one kernel launch) per distinct order, over the same buffers
        per_size = []
        for b, m, (A, bb, out, st, diag) in zip(batches, modes, bufs):
            for nval in np.unique(b.n):
                idx = np.nonzero(b.n == nval)[0]
                sub = wl.Batch(b.kind, b.n[idx], b.offA[idx], b.A, b.offv[idx] if b.kind == "solve" else None, b.b)
                per_size.append((engine.Plan(sub, code[m]), (A, bb, out, st, diag)))
        one = sum(p.launches for p, _ in per_size)

        def per_size_step():
            for p, (A, bb, out, st, diag) in per_size:
                p.execute(A, out, st, b=bb, diag=diag, stream=stream)
        for _ in range(2):
            per_size_step()
        torch.cuda.synchronize(device)
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        for _ in range(args.steps):
            per_size_step()
        q1.record(stream)
        torch.cuda.synchronize(device)
        t_per = q0.elapsed_time(q1) / 1e3 / args.steps
        for p, _ in per_size:
            p.close()
        del graph
        launch_modes = {"bucketed_plans_ms": 1e3 * t / args.steps,
                        "bucketed_launches_per_step": sum(p.launches for p in plans),
                        "graph_replay_ms": 1e3 * t_graph, "graph_launches_per_step": 1,
                        "one_launch_per_size_ms": 1e3 * t_per, "one_launch_per_size_launches": one}

    # ---- accuracy of what was timed ------------------------------------
    acc = []
    for b, m, (A, bb, out, st, diag) in zip(batches, modes, bufs):
        err, codes_ok, what = accuracy(b, out.cpu().numpy(), st.cpu().numpy(), m)
        d = diag.cpu().numpy()
        acc.append({"kind": b.kind, "mode": m, "max_rel_err": err, "codes_match": codes_ok, "measure": what,
                    "exact_path_frac": float(np.mean((d & (1 << 8)) != 0))})

    # ---- dominant kernel: the size class with the most flops, timed alone --
    fl, db, dm, dc, didx = dominant_class(batches, modes)
    dom = db if didx.size == db.nsys else subset(db, didx)
    dplan = engine.Plan(dom, code[dm])
    dA = torch.from_numpy(dom.A).to(device)
    dout = torch.empty(dom.b.size if dom.kind == "solve" else dom.A.size, dtype=torch.float64, device=device)
    dst = torch.empty((dom.nsys,), dtype=torch.int32, device=device)
    dbb = torch.from_numpy(dom.b).to(device) if dom.kind == "solve" else None
    for _ in range(3):
        dplan.execute(dA, dout, dst, b=dbb, stream=stream)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=device) \
        if dom.A.nbytes < 2 * L2_BYTES else None
    times = []
    for _ in range(max(3, args.steps)):
        if flush is not None:
            flush.zero_()
        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k0.record(stream)
        dplan.execute(dA, dout, dst, b=dbb, stream=stream)
        k1.record(stream)
        torch.cuda.synchronize(device)
        times.append(k0.elapsed_time(k1) / 1e3)
    t_kernel = statistics.median(times)
    alg_bytes = dom.bytes()
    alg_flops = dom.flops()
    hbm_peak, peak_src = measured_peaks()
    fp64_peak = fp64_peak_tflops(device)
    traffic, traffic_src = args.traffic, "--traffic"
    if traffic is None:
        ratio, src = traffic_ratio(dc)
        if ratio is not None:
            traffic = ratio * alg_bytes
            traffic_src = f"{src}: DRAM bytes / algorithmic bytes of that capture ({ratio:.3f}) x this launch's bytes"
    # the roofline of the launch is the slower of matrix bytes at HBM bandwidth
    # and algorithmic flops at the FP64 peak; `roofline` reports the binding one
    t_hbm = alg_bytes / (hbm_peak * 1e9)
    t_fp64 = alg_flops / (fp64_peak * 1e12)
    hbm_line = {"bound": "hbm", "achieved": alg_bytes / t_kernel / 1e9, "peak": hbm_peak, "unit": "GB/s",
                "frac": t_hbm / t_kernel, "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)"}
    fp64_line = {"bound": "fp64", "achieved": alg_flops / t_kernel / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                 "frac": t_fp64 / t_kernel,
                 "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 via torch.matmul (MEASURED_PEAKS.json "
                                "has no FP64 entry)"}
    roofline = dict(fp64_line if t_fp64 >= t_hbm else hbm_line)
    roofline.update({"traffic": traffic, "traffic_source": traffic_src if traffic is not None else None,
                     "kernel": kernel_name(dom.kind, dc, dm), "size_class": dc, "launch_s": t_kernel,
                     "bytes_per_launch": alg_bytes, "flops_per_launch": alg_flops,
                     "systems_per_launch": dom.nsys})
    roofline_other = fp64_line if t_fp64 < t_hbm else hbm_line
    dplan.close()
    del flush

    # ---- end to end through the C ABI with pinned host buffers ------------
    e2e = None
    if not args.no_e2e:
        host = []
        for b in batches:
            hA = torch.from_numpy(b.A).pin_memory().numpy()
            hb = torch.from_numpy(b.b).pin_memory().numpy() if b.kind == "solve" else None
            hout = torch.empty(b.b.size if b.kind == "solve" else b.A.size, dtype=torch.float64).pin_memory().numpy()
            hst = torch.empty(b.nsys, dtype=torch.int32).pin_memory().numpy()
            hb_batch = wl.Batch(b.kind, b.n, b.offA, hA, b.offv, hb)
            host.append((hb_batch, hout, hst))
        h2d = sum(hb.A.nbytes + (hb.b.nbytes if hb.kind == "solve" else 0) for hb, _, _ in host)
        d2h = sum(ho.nbytes + hs.nbytes for _, ho, hs in host)

        def e2e_step():
            for (hb, hout, hst), m in zip(host, modes):
                eng_mode = code[m]
                if hb.kind == "solve":
                    _, st_ = engine.solve_batched(hb, eng_mode, x=hout)
                else:
                    _, st_ = engine.invert_batched(hb, eng_mode, out=hout)
        for _ in range(max(1, args.warmup // 2)):
            e2e_step()
        torch.cuda.synchronize(device)

        def e2e_block():
            barrier(dist, device)
            t0 = time.perf_counter()
            for _ in range(args.steps):
                e2e_step()
            torch.cuda.synchronize(device)
            te_ = reduce_max(dist, time.perf_counter() - t0, device)
            barrier(dist, device)
            return te_

        # a wall-clock window of a few milliseconds is at the mercy of one host
        # hiccup: short runs repeat the K-step block (every rank the same count)
        # and keep the median block
        blocks = [e2e_block()]
        reps = int(min(9, max(1, 0.3 // max(blocks[0], 1e-6))))
        if dist is not None:
            reps = int(reduce_max(dist, float(reps), device))
        blocks += [e2e_block() for _ in range(reps - 1)]
        te = statistics.median(blocks)
        e2e = {"value": world * nsys_step * args.steps / te, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "blocks": len(blocks),
               "block_s_min_max": [min(blocks), max(blocks)],
               "path": "solve_matrix_batched / invert_matrix_batched with pinned host buffers, wall clock, "
                       "median of the K-step blocks"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle
        threads = oracle.host_threads()
        t_sys, infos = 0.0, []
        for b in batches:
            r, info = cpu_reference_run(b, threads, args.cpu_seconds / len(batches))
            t_sys += b.nsys / r
            infos.append(info)
        cpu = dict(infos[0])
        if len(infos) > 1:
            cpu["sample"] = " + ".join(i["sample"] for i in infos)
        cpu["value"] = nsys_step / t_sys
        cpu["unit"] = UNIT

    # the reference's own GPU path (its cuSOLVER build), timed on a bounded sample
    cus = None
    if rank == 0 and world == 1 and not args.no_cusolver:
        t_sys, infos = 0.0, []
        for b in batches:
            r, info = cusolver_reference_run(b, args.cusolver_seconds / len(batches))
            if r is None:
                cus = {"unavailable": info}
                break
            t_sys += b.nsys / r
            infos.append(info)
        if cus is None:
            cus = {"value": nsys_step / t_sys, "unit": UNIT, "sample": " + ".join(i["sample"] for i in infos),
                   "max_rel_err_vs_gsl": max(i["max_rel_err_vs_gsl"] for i in infos)}

    # plain FP64 batched kernels (every system GSL-exact) on the same workload
    fp64_value = None
    if any(m != "fp64" for m in modes):
        fplans = [engine.Plan(b, engine.FP64) for b in batches]
        for _ in range(2):
            for p, (A, bb, out, st, diag) in zip(fplans, bufs):
                p.execute(A, out, st, b=bb, stream=stream)
        torch.cuda.synchronize(device)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            for p, (A, bb, out, st, diag) in zip(fplans, bufs):
                p.execute(A, out, st, b=bb, stream=stream)
        f1.record(stream)
        torch.cuda.synchronize(device)
        tf = reduce_max(dist, f0.elapsed_time(f1) / 1e3, device)
        fp64_value = world * nsys_step * args.steps / tf
        for p in fplans:
            p.close()

    if rank == 0:
        mode_names = {"fp64": "GSL-exact FP64 (SIROCCO_FP64)", "fast": "certified FP64 (SIROCCO_FAST)",
                      "mixed": "mixed FP32/FP64 (SIROCCO_MIXED)"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64" if any(m == "mixed" for m in modes) else "f64",
                "data": "synthetic (seeded generators with the reference's structure)",
                "config": {"workload": WORKLOADS[args.config], "config_index": args.config},
                "run": {"systems_per_step": nsys_step,
                        "modes": {b.kind: mode_names[m] for b, m in zip(batches, modes)},
                        "l2": (f"inputs {in_bytes / 2**20:.0f} MiB > 126 MiB L2: no flush needed"
                               if in_bytes > L2_BYTES else
                               f"inputs {in_bytes / 2**20:.0f} MiB < L2: not flushed between steps"),
                        "parallelism": f"replicas x{world}"},
                "accuracy": acc, "plain_fp64_value": fp64_value,
                "mixed_over_fp64": (value / fp64_value) if fp64_value else None,
                "mixed_over_fp64_note": ("value / plain_fp64_value: the timed modes against every system on the "
                                         "GSL-exact FP64 path"),
                "roofline": roofline, "roofline_other_bound": roofline_other, "cpu_baseline": cpu, "e2e": e2e,
                "cusolver_reference": cus, "launch_modes": launch_modes, "gpu_launches": launches,
                "clocks": clock_info}
        print(json.dumps(line), flush=True)
    for p in plans:
        p.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def dominant_class(batches, modes):
    """The size class with the most algorithmic flops: (flops, batch, mode, class, indices)."""
    best = None
    for b, m in zip(batches, modes):
        classes = np.array([size_class(int(n), b.kind, m) for n in b.n])
        for c in np.unique(classes):
            idx = np.nonzero(classes == c)[0]
            nn = b.n[idx].astype(np.float64)
            fl = float(np.sum(2.0 / 3.0 * nn ** 3 + 2 * nn ** 2 if b.kind == "solve" else 2.0 * nn ** 3))
            if best is None or fl > best[0]:
                best = (fl, b, m, c, idx)
    return best


def run_dominant(args, engine, batches, modes, code, device):
    """Profiling case (--only-dominant): the workload's dominant size class alone,
    W + K launches of its plan and nothing else, so that an ncu capture of that
    kernel can select launches by count."""
    import torch
    fl, db, dm, dc, didx = dominant_class(batches, modes)
    dom = db if didx.size == db.nsys else subset(db, didx)
    plan = engine.Plan(dom, code[dm])
    A = torch.from_numpy(dom.A).to(device)
    out = torch.empty(dom.b.size if dom.kind == "solve" else dom.A.size, dtype=torch.float64, device=device)
    st = torch.empty((dom.nsys,), dtype=torch.int32, device=device)
    bb = torch.from_numpy(dom.b).to(device) if dom.kind == "solve" else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        plan.execute(A, out, st, b=bb)
    e0.record()
    for _ in range(args.steps):
        plan.execute(A, out, st, b=bb)
    e1.record()
    torch.cuda.synchronize(device)
    t = e0.elapsed_time(e1) / 1e3 / max(1, args.steps)
    print(json.dumps({"profiling_case": kernel_name(dom.kind, dc, dm), "size_class": dc, "systems": dom.nsys,
                      "bytes": dom.bytes(), "flops": dom.flops(), "launch_s": t,
                      "launches_per_execute": plan.launches}), flush=True)
    plan.close()
    return 0


def run_sweep(args):
    """Config 2: the conditioning sweep.  Per generator and log10 kappa_2 group,
    the mixed path (equilibrated FP32 LU + FP64 refinement, solves n <= 32)
    against the plain FP64 path on the GPU: forward and backward error,
    refinement steps, fallback fraction and throughput of both."""
    import torch

    from python_b200 import engine
    rank, world, local = dist_env()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    engine.load()
    nsys = args.nsys or 2048
    stream = torch.cuda.current_stream(device)
    groups, mixed_rate, fp64_rate = [], [], []

    def timed(plan, A, out, st, b, diag):
        for _ in range(args.warmup):
            plan.execute(A, out, st, b=b, diag=diag, stream=stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            plan.execute(A, out, st, b=b, diag=diag, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize(device)
        return e0.elapsed_time(e1) / 1e3 / args.steps

    for gen in ("ion", "macro"):
        for lk in wl.KAPPA_GROUPS:
            batch, kap, reachable = wl.config2(gen, lk, nsys=nsys)
            A = torch.from_numpy(batch.A).to(device)
            b = torch.from_numpy(batch.b).to(device) if batch.kind == "solve" else None
            size = batch.b.size if batch.kind == "solve" else batch.A.size
            res = {"generator": gen, "kind": batch.kind, "log10_kappa_target": lk, "systems": batch.nsys,
                   "log10_kappa": {"min": float(kap.min()), "median": float(np.median(kap)), "max": float(kap.max())},
                   "target_band_reachable": reachable}
            outs = {}
            for mode in ("fp64", "mixed"):
                if mode == "mixed" and batch.kind != "solve":
                    res["mixed"] = "not built: a refined inverse needs the FP64 residual I - A X, as many FP64 flops as the FP64 inverse"
                    continue
                plan = engine.Plan(batch, engine.FP64 if mode == "fp64" else engine.MIXED)
                out = torch.empty(size, dtype=torch.float64, device=device)
                st = torch.empty(batch.nsys, dtype=torch.int32, device=device)
                diag = torch.zeros(batch.nsys, dtype=torch.int32, device=device)
                dt = timed(plan, A, out, st, b, diag)
                plan.close()
                outs[mode] = (out.cpu().numpy(), st.cpu().numpy(), diag.cpu().numpy(), batch.nsys / dt)
            # host-side error analysis (FP64 arithmetic, numpy)
            n = int(batch.n[0])
            M = batch.A.reshape(batch.nsys, n, n)
            xf, sf, _, rf = outs["fp64"]
            res["fp64"] = {"systems_per_s": rf, "singular": int(np.sum(sf == (4 if batch.kind == "solve" else 1)))}
            fp64_rate.append(rf)
            if batch.kind == "solve":
                B = batch.b.reshape(batch.nsys, n)
                XF = xf.reshape(batch.nsys, n)

                def backward(X):
                    r = np.abs(B - np.einsum("sij,sj->si", M, X)).max(axis=1)
                    return r / (np.abs(M).sum(axis=2).max(axis=1) * np.abs(X).max(axis=1))
                ok = sf != 4
                res["fp64"]["backward_err"] = {"median": float(np.median(backward(XF)[ok])), "max": float(backward(XF)[ok].max())}
                xm, sm, dm, rm = outs["mixed"]
                XM = xm.reshape(batch.nsys, n)
                fb = (dm & 0x100) != 0
                acc = ok & ~fb
                fwd = np.zeros(batch.nsys)
                for i in np.nonzero(ok)[0]:
                    sig = np.abs(XF[i]) > 1e-20 * np.abs(XF[i]).sum()
                    fwd[i] = np.max(np.abs(XM[i][sig] - XF[i][sig]) / np.abs(XF[i][sig])) if sig.any() else 0.0
                it = dm & 0xff
                res["mixed"] = {"systems_per_s": rm, "fallback_frac": float(fb.mean()),
                                "codes_match_fp64": bool(np.array_equal(sm, sf)),
                                "forward_err_vs_fp64": {"median_accepted": float(np.median(fwd[acc])) if acc.any() else None,
                                                        "max_accepted": float(fwd[acc].max()) if acc.any() else None,
                                                        "max_all": float(fwd[ok].max()) if ok.any() else None},
                                "backward_err": {"median": float(np.median(backward(XM)[ok])), "max": float(backward(XM)[ok].max())},
                                "refinement_steps": {"mean_accepted": float(it[acc].mean()) if acc.any() else None,
                                                     "max_accepted": int(it[acc].max()) if acc.any() else None}}
                mixed_rate.append(rm)
            else:
                XF = xf.reshape(batch.nsys, n, n)
                ok = sf == 0
                eye = np.eye(n)
                R = np.abs(eye - np.einsum("sij,sjk->sik", M, XF)).sum(axis=2).max(axis=1)
                bwd = R / (np.abs(M).sum(axis=2).max(axis=1) * np.abs(XF).sum(axis=2).max(axis=1))
                res["fp64"]["backward_err"] = {"median": float(np.median(bwd[ok])), "max": float(bwd[ok].max())}
                from oracle import oracle
                idx = np.arange(0, batch.nsys, max(1, batch.nsys // 256))
                sub = subset(batch, idx)
                ir, sr = oracle.invert(sub, "port", threads=oracle.host_threads())
                worst = 0.0
                for j, s_ in enumerate(idx):
                    if sr[j] == 0:
                        r = ir[sub.offA[j]:sub.offA[j] + n * n]
                        v = xf[batch.offA[s_]:batch.offA[s_] + n * n]
                        worst = max(worst, float(np.max(np.abs(v - r)) / np.max(np.abs(r))))
                res["fp64"]["max_rel_err_vs_gsl_sample"] = worst
            groups.append(res)
    if rank == 0:
        value = float(np.sum([nsys for _ in mixed_rate]) / np.sum([nsys / r for r in mixed_rate])) if mixed_rate else None
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
                "data": "synthetic (config-0 / config-1 generators, rate spread widened per kappa group, rejection-sampled)",
                "config": {"workload": WORKLOADS[2], "config_index": 2, "systems_per_group": nsys},
                "value_is": "mixed-mode solve throughput over the ion groups (harmonic mean)",
                "sweep": groups}
        print(json.dumps(line), flush=True)
    return 0


def run_rows(args):
    """The rows around the batched solve, each through its public call on one
    GPU, wall clock over --steps calls after --warmup (every call synchronises):
    the macro-atom epilogue and draws on the config-1 batch, the GPU-assembled
    ion lock-step, and both rate-matrix assemblies.  One JSON line."""
    import ctypes

    import torch

    from python_b200 import engine
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)

    def clock(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            fn()
        torch.cuda.synchronize(dev)
        return (time.perf_counter() - t0) / args.steps

    out = {"metric": "rows around the batched solve: throughput of each public call", "impl": "ours",
           "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "data": "synthetic (seeded generators)"}
    # macro-atom epilogue and draws: config-1 batch, device-resident
    b = wl.config1(nsys=8192)
    nsys = b.nsys
    dn = np.ascontiguousarray(b.n, np.int32)
    offv = (np.arange(nsys, dtype=np.int64) * 61)
    dA = torch.from_numpy(b.A).to(dev)
    dR = torch.rand(nsys * 61, dtype=torch.float64, device=dev)
    dB = torch.empty_like(dA)
    dC = torch.empty_like(dA)
    dst = torch.empty(nsys, dtype=torch.int32, device=dev)
    lib = engine.load()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())

    def matom():
        rc = lib.matom_matrices_batched(nsys, dn.ctypes.data, b.offA.ctypes.data, offv.ctypes.data, vp(dA), vp(dR),
                                        vp(dB), vp(dC), vp(dst))
        assert rc == 0, engine.last_error()
    engine.set_precision(engine.FP64)
    t_matom = clock(matom)
    engine.set_precision(engine.FAST)
    t_matom_fast = clock(matom)
    engine.set_precision(engine.FP64)
    dX = torch.empty_like(dA)
    plan = engine.Plan(b, engine.FP64)

    def inv_only():
        plan.execute(dA, dX, dst)
        torch.cuda.synchronize(dev)
    t_inv = clock(inv_only)
    plan.close()
    plan = engine.Plan(b, engine.FAST)
    t_inv_fast = clock(inv_only)
    plan.close()
    nq = 1 << 20
    rng = np.random.default_rng(5)
    sysi = torch.from_numpy(rng.integers(0, nsys, nq).astype(np.int32)).to(dev)
    lvl = torch.from_numpy(rng.integers(0, 61, nq).astype(np.int32)).to(dev)
    zz = torch.rand(nq, dtype=torch.float64, device=dev)
    tgt = torch.empty(nq, dtype=torch.int32, device=dev)

    def draws():
        rc = lib.matom_sample_batched(nq, nsys, dn.ctypes.data, b.offA.ctypes.data, vp(dC), vp(sysi), vp(lvl), vp(zz),
                                      vp(tgt))
        assert rc == 0, engine.last_error()
    t_draw = clock(draws)
    out["matom_epilogue"] = {"workload": "8192 x n=61 inverse + B = N^-1 diag(R) + row running totals",
                             "systems_per_s": nsys / t_matom, "ms": t_matom * 1e3, "inverse_alone_ms": t_inv * 1e3,
                             "certified_fused_ms": t_matom_fast * 1e3,
                             "certified_inverse_alone_ms": t_inv_fast * 1e3,
                             "certified_fused_systems_per_s": nsys / t_matom_fast,
                             "draws_per_s": nq / t_draw, "draws": nq}
    del dA, dR, dB, dC, dX
    # ion rate matrices: a 181-ion table (13 elements, H to Ni), 20,000 cells
    tab = wl.ion_table(zs=(1, 2, 6, 7, 8, 10, 12, 14, 16, 18, 20, 26, 28), seed=21)
    ncell = 20000
    rates = wl.ion_rates(tab, ncell, seed=22)
    ne = np.full(ncell, 1e10)
    nh1, nh2 = np.full(ncell, 1e4), np.full(ncell, 1e10)
    t_ion = clock(lambda: engine.ion_rate_matrices(tab, rates, ne, nh1, nh2))
    blk = int((tab.elem_n.astype(np.int64) ** 2).sum())
    out["ion_rate_matrices"] = {"workload": f"{ncell} cells x {tab.nions} ions ({tab.nelem} element blocks)",
                                "cells_per_s": ncell / t_ion, "ms": t_ion * 1e3,
                                "bytes_out": ncell * (blk + tab.nions) * 8,
                                "note": "host arrays in and out: the call uploads the coefficients and returns A"}
    # the lock-step with GPU assembly: 4096 cells of the 48-ion table
    tab2 = wl.ion_table()
    nc2 = 4096
    rates2 = wl.ion_rates(tab2, nc2, seed=300)
    rng = np.random.default_rng(301)
    nh = np.exp(rng.uniform(np.log(1e6), np.log(1e12), nc2))
    dens = nh[:, None] * np.array([1.0, 0.1, 3e-4, 5e-4, 3e-5])[None, :]
    rounds = []

    def lock():
        den0 = np.zeros((nc2, tab2.nions))
        den0[:, tab2.elem_first] = 1.0
        ne0 = 0.1 * nh
        st, it = engine.ion_populations_lockstep_rates(tab2, rates2, 0, dens, ne0, den0)
        rounds.append(int(it.max()))
    t_lock = clock(lock)
    out["ion_lockstep_rates"] = {"workload": f"{nc2} cells x {tab2.nions} ions, n_e iteration to convergence",
                                 "cells_per_s": nc2 / t_lock, "ms": t_lock * 1e3, "rounds": rounds[-1]}
    # macro-atom jump matrices: 8192 cells of a 58-level model, device outputs
    m = wl.matom_model()
    cells = [wl.matom_cell(m, 7000 + c) for c in range(64)]
    inp1 = wl.matom_jump_inputs(m, cells)
    rep = 128                                   # 8192 cells: the 64 coefficient sets repeated
    inp = dict(inp1)
    for k in engine.MATOM_RATE_FIELDS:
        inp[k] = np.tile(inp1[k], rep)
    inp["ncell"] = 64 * rep
    nr = m.nlev + 1
    dN = torch.empty((inp["ncell"], nr, nr), dtype=torch.float64, device=dev)
    dRr = torch.empty((inp["ncell"], nr), dtype=torch.float64, device=dev)
    t_mq = clock(lambda: engine.matom_rate_matrices(inp, dN, dRr))
    out["matom_rate_matrices"] = {"workload": f"{inp['ncell']} cells x {m.nlev} levels + k-packet",
                                  "cells_per_s": inp["ncell"] / t_mq, "ms": t_mq * 1e3,
                                  "note": "host coefficients in, N and R left on the device"}
    print(json.dumps(out), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=3, choices=sorted(WORKLOADS))
    ap.add_argument("--mode", choices=["auto", "fp64", "mixed", "fast"], default="auto")
    ap.add_argument("--nsys", type=int, default=None,
                    help="systems (cells for config 3) instead of the workload's own count (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--only-dominant", action="store_true",
                    help="profiling case: launch only the dominant size class's plan (W + K times)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cusolver", action="store_true",
                    help="skip timing the reference's cuSOLVER build")
    ap.add_argument("--cusolver-seconds", type=float, default=5.0)
    ap.add_argument("--ref-seconds", type=float, default=120.0)
    ap.add_argument("--rows", action="store_true",
                    help="time the rows around the batched solve (matom epilogue and draws, assemblies, lock-step)")
    ap.add_argument("--traffic", type=float, default=None,
                    help="DRAM bytes per launch of the dominant kernel from an ncu capture")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.rows:
        return run_rows(args)
    if args.config == 2:
        return run_sweep(args)
    return run_ours(args)


if __name__ == "__main__":
    raise SystemExit(main())
