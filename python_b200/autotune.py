"""Autotuner of the engine's size classes.

``--family cta`` (the default): the GSL-exact CTA kernel family.  For every
padded order P listed in ``csrc/tune_candidates.inc`` the tuner builds the
tuning library (``csrc/tune.cu`` -> ``libsirocco_tune.so``), times each
candidate configuration on a device-resident batch of macro-atom inverses at
two orders of the class (its middle and its top), checks that all candidates
return the same bits and codes, and keeps the fastest.  It writes
``csrc/cta_classes.inc``.

``--family cgj``: the certified Gauss-Jordan classes (SIROCCO_FAST).  Every
padded order P of ``csrc/tune_cgj_candidates.inc`` gets its own tuning library
(``csrc/tune_cgj.cu`` compiled with that order's candidates, under
``_build/tune_cgj``).  The tuner times every shape at two orders of the class,
checks codes and that every shape's inverses agree with the first one's to
1e-12 (shapes may order the MMA sums differently), keeps the fastest shape,
then sets the class edges: from the top down, a class whose orders the next
kept class's winner inverts faster is dropped.  It writes
``csrc/cgj_classes.inc``.

``--family small``: the warp-group kernels of orders up to 32.  Each
candidate of ``csrc/tune_small_candidates.inc`` (a padded row length NP and a
lane count G >= NP per system) solves batches of ion-balance systems at two
orders of its class; all candidates must return the same bits.  The fastest G
per NP is kept, class edges are chosen as for the certified classes, and
``csrc/small_classes.inc`` is written.

All three write every timing into ``tuned_classes.json`` and rebuild the engine.

    python -m python_b200.autotune [--family cgj|small]   # on a B200; then commit the written files
"""
from __future__ import annotations

import argparse
import concurrent.futures
import ctypes
import datetime
import json
import os
import re
import subprocess
import sys
from ctypes import POINTER, c_float, c_int, c_void_p
from pathlib import Path

import numpy as np

from . import build
from . import workloads as wl

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
TUNE_LIB = PKG / "libsirocco_tune.so"
CANDIDATES = CSRC / "tune_candidates.inc"
CLASS_INC = CSRC / "cta_classes.inc"
RECORD = PKG / "tuned_classes.json"
SMALLEST_CTA_ORDER = 33          # orders up to 32 go to the small-system family
WORK_FLOP = 2.0e11               # floating-point work per timed launch
MAX_BYTES = 3 << 30              # input matrices per timed batch

CGJ_CANDIDATES = CSRC / "tune_cgj_candidates.inc"
CGJ_CLASS_INC = CSRC / "cgj_classes.inc"
CGJ_BUILD = PKG / "_build" / "tune_cgj"
CGJ_MIN_ORDER = 33               # below this the exact path's warp-group kernels serve certified inverses too
CGJ_WORK_FLOP = 5.0e10           # floating-point work per timed launch (certified classes)
CGJ_AGREE = 1e-12                # largest difference between two shapes' inverses, relative to the largest entry

SMALL_CANDIDATES = CSRC / "tune_small_candidates.inc"
SMALL_CLASS_INC = CSRC / "small_classes.inc"
SMALL_TUNE_LIB = PKG / "_build" / "libsirocco_tune_small.so"
SMALL_SYSTEMS = 1 << 18          # solves per timed launch (a generated set, repeated)


def parse_candidates(path: Path = CANDIDATES):
    out = []
    for line in path.read_text().splitlines():
        m = re.match(r"SS_TUNE\((\d+), (\d+), (\d+), (\d+), (\d+), (true|false), (\d+)\)", line.strip())
        if m:
            out.append((int(m[1]), int(m[2]), int(m[3]), int(m[4]), int(m[5]), m[6] == "true", int(m[7])))
    return out


def parse_classes(path: Path = CLASS_INC):
    out = []
    for line in path.read_text().splitlines():
        m = re.match(r"SS_CTA_CLASS\((\d+), (\d+), (\d+), (\d+), (\d+), (\d+), (true|false), (\d+)\)", line.strip())
        if m:
            out.append((int(m[2]), int(m[3]), int(m[4]), int(m[5]), int(m[6]), m[7] == "true", int(m[8])))
    return out


def build_tune_lib() -> Path:
    deps = [CSRC / "tune.cu", CANDIDATES] + build.HEADERS
    if build._stale(TUNE_LIB, deps):
        tmp = TUNE_LIB.with_suffix(".so.tmp")
        subprocess.run([build.NVCC, *build.ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                        "--expt-relaxed-constexpr", "-cudart", "static", "-o", str(tmp), str(CSRC / "tune.cu")],
                       check=True, cwd=str(CSRC))
        tmp.replace(TUNE_LIB)
    return TUNE_LIB


def load_tune_lib():
    """The tuning library with its argument types, and its candidates as
    (index, (P, threads, RG, CC, panel warps, global memory, CTAs per SM asked))."""
    lib = ctypes.CDLL(str(build_tune_lib()))
    lib.sirocco_tune_info.argtypes = [c_int, POINTER(c_int)]
    lib.sirocco_tune_time.argtypes = [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                                      POINTER(c_float), POINTER(c_int)]
    cands = []
    for i in range(lib.sirocco_tune_count()):
        cfg = (c_int * 7)()
        lib.sirocco_tune_info(i, cfg)
        cands.append((i, tuple(cfg[:5]) + (bool(cfg[5]), cfg[6])))
    return lib, cands


def run_candidate(lib, i: int, batch, device, reps: int = 1):
    """Inverts a device copy of the batch with candidate i; returns (out, status, ms, CTAs per SM)."""
    import torch
    nsys = batch.nsys
    dn = torch.from_numpy(np.ascontiguousarray(batch.n, np.int32)).to(device)
    doff = torch.from_numpy(np.ascontiguousarray(batch.offA, np.int64)).to(device)
    dA = torch.from_numpy(batch.A).to(device)
    dlist = torch.arange(nsys, dtype=torch.int32, device=device)
    out = torch.empty_like(dA)
    st = torch.full((nsys,), -99, dtype=torch.int32, device=device)
    ms, res = c_float(), c_int()
    rc = lib.sirocco_tune_time(i, nsys, c_void_p(dn.data_ptr()), c_void_p(doff.data_ptr()), c_void_p(dA.data_ptr()),
                               c_void_p(out.data_ptr()), c_void_p(st.data_ptr()), c_void_p(dlist.data_ptr()), reps,
                               ctypes.byref(ms), ctypes.byref(res))
    torch.cuda.synchronize(device)
    if rc != 0:
        return None, None, rc, 0
    return out.cpu().numpy(), st.cpu().numpy(), ms.value, res.value


def test_orders(p: int, p_prev: int):
    lo = max(p_prev + 1, SMALLEST_CTA_ORDER)
    return sorted({(lo + p) // 2, p - max(1, (p - lo) // 8)})


def write_outputs(best: dict, record: dict) -> None:
    lines = ["// Size classes of the CTA-per-system kernel family (kernels_cta.cuh).",
             "// Written by `python -m python_b200.autotune` from its timings on a B200; the",
             "// record of every candidate it timed is python_b200/tuned_classes.json.",
             "// SS_CTA_CLASS(index, P, threads, RG, CC, panel warps, matrix in global memory, CTAs per SM asked)"]
    for i, p in enumerate(sorted(best)):
        P, NT, RG, CC, PW, GM, MINB = best[p]
        lines.append(f"SS_CTA_CLASS({i}, {P}, {NT}, {RG}, {CC}, {PW}, {'true' if GM else 'false'}, {MINB})")
    CLASS_INC.write_text("\n".join(lines) + "\n")
    if RECORD.exists():
        old = json.loads(RECORD.read_text())
        for key in ("cgj", "small"):   # the other families' records stay
            if key in old:
                record[key] = old[key]
    RECORD.write_text(json.dumps(record, indent=1) + "\n")


# ---------------------------------------------------------- certified classes --
def parse_cgj_candidates(path: Path = CGJ_CANDIDATES):
    """(P, WGR, WGC, CL, CTAs per SM asked, staged) per candidate line."""
    out = []
    for line in path.read_text().splitlines():
        m = re.match(r"SS_TUNE_CGJ\((\d+), (\d+), (\d+), (\d+), (\d+), (true|false)\)", line.strip())
        if m:
            out.append((int(m[1]), int(m[2]), int(m[3]), int(m[4]), int(m[5]), m[6] == "true"))
    return out


def parse_cgj_classes(path: Path = CGJ_CLASS_INC):
    out = []
    for line in path.read_text().splitlines():
        m = re.match(r"SS_CGJ_CLASS\((\d+), (\d+), (\d+), (\d+), (\d+), (\d+), (true|false)\)", line.strip())
        if m:
            out.append((int(m[2]), int(m[3]), int(m[4]), int(m[5]), int(m[6]), m[7] == "true"))
    return out


def _cgj_line(c) -> str:
    return f"SS_TUNE_CGJ({c[0]}, {c[1]}, {c[2]}, {c[3]}, {c[4]}, {'true' if c[5] else 'false'})"


def build_cgj_tune_libs(jobs: int | None = None) -> dict:
    """One tuning library per padded order of the candidate list, compiled in
    parallel; returns {P: path}."""
    by_p: dict = {}
    for c in parse_cgj_candidates():
        by_p.setdefault(c[0], []).append(c)
    CGJ_BUILD.mkdir(parents=True, exist_ok=True)
    src = CSRC / "tune_cgj.cu"
    todo, libs = [], {}
    for p, cs in sorted(by_p.items()):
        lst = CGJ_BUILD / f"candidates_{p}.inc"
        text = "\n".join(_cgj_line(c) for c in cs) + "\n"
        if not lst.exists() or lst.read_text() != text:
            lst.write_text(text)
        lib = CGJ_BUILD / f"libtune_cgj_{p}.so"
        libs[p] = lib
        if build._stale(lib, [src, lst] + build.HEADERS):
            todo.append((lst, lib))

    def compile_one(item):
        lst, lib = item
        tmp = lib.with_suffix(".so.tmp")
        subprocess.run([build.NVCC, *build.ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                        "--expt-relaxed-constexpr", "-cudart", "static", f"-DSS_TUNE_CGJ_LIST=\"{lst}\"",
                        "-o", str(tmp), str(src)], check=True, cwd=str(CSRC))
        tmp.replace(lib)

    if todo:
        with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            list(ex.map(compile_one, todo))
    return libs


def load_cgj_lib(path: Path):
    """A certified-class tuning library and its candidates as (index, config)."""
    lib = ctypes.CDLL(str(path))
    lib.sirocco_tune_info.argtypes = [c_int, POINTER(c_int)]
    lib.sirocco_tune_time.argtypes = [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                      c_void_p, c_int, POINTER(c_float), POINTER(c_int)]
    cands = []
    for i in range(lib.sirocco_tune_count()):
        cfg = (c_int * 6)()
        lib.sirocco_tune_info(i, cfg)
        cands.append((i, tuple(cfg[:5]) + (bool(cfg[5]),)))
    return lib, cands


class _DeviceBatch:
    """A batch of certified matrices resident on the device."""

    def __init__(self, batch, device):
        import torch
        self.batch = batch
        self.n = torch.from_numpy(np.ascontiguousarray(batch.n, np.int32)).to(device)
        self.off = torch.from_numpy(np.ascontiguousarray(batch.offA, np.int64)).to(device)
        self.A = torch.from_numpy(batch.A).to(device)
        self.list = torch.arange(batch.nsys, dtype=torch.int32, device=device)
        self.out = torch.empty_like(self.A)
        self.st = torch.empty((batch.nsys,), dtype=torch.int32, device=device)
        self.scratch = torch.empty((2 * batch.nsys + 4,), dtype=torch.int32, device=device)


def run_cgj(lib, i: int, db: _DeviceBatch, reps: int):
    """Candidate i on the device batch: (inverses, status, fastest ms, CTAs per SM), or an error code."""
    import torch
    db.out.fill_(float("nan"))
    db.st.fill_(-99)
    ms, res = c_float(), c_int()
    rc = lib.sirocco_tune_time(i, db.batch.nsys, c_void_p(db.n.data_ptr()), c_void_p(db.off.data_ptr()),
                               c_void_p(db.A.data_ptr()), c_void_p(db.out.data_ptr()), c_void_p(db.st.data_ptr()),
                               c_void_p(db.list.data_ptr()), c_void_p(db.scratch.data_ptr()), reps,
                               ctypes.byref(ms), ctypes.byref(res))
    torch.cuda.synchronize()
    if rc != 0:
        return None, None, rc, 0
    return db.out.cpu().numpy(), db.st.cpu().numpy(), ms.value, res.value


def cgj_test_orders(p: int, p_prev: int):
    lo = max(p_prev + 1, CGJ_MIN_ORDER)
    return sorted({(lo + p) // 2, p - max(1, (p - lo) // 8)})


def cgj_batch(n: int):
    nsys = int(min(8192, max(592, CGJ_WORK_FLOP / (2.0 * n ** 3)), MAX_BYTES // (8 * n * n)))
    return wl.macro_batch([n] * nsys, seed=2000 + n)


def write_cgj_outputs(classes: list, notes: dict, record: dict) -> None:
    lines = ["// Size classes of the certified Gauss-Jordan inverse (kernels_cert.cuh).",
             "// Written by `python -m python_b200.autotune --family cgj` from its timings on a",
             "// B200 (every candidate of tune_cgj_candidates.inc; the record is",
             "// python_b200/tuned_classes.json, key \"cgj\").",
             "// SS_CGJ_CLASS(index, P, tile-warp rows WGR, tile-warp columns WGC, CTAs per matrix CL,",
             "//              CTAs per SM asked, rows staged by TMA)",
             "// Each CTA runs WGR x WGC tile warps plus one pivot warp; a tile warp holds",
             "// (P / CL / 8 / WGR) x (P / 8 / WGC) sub-blocks of 8 x 8 doubles.  A single row of",
             "// tile warps (WGR = 1) forms R' in registers.  Orders above 128 deal their rows to a",
             "// cluster of CL CTAs.  Orders up to 32 stay on the kernels of the exact path, orders",
             "// above the last class on the streamed certified kernel.  After each class: the",
             "// winner's rate at the tuner's test orders, and the runner-up."]
    for i, c in enumerate(classes):
        lines.append(f"SS_CGJ_CLASS({i}, {c[0]}, {c[1]}, {c[2]}, {c[3]}, {c[4]}, {'true' if c[5] else 'false'})"
                     + (f"  // {notes[c[0]]}" if c[0] in notes else ""))
    CGJ_CLASS_INC.write_text("\n".join(lines) + "\n")
    old = json.loads(RECORD.read_text()) if RECORD.exists() else {}
    old["cgj"] = record
    RECORD.write_text(json.dumps(old, indent=1) + "\n")


def tune_cgj(args) -> int:
    import torch
    dev = torch.device("cuda", 0)
    libs = build_cgj_tune_libs()
    loaded = {p: load_cgj_lib(path) for p, path in libs.items()}
    orders = sorted(loaded)
    record = {"device": torch.cuda.get_device_name(0), "when": datetime.datetime.now(datetime.timezone.utc).isoformat(),
              "work_flop_per_launch": CGJ_WORK_FLOP, "reps": args.reps, "classes": [], "edges": []}
    win, scores, tests = {}, {}, {}
    batches = {}

    def dbatch(n):
        if n not in batches:
            batches.clear()   # one batch on the device at a time
            batches[n] = _DeviceBatch(cgj_batch(n), dev)
        return batches[n]

    for k, p in enumerate(orders):
        p_prev = orders[k - 1] if k else CGJ_MIN_ORDER - 1
        lib, cands = loaded[p]
        tests[p] = cgj_test_orders(p, p_prev)
        entry = {"P": p, "orders": tests[p], "candidates": []}
        tot = {i: 0.0 for i, _ in cands}
        ok = {i: True for i, _ in cands}
        for n in tests[p]:
            db = dbatch(n)
            ref = None
            for i, cfg in cands:
                out, st, ms, res = run_cgj(lib, i, db, args.reps)
                if out is None or not (st == 0).all():
                    ok[i] = False
                    entry["candidates"].append({"config": cfg, "n": n, "error": ms if out is None else "status"})
                    continue
                if ref is None:
                    ref = out
                else:
                    dev_ = float(np.max(np.abs(out - ref)) / np.max(np.abs(ref)))
                    if not dev_ <= CGJ_AGREE:
                        raise SystemExit(f"shape {cfg} differs from {cands[0][1]} by {dev_:.2e} at n={n}")
                tot[i] += ms
                entry["candidates"].append({"config": cfg, "n": n, "nsys": db.batch.nsys, "ms": ms, "ctas_per_sm": res,
                                            "tflops": db.batch.flops() / (ms * 1e-3) / 1e12})
        good = sorted((i for i, _ in cands if ok[i]), key=lambda i: tot[i])
        if not good:
            raise SystemExit(f"no candidate of P={p} ran")
        win[p] = (good[0], dict(cands)[good[0]])
        scores[p] = tot[good[0]]
        entry["chosen"] = win[p][1]
        entry["runner_up"] = dict(cands)[good[1]] if len(good) > 1 else None
        record["classes"].append(entry)
        print(f"P={p:4d} orders {tests[p]}: " + ", ".join(f"{dict(cands)[i][1:]}={tot[i]:.3f}ms" for i in good)
              + f"  -> {win[p][1]}", flush=True)

    # class edges, from the top down: drop a class whose orders the next kept
    # class's winner inverts faster
    kept = [orders[-1]]
    for p in reversed(orders[:-1]):
        nxt = kept[0]
        lib, _ = loaded[nxt]
        t_next = 0.0
        for n in tests[p]:
            out, st, ms, _ = run_cgj(lib, win[nxt][0], dbatch(n), args.reps)
            t_next = float("inf") if out is None or not (st == 0).all() else t_next + ms
        drop = t_next < scores[p]
        record["edges"].append({"P": p, "next": nxt, "ms_own": scores[p], "ms_next": t_next, "dropped": drop})
        print(f"edge P={p}: own {scores[p]:.3f} ms, by P={nxt} {t_next:.3f} ms -> {'drop' if drop else 'keep'}",
              flush=True)
        if not drop:
            kept.insert(0, p)
    classes = [win[p][1] for p in kept]
    notes = {}
    for e in record["classes"]:
        if e["P"] in kept:
            rates = [c["tflops"] for c in e["candidates"] if c.get("config") == e["chosen"] and "tflops" in c]
            ru = e["runner_up"]
            notes[e["P"]] = (f"{min(rates):.1f}-{max(rates):.1f} TF/s at orders {e['orders']}"
                             + (f"; runner-up {tuple(ru[1:])}" if ru else ""))
    if args.dry_run:
        print("classes:", classes)
        return 0
    write_cgj_outputs(classes, notes, record)
    if not args.no_build:
        build.build_engine(force=True)
    print(f"wrote {CGJ_CLASS_INC.relative_to(PKG.parent)} and {RECORD.relative_to(PKG.parent)}")
    return 0


# ------------------------------------------------------------- small systems --
def parse_small_candidates(path: Path = SMALL_CANDIDATES):
    return [(int(m[1]), int(m[2])) for m in re.finditer(r"^SS_TUNE_SMALL\((\d+), (\d+)\)", path.read_text(), re.M)]


def parse_small_classes(path: Path = SMALL_CLASS_INC):
    return [(int(m[1]), int(m[2])) for m in
            re.finditer(r"^SS_SMALL_CLASS\(\d+, (\d+), (\d+)\)", path.read_text(), re.M)]


def build_small_tune_lib() -> Path:
    deps = [CSRC / "tune_small.cu", SMALL_CANDIDATES] + build.HEADERS
    if build._stale(SMALL_TUNE_LIB, deps):
        SMALL_TUNE_LIB.parent.mkdir(parents=True, exist_ok=True)
        tmp = SMALL_TUNE_LIB.with_suffix(".so.tmp")
        subprocess.run([build.NVCC, *build.ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                        "--expt-relaxed-constexpr", "-cudart", "static", "-o", str(tmp),
                        str(CSRC / "tune_small.cu")], check=True, cwd=str(CSRC))
        tmp.replace(SMALL_TUNE_LIB)
    return SMALL_TUNE_LIB


def load_small_lib():
    lib = ctypes.CDLL(str(build_small_tune_lib()))
    lib.sirocco_tune_info.argtypes = [c_int, POINTER(c_int)]
    lib.sirocco_tune_time.argtypes = [c_int, c_int] + [c_void_p] * 8 + [c_int, POINTER(c_float), POINTER(c_int)]
    cands = []
    for i in range(lib.sirocco_tune_count()):
        cfg = (c_int * 2)()
        lib.sirocco_tune_info(i, cfg)
        cands.append((i, (cfg[0], cfg[1])))
    return lib, cands


class _DeviceSolves:
    """SMALL_SYSTEMS ion-balance solves of order n on the device: a generated
    set of 4,096 systems, repeated."""

    def __init__(self, n: int, device):
        import torch
        base = wl.ion_batch([n] * 4096, seed=3000 + n)
        reps = SMALL_SYSTEMS // base.nsys
        self.nsys = base.nsys * reps
        self.flops = base.flops() * reps
        a, b = base.A.size, base.b.size
        self.n = torch.full((self.nsys,), n, dtype=torch.int32, device=device)
        k = torch.arange(reps, dtype=torch.int64, device=device).repeat_interleave(base.nsys)
        self.offA = torch.from_numpy(base.offA).to(device).repeat(reps) + k * a
        self.offv = torch.from_numpy(base.offv).to(device).repeat(reps) + k * b
        self.A = torch.from_numpy(base.A).to(device).repeat(reps)
        self.b = torch.from_numpy(base.b).to(device).repeat(reps)
        self.x = torch.empty_like(self.b)
        self.st = torch.empty((self.nsys,), dtype=torch.int32, device=device)
        self.list = torch.arange(self.nsys, dtype=torch.int32, device=device)


def run_small(lib, i: int, ds: _DeviceSolves, reps: int):
    import torch
    ds.x.fill_(float("nan"))
    ds.st.fill_(-99)
    ms, res = c_float(), c_int()
    rc = lib.sirocco_tune_time(i, ds.nsys, *(c_void_p(t.data_ptr()) for t in
                                             (ds.n, ds.offA, ds.offv, ds.A, ds.b, ds.x, ds.st, ds.list)),
                               reps, ctypes.byref(ms), ctypes.byref(res))
    torch.cuda.synchronize()
    if rc != 0:
        return None, None, rc, 0
    return ds.x.cpu().numpy(), ds.st.cpu().numpy(), ms.value, res.value


def write_small_outputs(classes: list, notes: dict, record: dict) -> None:
    lines = ["// Size classes of the small-system family (kernels_small.cuh, kernels_mixed.cuh).",
             "// Written by `python -m python_b200.autotune --family small` from its timings on a",
             "// B200 (every candidate of tune_small_candidates.inc; the record is",
             "// python_b200/tuned_classes.json, key \"small\").",
             "// SS_SMALL_CLASS(index, padded row length NP, lanes per system G)",
             "// A system of order n <= NP runs on G >= NP lanes of a warp (lane r holds row r),",
             "// 128 / G systems per CTA of 128 threads.  After each class: the winner's rate at",
             "// the tuner's test orders."]
    for i, (np_, g) in enumerate(classes):
        lines.append(f"SS_SMALL_CLASS({i}, {np_}, {g})" + (f"  // {notes[np_]}" if np_ in notes else ""))
    SMALL_CLASS_INC.write_text("\n".join(lines) + "\n")
    old = json.loads(RECORD.read_text()) if RECORD.exists() else {}
    old["small"] = record
    RECORD.write_text(json.dumps(old, indent=1) + "\n")


def tune_small(args) -> int:
    import torch
    dev = torch.device("cuda", 0)
    lib, cands = load_small_lib()
    orders = sorted({c[0] for _, c in cands})
    record = {"device": torch.cuda.get_device_name(0), "when": datetime.datetime.now(datetime.timezone.utc).isoformat(),
              "systems_per_launch": SMALL_SYSTEMS, "reps": args.reps, "classes": [], "edges": []}
    win, scores, tests, cache = {}, {}, {}, {}

    def solves(n):
        if n not in cache:
            cache.clear()
            cache[n] = _DeviceSolves(n, dev)
        return cache[n]

    for k, np_ in enumerate(orders):
        lo = orders[k - 1] + 1 if k else 2
        tests[np_] = sorted({(lo + np_) // 2, np_})
        mine = [(i, c) for i, c in cands if c[0] == np_]
        entry = {"NP": np_, "orders": tests[np_], "candidates": []}
        tot = {i: 0.0 for i, _ in mine}
        for n in tests[np_]:
            ds = solves(n)
            ref = None
            for i, cfg in mine:
                x, st, ms, res = run_small(lib, i, ds, args.reps)
                if x is None:
                    raise SystemExit(f"candidate {cfg} failed to run: {ms}")
                got = (x.tobytes(), st.tobytes())
                if ref is None:
                    ref = got
                elif got != ref:
                    raise SystemExit(f"candidate {cfg} disagrees with {mine[0][1]} at n={n}")
                tot[i] += ms
                entry["candidates"].append({"config": cfg, "n": n, "ms": ms, "ctas_per_sm": res,
                                            "systems_per_s": ds.nsys / (ms * 1e-3)})
        best = min(tot, key=tot.get)
        win[np_] = (best, dict(mine)[best])
        scores[np_] = tot[best]
        entry["chosen"] = win[np_][1]
        record["classes"].append(entry)
        print(f"NP={np_:3d} orders {tests[np_]}: " + ", ".join(f"G={dict(mine)[i][1]}:{tot[i]:.3f}ms" for i in tot)
              + f"  -> {win[np_][1]}", flush=True)

    kept = [orders[-1]]
    for np_ in reversed(orders[:-1]):
        nxt = kept[0]
        t_next = sum(run_small(lib, win[nxt][0], solves(n), args.reps)[2] for n in tests[np_])
        drop = t_next < scores[np_]
        record["edges"].append({"NP": np_, "next": nxt, "ms_own": scores[np_], "ms_next": t_next, "dropped": drop})
        print(f"edge NP={np_}: own {scores[np_]:.3f} ms, by NP={nxt} {t_next:.3f} ms -> {'drop' if drop else 'keep'}",
              flush=True)
        if not drop:
            kept.insert(0, np_)
    classes = [win[np_][1] for np_ in kept]
    notes = {}
    for e in record["classes"]:
        if e["NP"] in kept:
            rates = [c["systems_per_s"] for c in e["candidates"] if tuple(c["config"]) == tuple(e["chosen"])]
            notes[e["NP"]] = f"{min(rates) / 1e6:.0f}-{max(rates) / 1e6:.0f} M solves/s at orders {e['orders']}"
    if args.dry_run:
        print("classes:", classes)
        return 0
    write_small_outputs(classes, notes, record)
    if not args.no_build:
        build.build_engine(force=True)
    print(f"wrote {SMALL_CLASS_INC.relative_to(PKG.parent)} and {RECORD.relative_to(PKG.parent)}")
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--family", choices=("cta", "cgj", "small"), default="cta")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--only", type=int, nargs="*", help="tune only these padded orders (others keep their entry)")
    ap.add_argument("--dry-run", action="store_true", help="time and print, write nothing")
    ap.add_argument("--no-build", action="store_true", help="write the table but do not rebuild the engine")
    args = ap.parse_args(argv)
    if args.family == "cgj":
        return tune_cgj(args)
    if args.family == "small":
        return tune_small(args)
    import torch

    lib, cands = load_tune_lib()
    orders = sorted({c[1][0] for c in cands})
    current = {c[0]: c for c in parse_classes()}
    best = {p: current[p] for p in current if p in orders}
    record = {"device": torch.cuda.get_device_name(0), "when": datetime.datetime.now(datetime.timezone.utc).isoformat(),
              "work_flop_per_launch": WORK_FLOP, "reps": args.reps, "classes": []}
    dev = torch.device("cuda", 0)
    for k, p in enumerate(orders):
        if args.only and p not in args.only:
            continue
        p_prev = orders[k - 1] if k else SMALLEST_CTA_ORDER - 1
        mine = [c for c in cands if c[1][0] == p]
        entry = {"P": p, "orders": test_orders(p, p_prev), "candidates": []}
        scores = {i: 0.0 for i, _ in mine}
        ok = {i: True for i, _ in mine}
        for n in entry["orders"]:
            nsys = int(min(8192, max(296, WORK_FLOP / (2.0 * n ** 3)), MAX_BYTES // (8 * n * n)))
            batch = wl.macro_batch([n] * nsys, seed=1000 + n, density=0.25 if n <= 256 else 0.10)
            ref = None
            for i, cfg in mine:
                out, st, ms, res = run_candidate(lib, i, batch, dev, args.reps)
                if out is None:
                    ok[i] = False
                    entry["candidates"].append({"config": cfg, "n": n, "error": ms})
                    continue
                got = (out.tobytes(), st.tobytes())
                if ref is None:
                    ref = got
                elif got != ref:
                    raise SystemExit(f"candidate {cfg} disagrees with {mine[0][1]} at n={n}")
                scores[i] += ms
                entry["candidates"].append({"config": cfg, "n": n, "nsys": nsys, "ms": ms, "ctas_per_sm": res,
                                            "tflops": 2.0 * n ** 3 * nsys / (ms * 1e-3) / 1e12})
        good = [i for i, _ in mine if ok[i]]
        win = min(good, key=lambda i: scores[i])
        best[p] = dict(mine)[win]
        entry["chosen"] = best[p]
        record["classes"].append(entry)
        print(f"P={p:5d} orders {entry['orders']}: " + ", ".join(
            f"{dict(mine)[i][1:]}={scores[i]:.2f}ms" for i in good) + f"  -> {best[p]}", flush=True)
    if args.dry_run:
        return 0
    if args.only and RECORD.exists():
        # classes not re-tuned keep their earlier timings in the record
        kept = [e for e in json.loads(RECORD.read_text()).get("classes", []) if e["P"] not in args.only]
        record["classes"] = sorted(kept + record["classes"], key=lambda e: e["P"])
    write_outputs(best, record)
    if not args.no_build:
        build.build_engine(force=True)
    print(f"wrote {CLASS_INC.relative_to(PKG.parent)} and {RECORD.relative_to(PKG.parent)}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
