"""Autotuner of the CTA kernel family's size classes.

For every padded order P listed in ``csrc/tune_candidates.inc`` the tuner
builds the tuning library (``csrc/tune.cu`` -> ``libsirocco_tune.so``), times
each candidate configuration on a device-resident batch of macro-atom
inverses at two orders of the class (its middle and its top), checks that all
candidates return the same bits and codes, and keeps the fastest.  It writes
``csrc/cta_classes.inc`` (the class table the engine compiles in) and
``tuned_classes.json`` (every timing), after which the engine is rebuilt.

    python -m python_b200.autotune            # on a B200; then commit the two files
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
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
    RECORD.write_text(json.dumps(record, indent=1) + "\n")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--only", type=int, nargs="*", help="tune only these padded orders (others keep their entry)")
    ap.add_argument("--dry-run", action="store_true", help="time and print, write nothing")
    ap.add_argument("--no-build", action="store_true", help="write the table but do not rebuild the engine")
    args = ap.parse_args(argv)
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
