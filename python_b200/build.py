"""Build the engine's shared library in-tree (``python_b200/libsirocco_solve.so``)
for sm_100a with nvcc, and the CPU oracle used by the tests (``oracle/``).

    python -m python_b200.build            # engine + oracle (+ reference build when its tree is present)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libsirocco_solve.so"
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = [CSRC / "engine.cu"]
HEADERS = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.inc")) + [ROOT / "include" / "sirocco_solve.h"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_engine(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale(LIB, SOURCES + HEADERS + [Path(__file__)]):
        return LIB
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr",
           "-cudart", "static", "-o", str(LIB), *map(str, SOURCES)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    tmp = LIB.with_suffix(".so.tmp")
    cmd[cmd.index("-o") + 1] = str(tmp)
    subprocess.run(cmd, check=True, cwd=str(PKG))
    os.replace(tmp, LIB)
    return LIB


def build_oracle(reference: bool = True) -> None:
    targets = ["port"]
    # the reference checkout: SIROCCO_REFERENCE, else a `reference` directory
    # beside this repository's root; without it only the restatement is built
    ref_tree = Path(os.environ.get("SIROCCO_REFERENCE", str(ROOT.parent / "reference")))
    if reference and (ref_tree / "source" / "matrix_cpu.c").exists():
        targets.append("ref")
        if (ref_tree / "source" / "matrix_ion.c").exists():
            targets.append("refion")
        if (ref_tree / "source" / "macro_accelerate.c").exists():
            targets.append("refmatom")
            if LIB.exists():
                targets.append("refmatom_dropin")   # links the engine built above
        if (ref_tree / "source" / "matrix_gpu.cu").exists():
            targets.append("refgpu")
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), f"REF={ref_tree}", *targets], check=True)


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    build_engine(force="--force" in argv, verbose="-v" in argv)
    build_oracle()
    print(LIB)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
