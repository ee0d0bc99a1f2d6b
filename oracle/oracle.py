"""CPU ORACLE -- test infrastructure only.

ctypes access to the two CPU builds made by oracle/Makefile:
  * ``port``: the plain-C restatement of the reference's GSL path
    (oracle/gsl_lu_oracle.c), buildable anywhere gcc is present;
  * ``ref`` : the reference's own source/matrix_cpu.c + vendored GSL 2.6
    compiled from the reference tree (oracle/_ref/, present only where the
    reference tree was available when it was built).
It also loads the reference's cuSOLVER build (source/matrix_gpu.cu,
oracle/_ref/libref_cusolver.so) for ``bench.py``'s timed comparison with the
reference's own GPU path; that build is never used as a checker.
Only tests, ``__graft_entry__.smoke`` and the baseline legs of ``bench.py``
use this module, always as the checker or a timed baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import c_int, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_matrix.so"
CUSOLVER_LIB = HERE / "_ref" / "libref_cusolver.so"

_libs: dict = {}


def build_port() -> Path:
    if not PORT_LIB.exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    return PORT_LIB


def available(which: str) -> bool:
    return (PORT_LIB if which == "port" else REF_LIB).exists()


def _lib(which: str) -> ctypes.CDLL:
    if which not in _libs:
        path = build_port() if which == "port" else REF_LIB
        if not path.exists():
            raise FileNotFoundError(f"oracle library {path} not built")
        lib = ctypes.CDLL(str(path))
        pre = which + "_"
        getattr(lib, pre + "batch_solve").argtypes = [c_int] + [c_void_p] * 7 + [c_int]
        getattr(lib, pre + "batch_invert").argtypes = [c_int] + [c_void_p] * 5 + [c_int]
        getattr(lib, pre + "error_string").restype = ctypes.c_char_p
        _libs[which] = lib
    return _libs[which]


def _p(a):
    return a.ctypes.data_as(c_void_p)


def solve(batch, which: str = "port", threads: int = 1):
    """Serial solve_matrix on every system; returns (x, status)."""
    lib = _lib(which)
    n = np.ascontiguousarray(batch.n, np.int32)
    x = np.full(batch.b.size, np.nan)
    st = np.full(batch.nsys, -99, np.int32)
    getattr(lib, which + "_batch_solve")(batch.nsys, _p(n), _p(batch.offA), _p(batch.A), _p(batch.offv),
                                         _p(batch.b), _p(x), _p(st), threads)
    return x, st


def invert(batch, which: str = "port", threads: int = 1):
    """Serial invert_matrix on every system; returns (inverses, status)."""
    lib = _lib(which)
    n = np.ascontiguousarray(batch.n, np.int32)
    out = np.full(batch.A.size, np.nan)
    st = np.full(batch.nsys, -99, np.int32)
    getattr(lib, which + "_batch_invert")(batch.nsys, _p(n), _p(batch.offA), _p(batch.A), _p(out), _p(st), threads)
    return out, st


def error_string(code: int, which: str = "port") -> str:
    return getattr(_lib(which), which + "_error_string")(code).decode()


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ------------------------------------------- reference cuSOLVER build (timed) --
def cusolver_available() -> bool:
    return CUSOLVER_LIB.exists()


def _cusolver_lib() -> ctypes.CDLL:
    if "cusolver" not in _libs:
        lib = ctypes.CDLL(str(CUSOLVER_LIB))
        lib.refgpu_batch_solve.argtypes = [c_int] + [c_void_p] * 7
        lib.refgpu_batch_invert.argtypes = [c_int] + [c_void_p] * 5
        if lib.refgpu_create() != 0:
            raise RuntimeError("cusolver_create of the reference build failed")
        _libs["cusolver"] = lib
    return _libs["cusolver"]


def cusolver_solve(batch):
    """The reference's gpu_solve_matrix once per system; returns (x, status)."""
    lib = _cusolver_lib()
    n = np.ascontiguousarray(batch.n, np.int32)
    x = np.full(batch.b.size, np.nan)
    st = np.full(batch.nsys, -99, np.int32)
    if lib.refgpu_batch_solve(batch.nsys, _p(n), _p(batch.offA), _p(batch.A), _p(batch.offv), _p(batch.b),
                              _p(x), _p(st)) != 0:
        raise MemoryError("host scratch")
    return x, st


def cusolver_invert(batch):
    """The reference's gpu_invert_matrix once per system; returns (inverses, status)."""
    lib = _cusolver_lib()
    n = np.ascontiguousarray(batch.n, np.int32)
    out = np.full(batch.A.size, np.nan)
    st = np.full(batch.nsys, -99, np.int32)
    if lib.refgpu_batch_invert(batch.nsys, _p(n), _p(batch.offA), _p(batch.A), _p(out), _p(st)) != 0:
        raise MemoryError("host scratch")
    return out, st
