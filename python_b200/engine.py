"""ctypes binding of the engine's C ABI (``include/sirocco_solve.h``).

This is the same boundary a C host links against; the Python side only moves
numpy / torch buffers across it.  The engine library is required: importing
this module on a machine where ``libsirocco_solve.so`` is missing raises.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int, c_int64, c_void_p
from pathlib import Path

import numpy as np

from .workloads import Batch

LIB_PATH = Path(__file__).resolve().parent / "libsirocco_solve.so"

FP64 = 0
MIXED = 1
FAST = 2
SOLVE = 0
INVERT = 1

# every symbol include/sirocco_solve.h declares
EXPORTS = (
    "solve_matrix", "invert_matrix", "get_matrix_error_string",
    "cusolver_create", "cusolver_destroy", "cusolver_get_error_string",
    "gpu_solve_matrix", "gpu_invert_matrix",
    "solve_matrix_batched", "invert_matrix_batched", "sirocco_set_precision",
    "sirocco_plan_create", "sirocco_plan_execute", "sirocco_plan_launches",
    "sirocco_plan_destroy", "sirocco_last_error", "solve_matrix_batched_noalloc",
    "matom_matrices_batched", "matom_sample_batched", "ion_populations_lockstep", "macro_pops_lockstep",
    "ion_rate_matrices_batched", "ion_populations_lockstep_rates", "matom_rate_matrices_batched",
)

_lib = None

# assembly callback of ion_populations_lockstep
MACRO_ASSEMBLE_FN = ctypes.CFUNCTYPE(c_int, c_void_p, c_int, POINTER(c_int), POINTER(c_int), POINTER(c_double))
ASSEMBLE_FN = ctypes.CFUNCTYPE(c_int, c_void_p, c_int, POINTER(c_int), POINTER(c_double), POINTER(c_double),
                               POINTER(c_double), POINTER(c_double), POINTER(c_double))


class IonTableC(ctypes.Structure):
    """sirocco_ion_table (include/sirocco_solve.h)."""
    _fields_ = [("nions", c_int), ("nelem", c_int), ("elem_z", c_void_p), ("elem_first", c_void_p),
                ("elem_n", c_void_p), ("elem_istate_max", c_void_p), ("ion_istate", c_void_p), ("ion_di", c_void_p),
                ("ion_dr", c_void_p), ("n_inner", c_int), ("inner_nion", c_void_p), ("inner_yield", c_void_p),
                ("n_yield", c_int), ("yield_prob", c_void_p), ("ncx", c_int), ("cx_nion1", c_void_p),
                ("cx_nion2", c_void_p)]


class IonRatesC(ctypes.Structure):
    """sirocco_ion_rates (include/sirocco_solve.h)."""
    _fields_ = [(k, c_void_p) for k in ("pi", "rr", "di", "qr", "dr", "cxr", "cxi", "inner")]


class MatomTableC(ctypes.Structure):
    """sirocco_matom_table (include/sirocco_solve.h)."""
    _fields_ = [("nlev", c_int), ("ex", c_void_p), ("bbd_start", c_void_p), ("bbd_target", c_void_p),
                ("aug_start", c_void_p), ("aug_target", c_void_p), ("aug_rate", c_void_p), ("bfd_start", c_void_p),
                ("bfd_target", c_void_p), ("bbu_start", c_void_p), ("bbu_target", c_void_p), ("bfu_start", c_void_p),
                ("bfu_target", c_void_p), ("n_kbb", c_int), ("n_kbf", c_int), ("kbb_target", c_void_p),
                ("kbf_target", c_void_p)]


MATOM_RATE_FIELDS = ("bbd_rad", "bbd_coll", "bfd_sp", "bfd_qrec", "bbu_rad", "bbu_coll", "bfu_gamma", "bfu_alpha",
                     "bfu_ratio", "bfu_qion", "kbb", "kbf", "kr", "ne")


class MatomRatesC(ctypes.Structure):
    """sirocco_matom_rates (include/sirocco_solve.h)."""
    _fields_ = [(k, c_void_p) for k in MATOM_RATE_FIELDS]


class EngineError(RuntimeError):
    pass


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise EngineError(f"engine library not built: {LIB_PATH} (run python -m python_b200.build)")
    lib = ctypes.CDLL(str(LIB_PATH))
    dp = POINTER(c_double)
    lib.solve_matrix.argtypes = [dp, dp, c_int, dp, c_int]
    lib.solve_matrix.restype = c_int
    lib.invert_matrix.argtypes = [dp, dp, c_int]
    lib.invert_matrix.restype = c_int
    lib.gpu_solve_matrix.argtypes = [dp, dp, c_int, dp]
    lib.gpu_solve_matrix.restype = c_int
    lib.gpu_invert_matrix.argtypes = [dp, dp, c_int]
    lib.gpu_invert_matrix.restype = c_int
    lib.get_matrix_error_string.argtypes = [c_int]
    lib.get_matrix_error_string.restype = c_char_p
    lib.cusolver_get_error_string.argtypes = [c_int]
    lib.cusolver_get_error_string.restype = c_char_p
    lib.cusolver_create.restype = c_int
    lib.cusolver_destroy.restype = c_int
    lib.solve_matrix_batched.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.solve_matrix_batched.restype = c_int
    lib.invert_matrix_batched.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.invert_matrix_batched.restype = c_int
    lib.sirocco_set_precision.argtypes = [c_int]
    lib.sirocco_set_precision.restype = c_int
    lib.sirocco_plan_create.argtypes = [POINTER(c_void_p), c_int, c_int, c_void_p, c_void_p, c_void_p, c_int]
    lib.sirocco_plan_create.restype = c_int
    lib.sirocco_plan_execute.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.sirocco_plan_execute.restype = c_int
    lib.sirocco_plan_launches.argtypes = [c_void_p]
    lib.sirocco_plan_launches.restype = c_int
    lib.sirocco_plan_destroy.argtypes = [c_void_p]
    lib.sirocco_plan_destroy.restype = c_int
    lib.sirocco_last_error.restype = c_char_p
    lib.solve_matrix_batched_noalloc.argtypes = [c_int, c_int] + [c_void_p] * 8
    lib.solve_matrix_batched_noalloc.restype = c_int
    lib.matom_matrices_batched.argtypes = [c_int] + [c_void_p] * 8
    lib.matom_matrices_batched.restype = c_int
    lib.matom_sample_batched.argtypes = [c_int, c_int] + [c_void_p] * 7
    lib.matom_sample_batched.restype = c_int
    lib.ion_populations_lockstep.argtypes = [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                                             c_void_p, c_void_p, ASSEMBLE_FN, c_void_p, c_void_p, c_void_p]
    lib.ion_populations_lockstep.restype = c_int
    lib.ion_rate_matrices_batched.argtypes = [POINTER(IonTableC), c_int, POINTER(IonRatesC)] + [c_void_p] * 5
    lib.ion_rate_matrices_batched.restype = c_int
    lib.ion_populations_lockstep_rates.argtypes = [POINTER(IonTableC), c_int, POINTER(IonRatesC), c_int] + \
        [c_void_p] * 5
    lib.ion_populations_lockstep_rates.restype = c_int
    lib.matom_rate_matrices_batched.argtypes = [POINTER(MatomTableC), c_int, POINTER(MatomRatesC), c_void_p, c_void_p]
    lib.matom_rate_matrices_batched.restype = c_int
    lib.macro_pops_lockstep.argtypes = [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                        MACRO_ASSEMBLE_FN, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.macro_pops_lockstep.restype = c_int
    _lib = lib
    return lib


def last_error() -> str:
    return load().sirocco_last_error().decode()


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise EngineError(f"{what} failed with {rc}: {last_error()}")


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(c_void_p)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_double))


# --------------------------------------------------------------- drop-in ----
def solve_matrix(a: np.ndarray, b: np.ndarray, x: np.ndarray | None = None, nplasma: int = 0):
    """Drop-in solve_matrix on one system; returns (code, x)."""
    lib = load()
    a = np.ascontiguousarray(a, np.float64).copy()
    b = np.ascontiguousarray(b, np.float64)
    n = b.size
    if x is None:
        x = np.full(n, np.nan)
    code = lib.solve_matrix(_dptr(a), _dptr(b), n, _dptr(x), nplasma)
    return code, x


def invert_matrix(m: np.ndarray, out: np.ndarray | None = None):
    """Drop-in invert_matrix on one system; returns (code, inverse)."""
    lib = load()
    m = np.ascontiguousarray(m, np.float64).copy()
    n = m.shape[0]
    if out is None:
        out = np.full((n, n), np.nan)
    code = lib.invert_matrix(_dptr(m), _dptr(out), n)
    return code, out


def error_string(code: int) -> str:
    return load().get_matrix_error_string(code).decode()


# --------------------------------------------------------------- batched ----
def set_precision(mode: int) -> None:
    _check(load().sirocco_set_precision(mode), "sirocco_set_precision")


def solve_batched(batch: Batch, mode: int = FP64, x: np.ndarray | None = None):
    """Host-buffer batched solve through solve_matrix_batched; returns (x, status)."""
    lib = load()
    set_precision(mode)
    n = np.ascontiguousarray(batch.n, np.int32)
    if x is None:
        x = np.full(batch.b.size, np.nan)
    st = np.full(batch.nsys, -99, np.int32)
    rc = lib.solve_matrix_batched(batch.nsys, _ptr(n), _ptr(batch.offA), _ptr(batch.A), _ptr(batch.offv),
                                  _ptr(batch.b), _ptr(x), _ptr(st))
    _check(rc, "solve_matrix_batched")
    return x, st


def invert_batched(batch: Batch, mode: int = FP64, out: np.ndarray | None = None):
    """Host-buffer batched inverse through invert_matrix_batched; returns (inverses, status)."""
    lib = load()
    set_precision(mode)
    n = np.ascontiguousarray(batch.n, np.int32)
    if out is None:
        out = np.full(batch.A.size, np.nan)
    st = np.full(batch.nsys, -99, np.int32)
    rc = lib.invert_matrix_batched(batch.nsys, _ptr(n), _ptr(batch.offA), _ptr(batch.A), _ptr(out), _ptr(st))
    _check(rc, "invert_matrix_batched")
    return out, st


def matom_matrices(batch: Batch, R: np.ndarray, offv: np.ndarray, cumulative: bool = True, mode: int = FP64):
    """B = N^-1 diag(R) per cell and its row running totals through
    matom_matrices_batched in precision mode `mode`; returns (B, C or None, status)."""
    lib = load()
    set_precision(mode)
    n = np.ascontiguousarray(batch.n, np.int32)
    offv = np.ascontiguousarray(offv, np.int64)
    R = np.ascontiguousarray(R, np.float64)
    B = np.full(batch.A.size, np.nan)
    C = np.full(batch.A.size, np.nan) if cumulative else None
    st = np.full(batch.nsys, -99, np.int32)
    rc = lib.matom_matrices_batched(batch.nsys, _ptr(n), _ptr(batch.offA), _ptr(offv), _ptr(batch.A), _ptr(R),
                                    _ptr(B), _ptr(C) if C is not None else None, _ptr(st))
    _check(rc, "matom_matrices_batched")
    return B, C, st


def matom_sample(n: np.ndarray, offA: np.ndarray, C: np.ndarray, sys: np.ndarray, level: np.ndarray,
                 z: np.ndarray) -> np.ndarray:
    """Deactivation targets of a batch of draws through matom_sample_batched."""
    lib = load()
    n = np.ascontiguousarray(n, np.int32)
    offA = np.ascontiguousarray(offA, np.int64)
    sys = np.ascontiguousarray(sys, np.int32)
    level = np.ascontiguousarray(level, np.int32)
    z = np.ascontiguousarray(z, np.float64)
    C = np.ascontiguousarray(C, np.float64)
    target = np.full(sys.size, -99, np.int32)
    rc = lib.matom_sample_batched(sys.size, n.size, _ptr(n), _ptr(offA), _ptr(C), _ptr(sys), _ptr(level), _ptr(z),
                                  _ptr(target))
    _check(rc, "matom_sample_batched")
    return target


def ion_populations_lockstep(elem_first, elem_n, istate, h_elem: int, elem_dens: np.ndarray, ne: np.ndarray,
                             den: np.ndarray, assemble):
    """The n_e iteration of every cell at once (ion_populations_lockstep).

    ``assemble(cells, ne, nh1, nh2, A, b)`` fills, in place, the per-element
    rate-matrix blocks of the listed cells (A, packed cell after cell, each
    block row-major) and their right-hand sides (b, nions per cell).
    ``ne`` [ncell] and ``den`` [ncell, nions] are updated in place for the cells
    that converge; returns (status, iters).
    """
    import traceback
    lib = load()
    elem_first = np.ascontiguousarray(elem_first, np.int32)
    elem_n = np.ascontiguousarray(elem_n, np.int32)
    istate = np.ascontiguousarray(istate, np.int32)
    elem_dens = np.ascontiguousarray(elem_dens, np.float64)
    assert ne.dtype == np.float64 and ne.flags.c_contiguous and den.dtype == np.float64 and den.flags.c_contiguous
    ncell, nions = den.shape
    blk = int((elem_n.astype(np.int64) ** 2).sum())

    def cb(user, n, cells, ne_p, nh1_p, nh2_p, a_p, b_p):
        try:
            assemble(np.ctypeslib.as_array(cells, (n,)).copy(), np.ctypeslib.as_array(ne_p, (n,)).copy(),
                     np.ctypeslib.as_array(nh1_p, (n,)).copy(), np.ctypeslib.as_array(nh2_p, (n,)).copy(),
                     np.ctypeslib.as_array(a_p, (n * blk,)), np.ctypeslib.as_array(b_p, (n * nions,)))
            return 0
        except Exception:
            traceback.print_exc()
            return 1
    fn = ASSEMBLE_FN(cb)
    status = np.full(ncell, -99, np.int32)
    iters = np.zeros(ncell, np.int32)
    rc = lib.ion_populations_lockstep(ncell, nions, elem_n.size, _ptr(elem_first), _ptr(elem_n), _ptr(istate), h_elem,
                                      _ptr(elem_dens), _ptr(ne), _ptr(den), fn, None, _ptr(status), _ptr(iters))
    _check(rc, "ion_populations_lockstep")
    return status, iters


def _ion_c(tab, rates):
    """The C views of a workloads.IonTable / IonRates and the arrays they point into."""
    i32 = lambda a: np.ascontiguousarray(a, np.int32)
    f64 = lambda a: np.ascontiguousarray(a, np.float64)
    keep = dict(elem_z=i32(tab.elem_z), elem_first=i32(tab.elem_first), elem_n=i32(tab.elem_n),
                elem_istate_max=i32(tab.elem_istate_max), ion_istate=i32(tab.ion_istate), ion_di=i32(tab.ion_di),
                ion_dr=i32(tab.ion_dr), inner_nion=i32(tab.inner_nion), inner_yield=i32(tab.inner_yield),
                yield_prob=f64(tab.yield_prob).reshape(-1), cx_nion1=i32(tab.cx_nion1), cx_nion2=i32(tab.cx_nion2))
    t = IonTableC(tab.nions, tab.nelem, *[keep[k].ctypes.data for k in (
        "elem_z", "elem_first", "elem_n", "elem_istate_max", "ion_istate", "ion_di", "ion_dr")],
        tab.n_inner, keep["inner_nion"].ctypes.data, keep["inner_yield"].ctypes.data, len(tab.yield_prob),
        keep["yield_prob"].ctypes.data, tab.ncx, keep["cx_nion1"].ctypes.data, keep["cx_nion2"].ctypes.data)
    rk = {k: f64(getattr(rates, k)) for k in ("pi", "rr", "di", "qr", "dr", "cxr", "cxi", "inner")}
    r = IonRatesC(*[rk[k].ctypes.data for k in ("pi", "rr", "di", "qr", "dr", "cxr", "cxi", "inner")])
    return t, r, (keep, rk)


def matom_rate_matrices(inp: dict, N=None, R=None):
    """The Q / R assembly and normalisation of calc_matom_matrix on the GPU
    (matom_rate_matrices_batched) from workloads.matom_jump_inputs arrays:
    returns (N [ncell, nlev+1, nlev+1], R [ncell, nlev+1]).  N and R may be
    given as device tensors (torch) to keep the result on the GPU."""
    lib = load()
    nlev, ncell = int(inp["nlev"]), int(inp["ncell"])
    a = {k: np.ascontiguousarray(v) for k, v in inp.items() if isinstance(v, np.ndarray)}
    ptr = lambda k: a[k].ctypes.data if a[k].size else None
    t = MatomTableC(nlev, ptr("ex"), ptr("bbd_start"), ptr("bbd_target"), ptr("aug_start"), ptr("aug_target"),
                    ptr("aug_rate"), ptr("bfd_start"), ptr("bfd_target"), ptr("bbu_start"), ptr("bbu_target"),
                    ptr("bfu_start"), ptr("bfu_target"), int(a["kbb_target"].size), int(a["kbf_target"].size),
                    ptr("kbb_target"), ptr("kbf_target"))
    r = MatomRatesC(*[ptr(k) for k in MATOM_RATE_FIELDS])
    nr = nlev + 1
    if N is None:
        N = np.empty((ncell, nr, nr), np.float64)
        R = np.empty((ncell, nr), np.float64)
        pn, pr = _ptr(N), _ptr(R)
    else:
        pn, pr = c_void_p(N.data_ptr()), c_void_p(R.data_ptr())
    rc = lib.matom_rate_matrices_batched(ctypes.byref(t), ncell, ctypes.byref(r), pn, pr)
    _check(rc, "matom_rate_matrices_batched")
    return N, R


def ion_rate_matrices(tab, rates, ne, nh1, nh2):
    """populate_ion_rate_matrix on the GPU for every cell of ``rates``
    (ion_rate_matrices_batched): returns (A, b), A the cells' element blocks
    packed cell after cell, b [ncell, nions]."""
    lib = load()
    t, r, keep = _ion_c(tab, rates)
    ncell = rates.ncell
    blk = int((np.asarray(tab.elem_n, np.int64) ** 2).sum())
    ne, nh1, nh2 = (np.ascontiguousarray(a, np.float64) for a in (ne, nh1, nh2))
    A = np.empty(ncell * blk, np.float64)
    b = np.empty((ncell, tab.nions), np.float64)
    rc = lib.ion_rate_matrices_batched(ctypes.byref(t), ncell, ctypes.byref(r), _ptr(ne), _ptr(nh1), _ptr(nh2),
                                       _ptr(A), _ptr(b))
    _check(rc, "ion_rate_matrices_batched")
    del keep
    return A, b


def ion_populations_lockstep_rates(tab, rates, h_elem: int, elem_dens: np.ndarray, ne: np.ndarray, den: np.ndarray):
    """ion_populations_lockstep with the rate matrices assembled on the GPU
    (ion_populations_lockstep_rates).  ``ne`` and ``den`` are updated in place
    for the cells that converge; returns (status, iters)."""
    lib = load()
    t, r, keep = _ion_c(tab, rates)
    elem_dens = np.ascontiguousarray(elem_dens, np.float64)
    assert ne.dtype == np.float64 and ne.flags.c_contiguous and den.dtype == np.float64 and den.flags.c_contiguous
    ncell = den.shape[0]
    status = np.full(ncell, -99, np.int32)
    iters = np.zeros(ncell, np.int32)
    rc = lib.ion_populations_lockstep_rates(ctypes.byref(t), ncell, ctypes.byref(r), h_elem, _ptr(elem_dens),
                                            _ptr(ne), _ptr(den), _ptr(status), _ptr(iters))
    _check(rc, "ion_populations_lockstep_rates")
    del keep
    return status, iters


def macro_pops_lockstep(ion_first, ion_nlte, g, radiative: np.ndarray, scale: np.ndarray, ncell: int, assemble):
    """Level populations of one macro element in every cell (macro_pops_lockstep).

    ``assemble(cells, attempt, A)`` fills, in place, the n x n rate matrices
    of the listed cells (A packed cell after cell).  Returns (pop [ncell, n],
    status, iters).
    """
    import traceback
    lib = load()
    ion_first = np.ascontiguousarray(ion_first, np.int32)
    ion_nlte = np.ascontiguousarray(ion_nlte, np.int32)
    g = np.ascontiguousarray(g, np.float64)
    rad = np.ascontiguousarray(radiative, np.uint8)
    scale = np.ascontiguousarray(scale, np.float64)
    n = g.size

    def cb(user, k, cells, att, a_p):
        try:
            assemble(np.ctypeslib.as_array(cells, (k,)).copy(), np.ctypeslib.as_array(att, (k,)).copy(),
                     np.ctypeslib.as_array(a_p, (k * n * n,)))
            return 0
        except Exception:
            traceback.print_exc()
            return 1
    fn = MACRO_ASSEMBLE_FN(cb)
    pop = np.full((ncell, n), np.nan)
    status = np.full(ncell, -99, np.int32)
    iters = np.zeros(ncell, np.int32)
    rc = lib.macro_pops_lockstep(ncell, n, ion_first.size, _ptr(ion_first), _ptr(ion_nlte), _ptr(g), _ptr(rad),
                                 _ptr(scale), fn, None, _ptr(pop), _ptr(status), _ptr(iters))
    _check(rc, "macro_pops_lockstep")
    return pop, status, iters


class Plan:
    """A device-resident plan (sirocco_plan_*) over one batch layout.

    ``execute`` takes torch CUDA tensors (or raw device addresses) and enqueues
    the whole batch on the given stream (default: torch's current stream).
    """

    def __init__(self, batch: Batch, mode: int = FP64):
        lib = load()
        self.kind = SOLVE if batch.kind == "solve" else INVERT
        self._n = np.ascontiguousarray(batch.n, np.int32)
        self._offA = np.ascontiguousarray(batch.offA, np.int64)
        self._offv = np.ascontiguousarray(batch.offv if batch.offv is not None else np.zeros(batch.nsys), np.int64)
        h = c_void_p()
        rc = lib.sirocco_plan_create(ctypes.byref(h), self.kind, batch.nsys, _ptr(self._n), _ptr(self._offA),
                                     _ptr(self._offv), mode)
        _check(rc, "sirocco_plan_create")
        self._h = h
        self.nsys = batch.nsys
        self.launches = lib.sirocco_plan_launches(h)

    def execute(self, A, out, status, b=None, diag=None, stream=None) -> None:
        def addr(t):
            if t is None:
                return None
            return c_void_p(t if isinstance(t, int) else t.data_ptr())
        if stream is None:
            import torch
            stream = torch.cuda.current_stream().cuda_stream
        elif not isinstance(stream, int):
            stream = stream.cuda_stream
        rc = load().sirocco_plan_execute(self._h, addr(A), addr(b), addr(out), addr(status), addr(diag),
                                         c_void_p(stream))
        _check(rc, "sirocco_plan_execute")

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().sirocco_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
