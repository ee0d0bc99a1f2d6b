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


# ------------------------------------------------------- ion rate matrices --
ION_LIB = HERE / "_ref" / "libref_ionmat.so"


def ion_rate_matrix(tab, rates, cell: int, xne: float, nh1: float, nh2: float):
    """Restatement of populate_ion_rate_matrix (source/matrix_ion.c:444-659)
    for one cell: the full nions x nions matrix and the right-hand side, each
    entry accumulated block by block in the routine's order (photoionisation,
    direct ionisation, radiative + three-body recombination, dielectronic
    recombination, charge-exchange recombination and ionisation, inner-shell
    ionisation), then each element's first row replaced by ones (:633-655).
    Python floats round every product and sum separately, as the reference's
    x86-64 build does.  `tab` and `rates` follow python_b200.workloads.IonTable
    / IonRates."""
    n = tab.nions
    elem_of = tab.elem_of()
    z = [int(tab.elem_z[elem_of[i]]) for i in range(n)]
    first = [int(tab.elem_first[elem_of[i]]) for i in range(n)]
    imax = [int(tab.elem_istate_max[elem_of[i]]) for i in range(n)]
    ist = [int(v) for v in tab.ion_istate]
    pi, rr = [float(v) for v in rates.pi[cell]], [float(v) for v in rates.rr[cell]]
    di, qr, dr = [float(v) for v in rates.di[cell]], [float(v) for v in rates.qr[cell]], [float(v) for v in rates.dr[cell]]
    cxr = [float(v) for v in rates.cxr[cell]]
    cxi = [float(v) for v in rates.cxi[cell]]
    inner = [float(v) for v in rates.inner[cell]]
    m = [[0.0] * n for _ in range(n)]
    for mm in range(n):                                   # PI depopulates (:477-483)
        if ist[mm] != imax[mm]:
            m[mm][mm] -= pi[mm]
    for nn in range(n - 1):                               # PI populates (:487-497)
        if ist[nn] != imax[nn] and z[nn + 1] == z[nn]:
            m[nn + 1][nn] += pi[nn]
    for mm in range(n):                                   # DI depopulates (:501-507)
        if ist[mm] != imax[mm] and tab.ion_di[mm] > 0:
            m[mm][mm] -= xne * di[mm]
    for nn in range(n - 1):                               # DI populates (:511-520)
        if ist[nn] != imax[nn] and z[nn + 1] == z[nn] and tab.ion_di[nn] > 0:
            m[nn + 1][nn] += xne * di[nn]
    for mm in range(n):                                   # RR depopulates (:525-531)
        if mm != first[mm]:
            m[mm][mm] -= xne * (rr[mm] + xne * qr[mm])
    for nn in range(1, n):                                # RR populates (:535-544)
        if nn != first[nn] and z[nn - 1] == z[nn]:
            m[nn - 1][nn] += xne * (rr[nn] + xne * qr[nn])
    for mm in range(n):                                   # DR depopulates (:548-554)
        if mm != first[mm] and tab.ion_dr[mm] > 0:
            m[mm][mm] -= xne * dr[mm]
    for nn in range(1, n):                                # DR populates, flag of the lower ion (:562-572)
        if nn != first[nn] and z[nn - 1] == z[nn] and tab.ion_dr[nn - 1] > 0:
            m[nn - 1][nn] += xne * dr[nn]
    if tab.ncx > 0:                                       # charge-exchange recombination (:576-586)
        for mm in range(n):
            if z[mm] != 1 and ist[mm] != 0:
                m[mm][mm] -= cxr[mm] * nh1
                m[mm - 1][mm] += cxr[mm] * nh1
    for k in range(tab.ncx):                              # charge-exchange ionisation (:590-596)
        if z[int(tab.cx_nion2[k])] == 1:
            o = int(tab.cx_nion1[k])
            m[o][o] -= cxi[k] * nh2
            m[o + 1][o] += cxi[k] * nh2
    for k in range(tab.n_inner):                          # inner-shell ionisation (:599-613)
        y = int(tab.inner_yield[k])
        if y != -1:
            o = int(tab.inner_nion[k])
            m[o][o] -= inner[k]
            ne_ = min(z[o] - ist[o] + 1, 11)
            for d in range(1, ne_):
                m[o + d][o] += inner[k] * float(tab.yield_prob[y][d - 1])
    b = [0.0] * n
    for nn in range(n):                                   # first row of each element (:633-655)
        if nn == first[nn]:
            b[nn] = 1.0
            for mm in range(n):
                m[nn][mm] = 1.0 if z[mm] == z[nn] else 0.0
    return np.array(m, dtype=np.float64), np.array(b, dtype=np.float64)


def ion_reference_available() -> bool:
    return ION_LIB.exists()


def ref_ion_rate_matrix(tab, rates, cell: int, xne: float, nh1: float, nh2: float):
    """The reference's own populate_ion_rate_matrix (oracle/_ref/libref_ionmat.so)
    on the same inputs: (A, b, return value)."""
    lib = ctypes.CDLL(str(ION_LIB))
    f = lib.refion_assemble
    f.restype = c_int
    n = tab.nions
    A = np.zeros((n, n), dtype=np.float64)
    b = np.zeros(n, dtype=np.float64)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    elem_of = i32(tab.elem_of())
    args = [i32(tab.elem_z), i32(tab.elem_first), i32(tab.elem_istate_max), elem_of, i32(tab.ion_istate),
            i32(tab.ion_di), i32(tab.ion_dr)]
    inner_nion, inner_yield = i32(tab.inner_nion), i32(tab.inner_yield)
    yp = f64(tab.yield_prob).reshape(-1)
    cx1, cx2 = i32(tab.cx_nion1), i32(tab.cx_nion2)
    cells = [f64(getattr(rates, k)[cell]) for k in ("pi", "rr", "di", "qr", "dr", "cxr", "cxi", "inner")]
    keep = args + [inner_nion, inner_yield, yp, cx1, cx2] + cells + [A, b]
    rc = f(c_int(n), c_int(tab.nelem), *[_p(a) for a in args], c_int(tab.n_inner), _p(inner_nion), _p(inner_yield),
           c_int(len(tab.yield_prob)), _p(yp), c_int(tab.ncx), _p(cx1), _p(cx2), *[_p(a) for a in cells],
           ctypes.c_double(xne), ctypes.c_double(nh1), ctypes.c_double(nh2), _p(A), _p(b))
    del keep
    return A, b, rc


# ------------------------------------------------- macro-atom jump matrices --
MATOM_LIB = HERE / "_ref" / "libref_matom.so"
# the same reference routine with its invert_matrix resolved by the engine
# (python_b200/libsirocco_solve.so) through the drop-in C ABI
MATOM_DROPIN_LIB = HERE / "_ref" / "libref_matom_dropin.so"


def matom_density_ratio(m, cell, density_phot_min: float = 1e-10):
    """Per upward bound-free jump, the upper / lower density ratio of
    calc_matom_matrix (macro_accelerate.c:203-210): zero below DENSITY_PHOT_MIN."""
    out = []
    for u in range(m.nlev):
        for i in m.bfu[u]:
            lo = float(cell.den[m.phot_lo[i]])
            out.append(float(cell.den[m.phot_up[i]]) / lo if lo >= density_phot_min else 0.0)
    return np.array(out, dtype=np.float64)


def matom_kr(m, cell) -> float:
    """The k-packet to r-packet rate of calc_matom_matrix (:224-254), summed in
    the routine's order: simple lines, simple continua, then the other coolings."""
    kr = 0.0
    for i in range(m.line_lo.size):
        if not m.line_macro[i]:
            kr += float(cell.cool_bb[i])
    for i in range(m.phot_lo.size):
        if not m.phot_macro[i]:
            kr += float(cell.cool_bf[i])
    kr += cell.cool_bftot
    kr += cell.cool_adiabatic
    kr += cell.cool_ff + cell.cool_ff_lofreq
    return kr


def matom_rate_matrix(m, cell, density_phot_min: float = 1e-10):
    """Restatement of the Q / R assembly and normalisation of calc_matom_matrix
    (source/macro_accelerate.c:82-300) for one cell: N = I - Q / Q_norm
    ((nlev + 1)^2, row-major, the k-packet row and column last) and the
    diagonal of R / Q_norm.  Each sum and product is rounded separately, in the
    routine's order."""
    n = m.nlev
    K = n
    ex = [float(v) for v in m.ex]
    ne = float(cell.ne)
    Q = [[0.0] * (n + 1) for _ in range(n + 1)]
    R = [0.0] * (n + 1)
    qn = [0.0] * (n + 1)
    ratio = matom_density_ratio(m, cell, density_phot_min)
    ibu = ifu = ifd = 0
    for u in range(n):
        for i in m.bbd[u]:                                   # bound-bound down (:98-123)
            rad = float(cell.a21[i]) * float(cell.pesc[i])
            coll = float(cell.q21[i])
            bb = rad + coll * ne
            t = int(m.line_lo[i])
            qc = bb * ex[t]
            Q[u][t] += qc
            qk = (coll * ne) * (ex[u] - ex[t])
            Q[u][K] += qk
            rc = rad * (ex[u] - ex[t])
            R[u] += rc
            qn[u] += qc + qk + rc
        if m.aug_idx[u] >= 0:                                # Auger (:126-145)
            a = int(m.aug_idx[u])
            for k in range(int(m.n_aug[u])):
                t = int(m.aug_target[a][k])
                rate = float(m.aug_A[a]) * float(m.aug_branch[a][k])
                qc = rate * ex[t]
                Q[u][t] += qc
                qk = rate * (ex[u] - ex[t])
                Q[u][K] += qk
                qn[u] += qc + qk
        for i in m.bfd[u]:                                   # bound-free down (:148-174)
            sp = float(cell.recomb_sp[ifd])
            ifd += 1
            qr = float(cell.qrec[i])
            bf = (sp + qr * ne) * ne
            t = int(m.phot_lo[i])
            if bf > 0.0:
                qc = bf * ex[t]
                Q[u][t] += qc
                qk = qr * ne * ne * (ex[u] - ex[t])
                Q[u][K] += qk
                rc = ne * sp * (ex[u] - ex[t])
                R[u] += rc
                qn[u] += qc + qk + rc
        for i in m.bbu[u]:                                   # bound-bound up (:179-191)
            rad = float(cell.b12[i]) * float(cell.jbar[ibu])
            ibu += 1
            coll = float(cell.q12[i])
            t = int(m.line_up[i])
            qc = (rad + coll * ne) * ex[u]
            Q[u][t] += qc
            qn[u] += qc
        for i in m.bfu[u]:                                   # bound-free up (:194-222)
            t = int(m.phot_up[i])
            qc = (float(cell.gamma[ifu]) - float(cell.alpha_st[ifu]) * ne * float(ratio[ifu]) +
                  float(cell.qion[i]) * ne) * ex[u]
            ifu += 1
            if qc < 0.0:
                qc = 0.0
            Q[u][t] += qc
            qn[u] += qc
    for i in range(m.line_lo.size):                          # k-packet row (:236-263)
        if m.line_macro[i]:
            qc = float(cell.cool_bb[i])
            Q[K][int(m.line_up[i])] += qc
            qn[K] += qc
    for i in range(m.phot_lo.size):
        if m.phot_macro[i]:
            qc = float(cell.cool_bf[i])
            Q[K][int(m.phot_up[i])] += qc
            qn[K] += qc
    kr = matom_kr(m, cell)
    R[K] += kr
    qn[K] += kr
    for u in range(n + 1):                                   # N = I - Q / Q_norm (:270-284)
        for t in range(n + 1):
            if qn[u] > 0.0:
                Q[u][t] = -1.0 * Q[u][t] / qn[u]
        Q[u][u] = 1.0
        if qn[u] > 0.0:
            R[u] = R[u] / qn[u]
    return np.array(Q, dtype=np.float64), np.array(R, dtype=np.float64)


def matom_reference_available() -> bool:
    return MATOM_LIB.exists()


def ref_matom_b(m, cell, density_phot_min: float = 1e-10, dropin: bool = False):
    """The reference's own calc_matom_matrix (oracle/_ref/libref_matom.so) on the
    same model and coefficients: B = N^-1 diag(R), (nlev + 1)^2 row-major.  With
    dropin, the build whose invert_matrix is the engine's (libref_matom_dropin.so)."""
    lib = ctypes.CDLL(str(MATOM_DROPIN_LIB if dropin else MATOM_LIB))
    f = lib.refmatom_b
    f.restype = c_int
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    n = m.nlev
    cnt = lambda L: i32([len(v) for v in L])
    flat = lambda L: i32([i for v in L for i in v] or [0])
    arrs = [f64(m.ex), cnt(m.bbd), flat(m.bbd), cnt(m.bbu), flat(m.bbu), cnt(m.bfd), flat(m.bfd), cnt(m.bfu),
            flat(m.bfu), i32(m.aug_idx), i32(m.n_aug)]
    aug = [i32(m.aug_target.reshape(-1) if m.aug_target.size else [0]), f64(m.aug_A if m.aug_A.size else [0.0]),
           f64(m.aug_branch.reshape(-1) if m.aug_branch.size else [0.0])]
    lines = [i32(m.line_lo), i32(m.line_up), i32(m.line_macro)]
    phots = [i32(m.phot_lo), i32(m.phot_up), i32(m.phot_macro)]
    coef = [f64(getattr(cell, k)) for k in ("a21", "pesc", "q21", "b12", "q12", "qrec", "qion", "jbar", "gamma",
                                             "alpha_st", "recomb_sp", "den", "cool_bb", "cool_bf")]
    coef = [c if c.size else f64([0.0]) for c in coef]
    B = np.zeros((n + 1) * (n + 1), dtype=np.float64)
    rc = f(c_int(n), *[_p(a) for a in arrs], c_int(int(m.aug_A.size)), *[_p(a) for a in aug],
           c_int(int(m.line_lo.size)), *[_p(a) for a in lines], c_int(int(m.phot_lo.size)), *[_p(a) for a in phots],
           *[_p(a) for a in coef], ctypes.c_double(cell.cool_bftot), ctypes.c_double(cell.cool_adiabatic),
           ctypes.c_double(cell.cool_ff), ctypes.c_double(cell.cool_ff_lofreq), ctypes.c_double(cell.t_e),
           ctypes.c_double(cell.ne), ctypes.c_double(density_phot_min), _p(B))
    if rc != 0:
        raise RuntimeError(f"refmatom_b returned {rc}")
    return B.reshape(n + 1, n + 1)
