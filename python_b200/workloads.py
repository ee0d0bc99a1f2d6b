"""Seeded synthetic batches with the shapes and value distributions of the
per-cell systems that the reference solves.

Ion-balance systems follow the rate-matrix layout that
``populate_ion_rate_matrix`` builds (reference ``source/matrix_ion.c:445-659``):
``A[j][k]`` is the rate from stage k to stage j, each diagonal entry is minus
its column sum, and one row is replaced by ones with ``b`` the unit vector on
that row (number conservation, ``matrix_ion.c:633-655``).

Macro-atom systems follow ``calc_matom_matrix``
(``source/macro_accelerate.c:269-284``): ``N = I - Q`` where each row of the
jumping matrix ``Q`` sums to ``1 - p_deact`` and rows with no transitions are
identity rows.

All batches are float64, row-major, packed one system after another; the
packing offsets are returned beside them (``offA`` in elements of A,
``offv`` in elements of b / x).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BASE_SEED = 20261203
ION_SIZES_PER_CELL = (2, 3, 7, 8, 9, 11, 13, 15, 17, 27)


@dataclass
class Batch:
    kind: str                  # "solve" or "invert"
    n: np.ndarray              # int32 [nsys]
    offA: np.ndarray           # int64 [nsys], element offset of each matrix
    A: np.ndarray              # float64 [sum n^2]
    offv: np.ndarray | None = None   # int64 [nsys], element offset of b / x
    b: np.ndarray | None = None      # float64 [sum n]

    @property
    def nsys(self) -> int:
        return int(self.n.size)

    def matrix(self, s: int) -> np.ndarray:
        n = int(self.n[s])
        return self.A[self.offA[s]:self.offA[s] + n * n].reshape(n, n)

    def rhs(self, s: int) -> np.ndarray:
        n = int(self.n[s])
        return self.b[self.offv[s]:self.offv[s] + n]

    def flops(self) -> float:
        n = self.n.astype(np.float64)
        if self.kind == "solve":
            return float(np.sum(2.0 / 3.0 * n ** 3 + 2.0 * n ** 2))
        return float(np.sum(2.0 * n ** 3))

    def bytes(self) -> float:
        n = self.n.astype(np.float64)
        if self.kind == "solve":
            return float(np.sum(8.0 * (n ** 2 + 2 * n)))
        return float(np.sum(16.0 * n ** 2))


def offsets(n: np.ndarray, square: bool) -> np.ndarray:
    sz = n.astype(np.int64) ** 2 if square else n.astype(np.int64)
    off = np.zeros(n.size, np.int64)
    if n.size > 1:
        off[1:] = np.cumsum(sz[:-1])
    return off


def _loguniform(rng, lo, hi, size=None):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))


def ion_matrix(rng, n: int, spread=(1e-14, 1e2), auger=(1e-16, 1e-6),
               auger_frac=0.1, conservation="last"):
    """One ion-balance system of n stages (config-0 generator).

    Stage k ionises to k+1 at rate I_k and k+1 recombines to k at rate R_k,
    both log-uniform in ``spread``; a fraction ``auger_frac`` of the
    k -> k+2..k+4 entries carry a rate log-uniform in ``auger``.
    """
    a = np.zeros((n, n))
    if n > 1:
        ion = _loguniform(rng, *spread, n - 1)
        rec = _loguniform(rng, *spread, n - 1)
        k = np.arange(n - 1)
        a[k + 1, k] = ion
        a[k, k + 1] = rec
    for d in (2, 3, 4):
        if n > d:
            k = np.arange(n - d)
            hit = rng.random(n - d) < auger_frac
            a[k[hit] + d, k[hit]] = _loguniform(rng, *auger, int(hit.sum()))
    a[np.diag_indices(n)] = 0.0
    a[np.diag_indices(n)] = -a.sum(axis=0)
    b = np.zeros(n)
    row = n - 1 if conservation == "last" else 0
    a[row, :] = 1.0
    b[row] = 1.0
    return a, b


def macro_matrix(rng, n: int, density=0.25, qrange=(1e-8, 1.0),
                 pdeact=(1e-4, 0.5), identity_frac=0.03):
    """One macro-atom N = I - Q of order n (config-1 generator)."""
    q = np.where(rng.random((n, n)) < density, _loguniform(rng, *qrange, (n, n)), 0.0)
    q[np.diag_indices(n)] = 0.0
    empty = rng.random(n) < identity_frac
    q[empty] = 0.0
    rs = q.sum(axis=1)
    p = rng.uniform(*pdeact, n)
    scale = np.where(rs > 0, (1.0 - p) / np.where(rs > 0, rs, 1.0), 0.0)
    q *= scale[:, None]
    return np.eye(n) - q


def matom_cells(sizes, seed, density=0.25):
    """Macro-atom cells for the B = N^-1 diag(R) epilogue: N = I - Q/Q_norm from
    the config-1 generator and R the normalised deactivation rate of each level,
    so that R_u - sum_t N_ut = 0 (the normalisation calc_matom_matrix checks,
    source/macro_accelerate.c:288-300).  Returns (invert batch of N, R, offv)."""
    rng = np.random.default_rng(seed)
    mats = [macro_matrix(rng, int(n), density=density) for n in sizes]
    R = np.concatenate([m.sum(axis=1) for m in mats]) if mats else np.zeros(0)
    b = _pack("invert", mats)
    return b, R, offsets(np.asarray(b.n), False)


def _pack(kind, mats, rhs=None) -> Batch:
    n = np.array([m.shape[0] for m in mats], np.int32)
    offA = offsets(n, True)
    A = np.concatenate([m.ravel() for m in mats]) if mats else np.zeros(0)
    if kind == "solve":
        offv = offsets(n, False)
        b = np.concatenate(rhs) if rhs else np.zeros(0)
        return Batch(kind, n, offA, np.ascontiguousarray(A), offv, np.ascontiguousarray(b))
    return Batch(kind, n, offA, np.ascontiguousarray(A))


def config0(nsys=4096, n=27, seed=BASE_SEED + 0, conservation="last") -> Batch:
    """4,096 ion-balance systems of order 27, solved (plain FP64 solve_matrix)."""
    rng = np.random.default_rng(seed)
    mats, rhs = [], []
    for _ in range(nsys):
        a, b = ion_matrix(rng, n, conservation=conservation)
        mats.append(a)
        rhs.append(b)
    return _pack("solve", mats, rhs)


def config1(nsys=8192, n=61, seed=BASE_SEED + 1) -> Batch:
    """8,192 macro-atom matrices N = I - Q of order 61, inverted."""
    rng = np.random.default_rng(seed)
    return _pack("invert", [macro_matrix(rng, n) for _ in range(nsys)])


KAPPA_GROUPS = (2, 4, 6, 8, 10, 12)
# ion-chain rate spreads (decades below 1e2) whose draws land near each target
# log10 kappa_2 for order 27; the chain's own spectrum keeps kappa_2 above
# ~10^2.6 at this order, so the lowest group takes the narrowest spread
_ION_DECADES = {2: (0.0, 0.0), 4: (0.5, 2.5), 6: (1.5, 4.5), 8: (2.5, 6.5), 10: (3.0, 8.5), 12: (4.0, 10.0)}


def config2(generator: str, log_kappa: int, nsys: int = 2048, seed: int = BASE_SEED + 2, tol: float = 0.5):
    """One group of the conditioning sweep.

    ``generator`` "ion" (config-0 systems, order 27, solved) or "macro"
    (config-1 matrices, order 61, inverted) with the rate spread widened until
    log10 kappa_2 = ``log_kappa`` +- ``tol`` (kappa_2 from an FP64 SVD on the
    host, rejection-sampled).  Returns (batch, log10 kappa_2 per system,
    whether the target band was reachable).
    """
    rng = np.random.default_rng([seed, log_kappa, 0 if generator == "ion" else 1])
    mats, rhs, kap = [], [], []
    reachable = True
    if generator == "ion":
        lo, hi = _ION_DECADES[log_kappa]
        tries = 0
        budget = 4 * nsys if hi == 0.0 else 200 * nsys
        while len(mats) < nsys and tries < budget:
            cand = []
            for _ in range(256):
                d = rng.uniform(lo, hi)
                cand.append(ion_matrix(rng, 27, spread=(10.0 ** (2.0 - d), 1e2)))
            tries += 256
            k = np.log10(np.linalg.cond(np.stack([a for a, _ in cand])))
            for (a, b), kk in zip(cand, k):
                if abs(kk - log_kappa) <= tol and len(mats) < nsys:
                    mats.append(a), rhs.append(b), kap.append(kk)
        if len(mats) < nsys:
            # band below what the chain allows: keep the best-conditioned draws
            reachable = False
            need = nsys - len(mats)
            cand = [ion_matrix(rng, 27, spread=(1e2, 1e2)) for _ in range(need)]
            k = np.log10(np.linalg.cond(np.stack([a for a, _ in cand])))
            for (a, b), kk in zip(cand, k):
                mats.append(a), rhs.append(b), kap.append(kk)
        return _pack("solve", mats, rhs), np.array(kap), reachable
    # macro: kappa_2 follows the smallest deactivation probability (no absorbing rows)
    t = log_kappa - 0.27
    while len(mats) < nsys:
        cand = [macro_matrix(rng, 61, pdeact=(10.0 ** (-t), 2 * 10.0 ** (-t)), identity_frac=0.0) for _ in range(64)]
        k = np.log10(np.linalg.cond(np.stack(cand)))
        for m, kk in zip(cand, k):
            if abs(kk - log_kappa) <= tol and len(mats) < nsys:
                mats.append(m), kap.append(kk)
    return _pack("invert", mats), np.array(kap), reachable


def config3(ncells=50_000, seed=BASE_SEED + 3, macro_range=(20, 200)):
    """Mixed-size batch: per cell 10 ion systems (orders ION_SIZES_PER_CELL)
    and one macro-atom inverse of order uniform in ``macro_range``; the order
    of systems is shuffled.  Returns (solve batch, invert batch)."""
    rng = np.random.default_rng(seed)
    sizes = np.tile(np.array(ION_SIZES_PER_CELL), ncells)
    rng.shuffle(sizes)
    mats, rhs = [], []
    for n in sizes:
        a, b = ion_matrix(rng, int(n))
        mats.append(a)
        rhs.append(b)
    msz = rng.integers(macro_range[0], macro_range[1] + 1, ncells)
    macro = [macro_matrix(rng, int(n)) for n in msz]
    return _pack("solve", mats, rhs), _pack("invert", macro)


def config4(nsys=2048, seed=BASE_SEED + 4, nrange=(256, 1024)) -> Batch:
    """Large macro atoms: orders uniform in ``nrange``, 10 % of Q nonzero."""
    rng = np.random.default_rng(seed)
    sz = rng.integers(nrange[0], nrange[1] + 1, nsys)
    return _pack("invert", [macro_matrix(rng, int(n), density=0.10) for n in sz])


def ion_batch(sizes, seed, conservation="last", spread=(1e-14, 1e2)) -> Batch:
    rng = np.random.default_rng(seed)
    mats, rhs = [], []
    for n in sizes:
        a, b = ion_matrix(rng, int(n), spread=spread, conservation=conservation)
        mats.append(a)
        rhs.append(b)
    return _pack("solve", mats, rhs)


def macro_batch(sizes, seed, density=0.25) -> Batch:
    rng = np.random.default_rng(seed)
    return _pack("invert", [macro_matrix(rng, int(n), density=density) for n in sizes])


def dense_batch(kind, sizes, seed, log_spread=0.0) -> Batch:
    """General dense systems (Gaussian entries times exp(U[-s, s]))."""
    rng = np.random.default_rng(seed)
    mats, rhs = [], []
    for n in sizes:
        n = int(n)
        m = rng.standard_normal((n, n)) * np.exp(rng.uniform(-log_spread, log_spread, (n, n)))
        mats.append(m)
        rhs.append(rng.standard_normal(n))
    return _pack(kind, mats, rhs if kind == "solve" else None)


def from_matrices(kind, mats, rhs=None) -> Batch:
    return _pack(kind, [np.ascontiguousarray(m, dtype=np.float64) for m in mats],
                 [np.ascontiguousarray(r, dtype=np.float64) for r in rhs] if rhs is not None else None)


# ------------------------------------------------ ion tables and rate sets --
@dataclass
class IonTable:
    """The atomic-data part of an ion rate matrix (source/atomic.h ele[] / ion[] /
    inner_cross[] / charge_exchange[] as populate_ion_rate_matrix reads them).
    Elements hold consecutive ions in stage order; ion stage 1 is neutral."""
    elem_z: np.ndarray            # [nelem] atomic number
    elem_first: np.ndarray        # [nelem] first ion of the element
    elem_n: np.ndarray            # [nelem] ions of the element
    elem_istate_max: np.ndarray   # [nelem] highest stage
    ion_istate: np.ndarray        # [nions] stage
    ion_di: np.ndarray            # [nions] dere_di_flag
    ion_dr: np.ndarray            # [nions] drflag
    inner_nion: np.ndarray        # [n_inner] ion an inner-shell rate depopulates
    inner_yield: np.ndarray       # [n_inner] row of yield_prob, -1 without yield data
    yield_prob: np.ndarray        # [n_yield, 10] probability of 1..10 ejected electrons
    cx_nion1: np.ndarray          # [ncx] ion ionised by charge exchange
    cx_nion2: np.ndarray          # [ncx] its partner (hydrogen for the rates that count)

    @property
    def nions(self) -> int:
        return int(self.ion_istate.size)

    @property
    def nelem(self) -> int:
        return int(self.elem_z.size)

    @property
    def n_inner(self) -> int:
        return int(self.inner_nion.size)

    @property
    def ncx(self) -> int:
        return int(self.cx_nion1.size)

    def elem_of(self) -> np.ndarray:
        e = np.empty(self.nions, dtype=np.int32)
        for k in range(self.nelem):
            e[self.elem_first[k]:self.elem_first[k] + self.elem_n[k]] = k
        return e


@dataclass
class IonRates:
    """Per-cell coefficients of populate_ion_rate_matrix: photoionisation (pi),
    radiative recombination (rr), direct-ionisation, three-body and dielectronic
    coefficients (di, qr, dr; the reference's di_coeffs / qrecomb_coeffs /
    dr_coeffs), charge-exchange recombination per ion (cxr) and ionisation per
    charge-exchange entry (cxi), inner-shell rates (inner)."""
    pi: np.ndarray
    rr: np.ndarray
    di: np.ndarray
    qr: np.ndarray
    dr: np.ndarray
    cxr: np.ndarray
    cxi: np.ndarray
    inner: np.ndarray

    @property
    def ncell(self) -> int:
        return int(self.pi.shape[0])


def ion_table(zs=(1, 2, 6, 8, 26), seed: int = BASE_SEED + 5) -> IonTable:
    """Synthetic atomic table: every stage of each element from neutral to bare
    (Z + 1 ions), random DI / DR flags, 0-3 inner-shell rates for ions with at
    least three electrons (a fifth without yield data), and charge-exchange
    ionisation of metal ions against H II plus entries with other partners
    (which the reference skips)."""
    rng = np.random.default_rng(seed)
    elem_z = np.array(zs, dtype=np.int32)
    elem_n = elem_z + 1
    elem_first = np.concatenate([[0], np.cumsum(elem_n)[:-1]]).astype(np.int32)
    nions = int(elem_n.sum())
    ion_istate = np.concatenate([np.arange(1, z + 2) for z in zs]).astype(np.int32)
    ion_di = (rng.random(nions) < 0.5).astype(np.int32)
    ion_dr = (rng.random(nions) < 0.6).astype(np.int32) * rng.integers(1, 3, nions).astype(np.int32)
    z_of = np.repeat(elem_z, elem_n)
    inner_nion, inner_yield, probs = [], [], []
    for i in range(nions):
        if z_of[i] - ion_istate[i] + 1 >= 3:
            for _ in range(int(rng.integers(0, 4))):
                inner_nion.append(i)
                if rng.random() < 0.2:
                    inner_yield.append(-1)
                else:
                    p = rng.random(10)
                    probs.append(p / p.sum() * rng.uniform(0.5, 1.0))
                    inner_yield.append(len(probs) - 1)
    h_ii = int(elem_first[list(zs).index(1)] + 1) if 1 in zs else 0
    cx1, cx2 = [], []
    for e, z in enumerate(zs):
        if z == 1:
            continue
        for i in range(int(elem_first[e]), int(elem_first[e] + elem_n[e]) - 1):
            if rng.random() < 0.3:
                cx1.append(i)
                cx2.append(h_ii if rng.random() < 0.8 else int(elem_first[e]))
    return IonTable(elem_z, elem_first, elem_n.astype(np.int32), (elem_z + 1).astype(np.int32), ion_istate, ion_di,
                    ion_dr, np.array(inner_nion, dtype=np.int32), np.array(inner_yield, dtype=np.int32),
                    np.array(probs, dtype=np.float64).reshape(-1, 10), np.array(cx1, dtype=np.int32),
                    np.array(cx2, dtype=np.int32))


def ion_rates(tab: IonTable, ncell: int, seed: int = BASE_SEED + 6) -> IonRates:
    """Log-uniform coefficients per cell; charge-exchange recombination is zero
    for hydrogen and neutral ions (nothing to recombine into)."""
    rng = np.random.default_rng(seed)
    n = tab.nions

    def lu(lo, hi, shape):
        return np.exp(rng.uniform(np.log(lo), np.log(hi), shape))
    cxr = lu(1e-12, 1e-8, (ncell, n))
    z_of = np.repeat(tab.elem_z, tab.elem_n)
    cxr[:, (z_of == 1) | (tab.ion_istate == 1)] = 0.0
    return IonRates(pi=lu(1e-8, 1e2, (ncell, n)), rr=lu(1e-14, 1e-10, (ncell, n)), di=lu(1e-16, 1e-8, (ncell, n)),
                    qr=lu(1e-30, 1e-24, (ncell, n)), dr=lu(1e-14, 1e-10, (ncell, n)), cxr=cxr,
                    cxi=lu(1e-12, 1e-8, (ncell, tab.ncx)), inner=lu(1e-6, 1e-1, (ncell, tab.n_inner)))


# ------------------------------------------- macro-atom jump tables and rates --
@dataclass
class MatomModel:
    """A macro-atom model as calc_matom_matrix (source/macro_accelerate.c:31-348)
    walks it: levels with energies, lines and continua between levels (macro
    or simple), per-level jump lists in the reference's order, Auger entries."""
    ex: np.ndarray           # [nlev] level energies
    line_lo: np.ndarray      # [nline]
    line_up: np.ndarray
    line_macro: np.ndarray
    phot_lo: np.ndarray      # [nphot]
    phot_up: np.ndarray
    phot_macro: np.ndarray
    bbd: list                # per level: line indices of its downward bound-bound jumps
    bbu: list                # per level: line indices of its upward ones
    bfd: list                # per level: continuum indices of its downward bound-free jumps
    bfu: list                # per level: upward ones
    aug_idx: np.ndarray      # [nlev] Auger entry of the level, -1 without
    n_aug: np.ndarray        # [nlev] Auger channels used
    aug_target: np.ndarray   # [naug, 4]
    aug_A: np.ndarray        # [naug]
    aug_branch: np.ndarray   # [naug, 4]

    @property
    def nlev(self) -> int:
        return int(self.ex.size)


@dataclass
class MatomCell:
    """One cell's coefficients: a21, p_escape, q21, b12, q12 per line; q_recomb,
    q_ioniz per continuum; jbar per upward bound-bound jump, gamma and alpha_st
    per upward bound-free jump, recomb_sp per downward bound-free jump (levels
    in order); den per level; the k-packet cooling rates; t_e and n_e."""
    a21: np.ndarray
    pesc: np.ndarray
    q21: np.ndarray
    b12: np.ndarray
    q12: np.ndarray
    qrec: np.ndarray
    qion: np.ndarray
    jbar: np.ndarray
    gamma: np.ndarray
    alpha_st: np.ndarray
    recomb_sp: np.ndarray
    den: np.ndarray
    cool_bb: np.ndarray
    cool_bf: np.ndarray
    cool_bftot: float
    cool_adiabatic: float
    cool_ff: float
    cool_ff_lofreq: float
    t_e: float
    ne: float


def matom_model(ion_levels=(12, 20, 16, 9, 1), seed: int = BASE_SEED + 7) -> MatomModel:
    """Synthetic macro atom: ions of the given level counts, energies rising
    within and across ions; lines between levels of one ion (one in six
    simple), continua from each level of an ion to levels of the next (all
    macro but the highest ion's), a few Auger-capable levels."""
    rng = np.random.default_rng(seed)
    first = np.concatenate([[0], np.cumsum(ion_levels)[:-1]]).astype(int)
    ex = []
    base = 0.0
    for k, nl in enumerate(ion_levels):
        ex += list(base + np.sort(rng.uniform(0.0, 1e-11, nl)) * (1 if nl > 1 else 0))
        base += 2e-11
    ex = np.array(ex)
    nlev = ex.size
    lo, up, mac = [], [], []
    for k, nl in enumerate(ion_levels):
        for a in range(nl):
            for b in range(a + 1, nl):
                if rng.random() < 0.35:
                    lo.append(first[k] + a)
                    up.append(first[k] + b)
                    mac.append(0 if rng.random() < 1 / 6 else 1)
    plo, pup, pmac = [], [], []
    for k in range(len(ion_levels) - 1):
        for a in range(ion_levels[k]):
            for b in range(min(2, ion_levels[k + 1])):
                if b == 0 or rng.random() < 0.3:
                    plo.append(first[k] + a)
                    pup.append(first[k + 1] + b)
                    pmac.append(1)
    line_lo, line_up, line_macro = (np.array(v, dtype=np.int32) for v in (lo, up, mac))
    phot_lo, phot_up, phot_macro = (np.array(v, dtype=np.int32) for v in (plo, pup, pmac))
    bbd = [[i for i in range(line_lo.size) if line_up[i] == u and line_macro[i]] for u in range(nlev)]
    bbu = [[i for i in range(line_lo.size) if line_lo[i] == u and line_macro[i]] for u in range(nlev)]
    bfd = [[i for i in range(phot_lo.size) if phot_up[i] == u and phot_macro[i]] for u in range(nlev)]
    bfu = [[i for i in range(phot_lo.size) if phot_lo[i] == u and phot_macro[i]] for u in range(nlev)]
    aug_idx = np.full(nlev, -1, dtype=np.int32)
    n_aug = np.zeros(nlev, dtype=np.int32)
    tg, A, br = [], [], []
    for u in rng.choice(nlev - ion_levels[-1], size=3, replace=False):
        k = int(np.searchsorted(first, u, side="right") - 1)
        if k + 2 >= len(ion_levels):
            continue
        aug_idx[u] = len(A)
        n_aug[u] = int(rng.integers(1, 5))
        tg.append([first[k + 2] + int(rng.integers(0, ion_levels[k + 2])) for _ in range(4)])
        A.append(float(10 ** rng.uniform(10, 14)))
        p = rng.random(4)
        br.append(p / p.sum())
    return MatomModel(ex, line_lo, line_up, line_macro, phot_lo, phot_up, phot_macro, bbd, bbu, bfd, bfu, aug_idx,
                      n_aug, np.array(tg, dtype=np.int32).reshape(-1, 4), np.array(A, dtype=np.float64),
                      np.array(br, dtype=np.float64).reshape(-1, 4))


def matom_cell(m: MatomModel, seed: int) -> MatomCell:
    """Log-uniform coefficients for one cell; a few upward bound-free jumps get
    a stimulated-recombination term large enough to make their rate negative
    (the reference clamps it to zero), a few downward ones a zero rate."""
    rng = np.random.default_rng(seed)
    nl, npht = m.line_lo.size, m.phot_lo.size
    nbu = sum(len(v) for v in m.bbu)
    nfu = sum(len(v) for v in m.bfu)
    nfd = sum(len(v) for v in m.bfd)

    def lu(lo, hi, k):
        return np.exp(rng.uniform(np.log(lo), np.log(hi), k))
    alpha = lu(1e-14, 1e-10, nfu)
    alpha[rng.random(nfu) < 0.1] = 1e6
    sp = lu(1e-14, 1e-11, nfd)
    sp[rng.random(nfd) < 0.1] = 0.0
    den = lu(1e-12, 1.0, m.nlev)
    den[rng.random(m.nlev) < 0.1] = 1e-14
    return MatomCell(a21=lu(1e3, 1e9, nl), pesc=rng.uniform(1e-4, 1.0, nl), q21=lu(1e-12, 1e-7, nl),
                     b12=lu(1e5, 1e12, nl), q12=lu(1e-14, 1e-8, nl), qrec=lu(1e-30, 1e-24, npht),
                     qion=lu(1e-14, 1e-9, npht), jbar=lu(1e-20, 1e-12, nbu), gamma=lu(1e-4, 1e2, nfu), alpha_st=alpha,
                     recomb_sp=sp, den=den, cool_bb=lu(1e-30, 1e-22, nl), cool_bf=lu(1e-30, 1e-22, npht),
                     cool_bftot=float(lu(1e-25, 1e-21, 1)[0]), cool_adiabatic=float(lu(1e-28, 1e-23, 1)[0]),
                     cool_ff=float(lu(1e-26, 1e-22, 1)[0]), cool_ff_lofreq=float(lu(1e-28, 1e-24, 1)[0]),
                     t_e=float(10 ** rng.uniform(3.5, 5.5)), ne=float(10 ** rng.uniform(6, 12)))


def matom_jump_inputs(m: MatomModel, cells, density_phot_min: float = 1e-10) -> dict:
    """The arrays matom_rate_matrices_batched takes for a model and its cells:
    per-level jump lists (starts and targets) and, cell after cell, one
    coefficient per jump, computed as calc_matom_matrix computes them on the
    host (a21 * p_escape, b12 * jbar, the density ratio, the k-packet to
    r-packet sum in the routine's order)."""
    nlev = m.nlev
    lists = {"bbd": ([], []), "aug": ([], []), "bfd": ([], []), "bbu": ([], []), "bfu": ([], [])}
    aug_rate = []
    for u in range(nlev):
        for key in lists:
            lists[key][0].append(len(lists[key][1]))
        lists["bbd"][1].extend(int(m.line_lo[i]) for i in m.bbd[u])
        if m.aug_idx[u] >= 0:
            a = int(m.aug_idx[u])
            for k in range(int(m.n_aug[u])):
                lists["aug"][1].append(int(m.aug_target[a][k]))
                aug_rate.append(float(m.aug_A[a]) * float(m.aug_branch[a][k]))
        lists["bfd"][1].extend(int(m.phot_lo[i]) for i in m.bfd[u])
        lists["bbu"][1].extend(int(m.line_up[i]) for i in m.bbu[u])
        lists["bfu"][1].extend(int(m.phot_up[i]) for i in m.bfu[u])
    out = {"nlev": nlev, "ex": np.ascontiguousarray(m.ex, np.float64), "aug_rate": np.array(aug_rate, np.float64)}
    for key, (st, tg) in lists.items():
        out[key + "_start"] = np.array(st + [len(tg)], np.int32)
        out[key + "_target"] = np.array(tg, np.int32)
    mac_l = [i for i in range(m.line_lo.size) if m.line_macro[i]]
    mac_p = [i for i in range(m.phot_lo.size) if m.phot_macro[i]]
    out["kbb_target"] = np.array([int(m.line_up[i]) for i in mac_l], np.int32)
    out["kbf_target"] = np.array([int(m.phot_up[i]) for i in mac_p], np.int32)
    cols = {k: [] for k in ("bbd_rad", "bbd_coll", "bfd_sp", "bfd_qrec", "bbu_rad", "bbu_coll", "bfu_gamma",
                            "bfu_alpha", "bfu_ratio", "bfu_qion", "kbb", "kbf", "kr", "ne")}
    for c in cells:
        ibu = ifu = ifd = 0
        for u in range(nlev):
            for i in m.bbd[u]:
                cols["bbd_rad"].append(float(c.a21[i]) * float(c.pesc[i]))
                cols["bbd_coll"].append(float(c.q21[i]))
            for i in m.bfd[u]:
                cols["bfd_sp"].append(float(c.recomb_sp[ifd]))
                cols["bfd_qrec"].append(float(c.qrec[i]))
                ifd += 1
            for i in m.bbu[u]:
                cols["bbu_rad"].append(float(c.b12[i]) * float(c.jbar[ibu]))
                cols["bbu_coll"].append(float(c.q12[i]))
                ibu += 1
            for i in m.bfu[u]:
                lo = float(c.den[m.phot_lo[i]])
                cols["bfu_gamma"].append(float(c.gamma[ifu]))
                cols["bfu_alpha"].append(float(c.alpha_st[ifu]))
                cols["bfu_ratio"].append(float(c.den[m.phot_up[i]]) / lo if lo >= density_phot_min else 0.0)
                cols["bfu_qion"].append(float(c.qion[i]))
                ifu += 1
        cols["kbb"].extend(float(c.cool_bb[i]) for i in mac_l)
        cols["kbf"].extend(float(c.cool_bf[i]) for i in mac_p)
        kr = 0.0
        for i in range(m.line_lo.size):
            if not m.line_macro[i]:
                kr += float(c.cool_bb[i])
        for i in range(m.phot_lo.size):
            if not m.phot_macro[i]:
                kr += float(c.cool_bf[i])
        kr += c.cool_bftot
        kr += c.cool_adiabatic
        kr += c.cool_ff + c.cool_ff_lofreq
        cols["kr"].append(kr)
        cols["ne"].append(float(c.ne))
    for k, v in cols.items():
        out[k] = np.array(v, np.float64)
    out["ncell"] = len(cells)
    return out
