"""CPU restatement of the PTB density-matrix step (TEST INFRASTRUCTURE ONLY).

This module is the oracle that the CUDA path is checked against.  Only the
test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product library never calls it.

Parity status: UNPINNED against reference outputs.  grimme-lab/ptb is a
Fortran program (ifx + MKL ILP64) with no test suite and no dumped H/S/P
fixtures; no Fortran compiler exists on the build host, so the reference
cannot be run to generate golden vectors.  The restatement is checked
instead against the invariants the reference's own run logs exhibit
(``runs/h2o_512_0/filter_0.0001/full_matrix/out``: the full_matrix partition
reproduces the dense ``solve2`` density exactly, N_el = tr(PS) to 1e-11) and
against independent LAPACK/numpy computations (see tests/test_oracle.py).

Arrays use Fortran semantics in numpy: ``M[row, col]``.  Packed storage is
the reference's 1-based ``ij = i(i-1)/2 + j`` (j <= i), i.e. column ``i``,
rows ``<= i`` (source/solve.f:149-200).  All eigensolves go through the same
LAPACK drivers the reference calls through MKL (``dsygvd`` itype 1 'V' 'U',
``dsyevd`` 'V' 'U'), here from scipy's OpenBLAS build.

Fortran single-precision literals: the reference writes thresholds such as
``1e-3`` or ``thrs%normal = 1e-4`` without a kind suffix, so they are REAL(4)
constants promoted to REAL(8).  ``_f4`` reproduces that rounding.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg.lapack as _lapack


def _f4(x: float) -> float:
    """A Fortran default-real literal promoted to real(8)."""
    return float(np.float32(x))


# ----------------------------------------------------------------------------
# thresholds (source/metrics.f90:82-113, adjust_thresholds_dp)
# ----------------------------------------------------------------------------
@dataclass(frozen=True)
class Thresholds:
    high: float
    normal: float
    low: float


def adjust_thresholds(ndim: int) -> Thresholds:
    """Size-dependent thresholds, source/metrics.f90:82-113."""
    if ndim < 300:
        v = (1e-10, 1e-9, 1e-8)
    elif ndim < 2000:
        v = (1e-7, 1e-6, 1e-5)
    elif ndim < 15000:
        v = (1e-5, 1e-4, 1e-3)
    else:
        v = (1e-3, 1e-2, 1e-1)
    return Thresholds(*(_f4(x) for x in v))


# ----------------------------------------------------------------------------
# packed storage (source/solve.f:149-200) and filtering (source/pgtb.f90:1532-1577)
# ----------------------------------------------------------------------------
def npacked(n: int) -> int:
    return n * (n + 1) // 2


def _tril(n):
    return np.tril_indices(n)


def blowsym(n: int, packed: np.ndarray) -> np.ndarray:
    """Packed -> full symmetric, source/solve.f:149-165."""
    r, c = _tril(n)          # r = column i (0-based), c = row j <= i
    full = np.empty((n, n), dtype=np.float64)
    full[c, r] = packed
    full[r, c] = packed
    return full


def packsym(full: np.ndarray) -> np.ndarray:
    """Full -> packed taking column i, rows <= i, source/solve.f:185-200."""
    n = full.shape[0]
    r, c = _tril(n)
    return np.ascontiguousarray(full[c, r])


def filter_matrix_sym(packed: np.ndarray, filt: float) -> np.ndarray:
    """|A_ij| < filter -> 0 (returns a filtered copy), source/pgtb.f90:1532-1547."""
    out = packed.copy()
    out[np.abs(out) < filt] = 0.0
    return out


def analyse_matrix_sym(packed: np.ndarray, n: int) -> dict:
    """Counts STRICTLY POSITIVE entries per column, source/pgtb.f90:1548-1577."""
    r, c = _tril(n)
    pos = packed > 0
    colcnt = np.bincount(r[pos], minlength=n) + np.bincount(c[pos & (r != c)], minlength=n)
    tot = int(colcnt.sum())
    return {"dimension": n, "nonzero": tot, "sparsity": tot / float(n) ** 2,
            "per_column": tot // n}


# ----------------------------------------------------------------------------
# LAPACK drivers with the reference's arguments
# ----------------------------------------------------------------------------
# Thread count of the small per-submatrix LAPACK/BLAS calls.  Multithreaded
# OpenBLAS on matrices of order ~100-500, alternating dsygvd with a small
# dgemm, runs dsygvd about 7x slower than one thread does (thread hand-over
# between routines); MKL, which the reference links, lowers its thread count
# for such sizes by itself.  Below this order the submatrix loop runs its
# calls on one thread, so the timed CPU baseline is not inflated.
SMALL_LAPACK_ORDER = 512
_TPC = None


def _blas_threads(m: int):
    """Context: one BLAS/LAPACK thread for a submatrix of order m < SMALL_LAPACK_ORDER."""
    global _TPC
    if _TPC is None:
        from threadpoolctl import ThreadpoolController
        _TPC = ThreadpoolController()
    return _TPC.limit(limits=1 if m < SMALL_LAPACK_ORDER else None)


def sygvd(a: np.ndarray, b: np.ndarray):
    """dsygvd(itype=1,'V','U'); source/lapack_eig.f90:305-368. Returns (w, U, info)."""
    w, v, info = _lapack.dsygvd(a, b, itype=1, jobz="V", uplo="U")
    return w, v, int(info)


def syevd(a: np.ndarray):
    """dsyevd('V','U'); source/lapack_eig.f90:453-515."""
    w, v, info = _lapack.dsyevd(a, compute_v=1, lower=0)
    return w, v, int(info)


# ----------------------------------------------------------------------------
# metrics (source/metrics.f90:182-360, source/norms.f90)
# ----------------------------------------------------------------------------
def get_nel(P: np.ndarray, S: np.ndarray) -> float:
    """tr(P S), source/metrics.f90:182-230 (full P may be non-symmetric)."""
    return float(np.einsum("ij,ji->", P, S))


def band_structure(P: np.ndarray, H: np.ndarray) -> float:
    """tr(P H), source/metrics.f90:233-277."""
    return float(np.einsum("ij,ji->", P, H))


def idempotency_deviation(P: np.ndarray, S: np.ndarray):
    """Returns (reference quirk value, true Frobenius norm) of 1/2 PSP - P.

    source/metrics.f90:316-360 evaluates ``sqrt(sum(mm2 - P)**2)`` which is
    |sum(1/2 PSP - P)|, not a norm.  Both values are returned.
    """
    mm2 = 0.5 * (P @ S @ P)
    d = mm2 - P
    return abs(float(d.sum())), float(np.linalg.norm(d))


def frobenius(m):
    return float(np.sqrt(np.sum(m * m)))


def gershgorin(m):
    """max column abs-sum, source/norms.f90:5-18."""
    return float(np.max(np.sum(np.abs(m), axis=0)))


def infinity(m):
    """max row abs-sum, source/norms.f90:32-49."""
    return float(np.max(np.sum(np.abs(m), axis=1)))


# ----------------------------------------------------------------------------
# occupations and Fermi smearing (source/fermi.f:5-124)
# ----------------------------------------------------------------------------
_BOLTZ = _f4(3.166808578545117e-06)


def occu(ndim: int, nel: int, nopen: int):
    """Restricted -> alpha/beta occupations, source/fermi.f:71-124."""
    focc = np.zeros(ndim, dtype=np.int64)
    if nel % 2 == 0:
        ihomo = nel // 2
        focc[:ihomo] = 2
        if 2 * ihomo != nel:        # unreachable for even nel; kept as written
            ihomo += 1
            focc[ihomo - 1] = 1
            if nopen == 0:
                nopen = 1
        if nopen > 1:
            for i in range(1, nopen // 2 + 1):
                focc[ihomo - i] -= 1
                focc[ihomo + i - 1] += 1
    else:
        na = nel // 2 + (nopen - 1) // 2 + 1
        nb = nel // 2 - (nopen - 1) // 2
        focc[:na] += 1
        focc[:nb] += 1
    focca = np.where(focc >= 1, 1.0, 0.0)
    foccb = np.where(focc == 2, 1.0, 0.0)
    ihomoa = int(np.max(np.nonzero(focca > 0.99)[0]) + 1) if np.any(focca > 0.99) else 0
    ihomob = int(np.max(np.nonzero(foccb > 0.99)[0]) + 1) if np.any(foccb > 0.99) else 0
    if ihomoa < 1:
        raise RuntimeError("internal error in occu")
    return ihomoa, ihomob, focca, foccb


def fermismear(norbs: int, nel: int, t: float, eig: np.ndarray):
    """Newton solve for E_F at temperature t, source/fermi.f:5-67. Returns occ, E_F."""
    bkt = _BOLTZ * t
    ef = 0.5 * (eig[nel - 1] + eig[nel])
    occt = float(nel)
    ncycle = 0
    while True:
        ncycle += 1
        x = (eig - ef) / bkt
        small = x < 50
        xs = np.where(small, x, 0.0)
        ex = np.exp(xs)
        ff = np.where(small, 1.0 / (ex + 1.0), 0.0)
        df = np.where(small, ex / (bkt * (ex + 1.0) ** 2), 0.0)
        tot = float(ff.sum())
        totd = float(df.sum())
        ef = ef + (occt - tot) / (totd + 1e-14)
        if not (abs(occt - tot) > 1e-9 and ncycle < 200):
            break
    return ff, ef


def dmat(occ: np.ndarray, C: np.ndarray) -> np.ndarray:
    """P = C diag(occ) C^T, source/solve.f:263-283."""
    return C @ (C * occ).T


# ----------------------------------------------------------------------------
# dense oracle solve2 (source/pgtb.f90:1066-1170)
# ----------------------------------------------------------------------------
def solve2(mode: int, ndim: int, nel: int, nopen: int, et: float,
           Hvec: np.ndarray, Svec: np.ndarray, glob15: float = 0.0, glob17: float = 0.0):
    """Dense FP64 generalized diagonalisation + Fermi smearing. Returns (Pvec, e, focc, fail)."""
    S = blowsym(ndim, Svec)
    H = blowsym(ndim, Hvec)
    e, U, info = sygvd(H, S)
    fail = info != 0
    if mode >= 2:
        e = e + glob15 + glob17 * e
    if nel > 0:
        ihomoa, ihomob, focca, foccb = occu(ndim, nel, nopen)
    else:
        ihomoa = ihomob = 0
        focca = np.zeros(ndim)
        foccb = np.zeros(ndim)
    if ihomoa + 1 <= ndim:
        focca, _ = fermismear(ndim, ihomoa, et, e)
    if ihomob + 1 <= ndim and nel > 1:
        foccb, _ = fermismear(ndim, ihomob, et, e)
    focc = focca + foccb
    P = dmat(focc, U)
    return packsym(P), e, focc, fail


def dense_projector(H: np.ndarray, S: np.ndarray, nel: int):
    """Exact ground-state projector: doubly occupy the lowest nel/2 generalized eigenvectors."""
    e, U, info = sygvd(H, S)
    if info != 0:
        raise RuntimeError(f"dsygvd info={info}")
    nocc = nel // 2
    occ = np.zeros(H.shape[0])
    occ[:nocc] = 2.0
    if nel % 2:
        occ[nocc] = 1.0
    return dmat(occ, U), e


# ----------------------------------------------------------------------------
# submatrix method (source/sm.f90:34-409)
# ----------------------------------------------------------------------------
SINGLE_COLUMNS, ATOMS_COLUMNS, FULL_MATRIX, KMEANS_R_HEURISTIC = 1, 2, 3, 4
SUBMATRIX_SIGN, SUBMATRIX_SYGV = 1, 2


def submatrix_columns(mode: int, ndim: int, aoat: np.ndarray, nat: int,
                      partition: np.ndarray | None = None):
    """Owned-column lists per submatrix (0-based), source/sm.f90:92-162.

    Mode 4 takes ``partition`` (atom -> cluster id, 1-based) instead of
    running the non-deterministic k-means; column order follows
    source/sm.f90:483-496 (cluster, then atom, then AO).
    """
    aoat = np.asarray(aoat)
    if mode == SINGLE_COLUMNS:
        return [np.array([i]) for i in range(ndim)]
    if mode == ATOMS_COLUMNS:
        groups, cur = [], [0]
        for i in range(1, ndim):
            if aoat[i] == aoat[i - 1]:
                cur.append(i)
            else:
                groups.append(np.array(cur))
                cur = [i]
        groups.append(np.array(cur))
        return groups
    if mode == FULL_MATRIX:
        return [np.arange(ndim)]
    if mode == KMEANS_R_HEURISTIC:
        if partition is None:
            raise ValueError("mode 4 needs an atom->cluster partition")
        partition = np.asarray(partition)
        nsm = int(partition.max())
        out = []
        for ism in range(1, nsm + 1):
            cols = []
            for a in range(1, nat + 1):
                if partition[a - 1] == ism:
                    cols.extend(np.nonzero(aoat == a)[0].tolist())
            out.append(np.array(cols, dtype=np.int64))
        return out
    raise ValueError("not implemented")


def submatrix_map(H: np.ndarray, S: np.ndarray, owned: np.ndarray) -> np.ndarray:
    """Row i belongs iff H(i,c) > 0 or S(i,c) > 0 or i == c for an owned c, source/sm.f90:210-228."""
    ndim = H.shape[0]
    st = np.any((H[:, owned] > 0) | (S[:, owned] > 0), axis=1)
    st[owned] = True
    return np.nonzero(st)[0]


@dataclass
class SubmatrixResult:
    Pvec: np.ndarray
    nsm: int
    dims: list
    mu: float
    nel: float
    mu_trace: list = field(default_factory=list)
    info: list = field(default_factory=list)


def sm_stupid_simple(ndim: int, nelref: int, Hvec: np.ndarray, Svec: np.ndarray,
                     nat: int, xyz: np.ndarray, aoat: np.ndarray,
                     columns: int, mode: int, partition=None) -> SubmatrixResult:
    """Submatrix density step with mu bisection, source/sm.f90:34-409."""
    if mode != SUBMATRIX_SYGV:
        raise NotImplementedError("submatrix_mode.eq.1 not implemented")
    H = blowsym(ndim, Hvec)
    S = blowsym(ndim, Svec)
    comb = submatrix_columns(columns, ndim, aoat, nat, partition)
    nsm = len(comb)
    eig = []
    dims = []
    infos = []
    for owned in comb:
        mp = submatrix_map(H, S, owned)
        m = len(mp)
        imap = np.full(ndim, -1, dtype=np.int64)
        imap[mp] = np.arange(m)
        Hs = H[np.ix_(mp, mp)]
        Ss = S[np.ix_(mp, mp)]
        with _blas_threads(m):
            e, U, info = sygvd(Hs, Ss)
            Psm = Ss @ U
        io = imap[owned]
        fe = np.sum(Psm[io, :] * U[io, :], axis=0)
        eig.append((mp, imap, owned, e, U, fe))
        dims.append(m)
        infos.append(info)

    mua, mub = -10.0, 10.0
    tol_mu, tol_nel = _f4(1e-3), _f4(1e-5)
    finaliter = False
    trace = []
    P = np.zeros((ndim, ndim))
    mu = nel = 0.0
    for muiter in range(1, 101):
        mu = (mua + mub) / 2
        nel = 0.0
        if finaliter:
            P[:, :] = 0.0
        for (mp, imap, owned, e, U, fe) in eig:
            occ = np.where(e < mu, 2.0, np.where(e == mu, 1.0, 0.0))
            nel += float(np.sum(fe * occ))
            if finaliter:
                with _blas_threads(len(mp)):
                    Psm = dmat(occ, U)
                P[np.ix_(mp, owned)] = Psm[:, imap[owned]]
        if finaliter:
            break
        trace.append((muiter, mu, nel))
        if abs(mua - mub) < tol_mu or abs(nel - nelref) < tol_nel:
            finaliter = True
        if not finaliter:
            if nel > nelref:
                mub = mu
            else:
                mua = mu
    return SubmatrixResult(packsym(P), nsm, dims, mu, nel, trace, infos)


# ----------------------------------------------------------------------------
# purification module (source/purification.f90, source/purification_settings.f90)
# ----------------------------------------------------------------------------
MCWEENY, SIGN_ITER_PADE, SIGN_ITER_NEWTON, SIGN_DIAGONALIZATION = 1, 2, 3, 4
INV, INV_SQRT, SQRT_ = 1, 2, 3


@dataclass
class PurificationSettings:
    """Mirror of tPurificationSet with its defaults, source/purification_settings.f90:29-86."""
    mode: int = 1
    type: int = SIGN_DIAGONALIZATION
    cycles: int = 40
    prlvl: int = 1
    nel: int = 0
    submatrix_mode: int = SUBMATRIX_SYGV
    submatrix_columns: int = ATOMS_COLUMNS
    metric_type: int = INV_SQRT
    metric_cycles: int = 50
    metric_iterative: bool = False
    chempot_cycles: int = 60
    chempot_guess: float = -1.5
    chempot_increment: float = 0.1


def get_transformation_matrix(pur: PurificationSettings, S: np.ndarray, thr: Thresholds):
    """X = S^-1 or S^-1/2, source/purification.f90:83-229."""
    n = S.shape[0]
    I = np.eye(n)
    if pur.metric_iterative:
        if pur.metric_type == INV:
            X = S / infinity(S) ** 2
            for _ in range(pur.metric_cycles):
                atmp = S @ X
                XsX = X @ atmp
                X = 2.0 * X - XsX
                check = X @ S
                if frobenius(I - check) < thr.low:
                    break
        elif pur.metric_type == INV_SQRT:
            X = S / frobenius(S) ** 2
            for _ in range(pur.metric_cycles):
                atmp = X @ X
                XsX = atmp @ S
                atmp2 = X @ XsX
                X = 0.5 * (3 * X - atmp2)
                if frobenius(I - XsX) < thr.low:
                    break
                if np.any(np.isnan(XsX)):
                    raise FloatingPointError("Error, NaN encountered")
        else:
            X = np.zeros_like(S)
        return X
    w, V, info = syevd(S.copy())
    D = np.zeros(n)
    if pur.metric_type == INV:
        D = 1.0 / w
    elif pur.metric_type == INV_SQRT:
        D = 1.0 / np.sqrt(w)
    return (V * D) @ V.T


def build_guess(pur, H, X, chempot):
    """source/purification.f90:355-436."""
    n = H.shape[0]
    I = np.eye(n)
    if pur.type == MCWEENY:
        term4 = chempot * X - X @ (H @ X)
        term5 = term4 / min(frobenius(term4), gershgorin(term4))
        return 0.5 * (term5 + X)
    if pur.metric_type == INV_SQRT:
        term4 = X @ (H @ X) - chempot * I
        return term4 / min(frobenius(term4), gershgorin(term4))
    if pur.metric_type == INV:
        term3 = X @ H - chempot * I
        return term3 / min(frobenius(term3), gershgorin(term3))
    return np.zeros_like(H)


def mcweeny_(pur, guess, S, thr):
    """P <- 3PSP - 2PSPSP, source/purification.f90:438-510."""
    g = guess.copy()
    norm = frobenius(g)
    P = g
    for _ in range(pur.cycles):
        t1 = S @ g
        t2 = g @ t1
        t3 = t2 @ t1
        P = 3 * t2 - 2 * t3
        if np.any(np.isnan(P)):
            raise FloatingPointError("Error: NaN is encountered during purification")
        if abs(frobenius(P) - norm) < thr.normal:
            break
        g = P
        norm = frobenius(P)
    return P * 2


def sign_to_density_matrix(pur, sign_, X):
    """source/purification.f90:603-647."""
    I = np.eye(sign_.shape[0])
    if pur.metric_type == INV_SQRT:
        P = 0.5 * (X @ ((I - sign_) @ X))
    elif pur.metric_type == INV:
        P = 0.5 * ((I - sign_) @ X)
    else:
        P = np.zeros_like(X)
    if np.any(np.isnan(P)):
        raise FloatingPointError("Error: NaN is encountered during purification")
    return P


def sign_iterative(pur, guess, X, thr):
    """Pade / Newton-Schulz sign iteration, source/purification.f90:512-601."""
    n = guess.shape[0]
    I = np.eye(n)
    Y = guess.copy()
    for _ in range(pur.cycles):
        norm = frobenius(Y)
        if pur.type == SIGN_ITER_PADE:
            t1 = Y @ Y
            t2 = t1 @ t1
            t3 = 15.0 * I - 10.0 * t1 + 3.0 * t2
            Y = 0.125 * (Y @ t3)
        else:
            t1 = Y @ Y
            t2 = Y @ t1
            Y = 0.5 * (3 * Y - t2)
        if np.any(np.isnan(Y)):
            raise FloatingPointError("Error: NaN is encountered during purification")
        if abs(frobenius(Y) - norm) < thr.normal:
            break
    return sign_to_density_matrix(pur, Y, X) * 2


def sign_diagonalization_(pur, chempot, guess, X, thr):
    """Eigen-sign with inner mu re-bisection, source/purification.f90:650-782.

    Returns (P, chempot) because the reference's chempot is intent(inout).
    """
    n = guess.shape[0]
    w, V, info = syevd(guess.copy())
    nel = float(np.float32(pur.nel))
    incr = pur.chempot_increment
    lower = upper = 0.0
    is_lower = is_upper = False
    colsq = np.sum(V * V, axis=0)
    sgn = np.zeros(n)
    for _ in range(pur.chempot_cycles):
        eg = w - chempot
        sgn = np.where(np.abs(eg) < thr.normal, 0.0, np.where(eg > 0.0, 1.0, -1.0))
        nelcalc = float(np.sum(1.0 - colsq * sgn))
        if abs(nelcalc - nel) < thr.normal:
            break
        if nelcalc < nel:
            is_lower, lower = True, chempot
            chempot = chempot + incr
        else:
            is_upper, upper = True, chempot
            chempot = chempot - incr
        bisection = is_lower and is_upper
        incr = incr * 2.0
        if bisection:
            chempot = (lower + upper) / 2.0
            if abs(upper - lower) < thr.high:
                break
    sign_ = V @ (sgn[:, None] * V.T)
    return sign_to_density_matrix(pur, sign_, X) * 2, chempot


def purification_search(pur, H, S, X, thr):
    """Outer chemical-potential search, source/purification.f90:232-353."""
    chempot = pur.chempot_guess
    incr = pur.chempot_increment
    nel = pur.nel
    lower = upper = 0.0
    is_lower = is_upper = bisection = False
    P = None
    steps = 0
    for _ in range(pur.chempot_cycles):
        if bisection:
            chempot = (lower + upper) / 2.0
            if abs(upper - lower) < thr.high:
                break
        guess = build_guess(pur, H, X, chempot)
        if pur.type == MCWEENY:
            P = mcweeny_(pur, guess, S, thr)
        elif pur.type in (SIGN_ITER_PADE, SIGN_ITER_NEWTON):
            P = sign_iterative(pur, guess, X, thr)
        elif pur.type == SIGN_DIAGONALIZATION:
            P, chempot = sign_diagonalization_(pur, chempot, guess, X, thr)
        steps += 1
        nel_calc = get_nel(P, S)
        if abs(nel_calc - float(np.float32(nel))) < thr.normal:
            break
        if nel_calc < nel:
            is_lower, lower = True, chempot
            chempot = chempot + incr
        else:
            is_upper, upper = True, chempot
            chempot = chempot - incr
        bisection = is_lower and is_upper
        incr = incr * 2.0
    return P, chempot, steps


def purification(pur: PurificationSettings, ndim: int, Hvec: np.ndarray, Svec: np.ndarray):
    """purification_wrapper, source/purification.f90:28-80. Returns packed P."""
    thr = adjust_thresholds(ndim)
    H = blowsym(ndim, Hvec)
    S = blowsym(ndim, Svec)
    X = get_transformation_matrix(pur, S, thr)
    P, mu, steps = purification_search(pur, H, S, X, thr)
    return packsym(P), mu, steps


# ----------------------------------------------------------------------------
# trace-correcting purification (new algorithm; FP64 restatement of the GPU path)
# ----------------------------------------------------------------------------
def sp2_trace_correcting(H: np.ndarray, S: np.ndarray, nel: int, max_iter: int = 100,
                         idem_tol: float = 1e-13):
    """Second-order trace-correcting purification (SP2/TC2) in the Cholesky basis.

    A = L^-1 H L^-T, X0 = (e_max - A)/(e_max - e_min) from Gershgorin bounds;
    each step X <- X^2 if |tr X^2 - N| <= |2 tr X - tr X^2 - N| else 2X - X^2,
    N = nel/2.  Stops once the idempotency error e_k = tr X - tr X^2 drops
    below ``idem_tol * n``, or, inside the asymptotic regime (e_k < 1e-2), once
    it no longer decreases over two steps (e_k >= e_{k-2}; the two-step
    look-back tolerates the alternation of the two polynomials).
    P = 2 L^-T X L^-1.
    """
    if nel % 2:
        raise ValueError("trace-correcting purification needs an even electron count")
    n = H.shape[0]
    N = nel // 2
    L = np.linalg.cholesky(S)
    Linv = np.linalg.inv(L)
    A = Linv @ H @ Linv.T
    A = 0.5 * (A + A.T)
    emin, emax = gershgorin_bounds(A)
    X = (emax * np.eye(n) - A) / (emax - emin)
    hist = []
    it = 0
    for it in range(1, max_iter + 1):
        X2 = X @ X
        trX = float(np.trace(X))
        trX2 = float(np.trace(X2))
        X = X2 if sp2_choose_square(trX, trX2, N) else 2 * X - X2
        err = abs(trX - trX2)
        hist.append(err)
        if err < idem_tol * n or (len(hist) > 2 and err < 1e-2 and err >= hist[-3]):
            break
    P = 2.0 * (Linv.T @ X @ Linv)
    return P, it


def gershgorin_bounds(A: np.ndarray):
    """Spectral bounds [min(a_ii - r_i), max(a_ii + r_i)], r_i = sum_{j != i} |a_ij|."""
    rad = np.sum(np.abs(A), axis=1) - np.abs(np.diag(A))
    return float(np.min(np.diag(A) - rad)), float(np.max(np.diag(A) + rad))


def sp2_choose_square(trX: float, trX2: float, N: float) -> bool:
    """SP2 branch rule: X^2 if it lands the trace closer to N than 2X - X^2 does."""
    return abs(trX2 - N) <= abs(2.0 * trX - trX2 - N)


# ---------------------------------------------------------------------------
# Mixed Mulliken/Loewdin population analysis (source/mlpop.f)
# ---------------------------------------------------------------------------
MULL_LOEW14 = 0.3333333333   # source/parcom.f90:26 (REAL(wp) parameter)


def mlpop14(nao: int, Svec: np.ndarray, x: float = MULL_LOEW14):
    """source/mlpop.f:142-190: s34 = S^(1-x), s14 = S^x in REAL*4.

    blowsym84 (packed FP64 -> full REAL*4), ssyev('V','U'), e1 = e**(1-x) and
    e2 = e**x (REAL*4 base, REAL(8) exponent, stored REAL*4), then
    sgemm('N','T') of X with X*diag(e).  Returns float32 (nao, nao) arrays in
    Fortran index order ([row, col])."""
    X = blowsym(nao, Svec).astype(np.float32)
    w, V, info = _lapack.ssyev(X, compute_v=1, lower=0)
    if info != 0:
        raise RuntimeError(f"ssyev info={info}")
    e1 = (w.astype(np.float64) ** (1.0 - x)).astype(np.float32)
    e2 = (w.astype(np.float64) ** x).astype(np.float32)
    s34 = (V @ (V * e1[None, :]).T).astype(np.float32)
    s14 = (V @ (V * e2[None, :]).T).astype(np.float32)
    return s34, s14


def mlpop2(n: int, nao: int, Pvec: np.ndarray, s1: np.ndarray, s2: np.ndarray, aoat: np.ndarray,
           shell2ao: np.ndarray, dtype=np.float32):
    """source/mlpop.f:198-235: X = s2 (P s1) with P blown up to REAL*4
    (blowsym84), ssymm then sgemm, q(aoat(i)) += X(i,i) and
    qsh(shell2ao(i), aoat(i)) += X(i,i) in REAL*8.  aoat and shell2ao are
    1-based (bascom).  dtype=np.float64 gives the same formula in FP64 (the
    error-free value the REAL*4 reference approximates).  Returns q (n,) and
    qsh (n, 10) (= Fortran qsh(10, n) in memory order)."""
    x = blowsym(nao, Pvec).astype(dtype)
    cc = (x @ s1.astype(dtype)).astype(dtype)
    xx = (s2.astype(dtype) @ cc).astype(dtype)
    q = np.zeros(n)
    qsh = np.zeros((n, 10))
    d = np.diag(xx).astype(np.float64)
    for i in range(nao):
        ia = int(aoat[i]) - 1
        q[ia] += d[i]
        qsh[ia, int(shell2ao[i]) - 1] += d[i]
    return q, qsh


# ---------------------------------------------------------------------------
# Deterministic k-means partition for submatrix columns mode 4
# (source/sm.f90:127-154,459-514 with source/kmpp.f; the reference draws from
# the Fortran global RNG inside an OpenMP loop, so its partition is not
# reproducible -- this restatement fixes the generator: splitmix64 seeded per
# cluster count)
# ---------------------------------------------------------------------------
_M64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Vigna): state += golden gamma, then two xor-shift-multiply
    rounds; uniform() = top 53 bits / 2^53 in [0, 1)."""

    def __init__(self, seed: int):
        self.s = seed & _M64

    def uniform(self) -> float:
        self.s = (self.s + 0x9E3779B97F4A7C15) & _M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        z ^= z >> 31
        return float(z >> 11) * (2.0 ** -53)


def kmeans_seed(seed: int, k: int) -> int:
    return (seed ^ ((k * 0xD1B54A32D192ED03) & _M64)) & _M64


def kmeans_pp(xyz: np.ndarray, k: int, seed: int, maxiter: int = 1000):
    """k-means++ seeding + Lloyd iterations as source/kmpp.f:24-178 (first
    centre at int(u N), the others with probability proportional to the
    squared distance to the nearest chosen centre; nearest centre with ties to
    the lower index; centres = sum * (1/count)).  Returns 0-based labels, or
    None when a cluster empties (IFAULT = 1 in the reference)."""
    x = [tuple(float(v) for v in p) for p in np.asarray(xyz, dtype=np.float64)]
    n = len(x)
    rng = SplitMix64(kmeans_seed(seed, k))
    big = 1e33
    work = [big] * n
    i1 = min(int(rng.uniform() * n), n - 1)
    C = [x[i1]]
    for _ in range(1, k):
        tot = 0.0
        c = C[-1]
        for i in range(n):
            d2 = (x[i][0] - c[0]) ** 2 + (x[i][1] - c[1]) ** 2 + (x[i][2] - c[2]) ** 2
            if d2 < work[i]:
                work[i] = d2
            tot += work[i]
        w = rng.uniform() * tot
        acc = 0.0
        i1 = n - 1
        for i in range(n):
            acc += work[i]
            if acc > w:
                i1 = i
                break
        C.append(x[i1])
    z = [-1] * n
    for _ in range(maxiter):
        change = False
        for i in range(n):
            best, l1 = big, 0
            for l in range(k):
                c = C[l]
                d2 = (x[i][0] - c[0]) ** 2 + (x[i][1] - c[1]) ** 2 + (x[i][2] - c[2]) ** 2
                if d2 < best:
                    best, l1 = d2, l
            if z[i] != l1:
                z[i] = l1
                change = True
        if not change:
            break
        cnt = [0] * k
        sums = [[0.0, 0.0, 0.0] for _ in range(k)]
        for i in range(n):
            cnt[z[i]] += 1
            for j in range(3):
                sums[z[i]][j] += x[i][j]
        if min(cnt) == 0:
            return None
        C = [tuple(sums[l][j] * (1.0 / cnt[l]) for j in range(3)) for l in range(k)]
    return np.array(z, dtype=np.int64)


def atom_pattern(ndim: int, H: np.ndarray, S: np.ndarray, aoat: np.ndarray, nat: int) -> np.ndarray:
    """R[i, A] = any column c of atom A with H(i,c) > 0 or S(i,c) > 0 or i == c
    (the index-set test of source/sm.f90:503-508, per atom)."""
    F = (H > 0) | (S > 0) | np.eye(ndim, dtype=bool)
    R = np.zeros((ndim, nat), dtype=bool)
    at = np.asarray(aoat) - 1
    for a in range(nat):
        R[:, a] = F[:, at == a].any(axis=1)
    return R


def kmeans_effort(R: np.ndarray, z: np.ndarray, k: int) -> float:
    """sum_k m_k^2.5 (source/sm.f90:498-512) with m_k = rows coupled to a
    column of cluster k; m^2.5 evaluated as m*m*sqrt(m)."""
    m = np.zeros(k, dtype=np.int64)
    for i in range(R.shape[0]):
        ks = np.unique(z[np.nonzero(R[i])[0]])
        m[ks] += 1
    e = 0.0
    for v in m:
        v = float(v)
        e += v * v * math.sqrt(v)
    return e


def kmeans_partition(ndim: int, H: np.ndarray, S: np.ndarray, nat: int, xyz: np.ndarray, aoat: np.ndarray,
                     seed: int = 42):
    """Mode-4 grouping, source/sm.f90:127-154: k-means for 1..min(64, nat)
    clusters, keep the least sum m_k^2.5 (ties: fewer clusters).  Returns the
    1-based atom -> cluster partition, the cluster count and the effort."""
    R = atom_pattern(ndim, H, S, aoat, nat)
    best = (math.inf, 0, None)
    for k in range(1, min(64, nat) + 1):
        z = kmeans_pp(xyz, k, seed)
        if z is None:
            continue
        e = kmeans_effort(R, z, k)
        if e < best[0]:
            best = (e, k, z)
    e, k, z = best
    return z + 1, k, e


# ---------------------------------------------------------------------------
# Iteration-2 XC long-range damping, the consumer of P in the next SCF
# iteration (source/pgtb.f90:482-513)
# ---------------------------------------------------------------------------
def xc_damping_loops(nat: int, ndim: int, aoat, rab, rad, hao, xdiag, Pvec, Hvec) -> np.ndarray:
    """The reference's two loops verbatim in Python (small cases only): xab over
    atom pairs (source/pgtb.f90:485-495), then the AO-pair update (:496-513).
    rad(a) stands for hi = shell_cnf3(10,at) + (cn - avcn) shell_resp(10,at,1),
    hao(i) for shell_cnf2(ish,ati) gq(ia), xdiag(i) for shell_xi(8,ati)."""
    xab = np.zeros(nat * (nat + 1) // 2)
    k = 0
    for i in range(nat):
        for j in range(i + 1):
            r = rad[i] + rad[j]
            t8 = (rab[k] - r) / r
            xab[k] = 0.5 * (1.0 + math.erf(-1.8 * t8))
            k += 1
    H = np.array(Hvec, dtype=np.float64, copy=True)
    k = 0
    for i in range(ndim):
        ia = int(aoat[i])
        hi = hao[i]
        for j in range(i):
            ib = int(aoat[j])
            hj = hao[j]
            H[k] = H[k] + Pvec[k] * (hi + hj) * xab[lin(ib, ia) - 1]
            k += 1
        H[k] = H[k] + 2.0 * Pvec[k] * xdiag[i] * hi * xab[lin(ia, ia) - 1]
        k += 1
    return H


def xc_damping(nat: int, ndim: int, aoat, rab, rad, hao, xdiag, Pvec, Hvec) -> np.ndarray:
    """Vectorised form of xc_damping_loops (same operations, same order)."""
    from scipy.special import erf
    rad = np.asarray(rad, dtype=np.float64)
    ca, rb = _packed_cols_rows(nat)
    r = rad[ca] + rad[rb]
    t8 = (np.asarray(rab, dtype=np.float64) - r) / r
    xab = 0.5 * (1.0 + erf(-1.8 * t8))
    ci, rj = _packed_cols_rows(ndim)
    a = np.asarray(aoat, dtype=np.int64) - 1
    ia, ib = a[ci], a[rj]
    hi, lo = np.maximum(ia, ib), np.minimum(ia, ib)
    x = xab[hi * (hi + 1) // 2 + lo]
    hao = np.asarray(hao, dtype=np.float64)
    xdiag = np.asarray(xdiag, dtype=np.float64)
    P = np.asarray(Pvec, dtype=np.float64)
    off = P * (hao[ci] + hao[rj]) * x
    dia = 2.0 * P * xdiag[ci] * hao[ci] * x
    return np.asarray(Hvec, dtype=np.float64) + np.where(rj < ci, off, dia)


def _packed_cols_rows(n: int):
    """0-based (column, row) of every packed element in storage order."""
    cols = np.repeat(np.arange(n, dtype=np.int64), np.arange(1, n + 1))
    starts = cols * (cols + 1) // 2
    rows = np.arange(n * (n + 1) // 2, dtype=np.int64) - starts
    return cols, rows


def lin(i1: int, i2: int) -> int:
    """1-based packed address of (i1, i2), source/lin.f:5-11."""
    a, b = max(i1, i2), min(i1, i2)
    return b + a * (a - 1) // 2
