"""Host-side mirror of the reference's density-step interface over the C-ABI.

The functions keep the reference's names and argument meaning:

* ``sm_stupid_simple``  -> source/sm.f90:34 (submatrix method)
* ``purification``      -> source/purification.f90:28 (purification_wrapper)
* ``solve2``            -> source/pgtb.f90:1066 (dense FP64 diagonalisation)
* ``filter_matrix_sym`` -> source/pgtb.f90:1532
* ``check_density`` / ``get_nel`` / ``band_structure`` / ``idempotent``
                        -> source/metrics.f90:144-360
plus ``tc_purify`` (trace-correcting purification, the B200 fast path of the
dense step).  Arrays are numpy float64 in the reference's packed layout;
default Fortran integers are int64.  Every call goes through libptbgpu.so;
there is no CPU fallback: a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .settings import PurificationSettings

_LIB = None
_PKG = Path(__file__).resolve().parent

# status codes (include/ptbgpu.h)
OK, EINVAL, ECUDA, ENOTSPD, ENAN, EITER, ENOTIMPL, ETIMEOUT, ENOMEM = range(9)
PREC_FP64, PREC_MIXED, PREC_MIXED_NOREFINE = 0, 1, 2
MULL_LOEW14 = 0.3333333333   # Mulliken/Loewdin mixing of the populations, source/parcom.f90:26


class PtbGpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class _Settings(C.Structure):
    _fields_ = [("mode", C.c_int64), ("type", C.c_int64), ("cycles", C.c_int64), ("prlvl", C.c_int64),
                ("nel", C.c_int64), ("submatrix_mode", C.c_int64), ("submatrix_columns", C.c_int64),
                ("metric_type", C.c_int64), ("metric_cycles", C.c_int64), ("metric_iterative", C.c_int64),
                ("chempot_cycles", C.c_int64), ("chempot_guess", C.c_double), ("chempot_increment", C.c_double)]


class _Opts(C.Structure):
    _fields_ = [("filter", C.c_double), ("precision", C.c_int64), ("print_level", C.c_int64),
                ("max_iter", C.c_int64), ("electronic_temp", C.c_double), ("glob_par15", C.c_double),
                ("glob_par17", C.c_double), ("split3_iters", C.c_int64),
                ("fp64_slices", C.c_int64), ("refine_rounds", C.c_int64), ("refine_tol", C.c_double)]


class _Stats(C.Structure):
    _fields_ = [("mu", C.c_double), ("nel", C.c_double), ("band_energy", C.c_double),
                ("idempotency_ref", C.c_double), ("idempotency_frob", C.c_double), ("nsm", C.c_int64),
                ("sum_dims", C.c_int64), ("max_dim", C.c_int64), ("iterations", C.c_int64),
                ("mu_iterations", C.c_int64), ("info", C.c_int64), ("ms_total", C.c_double),
                ("ms_h2d", C.c_double), ("ms_solve", C.c_double), ("ms_d2h", C.c_double), ("flops", C.c_double),
                ("ms_tc_sp2", C.c_double), ("n_tc_sp2", C.c_int64), ("ms_tc_full", C.c_double),
                ("n_tc_full", C.c_int64), ("kernel_launches", C.c_int64), ("ms_oz", C.c_double),
                ("n_oz", C.c_int64), ("oz_ops", C.c_double), ("tc_flops", C.c_double),
                ("refine_rounds", C.c_int64), ("fp64_fallback", C.c_int64)]


EXPORTED = ("ptbgpu_init", "ptbgpu_finalize", "ptbgpu_last_error", "ptbgpu_default_settings",
            "ptbgpu_default_opts", "ptbgpu_filter_packed", "ptbgpu_check_density", "ptbgpu_sm_density",
            "ptbgpu_purify", "ptbgpu_tc_purify", "ptbgpu_tc_purify_device", "ptbgpu_tc_purify_batch", "ptbgpu_tc_purify_grouped",
            "ptbgpu_eig_density_batch",
            "ptbgpu_solve2",
            "ptbgpu_symsq_bf16x3", "ptbgpu_symsq_bf16x6", "ptbgpu_symsq_split", "ptbgpu_runtime_info",
            "ptbgpu_density_traces_noalloc", "ptbgpu_oz_gemm", "ptbgpu_mlpop14", "ptbgpu_mlpop14_device",
            "ptbgpu_mlpop2", "ptbgpu_mlpop2_device", "ptbgpu_kmeans_partition", "ptbgpu_sm_plan",
            "ptbgpu_sm_prepare", "ptbgpu_sm_nel", "ptbgpu_sm_finish", "ptbgpu_xc_damping",
            "ptbgpu_xc_damping_device", "ptbgpu_selftest_bounded_wait", "ptbgpu_oz_tiles",
            "ptbgpu_sygv_batched")


def library_path() -> Path:
    return Path(os.environ.get("PTBGPU_LIB", _PKG / "libptbgpu.so"))


def load_library():
    """Loads libptbgpu.so (built by ptb_b200.build); raises if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not path.exists():
        raise PtbGpuError(ECUDA, f"{path} not found: build it with `python -m ptb_b200.build`")
    # RTLD_DEEPBIND: the library and the cuBLAS / cuSOLVER it was linked against
    # resolve their symbols inside their own tree first, so copies of the same
    # libraries that other packages (torch) load into the global scope are not
    # mixed into our calls.  Load this module before importing such packages.
    mode = C.RTLD_LOCAL | getattr(os, "RTLD_NOW", 2) | getattr(os, "RTLD_DEEPBIND", 8)
    lib = C.CDLL(str(path), mode=mode)
    P = C.POINTER
    d = P(C.c_double)
    i64 = C.c_int64
    lib.ptbgpu_init.argtypes = [C.c_int, P(C.c_void_p)]
    lib.ptbgpu_finalize.argtypes = [C.c_void_p]
    lib.ptbgpu_last_error.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
    lib.ptbgpu_default_settings.argtypes = [P(_Settings)]
    lib.ptbgpu_default_settings.restype = None
    lib.ptbgpu_default_opts.argtypes = [P(_Opts)]
    lib.ptbgpu_default_opts.restype = None
    lib.ptbgpu_filter_packed.argtypes = [C.c_void_p, i64, d, C.c_double]
    lib.ptbgpu_check_density.argtypes = [C.c_void_p, i64, d, d, d, P(_Stats)]
    lib.ptbgpu_sm_density.argtypes = [C.c_void_p, i64, i64, d, d, d, i64, d, P(i64), i64, i64, P(i64),
                                      P(_Opts), P(_Stats)]
    lib.ptbgpu_purify.argtypes = [C.c_void_p, P(_Settings), i64, d, d, d, P(_Opts), P(_Stats)]
    lib.ptbgpu_tc_purify.argtypes = [C.c_void_p, i64, i64, d, d, d, P(_Opts), P(_Stats)]
    lib.ptbgpu_tc_purify_device.argtypes = [C.c_void_p, i64, i64, C.c_void_p, C.c_void_p, C.c_void_p, P(_Opts),
                                            P(_Stats)]
    lib.ptbgpu_tc_purify_batch.argtypes = [C.c_void_p, i64, P(i64), P(i64), P(d), P(d), P(d), i64, P(_Opts),
                                           P(_Stats), d]
    lib.ptbgpu_tc_purify_grouped.argtypes = [C.c_void_p, i64, P(i64), P(i64), P(d), P(d), P(d), P(_Opts),
                                             P(_Stats), d]
    lib.ptbgpu_eig_density_batch.argtypes = [C.c_void_p, i64, P(i64), P(i64), P(d), P(d), P(d), P(_Opts),
                                             P(_Stats), d]
    lib.ptbgpu_solve2.argtypes = [C.c_void_p, i64, i64, i64, i64, d, d, d, d, d, P(_Opts), P(_Stats)]
    lib.ptbgpu_selftest_bounded_wait.argtypes = [C.c_void_p, i64]
    lib.ptbgpu_xc_damping.argtypes = [C.c_void_p, i64, i64, P(i64), d, d, d, d, d, d, d]
    lib.ptbgpu_xc_damping_device.argtypes = [C.c_void_p, i64, i64, P(i64), d, d, d, d, C.c_void_p, C.c_void_p, d]
    lib.ptbgpu_symsq_bf16x3.argtypes = [C.c_void_p, i64, d, P(C.c_float)]
    lib.ptbgpu_symsq_bf16x6.argtypes = [C.c_void_p, i64, d, P(C.c_float)]
    lib.ptbgpu_symsq_split.argtypes = [C.c_void_p, i64, i64, i64, d, P(C.c_float), d]
    lib.ptbgpu_oz_gemm.argtypes = [C.c_void_p, i64, i64, i64, i64, i64, i64, i64, d, d, d, d]
    lib.ptbgpu_oz_tiles.argtypes = [i64, i64, i64, i64, i64, i64, i64, P(C.c_int32), i64, P(i64), P(i64)]
    lib.ptbgpu_sygv_batched.argtypes = [C.c_void_p, i64, P(i64), d, d, P(i64), P(i64), C.c_double, d, d, d]
    lib.ptbgpu_kmeans_partition.argtypes = [C.c_void_p, i64, d, d, i64, d, P(i64), C.c_uint64, P(_Opts), P(i64),
                                            P(i64), d]
    lib.ptbgpu_sm_plan.argtypes = [C.c_void_p, i64, d, d, i64, d, P(i64), i64, i64, P(i64), P(_Opts), P(i64),
                                   P(i64)]
    lib.ptbgpu_sm_prepare.argtypes = [C.c_void_p, i64, P(i64), P(_Stats)]
    lib.ptbgpu_sm_nel.argtypes = [C.c_void_p, C.c_double, d]
    lib.ptbgpu_sm_finish.argtypes = [C.c_void_p, i64, C.c_double, d]
    f = P(C.c_float)
    lib.ptbgpu_mlpop14.argtypes = [C.c_void_p, i64, d, C.c_double, f, f]
    lib.ptbgpu_mlpop14_device.argtypes = [C.c_void_p, i64, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    lib.ptbgpu_mlpop2.argtypes = [C.c_void_p, i64, i64, d, f, f, P(i64), P(i64), d, d, P(_Stats)]
    lib.ptbgpu_mlpop2_device.argtypes = [C.c_void_p, i64, i64, C.c_void_p, C.c_void_p, C.c_void_p, P(i64), P(i64),
                                         d, d, P(_Stats)]
    lib.ptbgpu_runtime_info.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
    lib.ptbgpu_density_traces_noalloc.argtypes = [C.c_int, i64, C.c_void_p, C.c_void_p, C.c_void_p, d,
                                                  C.c_void_p, C.c_char_p, C.c_size_t]
    for name in EXPORTED:
        f = getattr(lib, name)
        if f.restype is not None and name not in ("ptbgpu_default_settings", "ptbgpu_default_opts"):
            f.restype = C.c_int
    _LIB = lib
    return lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def npacked(n: int) -> int:
    return n * (n + 1) // 2


# The C-ABI takes bare pointers and reads as many elements as the sizes say, so
# the lengths of the host arrays are checked here, before any call.
def _packed(a, ndim: int, what: str) -> np.ndarray:
    """A packed symmetric matrix of order ndim as a contiguous float64 array."""
    x = _f64(a)
    if x.size != npacked(max(int(ndim), 0)):
        raise PtbGpuError(EINVAL, f"{what} has {x.size} elements; a packed matrix of order {ndim} has "
                                  f"{npacked(max(int(ndim), 0))}")
    return x


def _out_packed(out, ndim: int) -> np.ndarray:
    """A caller-provided output array for a packed matrix of order ndim (for
    instance in pinned host memory, which the device-to-host copy needs for
    full speed), or a new one."""
    if out is None:
        return np.empty(npacked(ndim))
    if out.dtype != np.float64 or out.size != npacked(ndim) or not out.flags.c_contiguous:
        raise ValueError("out must be a contiguous float64 array of npacked(ndim) elements")
    return out


def _vec(a, count: int, what: str, conv=None) -> np.ndarray:
    """An array of exactly count elements (float64, or int64 with conv=_i64)."""
    x = (conv or _f64)(a)
    if x.size != max(int(count), 0):
        raise PtbGpuError(EINVAL, f"{what} has {x.size} elements, expected {max(int(count), 0)}")
    return x


@dataclass
class Stats:
    mu: float = 0.0
    nel: float = 0.0
    band_energy: float = 0.0
    idempotency_ref: float = 0.0
    idempotency_frob: float = 0.0
    nsm: int = 0
    sum_dims: int = 0
    max_dim: int = 0
    iterations: int = 0
    mu_iterations: int = 0
    info: int = 0
    ms_total: float = 0.0
    ms_h2d: float = 0.0
    ms_solve: float = 0.0
    ms_d2h: float = 0.0
    flops: float = 0.0
    ms_tc_sp2: float = 0.0
    n_tc_sp2: int = 0
    ms_tc_full: float = 0.0
    n_tc_full: int = 0
    kernel_launches: int = 0
    ms_oz: float = 0.0
    n_oz: int = 0
    oz_ops: float = 0.0
    tc_flops: float = 0.0
    refine_rounds: int = 0
    fp64_fallback: int = 0

    @classmethod
    def from_c(cls, s: _Stats) -> "Stats":
        return cls(**{k: getattr(s, k) for k, _ in _Stats._fields_})


@dataclass
class Options:
    """Options without a counterpart in the reference's argument lists."""
    filter: float = 0.0
    precision: int = PREC_MIXED
    print_level: int = 0
    max_iter: int = 100
    electronic_temp: float = 300.0
    glob_par15: float = 0.0
    glob_par17: float = 0.0
    split3_iters: int = -1
    fp64_slices: int = 8
    refine_rounds: int = 4
    refine_tol: float = 1e-7

    def to_c(self) -> _Opts:
        return _Opts(self.filter, self.precision, self.print_level, self.max_iter, self.electronic_temp,
                     self.glob_par15, self.glob_par17, self.split3_iters, self.fp64_slices, self.refine_rounds,
                     self.refine_tol)


class Context:
    """One library context (device buffers, stream, cuBLAS/cuSOLVER handles)."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        h = C.c_void_p()
        rc = self._lib.ptbgpu_init(int(device), C.byref(h))
        if rc != OK:
            raise PtbGpuError(rc, f"ptbgpu_init(device={device}) failed")
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ptbgpu_finalize(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != OK:
            buf = C.create_string_buffer(1024)
            self._lib.ptbgpu_last_error(self._h, buf, 1024)
            raise PtbGpuError(rc, buf.value.decode(errors="replace"))

    def runtime_info(self) -> str:
        """Device and the CUDA runtime / driver / cuBLAS / cuSOLVER versions in use."""
        buf = C.create_string_buffer(512)
        self._check(self._lib.ptbgpu_runtime_info(self._h, buf, 512))
        return buf.value.decode()

    # ---- reference entry points ------------------------------------------
    def filter_matrix_sym(self, A: np.ndarray, n: int, filter: float) -> np.ndarray:
        """source/pgtb.f90:1532-1547, returns the filtered packed copy."""
        out = _packed(A, n, "A").copy()
        self._check(self._lib.ptbgpu_filter_packed(self._h, int(n), _dptr(out), float(filter)))
        return out

    def check_density(self, ndim: int, P: np.ndarray, S: np.ndarray, H: np.ndarray | None = None) -> Stats:
        """get_nel, band_structure and idempotent (source/metrics.f90:144-360) on packed data."""
        st = _Stats()
        P, S = _packed(P, ndim, "P"), _packed(S, ndim, "S")
        Hp = _dptr(_packed(H, ndim, "H")) if H is not None else None
        self._check(self._lib.ptbgpu_check_density(self._h, int(ndim), _dptr(P), _dptr(S), Hp, C.byref(st)))
        return Stats.from_c(st)

    def sm_stupid_simple(self, ndim: int, nelref: int, Hvec: np.ndarray, Svec: np.ndarray, n: int,
                         xyz: np.ndarray, aoat: np.ndarray, submatrix_columns: int, submatrix_mode: int,
                         partition: np.ndarray | None = None, opts: Options | None = None,
                         out: np.ndarray | None = None):
        """Submatrix density step, source/sm.f90:34-409.  Returns (Pvec, Stats).
        out: a preallocated contiguous float64 array of npacked(ndim) elements
        for P (every element is written)."""
        H, S = _packed(Hvec, ndim, "Hvec"), _packed(Svec, ndim, "Svec")
        P = _out_packed(out, ndim)
        xyz_a = _vec(xyz, 3 * n, "xyz")
        ao = _vec(aoat, ndim, "aoat", _i64)
        part = _i64(partition) if partition is not None else None
        st = _Stats()
        o = (opts or Options()).to_c()
        self._check(self._lib.ptbgpu_sm_density(
            self._h, int(ndim), int(nelref), _dptr(H), _dptr(S), _dptr(P), int(n), _dptr(xyz_a),
            ao.ctypes.data_as(C.POINTER(C.c_int64)), int(submatrix_columns), int(submatrix_mode),
            part.ctypes.data_as(C.POINTER(C.c_int64)) if part is not None else None, C.byref(o), C.byref(st)))
        return P, Stats.from_c(st)

    # ---- the submatrix method in phases (one rank's share; ptb_b200.distributed) ----
    def sm_plan(self, ndim: int, Hvec: np.ndarray, Svec: np.ndarray, n: int, xyz: np.ndarray, aoat: np.ndarray,
                submatrix_columns: int, submatrix_mode: int, partition: np.ndarray | None = None,
                opts: Options | None = None) -> np.ndarray:
        """Grouping, pattern scan and maps of the whole system; returns the
        submatrix dimensions (nsm,)."""
        nsm = C.c_int64(0)
        dims = np.zeros(ndim, dtype=np.int64)
        o = (opts or Options()).to_c()
        H, S = _packed(Hvec, ndim, "Hvec"), _packed(Svec, ndim, "Svec")
        xyz_a = _vec(xyz, 3 * n, "xyz")
        ao = _vec(aoat, ndim, "aoat", _i64)
        part = _i64(partition) if partition is not None else None
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))
        self._check(self._lib.ptbgpu_sm_plan(
            self._h, int(ndim), _dptr(H), _dptr(S), int(n), _dptr(xyz_a), ip(ao),
            int(submatrix_columns), int(submatrix_mode), ip(part) if part is not None else None, C.byref(o),
            C.byref(nsm), ip(dims)))
        return dims[:nsm.value].copy()

    def sm_prepare(self, ids) -> "Stats":
        """Eigenpairs and fe weights of the listed submatrices (0-based)."""
        v = _i64(np.asarray(ids, dtype=np.int64).reshape(-1))
        st = _Stats()
        self._check(self._lib.ptbgpu_sm_prepare(self._h, int(v.shape[0]), v.ctypes.data_as(C.POINTER(C.c_int64)),
                                                C.byref(st)))
        return Stats.from_c(st)

    def sm_nel(self, mu: float) -> float:
        """Electron count of the prepared submatrices at mu."""
        v = C.c_double(0.0)
        self._check(self._lib.ptbgpu_sm_nel(self._h, float(mu), C.byref(v)))
        return v.value

    def sm_finish(self, ndim: int, mu: float) -> np.ndarray:
        """Owned columns of the prepared submatrices at mu (packed, zeros elsewhere)."""
        P = np.zeros(npacked(ndim))
        self._check(self._lib.ptbgpu_sm_finish(self._h, int(ndim), float(mu), _dptr(P)))
        return P

    def kmeans_partition(self, ndim: int, Hvec: np.ndarray, Svec: np.ndarray, n: int, xyz: np.ndarray,
                         aoat: np.ndarray, seed: int = 42, opts: Options | None = None):
        """Columns mode 4 grouping (source/sm.f90:127-154, clustering_kmeans
        :459-514): seeded k-means++ for 1..min(64, n) clusters, least sum of
        dim^2.5.  Returns (1-based atom -> cluster partition, nsm, effort)."""
        part = np.zeros(n, dtype=np.int64)
        nsm = C.c_int64(0)
        eff = C.c_double(0.0)
        o = (opts or Options()).to_c()
        H, S = _packed(Hvec, ndim, "Hvec"), _packed(Svec, ndim, "Svec")
        xyz_a = _vec(xyz, 3 * n, "xyz")
        ao = _vec(aoat, ndim, "aoat", _i64)
        self._check(self._lib.ptbgpu_kmeans_partition(
            self._h, int(ndim), _dptr(H), _dptr(S), int(n), _dptr(xyz_a),
            ao.ctypes.data_as(C.POINTER(C.c_int64)), C.c_uint64(seed), C.byref(o),
            part.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(nsm), C.byref(eff)))
        return part, int(nsm.value), float(eff.value)

    def purification(self, pur: PurificationSettings, ndim: int, H: np.ndarray, S: np.ndarray,
                     opts: Options | None = None):
        """purification_wrapper, source/purification.f90:28-80.  Returns (Pvec, Stats)."""
        Hh, Sh = _packed(H, ndim, "H"), _packed(S, ndim, "S")
        P = np.zeros(npacked(ndim))
        st = _Stats()
        cs = pur.to_c(_Settings)
        o = (opts or Options()).to_c()
        self._check(self._lib.ptbgpu_purify(self._h, C.byref(cs), int(ndim), _dptr(Hh), _dptr(Sh), _dptr(P),
                                            C.byref(o), C.byref(st)))
        return P, Stats.from_c(st)

    def tc_purify(self, ndim: int, nel: int, H: np.ndarray, S: np.ndarray, opts: Options | None = None,
                  out: np.ndarray | None = None):
        """Trace-correcting purification (FP64 or bf16x3 + FP64 refinement).  Returns (Pvec, Stats).
        out: a preallocated contiguous float64 array of npacked(ndim) elements for P (e.g. in
        pinned memory, which the device-to-host copy needs for full speed)."""
        Hh, Sh = _packed(H, ndim, "H"), _packed(S, ndim, "S")
        P = _out_packed(out, ndim)
        st = _Stats()
        o = (opts or Options()).to_c()
        self._check(self._lib.ptbgpu_tc_purify(self._h, int(ndim), int(nel), _dptr(Hh), _dptr(Sh), _dptr(P),
                                               C.byref(o), C.byref(st)))
        return P, Stats.from_c(st)

    def tc_purify_device(self, ndim: int, nel: int, dH: int, dS: int, dP: int, opts: Options | None = None):
        """Same on device-resident packed arrays (raw device pointers)."""
        st = _Stats()
        o = (opts or Options()).to_c()
        self._check(self._lib.ptbgpu_tc_purify_device(self._h, int(ndim), int(nel), C.c_void_p(dH),
                                                      C.c_void_p(dS), C.c_void_p(dP), C.byref(o), C.byref(st)))
        return Stats.from_c(st)

    def tc_purify_batch(self, systems, opts: Options | None = None, workers: int = 0):
        """tc_purify over many independent systems, `systems` a sequence of
        (ndim, nel, H, S).  Host worker threads with their own streams overlap
        the systems on the GPU.  Returns ([Pvec], [Stats], wall milliseconds)."""
        n = len(systems)
        m = max(n, 1)
        ndim = (C.c_int64 * m)(*[int(s[0]) for s in systems])
        nel = (C.c_int64 * m)(*[int(s[1]) for s in systems])
        Hs = [_packed(s[2], s[0], f"H of system {i}") for i, s in enumerate(systems)]
        Ss = [_packed(s[3], s[0], f"S of system {i}") for i, s in enumerate(systems)]
        Ps = [np.zeros(npacked(int(s[0]))) for s in systems]
        arr = lambda xs: (C.POINTER(C.c_double) * m)(*[_dptr(x) for x in xs])
        st = (_Stats * max(n, 1))()
        wall = C.c_double(0.0)
        o = (opts or Options()).to_c()
        self._check(self._lib.ptbgpu_tc_purify_batch(self._h, n, ndim, nel, arr(Hs), arr(Ss), arr(Ps),
                                                     int(workers), C.byref(o), st, C.byref(wall)))
        return Ps, [Stats.from_c(st[i]) for i in range(n)], wall.value

    def eig_density_batch(self, systems, opts: Options | None = None):
        """The density step of many independent systems in one launch of the
        FP64 eigensolver (ptbgpu_eig_density_batch): `systems` a sequence of
        (ndim, nel, H, S) packed; P = 2 sum of the nel/2 lowest generalized
        eigenvectors' outer products (opts.filter applied to H and S).  Returns
        ([Pvec], [Stats], wall milliseconds)."""
        n = len(systems)
        m = max(n, 1)
        for i, s in enumerate(systems):
            if int(s[1]) % 2:
                raise PtbGpuError(EINVAL, f"system {i}: odd electron count {int(s[1])} (the T = 0 projector "
                                          "here is closed-shell)")
        ndim = (C.c_int64 * m)(*[int(s[0]) for s in systems])
        nel = (C.c_int64 * m)(*[int(s[1]) for s in systems])
        Hs = [_packed(s[2], s[0], f"H of system {i}") for i, s in enumerate(systems)]
        Ss = [_packed(s[3], s[0], f"S of system {i}") for i, s in enumerate(systems)]
        Ps = [np.zeros(npacked(int(s[0]))) for s in systems]
        arr = lambda xs: (C.POINTER(C.c_double) * m)(*[_dptr(x) for x in xs])
        st = (_Stats * m)()
        wall = C.c_double(0.0)
        o = (opts or Options()).to_c()
        self._check(self._lib.ptbgpu_eig_density_batch(self._h, n, ndim, nel, arr(Hs), arr(Ss), arr(Ps),
                                                       C.byref(o), st, C.byref(wall)))
        return Ps, [Stats.from_c(st[i]) for i in range(n)], wall.value

    def xc_damping(self, nat: int, ndim: int, aoat, rab, rad, hao, xdiag, P: np.ndarray, H: np.ndarray,
                   timed: bool = False):
        """Iteration-2 XC long-range damping, source/pgtb.f90:482-513: returns H + the
        P-dependent term (packed); timed: (H, device ms of the AO-pair update)."""
        a = _vec(aoat, ndim, "aoat", _i64)
        Hout = _packed(H, ndim, "H").copy()
        rab_, rad_ = _packed(rab, nat, "rab"), _vec(rad, nat, "rad")
        hao_, xd_ = _vec(hao, ndim, "hao"), _vec(xdiag, ndim, "xdiag")
        Pp = _packed(P, ndim, "P")
        ms = C.c_double(0.0)
        self._check(self._lib.ptbgpu_xc_damping(self._h, int(nat), int(ndim), a.ctypes.data_as(C.POINTER(C.c_int64)),
                                                _dptr(rab_), _dptr(rad_), _dptr(hao_), _dptr(xd_), _dptr(Pp),
                                                _dptr(Hout), C.byref(ms)))
        return (Hout, ms.value) if timed else Hout

    def xc_damping_device(self, nat: int, ndim: int, aoat, rab, rad, hao, xdiag, dP: int, dH: int) -> float:
        """Same on device-resident packed P and H (raw device pointers, H updated in
        place); returns the device ms of the AO-pair update."""
        a = _vec(aoat, ndim, "aoat", _i64)
        rab_, rad_ = _packed(rab, nat, "rab"), _vec(rad, nat, "rad")
        hao_, xd_ = _vec(hao, ndim, "hao"), _vec(xdiag, ndim, "xdiag")
        ms = C.c_double(0.0)
        self._check(self._lib.ptbgpu_xc_damping_device(self._h, int(nat), int(ndim),
                                                       a.ctypes.data_as(C.POINTER(C.c_int64)), _dptr(rab_),
                                                       _dptr(rad_), _dptr(hao_), _dptr(xd_),
                                                       C.c_void_p(dP), C.c_void_p(dH), C.byref(ms)))
        return ms.value

    def tc_purify_grouped(self, systems, opts: Options | None = None):
        """tc_purify over many systems grouped into stacked launches per size
        bucket, `systems` a sequence of (ndim, nel, H, S).  Returns ([Pvec],
        [Stats], wall milliseconds)."""
        n = len(systems)
        m = max(n, 1)
        ndim = (C.c_int64 * m)(*[int(s[0]) for s in systems])
        nel = (C.c_int64 * m)(*[int(s[1]) for s in systems])
        Hs = [_packed(s[2], s[0], f"H of system {i}") for i, s in enumerate(systems)]
        Ss = [_packed(s[3], s[0], f"S of system {i}") for i, s in enumerate(systems)]
        Ps = [np.zeros(npacked(int(s[0]))) for s in systems]
        arr = lambda xs: (C.POINTER(C.c_double) * m)(*[_dptr(x) for x in xs])
        st = (_Stats * m)()
        wall = C.c_double(0.0)
        o = (opts or Options()).to_c()
        self._check(self._lib.ptbgpu_tc_purify_grouped(self._h, n, ndim, nel, arr(Hs), arr(Ss), arr(Ps), C.byref(o),
                                                       st, C.byref(wall)))
        return Ps, [Stats.from_c(st[i]) for i in range(n)], wall.value

    def selftest_bounded_wait(self, limit_us: int = 20000):
        """One bounded device wait on a flag nothing sets: raises PtbGpuError with
        code ETIMEOUT through the library's device-error path."""
        self._check(self._lib.ptbgpu_selftest_bounded_wait(self._h, int(limit_us)))

    def solve2(self, mode: int, ndim: int, nel: int, nopen: int, H: np.ndarray, S: np.ndarray,
               opts: Options | None = None):
        """Dense FP64 diagonalisation + Fermi smearing, source/pgtb.f90:1066-1170.

        Returns (Pvec, e, focc, Stats)."""
        Hh, Sh = _packed(H, ndim, "H"), _packed(S, ndim, "S")
        P = np.zeros(npacked(ndim))
        e = np.zeros(ndim)
        focc = np.zeros(ndim)
        st = _Stats()
        o = (opts or Options()).to_c()
        self._check(self._lib.ptbgpu_solve2(self._h, int(mode), int(ndim), int(nel), int(nopen), _dptr(Hh),
                                            _dptr(Sh), _dptr(P), _dptr(e), _dptr(focc), C.byref(o), C.byref(st)))
        return P, e, focc, Stats.from_c(st)

    # ---- kernel level ------------------------------------------------------
    def symsq_bf16x3(self, X: np.ndarray) -> np.ndarray:
        """C = X X (symmetric X) on the tcgen05 kernel with bf16x3 operands; FP32 result."""
        return self._symsq(X, self._lib.ptbgpu_symsq_bf16x3)

    def symsq_bf16x6(self, X: np.ndarray) -> np.ndarray:
        """C = X X with the three-plane split (bf16x6 products); FP32 result."""
        return self._symsq(X, self._lib.ptbgpu_symsq_bf16x6)

    def symsq_split(self, X: np.ndarray, planes: int, kblock: int, timed: bool = False):
        """C = X X with an explicit plane count (2 or 3) and kernel: K block 32 /
        64 (one CTA), 1032 / 1064 (CTA pair, two planes), 0 = tuned.  timed:
        returns (C, device milliseconds of the product launches)."""
        ms = C.c_double(0.0)
        out = self._symsq(X, lambda h, n, x, o: self._lib.ptbgpu_symsq_split(h, n, planes, kblock, x, o,
                                                                              C.byref(ms)))
        return (out, ms.value) if timed else out

    def oz_gemm(self, A: np.ndarray, B: np.ndarray, slices: int = 7, kblock: int = 0, tri_a: int = 0,
                tri_b: int = 0, symmetric: bool = False, timed: bool = False, variant: int = 0):
        """C = A B in FP64 on the int8 tensor cores (4 or 6..8 slices per
        operand row); tri_*: 0 full, 1 lower, 2 upper triangular operand;
        symmetric: only the upper triangle of C is computed and mirrored;
        variant: 0 default, 1 A from shared memory, 2 A in tensor memory,
        3 A from shared memory on a CTA pair (256-row tiles), 4 128-column
        tiles summed in two passes over K (kblock 0 or 32), 5 variant 4 on a
        CTA pair (256 x 128 tiles).
        timed: returns (C, device milliseconds of the product kernel)."""
        Ah, Bh = _f64(A), _f64(B)
        n = Ah.shape[0]
        out = np.zeros((n, n), dtype=np.float64)
        ms = C.c_double(0.0)
        self._check(self._lib.ptbgpu_oz_gemm(self._h, int(n), int(slices), int(kblock), int(variant), int(tri_a),
                                             int(tri_b), int(bool(symmetric)), _dptr(Ah), _dptr(Bh), _dptr(out),
                                             C.byref(ms)))
        return (out, ms.value) if timed else out

    def sygv_batched(self, problems, mu: float | None = None):
        """The submatrix method's batched generalized eigensolver on dense problems
        (ptbgpu_sygv_batched): problems = [(H_k, S_k, owned_k)] with (m, m) arrays
        and 0-based local owned indices.  Returns per problem (e, fe) (the
        solver's order), and with mu given also the owned columns of
        P = U occ U^T as an (m, len(owned)) array."""
        dims = np.array([np.asarray(h).shape[0] for h, _, _ in problems], dtype=np.int64)
        for (h, s_, o), m in zip(problems, dims):
            if np.asarray(h).shape != (m, m) or np.asarray(s_).shape != (m, m) or len(o) == 0:
                raise PtbGpuError(EINVAL, "problem arrays must be (m, m) with at least one owned index")
        H = np.concatenate([np.asarray(h, dtype=np.float64).ravel(order="F") for h, _, _ in problems])
        S = np.concatenate([np.asarray(s_, dtype=np.float64).ravel(order="F") for _, s_, _ in problems])
        nown = np.array([len(o) for _, _, o in problems], dtype=np.int64)
        owned = np.concatenate([np.asarray(o, dtype=np.int64) for _, _, o in problems])
        tot = int(dims.sum())
        e = np.zeros(tot)
        fe = np.zeros(tot)
        pc = np.zeros(int(np.sum(dims * nown))) if mu is not None else None
        self._check(self._lib.ptbgpu_sygv_batched(
            self._h, len(problems), dims.ctypes.data_as(C.POINTER(C.c_int64)), _dptr(H), _dptr(S),
            nown.ctypes.data_as(C.POINTER(C.c_int64)), owned.ctypes.data_as(C.POINTER(C.c_int64)),
            float(mu if mu is not None else 0.0), _dptr(e), _dptr(fe), _dptr(pc) if pc is not None else None))
        out, o0, p0 = [], 0, 0
        for m, no in zip(dims, nown):
            item = [e[o0:o0 + m], fe[o0:o0 + m]]
            if pc is not None:
                item.append(pc[p0:p0 + m * no].reshape((m, no), order="F"))
            out.append(tuple(item))
            o0 += m
            p0 += m * no
        return out

    # ---- population analysis (source/mlpop.f) ----
    def mlpop14(self, nao: int, Svec: np.ndarray, x: float = MULL_LOEW14):
        """mlpop14 (source/mlpop.f:142): (s34, s14) = (S^(1-x), S^x) as float32
        (nao, nao) arrays indexed [row, col] (column-major in memory)."""
        s34 = np.zeros((nao, nao), dtype=np.float32, order="F")
        s14 = np.zeros((nao, nao), dtype=np.float32, order="F")
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        Sp = _packed(Svec, nao, "Svec")
        self._check(self._lib.ptbgpu_mlpop14(self._h, int(nao), _dptr(Sp), float(x), fp(s34), fp(s14)))
        return s34, s14

    def mlpop2(self, n: int, nao: int, Pvec: np.ndarray, s1: np.ndarray, s2: np.ndarray, aoat: np.ndarray,
               shell2ao: np.ndarray):
        """mlpop2 (source/mlpop.f:198): atomic populations q (n,) and shell
        populations qsh (n, 10) (Fortran qsh(10, n)); s1 = S^(1-x), s2 = S^x
        indexed [row, col]; aoat / shell2ao 1-based."""
        f1 = np.asfortranarray(s1, dtype=np.float32)
        f2 = np.asfortranarray(s2, dtype=np.float32)
        for name, f in (("s1", f1), ("s2", f2)):
            if f.shape != (nao, nao):
                raise PtbGpuError(EINVAL, f"{name} has shape {f.shape}, expected ({nao}, {nao})")
        q = np.zeros(n)
        qsh = np.zeros((n, 10))
        st = _Stats()
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))
        a, sh = _vec(aoat, nao, "aoat", _i64), _vec(shell2ao, nao, "shell2ao", _i64)
        Pp = _packed(Pvec, nao, "Pvec")
        self._check(self._lib.ptbgpu_mlpop2(self._h, int(n), int(nao), _dptr(Pp), fp(f1), fp(f2), ip(a),
                                            ip(sh), _dptr(q), _dptr(qsh), C.byref(st)))
        return q, qsh, Stats.from_c(st)

    def mlpop2_device(self, n: int, nao: int, dP: int, ds1: int, ds2: int, aoat: np.ndarray,
                      shell2ao: np.ndarray):
        """mlpop2 on device-resident packed P and column-major float32 s1, s2
        (raw device pointers)."""
        q = np.zeros(n)
        qsh = np.zeros((n, 10))
        st = _Stats()
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))
        a, sh = _vec(aoat, nao, "aoat", _i64), _vec(shell2ao, nao, "shell2ao", _i64)
        self._check(self._lib.ptbgpu_mlpop2_device(self._h, int(n), int(nao), C.c_void_p(dP), C.c_void_p(ds1),
                                                   C.c_void_p(ds2), ip(a), ip(sh), _dptr(q), _dptr(qsh),
                                                   C.byref(st)))
        return q, qsh, Stats.from_c(st)

    def _symsq(self, X, fn):
        Xh = _f64(X)
        n = Xh.shape[0]
        out = np.zeros((n, n), dtype=np.float32)
        self._check(fn(self._h, int(n), _dptr(Xh), out.ctypes.data_as(C.POINTER(C.c_float))))
        return out


def density_traces_noalloc(device: int, ndim: int, dP: int, dS: int, dH: int | None = None,
                           stream: int | None = None) -> tuple[float, float]:
    """(tr(PS), tr(PH)) of device-resident packed P, S, H (raw device pointers)
    through ptbgpu_density_traces_noalloc: no context and no device allocation,
    for callers that cannot allocate device memory; ndim <= 65536."""
    lib = load_library()
    out = np.zeros(2)
    err = C.create_string_buffer(512)
    rc = lib.ptbgpu_density_traces_noalloc(int(device), int(ndim), C.c_void_p(dP), C.c_void_p(dS),
                                           C.c_void_p(dH) if dH else None, _dptr(out),
                                           C.c_void_p(stream) if stream else None, err, 512)
    if rc != OK:
        raise PtbGpuError(rc, err.value.decode(errors="replace"))
    return float(out[0]), float(out[1])


def oz_tiles(n: int, slices: int = 8, kblock: int = 0, variant: int = 0, a_tri: int = 0, b_tri: int = 0,
             symmetric: bool = False) -> tuple[np.ndarray, dict]:
    """Tile list of the int8-sliced product (ptbgpu_oz_tiles; host logic, no
    device): an (m, 4) int32 array of {row block (pair row block for the
    CTA-pair variants), column block, k0, k1} and a dict with the resolved
    variant, columns per tile, CTAs launched and rows per tile entry.  a_tri /
    b_tri mask the rows of A and of B^T: 0 none, 1 k <= i, 2 k >= i."""
    lib = load_library()
    cnt = C.c_int64(0)
    info = np.zeros(4, dtype=np.int64)
    args = (int(n), int(slices), int(kblock), int(variant), int(a_tri), int(b_tri), int(bool(symmetric)))
    ip = info.ctypes.data_as(C.POINTER(C.c_int64))
    rc = lib.ptbgpu_oz_tiles(*args, None, 0, C.byref(cnt), ip)
    if rc != OK:
        raise PtbGpuError(rc, "ptbgpu_oz_tiles: bad arguments")
    tiles = np.zeros((cnt.value, 4), dtype=np.int32)
    rc = lib.ptbgpu_oz_tiles(*args, tiles.ctypes.data_as(C.POINTER(C.c_int32)), cnt.value, C.byref(cnt), ip)
    if rc != OK:
        raise PtbGpuError(rc, "ptbgpu_oz_tiles failed")
    return tiles, {"variant": int(info[0]), "tile_n": int(info[1]), "ctas": int(info[2]), "rows": int(info[3])}


# module-level conveniences with the reference's names -----------------------
def get_nel(ctx: Context, ndim: int, P: np.ndarray, S: np.ndarray) -> float:
    """tr(PS) of packed P, S (source/metrics.f90:202-230)."""
    return ctx.check_density(ndim, P, S).nel


def band_structure(ctx: Context, ndim: int, P: np.ndarray, H: np.ndarray, S: np.ndarray) -> float:
    """tr(PH) of packed P, H (source/metrics.f90:253-277)."""
    return ctx.check_density(ndim, P, S, H).band_energy
