"""GPU parity of the int8-sliced FP64 product (tcgen05 kind::i8) through the
C-ABI, and of the mixed purification path that uses it.

Error model of the product with S slices: each operand row i is cut at
2^(e_i - 7S) (e_i: |row max| < 2^e_i) and slice pairs of weight below
2^(-7S) are dropped, so |C - AB|(i,j) <= 3 K 2^(-7S) 2^(e_i + f_j).  The int32
sums are exact, so the result does not depend on the K blocking.
"""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import PREC_FP64, PREC_MIXED, Options, PtbGpuError, synth

pytestmark = pytest.mark.gpu


def row_exp(M):
    m = np.max(np.abs(M), axis=1)
    e = np.zeros(len(m))
    nz = m > 0
    e[nz] = np.frexp(m[nz])[1]
    return e


def bound(A, B, S):
    """3 K 2^(-7S) 2^(e_i + f_j) with e from the rows of A and f from the columns of B."""
    K = A.shape[1]
    return 3.0 * K * 2.0 ** (-7 * S) * np.exp2(row_exp(A)[:, None] + row_exp(B.T)[None, :])


@pytest.mark.parametrize("n", [128, 300, 777])
@pytest.mark.parametrize("S", [6, 7, 8])
def test_oz_gemm_general(ctx, n, S):
    rng = np.random.default_rng(n + S)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, n))
    C = ctx.oz_gemm(A, B, slices=S)
    ref = (A.astype(np.longdouble) @ B.astype(np.longdouble)).astype(np.float64)
    err = np.abs(C - ref)
    assert np.all(err <= bound(A, B, S) + 2.0 ** -52 * np.abs(ref))
    if S == 8:
        assert np.max(err) < 1e-12


def test_oz_gemm_row_scales(ctx):
    """Rows and columns spread over 20 decades: the per-row exponents keep the
    error relative to each row's and column's own magnitude."""
    n = 400
    rng = np.random.default_rng(3)
    A = rng.standard_normal((n, n)) * (10.0 ** rng.uniform(-10, 10, n))[:, None]
    B = rng.standard_normal((n, n)) * (10.0 ** rng.uniform(-10, 10, n))[None, :]
    A[5] = 0.0   # a zero row
    C = ctx.oz_gemm(A, B, slices=7)
    ref = A @ B
    assert np.all(np.abs(C - ref) <= bound(A, B, 7))
    assert np.all(C[5] == 0.0)


def test_oz_gemm_k_blocking_is_bit_exact(ctx):
    n = 512
    rng = np.random.default_rng(9)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, n))
    C32 = ctx.oz_gemm(A, B, slices=7, kblock=32)
    C64 = ctx.oz_gemm(A, B, slices=7, kblock=64)
    assert np.array_equal(C32, C64)


@pytest.mark.parametrize("tri_a,tri_b", [(1, 0), (2, 0), (0, 1), (0, 2), (1, 2)])
def test_oz_gemm_triangular(ctx, tri_a, tri_b):
    """A triangular operand is read only inside its triangle (the rest may hold
    anything) and its K blocks past the diagonal are skipped."""
    n = 640
    rng = np.random.default_rng(10 * tri_a + tri_b)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, n))
    mask = {0: lambda M: M, 1: np.tril, 2: np.triu}
    Am, Bm = mask[tri_a](A), mask[tri_b](B)
    C = ctx.oz_gemm(A, B, slices=7, tri_a=tri_a, tri_b=tri_b)
    ref = Am @ Bm
    assert np.all(np.abs(C - ref) <= bound(Am, Bm, 7))


def test_oz_gemm_symmetric_output(ctx):
    n = 600
    rng = np.random.default_rng(11)
    X = rng.standard_normal((n, n))
    X = 0.5 * (X + X.T)
    C = ctx.oz_gemm(X, X, slices=7, symmetric=True)
    ref = X @ X
    assert np.array_equal(C, C.T)
    assert np.all(np.abs(C - ref) <= bound(X, X, 7))


def test_oz_gemm_rejects_bad_arguments(ctx):
    A = np.eye(64)
    with pytest.raises(PtbGpuError):
        ctx.oz_gemm(A, A, slices=5)
    with pytest.raises(PtbGpuError):
        ctx.oz_gemm(A, A, slices=7, kblock=48)


def test_mixed_path_int8_fp64_matches_cublas_fp64(ctx, water32):
    """The mixed path with its FP64 products on the int8 tensor cores agrees
    with the same path on cuBLAS/cuSOLVER FP64, and both meet the tolerances
    against the dense FP64 projector."""
    s = water32
    n = s.ndim
    Hf = O.blowsym(n, O.filter_matrix_sym(s.Hvec, 1e-5))
    Sf = O.blowsym(n, O.filter_matrix_sym(s.Svec, 1e-5))
    Pd, _ = O.dense_projector(Hf, Sf, s.nel)
    res = {}
    for S in (0, 7, 8):
        P, st = ctx.tc_purify(n, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=PREC_MIXED, fp64_slices=S))
        Pf = O.blowsym(n, P)
        assert np.max(np.abs(Pf - Pd)) <= 1e-6
        assert abs(O.band_structure(Pf, Hf) - O.band_structure(Pd, Hf)) <= 1e-6
        assert abs(O.get_nel(Pf, Sf) - s.nel) <= 1e-8
        assert (st.n_oz > 0) == (S > 0)
        res[S] = P
    assert np.max(np.abs(res[7] - res[0])) < 1e-8
    assert np.max(np.abs(res[8] - res[0])) < 1e-8


def test_fp64_slices_validated(ctx, water8):
    s = water8
    with pytest.raises(PtbGpuError):
        ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(precision=PREC_MIXED, fp64_slices=3))


@pytest.mark.parametrize("S", [4, 6, 7, 8])
@pytest.mark.parametrize("kblock", [32, 64])
def test_oz_gemm_tmem_a_variant_is_bit_exact(ctx, S, kblock):
    """The kernel that keeps the A slices in tensor memory (48- or 64-column
    tiles) sums the same exact int32 products as the shared-memory one."""
    n = 700   # not a multiple of 48, 64 or 128: overhanging tiles
    rng = np.random.default_rng(S * 100 + kblock)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, n))
    X = 0.5 * (A + A.T)
    for kw in ({}, {"symmetric": True}, {"tri_a": 1, "tri_b": 2}, {"tri_a": 2}, {"tri_b": 1}):
        M = X if kw.get("symmetric") else A
        N = X if kw.get("symmetric") else B
        C1 = ctx.oz_gemm(M, N, slices=S, kblock=kblock, variant=1, **kw)
        C2 = ctx.oz_gemm(M, N, slices=S, kblock=kblock, variant=2, **kw)
        assert np.array_equal(C1, C2), kw


@pytest.mark.parametrize("S", [4, 6, 7, 8])
@pytest.mark.parametrize("kblock", [32, 64])
@pytest.mark.parametrize("n", [300, 700])
def test_oz_gemm_pair_variant_is_bit_exact(ctx, S, kblock, n):
    """The CTA-pair kernel (256-row tiles, K ranges merged over both halves)
    sums the same exact int32 products as the one-CTA kernel; n = 300 gives an
    odd count of 128-row blocks, so the last pair has a half past the operand."""
    rng = np.random.default_rng(S * 1000 + kblock + n)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, n))
    X = 0.5 * (A + A.T)
    for kw in ({}, {"symmetric": True}, {"tri_a": 1, "tri_b": 2}, {"tri_a": 2}, {"tri_b": 1},
               {"tri_a": 1, "symmetric": True}):
        M = X if kw.get("symmetric") else A
        N = X if kw.get("symmetric") else B
        C1 = ctx.oz_gemm(M, N, slices=S, kblock=kblock, variant=1, **kw)
        C3 = ctx.oz_gemm(M, N, slices=S, kblock=kblock, variant=3, **kw)
        assert np.array_equal(C1, C3), kw


@pytest.mark.parametrize("variant", [4, 5])
@pytest.mark.parametrize("S", [4, 6, 7, 8])
@pytest.mark.parametrize("n", [300, 700, 1000])
def test_oz_gemm_wide_variant_is_bit_exact(ctx, S, n, variant):
    """The 128-column kernel (variant 4; variant 5 on a CTA pair, 256 x 128
    tiles) sums the low-weight accumulator groups in a first pass over K,
    parks their FP64 sum in the output and continues it with the other groups
    in a second pass: the same FP64 sum in the same order as the 64-column
    kernel, so bit-identical results, for general, symmetric and triangular
    products; n = 300 leaves the last CTA pair with a half past the operand."""
    rng = np.random.default_rng(S * 7 + n)
    A = rng.standard_normal((n, n)) * np.exp2(rng.integers(-20, 20, size=(n, 1)))
    B = rng.standard_normal((n, n))
    X = 0.5 * (A + A.T)
    for kw in ({}, {"symmetric": True}, {"tri_a": 1, "tri_b": 2}, {"tri_a": 2}, {"tri_b": 1},
               {"tri_a": 1, "symmetric": True}):
        M = X if kw.get("symmetric") else A
        N = X if kw.get("symmetric") else B
        C1 = ctx.oz_gemm(M, N, slices=S, kblock=64, variant=1, **kw)
        C4 = ctx.oz_gemm(M, N, slices=S, variant=variant, **kw)
        assert np.array_equal(C1, C4), kw
    with pytest.raises(PtbGpuError):
        ctx.oz_gemm(A, B, slices=S, kblock=64, variant=variant)


def test_mixed_path_with_int8_triangular_inverse(ctx):
    """ndim 5888 = 2 x 2944: the triangular inverse of the Cholesky factor takes
    its top-level off-diagonal products on the int8 tensor cores.  The mixed
    result agrees with the library's FP64 path (itself checked against the
    oracle at smaller sizes) to the mixed-precision tolerances."""
    s = synth.water_cluster(256, seed=2)
    assert s.ndim == 5888
    P, st = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=PREC_MIXED))
    P64, _ = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=PREC_FP64))
    assert np.max(np.abs(P - P64)) <= 1e-6
    chk = ctx.check_density(s.ndim, P, ctx.filter_matrix_sym(s.Svec, s.ndim, 1e-5),
                            ctx.filter_matrix_sym(s.Hvec, s.ndim, 1e-5))
    assert abs(chk.nel - s.nel) <= 1e-8
