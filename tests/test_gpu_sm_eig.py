"""The submatrix method's batched generalized eigensolver (ptbgpu_sygv_batched)
against LAPACK (scipy's dsygvd, the routine the reference calls per submatrix,
source/sm.f90:296-299), stage by stage through what leaves the solver:

* eigenvalues of H c = e S c (the solver's order is not sorted: compared sorted),
* fe_j = sum_c (S U)_{c,j} U_{c,j} over the owned rows (source/sm.f90:305-310),
* the owned columns of P = U occ U^T with occ 2 / 1 / 0 for e < / = / > mu
  (source/sm.f90:322-362).

Orders 1 to 1024 (one CTA per problem) in one batch, uneven owned counts, an
exactly degenerate spectrum, and a non-positive-definite overlap; orders above
1024 (one thread-block cluster per problem) alone and mixed with small ones,
with a degenerate spectrum and a non-positive-definite overlap of their own.
FP64 throughout: eigenvalues to 1e-11 of the spectral range, fe and P to 1e-10.
"""
import numpy as np
import pytest
import scipy.linalg as sl

from ptb_b200 import PtbGpuError, api

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 5, 31, 32, 33, 64, 65, 100, 257, 600, 1024]


def _problem(m, rng, nown):
    A = rng.standard_normal((m, m))
    S = A @ A.T / m + np.eye(m)                # SPD, condition ~ 5
    H = rng.uniform(-1, 1, (m, m))
    H = 0.5 * (H + H.T) + np.diag(rng.uniform(-2, 2, m))
    own = np.sort(rng.choice(m, size=min(nown, m), replace=False))
    return H, S, own


def _reference(H, S, own, mu):
    e, U = sl.eigh(H, S)                       # S-orthonormal eigenvectors, ascending
    fe = np.sum((S @ U)[own, :] * U[own, :], axis=0)
    occ = np.where(e < mu, 2.0, np.where(e == mu, 1.0, 0.0))
    P = (U * occ) @ U[own, :].T
    return e, fe, P


def test_batched_eigensolver_matches_lapack(ctx):
    rng = np.random.default_rng(17)
    probs = [_problem(m, rng, 1 + (m % 13)) for m in SIZES]
    mu = 0.05
    out = ctx.sygv_batched(probs, mu=mu)
    for (H, S, own), (e, fe, Pc) in zip(probs, out):
        m = H.shape[0]
        er, fer, Pr = _reference(H, S, own, mu)
        order = np.argsort(e, kind="stable")
        scale = max(1.0, np.max(np.abs(er)))
        assert np.max(np.abs(e[order] - er)) <= 1e-11 * scale * max(1.0, np.sqrt(m)), m
        assert np.max(np.abs(fe[order] - fer)) <= 1e-10, m
        assert np.max(np.abs(Pc - Pr)) <= 1e-10, m
        assert abs(np.sum(fe) - len(own)) <= 1e-10 * m    # sum_j fe_j = number of owned rows


def test_degenerate_spectrum(ctx):
    """Repeated identical blocks give exactly repeated eigenvalues; the owned
    columns of P depend only on the occupied subspace, which must come out
    right whichever basis of each degenerate cluster the solver lands on."""
    rng = np.random.default_rng(5)
    b = 40
    Hb = rng.uniform(-1, 1, (b, b))
    Hb = 0.5 * (Hb + Hb.T)
    Ab = rng.standard_normal((b, b))
    Sb = Ab @ Ab.T / b + np.eye(b)
    H = np.kron(np.eye(4), Hb)
    S = np.kron(np.eye(4), Sb)
    own = np.array([0, 3, 41, 100, 159])
    e_b = sl.eigh(Hb, Sb, eigvals_only=True)
    mu = 0.5 * (e_b[17] + e_b[18])             # between two quadruplets
    (e, fe, Pc), = ctx.sygv_batched([(H, S, own)], mu=mu)
    er, fer, Pr = _reference(H, S, own, mu)
    assert np.max(np.abs(np.sort(e) - er)) <= 1e-12 * max(1.0, np.max(np.abs(er))) * 10
    assert np.max(np.abs(Pc - Pr)) <= 1e-10
    # per cluster of four equal eigenvalues the fe sums are basis independent
    occ_fe = np.sum(fe[e < mu])
    assert abs(occ_fe - np.sum(fer[er < mu])) <= 1e-10


def test_non_positive_definite_overlap_is_reported(ctx):
    rng = np.random.default_rng(2)
    H, S, own = _problem(70, rng, 3)
    S = S.copy()
    S[40, 40] = -5.0
    with pytest.raises(PtbGpuError) as ei:
        ctx.sygv_batched([_problem(30, rng, 2), (H, S, own)])
    assert ei.value.code == api.ENOTSPD and "submatrix 2" in str(ei.value)


LARGE = [1025, 1100, 1537, 2100]


def test_cluster_orders_match_lapack(ctx):
    """Orders above 1024 go to the cluster solver (Cholesky, reduction,
    tridiagonalisation, divide and conquer and owned rows each spread over the
    CTAs of a cluster); owned counts as the k-means partitions have them (one to
    a few hundred columns)."""
    rng = np.random.default_rng(23)
    nowns = [1, 37, 310, 120]
    probs = [_problem(m, rng, no) for m, no in zip(LARGE, nowns)]
    mu = -0.1
    out = ctx.sygv_batched(probs, mu=mu)
    for (H, S, own), (e, fe, Pc) in zip(probs, out):
        m = H.shape[0]
        er, fer, Pr = _reference(H, S, own, mu)
        order = np.argsort(e, kind="stable")
        scale = max(1.0, np.max(np.abs(er)))
        assert np.max(np.abs(e[order] - er)) <= 1e-11 * scale * np.sqrt(m), m
        assert np.max(np.abs(fe[order] - fer)) <= 1e-10, m
        assert np.max(np.abs(Pc - Pr)) <= 1e-10, m
        assert abs(np.sum(fe) - len(own)) <= 1e-10 * m


def test_cluster_and_batched_orders_in_one_call(ctx):
    """Small and large problems of one call run on both solvers at once (the
    persistent launch and the clusters side by side); each result lands at its
    own offsets."""
    rng = np.random.default_rng(29)
    sizes = [700, 1300, 33, 1030, 256]
    probs = [_problem(m, rng, 1 + (m % 29)) for m in sizes]
    out = ctx.sygv_batched(probs, mu=0.2)
    for (H, S, own), (e, fe, Pc) in zip(probs, out):
        er, fer, Pr = _reference(H, S, own, 0.2)
        order = np.argsort(e, kind="stable")
        assert np.max(np.abs(e[order] - er)) <= 1e-11 * max(1.0, np.max(np.abs(er))) * np.sqrt(len(e))
        assert np.max(np.abs(fe[order] - fer)) <= 1e-10
        assert np.max(np.abs(Pc - Pr)) <= 1e-10


def test_cluster_degenerate_spectrum(ctx):
    """Four identical 300-blocks: every eigenvalue four times, so the top merges
    of the divide and conquer (run by the whole cluster) deflate by rotations."""
    rng = np.random.default_rng(31)
    b = 300
    Hb = rng.uniform(-1, 1, (b, b))
    Hb = 0.5 * (Hb + Hb.T)
    Ab = rng.standard_normal((b, b))
    Sb = Ab @ Ab.T / b + np.eye(b)
    H = np.kron(np.eye(4), Hb)
    S = np.kron(np.eye(4), Sb)
    own = np.array([0, 7, 299, 300, 650, 1199])
    e_b = sl.eigh(Hb, Sb, eigvals_only=True)
    mu = 0.5 * (e_b[140] + e_b[141])
    (e, fe, Pc), = ctx.sygv_batched([(H, S, own)], mu=mu)
    er, fer, Pr = _reference(H, S, own, mu)
    assert np.max(np.abs(np.sort(e) - er)) <= 1e-11 * max(1.0, np.max(np.abs(er))) * 40
    assert np.max(np.abs(Pc - Pr)) <= 1e-10
    assert abs(np.sum(fe[e < mu]) - np.sum(fer[er < mu])) <= 1e-10


def test_cluster_non_positive_definite_overlap_is_reported(ctx):
    rng = np.random.default_rng(3)
    H, S, own = _problem(1200, rng, 5)
    S = S.copy()
    S[900, 900] = -5.0
    with pytest.raises(PtbGpuError) as ei:
        ctx.sygv_batched([_problem(40, rng, 2), (H, S, own)])
    assert ei.value.code == api.ENOTSPD and "submatrix 2" in str(ei.value)


def test_dense_solve2_on_one_cluster(ctx):
    """solve2's generalized eigensolve (source/pgtb.f90:1066-1170) runs the same
    solver on one thread-block cluster up to order 4096: P, the eigenvalues and
    the Fermi occupations of an 80-H2O cluster (ndim 1840) against the oracle's
    dsygvd."""
    from oracle import ptb_oracle as O
    from ptb_b200 import Options, synth

    s = synth.water_cluster(80, seed=3)
    n = s.ndim
    P, e, focc, st = ctx.solve2(1, n, s.nel, 0, s.Hvec, s.Svec, Options(filter=1e-4))
    ref, e_ref, f_ref, _ = O.solve2(1, n, s.nel, 0, 300.0, O.filter_matrix_sym(s.Hvec, 1e-4),
                                    O.filter_matrix_sym(s.Svec, 1e-4))
    assert np.max(np.abs(e - e_ref)) < 1e-10
    assert np.max(np.abs(focc - f_ref)) < 1e-10
    assert np.max(np.abs(P - ref)) < 1e-10


def test_dense_solve2_on_the_whole_gpu(ctx):
    """Above order 4096 the same solver runs as one cooperative launch over a
    grid of CTAs (a bounded software barrier between dependent steps): solve2 of
    a 180-H2O cluster (ndim 4140) against the oracle's dsygvd."""
    from oracle import ptb_oracle as O
    from ptb_b200 import Options, synth

    s = synth.water_cluster(180, seed=4)
    n = s.ndim
    assert n > 4096
    P, e, focc, st = ctx.solve2(1, n, s.nel, 0, s.Hvec, s.Svec, Options(filter=1e-4))
    ref, e_ref, f_ref, _ = O.solve2(1, n, s.nel, 0, 300.0, O.filter_matrix_sym(s.Hvec, 1e-4),
                                    O.filter_matrix_sym(s.Svec, 1e-4))
    assert np.max(np.abs(e - e_ref)) < 1e-10
    assert np.max(np.abs(focc - f_ref)) < 1e-10
    assert np.max(np.abs(P - ref)) < 1e-9


@pytest.mark.parametrize("G", [2, 16])
def test_cluster_solver_at_other_cluster_sizes(G):
    """The cluster solver is written for any number of CTAs per cluster: the
    batch rule picks 2 for many large problems, and 16 is the largest size.  The
    size is read once per process, so the cluster tests rerun in a child pytest
    with PTBGPU_EIG_CLUSTER set."""
    import os
    import subprocess
    import sys
    from pathlib import Path

    here = Path(__file__).resolve()
    env = dict(os.environ, PTBGPU_EIG_CLUSTER=str(G))
    r = subprocess.run([sys.executable, "-m", "pytest", str(here), "-m", "gpu", "-q", "-p", "no:cacheprovider",
                        "-k", "cluster_ and not other_cluster_sizes"],
                       cwd=here.parent.parent, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and "4 passed" in r.stdout, r.stdout[-1000:]
