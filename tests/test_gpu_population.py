"""GPU parity of the population analysis on the produced density matrix
(mlpop14 / mlpop2, source/mlpop.f) through the C-ABI.

The reference evaluates both in REAL*4.  mlpop14 is compared with the oracle's
REAL*4 restatement to FP32 accuracy; mlpop2 forms diag(s2 P s1) from an exact
int8-sliced product, so it is compared with the FP64 evaluation of the same
formula tightly and with the REAL*4 restatement to FP32 accuracy.
"""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import PREC_MIXED, Options, PtbGpuError, synth

pytestmark = pytest.mark.gpu


def test_mlpop14_matches_oracle(ctx, water8):
    s = water8
    n = s.ndim
    s34, s14 = ctx.mlpop14(n, s.Svec)
    r34, r14 = O.mlpop14(n, s.Svec)
    assert np.max(np.abs(s34 - r34)) < 2e-5
    assert np.max(np.abs(s14 - r14)) < 2e-5
    S = O.blowsym(n, s.Svec)
    assert np.max(np.abs(s34.astype(np.float64) @ s14 - S)) < 1e-4


@pytest.mark.parametrize("nmol", [8, 32])
def test_mlpop2_matches_oracle(ctx, nmol):
    """Non-symmetric s1, s2 so that a transposed operand would show."""
    s = synth.water_cluster(nmol, seed=2)
    n = s.ndim
    sh = synth.shell2ao(s.aoat)
    P, _ = ctx.tc_purify(n, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=PREC_MIXED))
    rng = np.random.default_rng(nmol)
    s34, s14 = O.mlpop14(n, s.Svec)
    s1 = (s34 + 1e-3 * rng.standard_normal((n, n))).astype(np.float32)
    s2 = (s14 + 1e-3 * rng.standard_normal((n, n))).astype(np.float32)
    q, qsh, st = ctx.mlpop2(s.nat, n, P, s1, s2, s.aoat, sh)
    q64, qsh64 = O.mlpop2(s.nat, n, P, s1, s2, s.aoat, sh, dtype=np.float64)
    q32, qsh32 = O.mlpop2(s.nat, n, P, s1, s2, s.aoat, sh)
    assert np.max(np.abs(q - q64)) < 1e-9
    assert np.max(np.abs(qsh - qsh64)) < 1e-9
    assert np.max(np.abs(q - q32)) < 1e-4
    assert np.max(np.abs(qsh - qsh32)) < 1e-4
    assert np.allclose(qsh.sum(axis=1), q, rtol=0, atol=1e-12)
    assert st.n_oz == 1


def test_mlpop2_populations_sum_to_electrons(ctx, water32):
    s = water32
    n = s.ndim
    P, _ = ctx.tc_purify(n, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=PREC_MIXED))
    s34, s14 = ctx.mlpop14(n, ctx.filter_matrix_sym(s.Svec, n, 1e-5))
    q, qsh, _ = ctx.mlpop2(s.nat, n, P, s34, s14, s.aoat, synth.shell2ao(s.aoat))
    # sum_A q_A = tr(S^x P S^(1-x)) = tr(PS) up to the REAL*4 powers of S
    assert abs(q.sum() - s.nel) < 1e-3
    assert np.all(qsh[:, 5:] == 0.0)


def test_mlpop2_device_matches_host(ctx, water8):
    import torch
    s = water8
    n = s.ndim
    sh = synth.shell2ao(s.aoat)
    P, _ = ctx.tc_purify(n, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=PREC_MIXED))
    s34, s14 = ctx.mlpop14(n, s.Svec)
    qh, qshh, _ = ctx.mlpop2(s.nat, n, P, s34, s14, s.aoat, sh)
    dP = torch.from_numpy(P).cuda()
    # column-major device copies: the transpose of a C-contiguous array
    d1 = torch.from_numpy(np.ascontiguousarray(s34.T)).cuda()
    d2 = torch.from_numpy(np.ascontiguousarray(s14.T)).cuda()
    torch.cuda.synchronize()
    qd, qshd, _ = ctx.mlpop2_device(s.nat, n, dP.data_ptr(), d1.data_ptr(), d2.data_ptr(), s.aoat, sh)
    assert np.array_equal(qh, qd)
    assert np.array_equal(qshh, qshd)


def test_mlpop2_rejects_bad_maps(ctx, water8):
    s = water8
    n = s.ndim
    s34, s14 = O.mlpop14(n, s.Svec)
    P = O.packsym(np.eye(n))
    bad = s.aoat.copy()
    bad[3] = s.nat + 1
    with pytest.raises(PtbGpuError):
        ctx.mlpop2(s.nat, n, P, s34, s14, bad, synth.shell2ao(s.aoat))
    sh = synth.shell2ao(s.aoat)
    sh[0] = 11
    with pytest.raises(PtbGpuError):
        ctx.mlpop2(s.nat, n, P, s34, s14, s.aoat, sh)
