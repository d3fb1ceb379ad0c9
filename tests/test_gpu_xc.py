"""The iteration-2 XC long-range damping term (source/pgtb.f90:482-513) on the
GPU against the oracle: relative agreement 1e-14 (CUDA's and scipy's erf may
differ in the last bit; every product and sum is rounded in the reference's
order without fused multiply-adds), device-pointer entry bit-identical to the
host entry, and argument checks."""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import PtbGpuError, synth

pytestmark = pytest.mark.gpu

BOHR = 1.0 / 0.52917721092


def _inputs(s, seed=0):
    rng = np.random.default_rng(seed)
    nat, ndim = s.nat, s.ndim
    xyz = s.xyz * BOHR
    ca, rb = O._packed_cols_rows(nat)
    rab = np.sqrt(np.sum((xyz[ca] - xyz[rb]) ** 2, axis=1))
    rad = rng.uniform(2.0, 4.0, nat)             # special radii (Bohr)
    hao = rng.uniform(-0.5, 0.5, ndim)           # shell_cnf2 * gq
    xdiag = rng.uniform(0.5, 1.5, ndim)          # shell_xi(8, element)
    P = rng.normal(0.0, 0.1, ndim * (ndim + 1) // 2)
    H = rng.normal(0.0, 0.2, ndim * (ndim + 1) // 2)
    return nat, ndim, s.aoat, rab, rad, hao, xdiag, P, H


@pytest.mark.parametrize("nmol", [8, 32])
def test_xc_damping_matches_oracle(ctx, nmol):
    s = synth.water_cluster(nmol, seed=2)
    args = _inputs(s)
    ref = O.xc_damping(*args)
    out = ctx.xc_damping(*args)
    np.testing.assert_allclose(out, ref, rtol=1e-14, atol=1e-16)
    # the input H is left unchanged by the host entry
    assert not np.shares_memory(out, args[-1])


def test_xc_damping_device_entry_matches_host(ctx):
    import torch
    s = synth.water_cluster(32, seed=3)
    nat, ndim, aoat, rab, rad, hao, xdiag, P, H = _inputs(s, seed=1)
    host = ctx.xc_damping(nat, ndim, aoat, rab, rad, hao, xdiag, P, H)
    dP = torch.from_numpy(P).cuda()
    dH = torch.from_numpy(H.copy()).cuda()
    ms = ctx.xc_damping_device(nat, ndim, aoat, rab, rad, hao, xdiag, dP.data_ptr(), dH.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(dH.cpu().numpy(), host)
    assert ms > 0.0


def test_xc_damping_rejects_bad_atom_index(ctx):
    s = synth.water_cluster(8, seed=2)
    nat, ndim, aoat, rab, rad, hao, xdiag, P, H = _inputs(s)
    bad = aoat.copy()
    bad[5] = nat + 1
    with pytest.raises(PtbGpuError, match="aoat"):
        ctx.xc_damping(nat, ndim, bad, rab, rad, hao, xdiag, P, H)
    bad[5] = 0
    with pytest.raises(PtbGpuError, match="aoat"):
        ctx.xc_damping(nat, ndim, bad, rab, rad, hao, xdiag, P, H)


def test_xc_damping_odd_packed_length(ctx):
    """ndim = 6 has 21 packed elements: the odd last element takes its own path."""
    rng = np.random.default_rng(5)
    nat, ndim = 3, 6
    aoat = np.array([1, 1, 2, 2, 3, 3])
    rab = rng.uniform(1.0, 5.0, 6)
    rad = rng.uniform(1.0, 2.0, 3)
    hao, xd = rng.normal(size=ndim), rng.normal(size=ndim)
    P, H = rng.normal(size=21), rng.normal(size=21)
    out = ctx.xc_damping(nat, ndim, aoat, rab, rad, hao, xd, P, H)
    np.testing.assert_allclose(out, O.xc_damping(nat, ndim, aoat, rab, rad, hao, xd, P, H), rtol=1e-14, atol=1e-16)


def test_xc_damping_device_rejects_misaligned(ctx):
    import torch
    s = synth.water_cluster(8, seed=2)
    nat, ndim, aoat, rab, rad, hao, xdiag, P, H = _inputs(s)
    buf = torch.zeros(P.size + 1, dtype=torch.float64, device="cuda")
    dH = torch.from_numpy(H).cuda()
    with pytest.raises(PtbGpuError, match="16-byte"):
        ctx.xc_damping_device(nat, ndim, aoat, rab, rad, hao, xdiag, buf.data_ptr() + 8, dH.data_ptr())
