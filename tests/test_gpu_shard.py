"""The submatrix method in phases through the C-ABI (ptbgpu_sm_plan /
_prepare / _nel / _finish) and the rank protocol of ptb_b200.distributed on
one GPU: one rank preparing every submatrix reproduces ptbgpu_sm_density
exactly, and shares of the submatrices add up to it."""
import numpy as np
import pytest

from ptb_b200 import Options, synth
from ptb_b200.distributed import DeviceShard, assign_submatrices, sm_stupid_simple_sharded

pytestmark = pytest.mark.gpu

FILTER = 1e-4


@pytest.mark.parametrize("columns", [1, 2, 4])
def test_one_rank_reproduces_sm_density(ctx, columns):
    s = synth.alkane(20, seed=2)
    n = s.ndim
    o = Options(filter=FILTER)
    part = None
    if columns == 4:
        part, _, _ = ctx.kmeans_partition(n, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, opts=o)
    Pd, st = ctx.sm_stupid_simple(n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, columns, 2, partition=part, opts=o)
    Ps, info = sm_stupid_simple_sharded(DeviceShard(ctx), n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, columns, 2,
                                        partition=part, opts=o)
    assert info.mu == st.mu and info.nsm == st.nsm
    assert np.array_equal(Ps, Pd)


def test_shares_add_up(ctx):
    """Four ranks' shares, prepared one after the other on this GPU, with the
    electron count summed over the shares at every bisection step."""
    s = synth.alkane(20, seed=2)
    n = s.ndim
    o = Options(filter=FILTER)
    Pd, st = ctx.sm_stupid_simple(n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, 1, 2, opts=o)
    dims = ctx.sm_plan(n, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, 1, 2, opts=o)
    parts = assign_submatrices(dims, 4)
    # eigenvalues / fe of each share: nel(mu) as the sum of the shares' counts
    nel_by_share = []
    for ids in parts:
        ctx.sm_prepare(ids)
        nel_by_share.append([ctx.sm_nel(mu) for mu in (st.mu - 0.05, st.mu, st.mu + 0.05)])
    ctx.sm_prepare(list(range(len(dims))))
    whole = [ctx.sm_nel(mu) for mu in (st.mu - 0.05, st.mu, st.mu + 0.05)]
    assert np.allclose(np.sum(nel_by_share, axis=0), whole, rtol=0, atol=1e-10)
    P = np.zeros_like(Pd)
    for ids in parts:
        ctx.sm_prepare(ids)
        P += ctx.sm_finish(n, st.mu)
    # a share batches its submatrices differently (the batched eigensolver's
    # result can differ in the last bits with the batch): FP64 rounding only
    assert np.max(np.abs(P - Pd)) < 1e-12
