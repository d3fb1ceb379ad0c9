"""GPU parity of the seeded k-means partition of submatrix columns mode 4
(source/sm.f90:127-154,459-514, source/kmpp.f) through the C-ABI.

The partition is integer work on a fixed generator stream, so the library and
the oracle's restatement must agree exactly (labels and the effort value).
"""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import Options, synth

pytestmark = pytest.mark.gpu

FILTER = 1e-4


def _filtered(s):
    n = s.ndim
    H = O.blowsym(n, O.filter_matrix_sym(s.Hvec, FILTER))
    S = O.blowsym(n, O.filter_matrix_sym(s.Svec, FILTER))
    return H, S


@pytest.mark.parametrize("system", ["water32", "alkane"])
def test_kmeans_partition_matches_oracle(ctx, system):
    s = synth.water_cluster(32, seed=1) if system == "water32" else synth.alkane(40, seed=2)
    n = s.ndim
    H, S = _filtered(s)
    part, nsm, eff = ctx.kmeans_partition(n, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, seed=42,
                                          opts=Options(filter=FILTER))
    rpart, rk, reff = O.kmeans_partition(n, H, S, s.nat, s.xyz, s.aoat, seed=42)
    assert nsm == rk
    assert eff == reff
    assert np.array_equal(part, rpart)
    assert part.min() == 1 and part.max() == nsm


def test_kmeans_partition_is_reproducible(ctx, water32):
    s = water32
    a = ctx.kmeans_partition(s.ndim, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, seed=7, opts=Options(filter=FILTER))
    b = ctx.kmeans_partition(s.ndim, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, seed=7, opts=Options(filter=FILTER))
    assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]


def test_sm_mode4_without_partition_uses_seeded_kmeans(ctx):
    s = synth.alkane(40, seed=2)   # a chain: 4 clusters win (a compact water box keeps 1)
    n = s.ndim
    o = Options(filter=FILTER)
    part, nsm, _ = ctx.kmeans_partition(n, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, seed=42, opts=o)
    P1, st1 = ctx.sm_stupid_simple(n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, 4, 2, partition=None, opts=o)
    P2, st2 = ctx.sm_stupid_simple(n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, 4, 2, partition=part, opts=o)
    assert st1.nsm == nsm == st2.nsm
    assert np.array_equal(P1, P2)
    ref = O.sm_stupid_simple(n, s.nel, O.filter_matrix_sym(s.Hvec, FILTER), O.filter_matrix_sym(s.Svec, FILTER),
                             s.nat, s.xyz, s.aoat, 4, 2, partition=part)
    assert np.max(np.abs(P1 - ref.Pvec)) < 1e-9
