"""Submatrix method with submatrices above the batched limit (1024): each is
one generalized eigensolve, several at once on the library's side streams.
Checked against the oracle with the same partition as the other submatrix
tests (equal bisection trace, max|dP| < 1e-9), and run twice to check that the
cached side streams give the same result."""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import Options, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nslab", [3, 5])
def test_large_submatrices_match_oracle(ctx, nslab):
    s = synth.water_cluster(80, seed=3)
    n = s.ndim
    # atoms in nslab slabs along x (1-based cluster ids)
    rank = np.argsort(np.argsort(s.xyz[:, 0]))
    part = (rank * nslab // s.nat + 1).astype(np.int64)
    H = O.filter_matrix_sym(s.Hvec, 1e-4)
    S = O.filter_matrix_sym(s.Svec, 1e-4)
    ref = O.sm_stupid_simple(n, s.nel, H, S, s.nat, s.xyz, s.aoat, 4, 2, part)
    assert max(ref.dims) > 1024
    for _ in range(2):
        P, st = ctx.sm_stupid_simple(n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, 4, 2, part,
                                     Options(filter=1e-4))
        assert st.nsm == ref.nsm == nslab
        assert st.sum_dims == sum(ref.dims)
        assert st.mu == ref.mu
        assert st.mu_iterations == len(ref.mu_trace)
        assert abs(st.nel - ref.nel) < 1e-9
        assert np.max(np.abs(P - ref.Pvec)) < 1e-9
