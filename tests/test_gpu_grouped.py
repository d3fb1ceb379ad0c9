"""Grouped purification (ptbgpu_tc_purify_grouped): systems bucketed by their
dimension rounded up to 256, padded and stacked, every step one launch per
bucket.  Checked per system against the FP64 dense projector with the
mixed-precision tolerances (max|dP| <= 1e-6, |dE| <= 1e-6 Eh,
|tr(PS) - nel| <= 1e-8), and against the single-system call.
"""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import PREC_FP64, PREC_MIXED, Options, PtbGpuError, synth

pytestmark = pytest.mark.gpu

TOL_P = 1e-6
TOL_E = 1e-6
TOL_NEL = 1e-8

# three systems in the 256 bucket (ndim 166-240), three in the 512 bucket
# (304-511), two in the 768 bucket, and single systems of 1357 and 2553
INDICES = (5, 56, 104, 8, 13, 107, 1, 10, 2, 19)


@pytest.fixture(scope="module")
def systems():
    return [synth.lattice_instance(i) for i in INDICES]


def _check(s, P):
    n = s.ndim
    Hf, Sf = O.blowsym(n, s.Hvec), O.blowsym(n, s.Svec)
    Pd, _ = O.dense_projector(Hf, Sf, s.nel)
    Pf = O.blowsym(n, P)
    assert np.max(np.abs(Pf - Pd)) <= TOL_P, s.name
    assert abs(O.band_structure(Pf, Hf) - O.band_structure(Pd, Hf)) <= TOL_E, s.name
    assert abs(O.get_nel(Pf, Sf) - s.nel) <= TOL_NEL, s.name


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_grouped_against_dense(ctx, systems, precision):
    Ps, stats, wall = ctx.tc_purify_grouped([(s.ndim, s.nel, s.Hvec, s.Svec) for s in systems],
                                            Options(precision=precision))
    assert wall > 0.0
    for s, P, st in zip(systems, Ps, stats):
        _check(s, P)
        assert st.iterations > 5
        if precision == PREC_MIXED and not st.fp64_fallback:
            assert st.refine_rounds >= 1


def test_grouped_matches_single_calls(ctx, systems):
    """Same systems through the single-system entry: both meet the tolerances,
    so they agree to twice the tolerance (not bit for bit: the padded FP64
    steps and the stacked products round differently)."""
    picked = systems[:6]
    Ps, _, _ = ctx.tc_purify_grouped([(s.ndim, s.nel, s.Hvec, s.Svec) for s in picked], Options())
    for s, P in zip(picked, Ps):
        P1, _ = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options())
        assert np.max(np.abs(P - P1)) <= 2 * TOL_P, s.name


def test_grouped_water_and_filter(ctx):
    """Gapped molecular systems of two sizes with the library's filter."""
    sys_ = [synth.water_cluster(8, seed=5), synth.water_cluster(32, seed=1), synth.water_cluster(8, seed=6)]
    o = Options(filter=1e-5, precision=PREC_MIXED)
    Ps, stats, _ = ctx.tc_purify_grouped([(s.ndim, s.nel, s.Hvec, s.Svec) for s in sys_], o)
    for s, P in zip(sys_, Ps):
        n = s.ndim
        Hf = O.blowsym(n, O.filter_matrix_sym(s.Hvec, 1e-5))
        Sf = O.blowsym(n, O.filter_matrix_sym(s.Svec, 1e-5))
        Pd, _ = O.dense_projector(Hf, Sf, s.nel)
        assert np.max(np.abs(O.blowsym(n, P) - Pd)) <= TOL_P


def test_grouped_fallback_and_errors(ctx, systems):
    s = systems[-1]   # lattice 19: needs three rounds
    Ps, stats, _ = ctx.tc_purify_grouped([(s.ndim, s.nel, s.Hvec, s.Svec)],
                                         Options(precision=PREC_MIXED, refine_rounds=1, refine_tol=1e-13))
    assert stats[0].fp64_fallback == 1
    _check(s, Ps[0])
    bad = systems[0]
    with pytest.raises(PtbGpuError, match="system 1"):
        ctx.tc_purify_grouped([(s.ndim, s.nel, s.Hvec, s.Svec), (bad.ndim, bad.nel + 1, bad.Hvec, bad.Svec)])
    Ps, stats, _ = ctx.tc_purify_grouped([])
    assert Ps == [] and stats == []
