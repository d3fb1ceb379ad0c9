"""Refinement rounds of the mixed-precision trace-correcting purification on
systems with small HOMO-LUMO gaps (cubic-lattice instances, range/gap up to
~3e4), against the FP64 dense projector.

Tolerances as for every mixed-precision result: max|dP| <= 1e-6,
|dE| <= 1e-6 Eh, |tr(PS) - nel| <= 1e-8.
"""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import PREC_FP64, PREC_MIXED, Options, PtbGpuError, synth

pytestmark = pytest.mark.gpu

TOL_P = 1e-6
TOL_E = 1e-6
TOL_NEL = 1e-8


def _dense(s):
    n = s.ndim
    Hf, Sf = O.blowsym(n, s.Hvec), O.blowsym(n, s.Svec)
    Pd, _ = O.dense_projector(Hf, Sf, s.nel)
    return Hf, Sf, Pd


def _check(s, P, Hf, Sf, Pd):
    Pf = O.blowsym(s.ndim, P)
    assert np.max(np.abs(Pf - Pd)) <= TOL_P, s.name
    assert abs(O.band_structure(Pf, Hf) - O.band_structure(Pd, Hf)) <= TOL_E, s.name
    assert abs(O.get_nel(Pf, Sf) - s.nel) <= TOL_NEL, s.name
    return np.max(np.abs(Pf - Pd))


# range/gap: lattice_19 6.9e3, lattice_68 2.7e4 (the second and third largest of
# the 256 lattice instances), lattice_2 7.1e3
@pytest.mark.parametrize("index", [2, 19, 68])
@pytest.mark.parametrize("slices", [8, 0])
def test_small_gap_needs_more_rounds(ctx, index, slices):
    s = synth.lattice_instance(index)
    Hf, Sf, Pd = _dense(s)
    P, st = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(precision=PREC_MIXED, fp64_slices=slices))
    _check(s, P, Hf, Sf, Pd)
    assert st.refine_rounds >= 2
    assert st.fp64_fallback == 0


def test_one_round_for_a_large_gap(ctx):
    s = synth.water_cluster(32, seed=1)
    H = O.filter_matrix_sym(s.Hvec, 1e-4)
    S = O.filter_matrix_sym(s.Svec, 1e-4)
    Hf, Sf = O.blowsym(s.ndim, H), O.blowsym(s.ndim, S)
    Pd, _ = O.dense_projector(Hf, Sf, s.nel)
    P, st = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(filter=1e-4, precision=PREC_MIXED))
    Pf = O.blowsym(s.ndim, P)
    assert np.max(np.abs(Pf - Pd)) <= TOL_P
    assert st.refine_rounds == 1 and st.fp64_fallback == 0


@pytest.mark.parametrize("slices", [8, 0])
def test_unreachable_tolerance_falls_back_to_fp64(ctx, slices):
    """One round allowed and a tolerance no round can meet: the purification is
    redone in FP64 (with the matching back-transform) and flagged."""
    s = synth.lattice_instance(19)
    Hf, Sf, Pd = _dense(s)
    o = Options(precision=PREC_MIXED, fp64_slices=slices, refine_rounds=1, refine_tol=1e-13)
    P, st = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, o)
    assert st.fp64_fallback == 1 and st.refine_rounds == 1
    err = _check(s, P, Hf, Sf, Pd)
    assert err <= 1e-9   # FP64 quality (the int8 back-transform with 8 slices included)
    Pfp, _ = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(precision=PREC_FP64))
    assert np.max(np.abs(P - Pfp)) <= 1e-9


def test_refine_options_validated(ctx, water8):
    s = water8
    with pytest.raises(PtbGpuError, match="refine_rounds"):
        ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(precision=PREC_MIXED, refine_rounds=17))
    with pytest.raises(PtbGpuError, match="refine_rounds"):
        ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(precision=PREC_MIXED, refine_tol=-1.0))


@pytest.mark.parametrize("split3", [-1, 0, 4])
def test_three_plane_leading_iterations(ctx, split3):
    """Pass 1 with no, all, or the first four iterations on three-plane products
    (the trajectory then keeps a third bf16 plane per iterate): every variant
    meets the tolerances, single-system and grouped."""
    s = synth.lattice_instance(2)
    Hf, Sf, Pd = _dense(s)
    o = Options(precision=PREC_MIXED, split3_iters=split3)
    P, st = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, o)
    _check(s, P, Hf, Sf, Pd)
    Ps, _, _ = ctx.tc_purify_grouped([(s.ndim, s.nel, s.Hvec, s.Svec)], o)
    _check(s, Ps[0], Hf, Sf, Pd)
