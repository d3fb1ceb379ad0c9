"""GPU parity at the benchmark configurations, through the C-ABI, against the
CPU oracle.

* 32-H2O cluster (ndim 736) and C200H402 (ndim 4610), submatrix method with
  per-atom columns, filter 1e-4 (source/sm.f90:34-409): the same submatrices,
  the same bisection (mu equal to the oracle's bit for bit, the same number of
  steps) and max|dP| < 1e-9 against the oracle's sm_stupid_simple; C200H402
  also with one column per submatrix (4610 submatrices).
* 512-H2O box (ndim 11776, nel 4096), filter 1e-5: the trace-correcting
  purification in mixed precision and in FP64 against the oracle's dense FP64
  projector (dsygvd, the lowest nel/2 generalized eigenvectors doubly
  occupied): max|dP| <= 1e-6, |d tr(PH)| <= 1e-6 Eh, |tr(PS) - nel| <= 1e-8.
* The uneven multi-instance batch (256 cubic-lattice systems): a committed
  stratified subset (tests/golden/lattice_subset.json, every system with
  range/gap above 1e4 plus small, median and large ones of each ndim quartile)
  through the batch entry, each system against its dense projector with the
  same tolerances.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import PREC_FP64, PREC_MIXED, Options, synth

pytestmark = pytest.mark.gpu

TOL_P = 1e-6        # max |dP| (mixed precision against the FP64 oracle)
TOL_E = 1e-6        # |d tr(PH)| in Eh
TOL_NEL = 1e-8      # |tr(PS) - nel|
TOL_SM = 1e-9       # max |dP| of the FP64 submatrix method against the oracle

SUBSET = Path(__file__).resolve().parent / "golden" / "lattice_subset.json"


def _sm_parity(ctx, s, columns, filt=1e-4):
    n = s.ndim
    H = O.filter_matrix_sym(s.Hvec, filt)
    S = O.filter_matrix_sym(s.Svec, filt)
    ref = O.sm_stupid_simple(n, s.nel, H, S, s.nat, s.xyz, s.aoat, columns, 2)
    P, st = ctx.sm_stupid_simple(n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, columns, 2, None,
                                 Options(filter=filt))
    assert st.nsm == ref.nsm
    assert st.sum_dims == sum(ref.dims)
    assert st.max_dim == max(ref.dims)
    assert st.mu == ref.mu
    assert st.mu_iterations == len(ref.mu_trace)
    assert abs(st.nel - ref.nel) < 1e-9
    assert np.max(np.abs(P - ref.Pvec)) < TOL_SM
    return st


def test_water32_per_atom_submatrix_method(ctx):
    st = _sm_parity(ctx, synth.make_config(0), 2)
    assert st.nsm == 96


def test_alkane_per_atom_submatrix_method(ctx):
    st = _sm_parity(ctx, synth.make_config(2), 2)
    assert st.nsm == 602


def test_alkane_per_column_submatrix_method(ctx):
    st = _sm_parity(ctx, synth.make_config(2), 1)
    assert st.nsm == 4610


@pytest.fixture(scope="module")
def water512_dense():
    s = synth.make_config(1)
    n = s.ndim
    Hf = O.blowsym(n, O.filter_matrix_sym(s.Hvec, 1e-5))
    Sf = O.blowsym(n, O.filter_matrix_sym(s.Svec, 1e-5))
    Pd, _ = O.dense_projector(Hf, Sf, s.nel)
    return s, Hf, Sf, Pd, O.band_structure(Pd, Hf)


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_water512_trace_correcting_against_dense_projector(ctx, water512_dense, precision):
    s, Hf, Sf, Pd, e_ref = water512_dense
    n = s.ndim
    assert n == 11776 and s.nel == 4096
    P, st = ctx.tc_purify(n, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=precision))
    Pf = O.blowsym(n, P)
    assert np.max(np.abs(Pf - Pd)) <= TOL_P
    assert abs(O.band_structure(Pf, Hf) - e_ref) <= TOL_E
    assert abs(O.get_nel(Pf, Sf) - s.nel) <= TOL_NEL
    if precision == PREC_MIXED:
        assert st.n_tc_sp2 > 0 and st.fp64_fallback == 0


def test_lattice_batch_subset_against_dense_projector(ctx):
    meta = json.loads(SUBSET.read_text())
    idx = meta["subset"]
    hard = [r["index"] for r in meta["systems"] if r["range_over_gap"] > meta["hard_threshold"]]
    assert set(hard) <= set(idx) and len(idx) >= 12
    systems = [synth.lattice_instance(i) for i in idx]
    for s, r in zip(systems, (meta["systems"][i] for i in idx)):
        assert s.ndim == r["ndim"] and s.nel == r["nel"]
    Ps, stats, _ = ctx.tc_purify_batch([(s.ndim, s.nel, s.Hvec, s.Svec) for s in systems],
                                       Options(precision=PREC_MIXED), workers=4)
    for s, P in zip(systems, Ps):
        n = s.ndim
        Hf, Sf = O.blowsym(n, s.Hvec), O.blowsym(n, s.Svec)
        Pd, _ = O.dense_projector(Hf, Sf, s.nel)
        Pf = O.blowsym(n, P)
        assert np.max(np.abs(Pf - Pd)) <= TOL_P, s.name
        assert abs(O.band_structure(Pf, Hf) - O.band_structure(Pd, Hf)) <= TOL_E, s.name
        assert abs(O.get_nel(Pf, Sf) - s.nel) <= TOL_NEL, s.name
