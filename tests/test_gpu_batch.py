"""Multi-instance batch of the trace-correcting purification
(ptbgpu_tc_purify_batch) against the FP64 dense projector of each system.

The batch runs one system per worker thread with its own context and stream,
so every system must come out exactly as the single-system call gives it:
the same mixed-precision tolerances (max|dP| <= 1e-6, |dE| <= 1e-6 Eh,
|tr(PS) - nel| <= 1e-8) against the dense oracle, and bit-identical to
ptbgpu_tc_purify on the same system.
"""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import PREC_FP64, PREC_MIXED, Options, PtbGpuError, synth

pytestmark = pytest.mark.gpu

TOL_P = 1e-6
TOL_E = 1e-6
TOL_NEL = 1e-8

# lattice systems of 25 to 220 atoms (about 190 to 1700 AOs), mixed sizes
INDICES = (5, 8, 1, 0, 2, 7)


@pytest.fixture(scope="module")
def lattice_systems():
    return [synth.lattice_instance(i) for i in INDICES]


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_batch_against_dense(ctx, lattice_systems, precision):
    systems = [(s.ndim, s.nel, s.Hvec, s.Svec) for s in lattice_systems]
    Ps, stats, wall = ctx.tc_purify_batch(systems, Options(precision=precision), workers=3)
    assert wall > 0.0
    for s, P, st in zip(lattice_systems, Ps, stats):
        n = s.ndim
        Hf, Sf = O.blowsym(n, s.Hvec), O.blowsym(n, s.Svec)
        Pd, _ = O.dense_projector(Hf, Sf, s.nel)
        Pf = O.blowsym(n, P)
        assert np.max(np.abs(Pf - Pd)) <= TOL_P, s.name
        assert abs(O.band_structure(Pf, Hf) - O.band_structure(Pd, Hf)) <= TOL_E, s.name
        assert abs(O.get_nel(Pf, Sf) - s.nel) <= TOL_NEL, s.name
        assert st.iterations > 5


def test_batch_matches_single_calls(ctx, lattice_systems):
    """Each system of a batch is bit-identical to its own single call."""
    picked = lattice_systems[:4]
    o = Options(precision=PREC_MIXED)
    Ps, _, _ = ctx.tc_purify_batch([(s.ndim, s.nel, s.Hvec, s.Svec) for s in picked], o, workers=4)
    for s, P in zip(picked, Ps):
        P1, _ = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, o)
        assert np.array_equal(P, P1), s.name


def test_batch_one_worker_and_empty(ctx, lattice_systems):
    s = lattice_systems[0]
    Ps, stats, _ = ctx.tc_purify_batch([(s.ndim, s.nel, s.Hvec, s.Svec)] * 2, Options(), workers=1)
    assert np.array_equal(Ps[0], Ps[1])
    assert stats[0].iterations == stats[1].iterations
    Ps, stats, _ = ctx.tc_purify_batch([], Options())
    assert Ps == [] and stats == []


def test_batch_reports_the_failing_system(ctx, lattice_systems):
    """An odd electron count in one system fails the batch with its index."""
    good = lattice_systems[0]
    bad = lattice_systems[1]
    systems = [(good.ndim, good.nel, good.Hvec, good.Svec), (bad.ndim, bad.nel + 1, bad.Hvec, bad.Svec)]
    with pytest.raises(PtbGpuError, match="system 1"):
        ctx.tc_purify_batch(systems, Options(), workers=2)
    # the context stays usable
    Ps, _, _ = ctx.tc_purify_batch(systems[:1], Options(), workers=2)
    P1, _ = ctx.tc_purify(good.ndim, good.nel, good.Hvec, good.Svec, Options())
    assert np.array_equal(Ps[0], P1)
