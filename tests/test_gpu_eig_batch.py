"""The density step of many independent systems in one launch of the FP64
eigensolver (ptbgpu_eig_density_batch), against the oracle's dense projector
(LAPACK dsygvd, P = 2 sum of the nel/2 lowest S-orthonormal eigenvectors'
outer products; the reference's solve2 without Fermi smearing,
source/pgtb.f90:1066-1170).

The committed stratified subset of the 256-system lattice batch
(tests/golden/lattice_subset.json: every system with range/gap above 1e4 plus
small, median and large ones per ndim quartile; orders 166-3064, so both the
one-CTA solver and the cluster solver run in the same call), molecular systems
with the filter applied, a non-positive-definite overlap and an empty batch.
FP64 throughout: max|dP| <= 1e-8, |dE| <= 1e-9 Eh, |tr(PS) - nel| <= 1e-9.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import Options, PtbGpuError, api, synth

pytestmark = pytest.mark.gpu

SUBSET = Path(__file__).resolve().parent / "golden" / "lattice_subset.json"
TOL_P, TOL_E, TOL_NEL = 1e-8, 1e-9, 1e-9


def _check(s, P, filt=0.0):
    n = s.ndim
    Hf = O.blowsym(n, O.filter_matrix_sym(s.Hvec, filt) if filt else s.Hvec)
    Sf = O.blowsym(n, O.filter_matrix_sym(s.Svec, filt) if filt else s.Svec)
    Pd, _ = O.dense_projector(Hf, Sf, s.nel)
    Pf = O.blowsym(n, P)
    assert np.max(np.abs(Pf - Pd)) <= TOL_P, s.name
    assert abs(O.band_structure(Pf, Hf) - O.band_structure(Pd, Hf)) <= TOL_E, s.name
    assert abs(O.get_nel(Pf, Sf) - s.nel) <= TOL_NEL, s.name


def test_lattice_subset_in_one_launch(ctx):
    meta = json.loads(SUBSET.read_text())
    systems = [synth.lattice_instance(i) for i in meta["subset"]]
    assert max(s.ndim for s in systems) > 1024 and min(s.ndim for s in systems) <= 1024
    Ps, stats, wall = ctx.eig_density_batch([(s.ndim, s.nel, s.Hvec, s.Svec) for s in systems])
    assert wall > 0.0
    for s, P in zip(systems, Ps):
        _check(s, P)


def test_molecules_with_filter(ctx, water8, water32):
    alkane = synth.make_config(2)
    systems = [water32, water8, alkane]
    Ps, _, _ = ctx.eig_density_batch([(s.ndim, s.nel, s.Hvec, s.Svec) for s in systems], Options(filter=1e-4))
    for s, P in zip(systems, Ps):
        _check(s, P, 1e-4)


def test_non_positive_definite_overlap_names_the_system(ctx, water8):
    s = water8
    bad = s.Svec.copy()
    bad[0] = -1.0                                   # S_11 < 0
    with pytest.raises(PtbGpuError) as ei:
        ctx.eig_density_batch([(s.ndim, s.nel, s.Hvec, s.Svec), (s.ndim, s.nel, s.Hvec, bad)])
    assert ei.value.code == api.ENOTSPD and "system 2" in str(ei.value)


def test_empty_batch(ctx):
    Ps, stats, _ = ctx.eig_density_batch([])
    assert Ps == [] and stats == []
