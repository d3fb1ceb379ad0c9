"""The oracle reproduces the committed golden vectors (tests/golden/make_golden.py)."""
from pathlib import Path

import numpy as np
import pytest

from oracle import ptb_oracle as O

G = np.load(Path(__file__).resolve().parent / "golden" / "water4.npz")


def test_golden_inputs_are_the_seeded_system():
    from ptb_b200 import synth
    s = synth.water_cluster(4, seed=2)
    assert np.array_equal(s.Hvec, G["Hvec"]) and np.array_equal(s.Svec, G["Svec"])
    assert int(G["nel"]) == s.nel


@pytest.mark.parametrize("cols", [1, 2, 3])
def test_oracle_submatrix_matches_golden(cols):
    n = G["aoat"].shape[0]
    H = O.filter_matrix_sym(G["Hvec"], float(G["filter"]))
    S = O.filter_matrix_sym(G["Svec"], float(G["filter"]))
    r = O.sm_stupid_simple(n, int(G["nel"]), H, S, G["xyz"].shape[0], G["xyz"], G["aoat"], cols, 2)
    assert np.array_equal(np.array([m for _, m, _ in r.mu_trace]), G[f"mu_sm{cols}"])
    assert np.array_equal(np.array(r.dims), G[f"dims_sm{cols}"])
    assert np.max(np.abs(r.Pvec - G[f"P_sm{cols}"])) < 1e-12


def test_oracle_dense_and_sp2_match_golden():
    n = G["aoat"].shape[0]
    Hf = O.blowsym(n, O.filter_matrix_sym(G["Hvec"], float(G["filter"])))
    Sf = O.blowsym(n, O.filter_matrix_sym(G["Svec"], float(G["filter"])))
    Pd, e = O.dense_projector(Hf, Sf, int(G["nel"]))
    assert np.max(np.abs(O.packsym(Pd) - G["P_dense"])) < 1e-12
    P, it = O.sp2_trace_correcting(Hf, Sf, int(G["nel"]))
    assert np.max(np.abs(O.packsym(P) - G["P_sp2"])) < 1e-12
    # full_matrix partition == dense (the invariant of the reference's full_matrix runs)
    assert np.max(np.abs(G["P_sm3"] - G["P_dense"])) < 1e-11
    assert np.max(np.abs(G["P_solve2"] - G["P_dense"])) < 1e-11
