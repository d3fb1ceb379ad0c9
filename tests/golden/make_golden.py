"""Generates the committed golden fixtures of the density step.

    python tests/golden/make_golden.py

The reference (Fortran, ifx + MKL) cannot be built on this host and its
repository ships no H/S/P dumps, so these vectors come from the CPU oracle
(oracle/ptb_oracle.py, itself pinned by the known-answer tests in
tests/test_oracle.py).  They freeze the oracle's outputs on small seeded
systems so that (a) oracle regressions are caught and (b) the GPU tests on a
box without scipy-level reruns still have exact targets.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ptb_oracle as O  # noqa: E402
from ptb_b200 import synth  # noqa: E402

OUT = Path(__file__).resolve().parent / "water4.npz"


def main():
    s = synth.water_cluster(4, seed=2)
    n = s.ndim
    H = O.filter_matrix_sym(s.Hvec, 1e-4)
    S = O.filter_matrix_sym(s.Svec, 1e-4)
    Hf, Sf = O.blowsym(n, H), O.blowsym(n, S)
    Pd, e = O.dense_projector(Hf, Sf, s.nel)
    out = dict(Hvec=s.Hvec, Svec=s.Svec, aoat=s.aoat, xyz=s.xyz, nel=s.nel, filter=1e-4,
               P_dense=O.packsym(Pd), eig=e)
    for cols in (1, 2, 3):
        r = O.sm_stupid_simple(n, s.nel, H, S, s.nat, s.xyz, s.aoat, cols, 2)
        out[f"P_sm{cols}"] = r.Pvec
        out[f"mu_sm{cols}"] = np.array([m for _, m, _ in r.mu_trace])
        out[f"nel_sm{cols}"] = np.array([x for _, _, x in r.mu_trace])
        out[f"dims_sm{cols}"] = np.array(r.dims)
    P2, e2, focc, fail = O.solve2(1, n, s.nel, 0, 300.0, H, S)
    out["P_solve2"] = P2
    out["focc_solve2"] = focc
    P, it = O.sp2_trace_correcting(Hf, Sf, s.nel)
    out["P_sp2"] = O.packsym(P)
    for t in (1, 2, 3, 4):
        pur = O.PurificationSettings(type=t, metric_type=O.INV if t == 1 else O.INV_SQRT, nel=s.nel, cycles=100)
        Pv, mu, steps = O.purification(pur, n, s.Hvec, s.Svec)
        out[f"P_pur{t}"] = Pv
        out[f"mu_pur{t}"] = np.array([mu, steps])
    np.savez_compressed(OUT, **out)
    print(OUT, OUT.stat().st_size)


if __name__ == "__main__":
    main()
