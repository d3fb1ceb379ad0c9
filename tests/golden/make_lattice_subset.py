"""Writes tests/golden/lattice_subset.json: the spectral range / HOMO-LUMO gap
of every system of the uneven multi-instance batch (the 256 seeded cubic-lattice
systems of ptb_b200.synth, 20-400 atoms) and the stratified subset that the GPU
parity test of that batch runs against the oracle's dense projector.

The subset holds every system whose range/gap exceeds 1e4 (the hardest cases
for the mixed-precision refinement) plus, for each quartile of ndim, the
systems of smallest and largest ndim and of median range/gap in it.

    python tests/golden/make_lattice_subset.py
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import ptb_oracle as O  # noqa: E402
from ptb_b200 import synth  # noqa: E402

HARD = 1e4


def range_over_gap(s) -> float:
    e, _, info = O.sygvd(O.blowsym(s.ndim, s.Hvec), O.blowsym(s.ndim, s.Svec))
    assert info == 0
    nocc = s.nel // 2
    return float((e[-1] - e[0]) / (e[nocc] - e[nocc - 1]))


def main():
    t0 = time.time()
    systems = synth.make_config(4)
    rows = []
    for i, s in enumerate(systems):
        rows.append({"index": i, "ndim": int(s.ndim), "nel": int(s.nel), "range_over_gap": range_over_gap(s)})
    picked = {r["index"] for r in rows if r["range_over_gap"] > HARD}
    by_n = sorted(rows, key=lambda r: r["ndim"])
    q = len(by_n) // 4
    for k in range(4):
        part = by_n[k * q:(k + 1) * q] if k < 3 else by_n[3 * q:]
        picked.add(part[0]["index"])
        picked.add(part[-1]["index"])
        med = sorted(part, key=lambda r: r["range_over_gap"])[len(part) // 2]
        picked.add(med["index"])
    out = {"hard_threshold": HARD, "subset": sorted(picked), "systems": rows,
           "note": "range/gap = (e_max - e_min) / (e_LUMO - e_HOMO) of the generalized problem H c = e S c"}
    (HERE / "lattice_subset.json").write_text(json.dumps(out, indent=1) + "\n")
    rg = np.array([r["range_over_gap"] for r in rows])
    print(f"{len(picked)} systems picked; range/gap median {np.median(rg):.3g}, max {rg.max():.3g}; "
          f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
