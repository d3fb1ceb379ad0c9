"""CPU checks that the synthetic workloads are the configured systems: atom
counts, basis sizes, electron counts and box edges of the five density-step
configurations, and the stated recipe of the synthetic (H, S) pairs."""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import synth

# (molecules, ndim, nel, box edge in Angstrom) of the water configurations
WATER = {32: (736, 256, 9.855), 512: (11776, 4096, 24.84), 2048: (47104, 16384, 39.42)}


@pytest.mark.parametrize("nmol", sorted(WATER))
def test_water_boxes(nmol):
    ndim, nel, edge = WATER[nmol]
    sym, xyz, L = synth.water_cluster_geometry(nmol, seed=1)
    assert len(sym) == 3 * nmol and abs(L - edge) < 0.01
    aoat, slots, occ = synth.basis_layout(sym)
    assert aoat.shape[0] == ndim and 2 * int(occ.sum()) == nel
    w = xyz.reshape(nmol, 3, 3)
    oxy = w[:, 0, :]
    assert oxy.min() >= 0.0 and oxy.max() <= L
    d = np.sqrt(np.sum((oxy[:, None] - oxy[None]) ** 2, axis=-1)) + 1e9 * np.eye(nmol)
    assert d.min() >= 2.5
    r1 = np.linalg.norm(w[:, 1] - w[:, 0], axis=1)
    r2 = np.linalg.norm(w[:, 2] - w[:, 0], axis=1)
    assert np.allclose(r1, 0.96) and np.allclose(r2, 0.96)
    cosang = np.sum((w[:, 1] - w[:, 0]) * (w[:, 2] - w[:, 0]), axis=1) / (r1 * r2)
    assert np.allclose(np.degrees(np.arccos(cosang)), 104.5)


def test_alkane_chain():
    sym, xyz = synth.alkane_geometry(200, seed=3)
    assert sym.count("C") == 200 and sym.count("H") == 402
    aoat, _, occ = synth.basis_layout(sym)
    # the synthetic occupation rule (four occupied-type AOs per 13-AO atom, none on a
    # 5-AO atom) fills 800 orbitals, not the 601 of the valence count 1202: in this
    # model a filling of 601 would put mu inside the occupied-type band
    assert aoat.shape[0] == 4610 and 2 * int(occ.sum()) == 1600
    C = xyz[[k for k, s in enumerate(sym) if s == "C"]]
    cc = np.linalg.norm(np.diff(C, axis=0), axis=1)
    assert abs(cc.mean() - 1.54) < 0.01 and cc.std() < 0.05   # 0.02 A Gaussian jitter per atom
    H = xyz[[k for k, s in enumerate(sym) if s == "H"]]
    ch = np.min(np.linalg.norm(H[:, None] - C[None], axis=-1), axis=1)
    assert abs(ch.mean() - 1.09) < 0.01


def test_lattice_instances():
    counts = [synth.lattice_instance(i).nat for i in range(0, 256, 37)]
    assert all(20 <= c <= 400 for c in counts)
    s = synth.lattice_instance(5)
    heavy = sum(1 for x in s.symbols if x == "O")
    assert heavy == s.nat // 3
    assert s.ndim == 13 * heavy + 5 * (s.nat - heavy)
    assert s.nel == 2 * 4 * heavy   # four occupied-type AOs per 13-AO atom, none on a 5-AO atom


@pytest.mark.parametrize("make", [lambda: synth.water_cluster(32, seed=1), lambda: synth.alkane(20),
                                  lambda: synth.lattice_instance(3)])
def test_hamiltonian_and_overlap_recipe(make):
    s = make()
    n = s.ndim
    amp = synth.LATTICE_AMP if s.name.startswith("lattice") else synth.MOLECULAR_AMP
    H, S = O.blowsym(n, s.Hvec), O.blowsym(n, s.Svec)
    at = s.aoat - 1
    d = np.sqrt(np.sum((s.xyz[at][:, None] - s.xyz[at][None]) ** 2, axis=-1))
    off = ~np.eye(n, dtype=bool)
    # |F_uv| <= amp exp(-r_AB) off the diagonal
    assert np.all(np.abs(H[off]) <= amp * np.exp(-d[off]) + 1e-15)
    # S: exp(-r^2/2) for the same slot on different atoms, 0 otherwise, 1 on the diagonal
    same = (s.slots[:, None] == s.slots[None]) & (at[:, None] != at[None])
    assert np.allclose(S[same], np.exp(-0.5 * d[same] ** 2)) and np.all(S[off & ~same] == 0.0)
    assert np.all(np.diag(S) == 1.0)
    # symmetric positive definite S
    assert np.linalg.eigvalsh(S).min() > 0.0
    # onsite energies: occupied-type around -0.5 Eh, virtual-type around +0.3 Eh
    e = np.diag(H)
    assert abs(e[s.occ_type].mean() + 0.5) < 0.05 and abs(e[~s.occ_type].mean() - 0.3) < 0.05


def test_configurations_match_the_workload_table():
    assert synth.CONFIGS[0]["nmol"] == 32 and synth.CONFIGS[0]["filter"] == 1e-4
    assert synth.CONFIGS[1]["nmol"] == 512 and synth.CONFIGS[1]["filter"] == 1e-5
    assert synth.CONFIGS[2]["ncarbon"] == 200 and synth.CONFIGS[2]["filter"] == 1e-4
    assert synth.CONFIGS[3]["nmol"] == 2048 and synth.CONFIGS[3]["filter"] == 1e-4
    assert synth.CONFIGS[4]["count"] == 256
