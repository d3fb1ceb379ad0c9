"""Seeded synthetic systems for the density-matrix step.

The PTB Hamiltonian build (Fortran, integrals + EEQ + dftd4) is not part of
this library, so benchmark and test inputs are synthetic tight-binding pairs
(H, S) placed on real molecular geometries:

* geometry: water clusters at 1.0 g/cm^3 (29.915 A^3 per molecule, O-O >= 2.5 A,
  r(OH) = 0.96 A, HOH = 104.5 deg, random orientations), the all-trans alkane
  C_nH_{2n+2} (C-C 1.54 A, C-H 1.09 A, tetrahedral angles, 0.02 A Gaussian
  jitter), or jittered 1.5 A cubic lattices;
* basis: vDZP counts per element (H 2s1p = 5 AOs; C/N/O 2s2p1d = 13 AOs;
  .basis_vDZP), AO slots s,s',p(3),p'(3),d(5) in that order;
* F_{mu nu} = amp * exp(-r_AB / 1 A) * U[-1,1] (symmetric, mu != nu), onsite
  N(-0.5, 0.1) Eh for occupied-type AOs (slot s and the first p shell of a
  heavy atom) and N(+0.3, 0.1) Eh for virtual-type AOs;
* S_{mu nu} = exp(-0.5 r_AB^2) for AOs of different atoms in the same slot,
  1 on the diagonal, 0 otherwise.  This is a direct sum of principal
  submatrices of a Gaussian-kernel matrix, hence symmetric positive definite;
* nel = 2 * (number of occupied-type AOs).

Matrices are returned in the reference's packed layout (column i, rows <= i).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

AO_PER_ELEMENT = {"H": 5, "C": 13, "N": 13, "O": 13}
OCC_SLOTS_HEAVY = (0, 2, 3, 4)
# Coupling amplitude.  The multi-instance lattice batch uses 0.3 as specified
# for it (its generalized HOMO-LUMO gaps are then 1e-3..1e-2 Eh).  On the
# molecular geometries 0.3 closes the gap (32 H2O: 8e-4 Eh), unlike PTB water
# whose logged chemical-potential trace brackets a gap of several tenths of an
# Eh, so the molecular systems use 0.1 (32 H2O: gap 0.20 Eh).
LATTICE_AMP = 0.3
MOLECULAR_AMP = 0.1
DEFAULT_AMP = MOLECULAR_AMP


@dataclass
class System:
    name: str
    symbols: list
    xyz: np.ndarray          # (nat, 3) Angstrom
    aoat: np.ndarray         # (ndim,) 1-based atom index per AO (int64)
    slots: np.ndarray        # (ndim,) AO slot within its atom
    occ_type: np.ndarray     # (ndim,) bool
    Hvec: np.ndarray         # packed
    Svec: np.ndarray         # packed
    nel: int

    @property
    def ndim(self) -> int:
        return int(self.aoat.shape[0])

    @property
    def nat(self) -> int:
        return int(self.xyz.shape[0])


def _random_rotations(rng, k):
    q = rng.normal(size=(k, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((k, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def water_cluster_geometry(nmol: int, seed: int, min_oo: float = 2.5):
    """nmol waters, O centres uniform in a cube at 1.0 g/cm^3 with O-O >= min_oo."""
    rng = np.random.default_rng(seed)
    L = (nmol * 29.915) ** (1.0 / 3.0)
    ncell = max(1, int(L // min_oo))
    cell = L / ncell
    grid: dict = {}
    centres = []
    while len(centres) < nmol:
        p = rng.uniform(0.0, L, size=3)
        c = tuple((p // cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get((c[0] + dx, c[1] + dy, c[2] + dz), ()):
                        if np.sum((p - q) ** 2) < min_oo * min_oo:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            centres.append(p)
            grid.setdefault(c, []).append(p)
    centres = np.array(centres)
    half = np.deg2rad(104.5) / 2
    r = 0.96
    local = np.array([[0.0, 0.0, 0.0],
                      [r * np.sin(half), r * np.cos(half), 0.0],
                      [-r * np.sin(half), r * np.cos(half), 0.0]])
    R = _random_rotations(rng, nmol)
    xyz = np.einsum("kij,aj->kai", R, local) + centres[:, None, :]
    symbols = ["O", "H", "H"] * nmol
    return symbols, xyz.reshape(-1, 3), L


def alkane_geometry(ncarbon: int, seed: int, jitter: float = 0.02):
    """All-trans C_nH_{2n+2}: C-C 1.54 A, C-H 1.09 A, tetrahedral angles, Gaussian jitter."""
    rng = np.random.default_rng(seed)
    tet = np.arccos(-1.0 / 3.0)
    dcc, dch = 1.54, 1.09
    dx = dcc * np.sin(tet / 2)
    dy = dcc * np.cos(tet / 2)
    C = np.array([[k * dx, (k % 2) * dy, 0.0] for k in range(ncarbon)])
    symbols, pos = [], []
    z = np.array([0.0, 0.0, 1.0])
    for k in range(ncarbon):
        symbols.append("C")
        pos.append(C[k])
        nbrs = [C[j] for j in (k - 1, k + 1) if 0 <= j < ncarbon]
        bonds = [(q - C[k]) / np.linalg.norm(q - C[k]) for q in nbrs]
        if len(bonds) == 2:
            u = -(bonds[0] + bonds[1])
            u /= np.linalg.norm(u)
            a = tet / 2
            dirs = [u * np.cos(a) + z * np.sin(a), u * np.cos(a) - z * np.sin(a)]
        else:
            b = bonds[0] if bonds else np.array([1.0, 0.0, 0.0])
            ip = np.array([0.0, 1.0 if k % 2 == 0 else -1.0, 0.0])
            ip -= b * np.dot(ip, b)
            if np.linalg.norm(ip) < 1e-8:
                ip = np.array([0.0, 1.0, 0.0])
            ip /= np.linalg.norm(ip)
            w = np.cross(b, ip)
            th = np.pi - tet
            dirs = []
            for phi in (0.0, 2 * np.pi / 3, 4 * np.pi / 3):
                perp = ip * np.cos(phi) + w * np.sin(phi)
                dirs.append(-b * np.cos(th) + perp * np.sin(th))
            if not bonds:
                dirs.append(b)
        for d in dirs:
            symbols.append("H")
            pos.append(C[k] + dch * d)
    xyz = np.array(pos) + rng.normal(0.0, jitter, size=(len(pos), 3))
    return symbols, xyz


def lattice_geometry(nat: int, seed: int, spacing: float = 1.5, jitter: float = 0.1):
    """nat atoms on a jittered cubic lattice; 1/3 heavy (13 AOs) and 2/3 light (5 AOs)."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(nat ** (1.0 / 3.0)))
    g = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side),
                             indexing="ij"), -1).reshape(-1, 3)[:nat]
    xyz = g * spacing + rng.normal(0.0, jitter, size=(nat, 3))
    heavy = np.zeros(nat, dtype=bool)
    heavy[rng.permutation(nat)[: nat // 3]] = True
    symbols = ["O" if h else "H" for h in heavy]
    return symbols, xyz


def basis_layout(symbols):
    aoat, slots, occ = [], [], []
    for a, s in enumerate(symbols, start=1):
        nao = AO_PER_ELEMENT[s]
        for k in range(nao):
            aoat.append(a)
            slots.append(k)
            occ.append(nao == 13 and k in OCC_SLOTS_HEAVY)
    return (np.array(aoat, dtype=np.int64), np.array(slots, dtype=np.int64),
            np.array(occ, dtype=bool))


# Shells of the vDZP-sized synthetic basis, per AO of an atom (1-based, as
# bascom's shell2ao): H 5 AOs = s, s, p; C/N/O 13 AOs = s, s, p, p, d.
SHELLS_PER_AO = {5: (1, 2, 3, 3, 3), 13: (1, 2, 3, 3, 3, 4, 4, 4, 5, 5, 5, 5, 5)}


def shell2ao(aoat: np.ndarray) -> np.ndarray:
    """AO -> shell index within its atom (1-based) for an AO -> atom map."""
    aoat = np.asarray(aoat)
    out = np.empty(aoat.shape[0], dtype=np.int64)
    i = 0
    while i < aoat.shape[0]:
        j = i
        while j < aoat.shape[0] and aoat[j] == aoat[i]:
            j += 1
        out[i:j] = SHELLS_PER_AO[j - i]
        i = j
    return out


def _pack_upper(full: np.ndarray) -> np.ndarray:
    n = full.shape[0]
    r, c = np.tril_indices(n)
    return np.ascontiguousarray(full[c, r])


def build_hs(symbols, xyz, seed: int, amp: float = DEFAULT_AMP, name: str = "system") -> System:
    """Synthetic packed (H, S) on a geometry; see the module docstring for the recipe."""
    aoat, slots, occ = basis_layout(symbols)
    n = aoat.shape[0]
    rng = np.random.default_rng(seed + 7919)
    at = aoat - 1
    d = np.sqrt(np.sum((xyz[:, None, :] - xyz[None, :, :]) ** 2, axis=-1))
    npk = n * (n + 1) // 2
    hvec = np.empty(npk)
    svec = np.empty(npk)
    # packed order: column r, rows c <= r; built in column blocks of about 2^24
    # elements so that large systems fit in host memory (the uniform draws come
    # from the one generator in order, so the values do not depend on the blocking)
    r0 = 0
    while r0 < n:
        r1 = r0 + 1
        while r1 < n and (r1 + 1) * (r1 + 2) // 2 - r0 * (r0 + 1) // 2 <= (1 << 24):
            r1 += 1
        k0, k1 = r0 * (r0 + 1) // 2, r1 * (r1 + 1) // 2
        r = np.repeat(np.arange(r0, r1), np.arange(r0 + 1, r1 + 1))
        c = np.arange(k0, k1) - r * (r + 1) // 2
        rab = d[at[r], at[c]]
        u = rng.uniform(-1.0, 1.0, size=k1 - k0)
        hvec[k0:k1] = amp * np.exp(-rab) * u
        same_slot = (slots[r] == slots[c]) & (at[r] != at[c])
        svec[k0:k1] = np.where(same_slot, np.exp(-0.5 * rab * rab), 0.0)
        r0 = r1
    dk = np.arange(1, n + 1) * np.arange(2, n + 2) // 2 - 1   # diagonal positions
    onsite = np.where(occ, rng.normal(-0.5, 0.1, size=n), rng.normal(0.3, 0.1, size=n))
    hvec[dk] = onsite
    svec[dk] = 1.0
    nel = 2 * int(occ.sum())
    return System(name, list(symbols), np.asarray(xyz, dtype=np.float64), aoat, slots, occ,
                  np.ascontiguousarray(hvec), np.ascontiguousarray(svec), nel)


def water_cluster(nmol: int, seed: int = 1, amp: float = DEFAULT_AMP) -> System:
    sym, xyz, _ = water_cluster_geometry(nmol, seed)
    return build_hs(sym, xyz, seed, amp, name=f"h2o_{nmol}")


def alkane(ncarbon: int, seed: int = 3, amp: float = DEFAULT_AMP) -> System:
    sym, xyz = alkane_geometry(ncarbon, seed)
    return build_hs(sym, xyz, seed, amp, name=f"C{ncarbon}H{2 * ncarbon + 2}")


def lattice_instance(index: int, seed: int = 11, amp: float = LATTICE_AMP) -> System:
    rng = np.random.default_rng(seed * 1000003 + index)
    nat = int(rng.integers(20, 401))
    sym, xyz = lattice_geometry(nat, seed * 7777 + index)
    return build_hs(sym, xyz, seed * 31 + index, amp, name=f"lattice_{index}")


# Configurations of the density-step workloads (atoms, ndim, filter).
CONFIGS = {
    0: dict(kind="water", nmol=32, filter=1e-4, seed=1),
    1: dict(kind="water", nmol=512, filter=1e-5, seed=1),
    2: dict(kind="alkane", ncarbon=200, filter=1e-4, seed=3),
    3: dict(kind="water", nmol=2048, filter=1e-4, seed=1),
    4: dict(kind="batch", count=256, filter=0.0, seed=11),
}


def make_config(idx: int):
    cfg = CONFIGS[idx]
    if cfg["kind"] == "water":
        return water_cluster(cfg["nmol"], cfg["seed"])
    if cfg["kind"] == "alkane":
        return alkane(cfg["ncarbon"], cfg["seed"])
    return [lattice_instance(i, cfg["seed"]) for i in range(cfg["count"])]
