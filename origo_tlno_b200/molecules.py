"""Seeded synthetic molecules and contracted Gaussian bases (cfg0..cfg4).

Every workload the tests and the benchmark use is generated here from fixed
seeds, in bohr, as contracted shells in the reference's input convention:
one record per contracted shell (centre, L, exponents, raw contraction
coefficients); the library normalises each Cartesian component the way the
reference's ``make_shell`` does (core/shell/shell_contract.cpp:41-48) and
orders the spherical AOs shell by shell (2L+1 each).

Recipes of the synthetic workloads cfg0-cfg4 (the choices the workload
descriptions leave open made explicit):

* cfg0 -- water, O (0, 0, 0.117) A, H (0, +-0.757, -0.469) A.  O: s, s, p;
  each H: s; 3 primitives each; exponents log-uniform in [0.1, 200] and
  coefficients uniform in (0.1, 1), drawn from seed 0 shell by shell
  (exponents then coefficients).  D = C C^T, C 7x5 with N(0,1)/sqrt(7)
  entries (seed 1).
* cfg1 -- 24 atoms (14 heavy with Z drawn from {6,7,8}, 10 H) uniform in a
  10 A box with minimum pair distance 1.0 A (seed 2, rejection sampling).
  Heavy: s,s,s,p,p,d with 6/3/1/3/1/1 primitives; H: s,s,p with 3/1/1.
  "Exponents log-uniform in [0.08, 5000] scaled by shell rank": the k-th
  shell of angular momentum L on an element (k = 0, 1, ...) draws its
  exponents log-uniformly in [0.08, max(5000 * 10^-k * 20^-L, 0.32)].
  One basis per element (all atoms of an element share it), drawn in order
  of increasing Z.  D = C C^T with n_occ = 45, C ~ N(0,1)/sqrt(n_bf).
* cfg2 -- 60 atoms (40 heavy with Z in {6,7,8,16}, 20 H) in a 15 A box
  (seed 3).  Heavy: s x4 (8/4/2/1 primitives), p x3 (6/3/1), d x2 (2/1),
  f x1 (1); H: s x3 (4/2/1), p x2 (2/1), d x1 (1): 1-8 primitives.
  n_occ = 130.
* cfg3 -- 256 molecules with 3..30 atoms (seed 4; H/C/N/O 40/35/12/13 %),
  cubic box of side 1.6 * n_atoms^(1/3) + 2 A, minimum distance 1.0 A,
  cfg1 basis recipe (one basis per element, drawn from seed 4).
  n_occ = n_bf // 4 per molecule.
* cfg4 -- 400 rigid cfg0-geometry waters, uniformly random orientations,
  centres on 400 of the 448 sites of a 7x8x8 grid with 3.0 A spacing,
  jittered uniformly by +-0.25 A per axis (seed 5).  O: s x3, p x2, d x1;
  H: s x2, p x1 -- the shell composition of def2-SVP, whose contraction
  pattern the recipe follows: O s 5/1/1, p 3/1, d 1; H s 3/1, p 1
  primitives, exponents log-uniform per shell in def2-SVP-like ranges
  (O s1 [0.5, 2500], s2 [0.25, 1.0], s3 [0.1, 0.4], p1 [0.3, 15],
  p2 [0.1, 0.4], d [0.5, 1.5]; H s1 [0.4, 15], s2 [0.1, 0.2], p [0.5, 1.2]),
  coefficients U(0.1, 1); one basis per element from seed 5.
  n_occ = 2000, Schwarz threshold 1e-11;
  the SCF-like sequence is D_{k+1} = D_k + 1e-3 * (C_k C_k^T) with a fresh
  C_k ~ N(0,1)/sqrt(n_bf) per step (seed 1000 + k).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

ANGSTROM_TO_BOHR = 1.0 / 0.529177210903


@dataclass
class ShellSpec:
    """One contracted shell: centre (bohr), L, exponents, raw coefficients."""

    center: Tuple[float, float, float]
    L: int
    exponents: np.ndarray
    coefficients: np.ndarray
    atom: int = -1


@dataclass
class Molecule:
    name: str
    charges: np.ndarray           # (natom,) int
    coords: np.ndarray            # (natom, 3) bohr
    shells: List[ShellSpec] = field(default_factory=list)

    @property
    def n_sph(self) -> int:
        return sum(2 * s.L + 1 for s in self.shells)

    @property
    def n_cart(self) -> int:
        return sum((s.L + 1) * (s.L + 2) // 2 for s in self.shells)

    def soa(self):
        """Shell arrays in the C-ABI layout (see include/tlno_gpu.h)."""
        n = len(self.shells)
        centers = np.array([s.center for s in self.shells], dtype=np.float64).reshape(n, 3)
        L = np.array([s.L for s in self.shells], dtype=np.int32)
        nprim = np.array([len(s.exponents) for s in self.shells], dtype=np.int32)
        exps = np.concatenate([s.exponents for s in self.shells]).astype(np.float64)
        coefs = np.concatenate([s.coefficients for s in self.shells]).astype(np.float64)
        return centers, L, nprim, exps, coefs


# Element basis recipes: list of (L, nprim) in shell order.
_CFG1_HEAVY = [(0, 6), (0, 3), (0, 1), (1, 3), (1, 1), (2, 1)]
_CFG1_H = [(0, 3), (0, 1), (1, 1)]
_CFG2_HEAVY = [(0, 8), (0, 4), (0, 2), (0, 1), (1, 6), (1, 3), (1, 1),
               (2, 2), (2, 1), (3, 1)]
_CFG2_H = [(0, 4), (0, 2), (0, 1), (1, 2), (1, 1), (2, 1)]
# (L, nprim, lo, hi): def2-SVP-like contraction pattern for the water cluster
_CFG4_O = [(0, 5, 0.5, 2500.0), (0, 1, 0.25, 1.0), (0, 1, 0.1, 0.4), (1, 3, 0.3, 15.0),
           (1, 1, 0.1, 0.4), (2, 1, 0.5, 1.5)]
_CFG4_H = [(0, 3, 0.4, 15.0), (0, 1, 0.1, 0.2), (1, 1, 0.5, 1.2)]


def _rank_scaled_basis(rng, recipe, lo=0.08, hi=5000.0):
    """Exponents log-uniform in [lo, hi * 10^-k * 20^-L] for rank k of L."""
    out = []
    rank: Dict[int, int] = {}
    for L, nprim in recipe:
        k = rank.get(L, 0)
        rank[L] = k + 1
        top = max(hi * (10.0 ** -k) * (20.0 ** -L), 4.0 * lo)
        e = np.exp(rng.uniform(np.log(lo), np.log(top), size=nprim))
        e = np.sort(e)[::-1].copy()
        c = rng.uniform(0.1, 1.0, size=nprim)
        out.append((L, e, c))
    return out


def _plain_basis(rng, recipe, lo=0.1, hi=200.0):
    out = []
    for L, nprim in recipe:
        e = np.exp(rng.uniform(np.log(lo), np.log(hi), size=nprim))
        c = rng.uniform(0.1, 1.0, size=nprim)
        out.append((L, e, c))
    return out


def _ranged_basis(rng, recipe):
    out = []
    for L, nprim, lo, hi in recipe:
        e = np.sort(np.exp(rng.uniform(np.log(lo), np.log(hi), size=nprim)))[::-1].copy()
        c = rng.uniform(0.1, 1.0, size=nprim)
        out.append((L, e, c))
    return out


def _attach(mol: Molecule, element_basis: Dict[int, list]) -> Molecule:
    for a, (Z, xyz) in enumerate(zip(mol.charges, mol.coords)):
        for L, e, c in element_basis[int(Z)]:
            mol.shells.append(ShellSpec(tuple(float(v) for v in xyz), L,
                                        e.copy(), c.copy(), atom=a))
    return mol


def _random_positions(rng, n, box, dmin, max_tries=200000):
    pts: List[np.ndarray] = []
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place atoms with the minimum distance")
        p = rng.uniform(0.0, box, size=3)
        if all(np.linalg.norm(p - q) >= dmin for q in pts):
            pts.append(p)
    return np.array(pts)


_WATER_A = np.array([[0.0, 0.0, 0.117], [0.0, 0.757, -0.469], [0.0, -0.757, -0.469]])


def cfg0() -> Molecule:
    rng = np.random.default_rng(0)
    mol = Molecule("cfg0_water", np.array([8, 1, 1]), _WATER_A * ANGSTROM_TO_BOHR)
    recipes = {0: [(0, 3), (0, 3), (1, 3)], 1: [(0, 3)], 2: [(0, 3)]}
    for a in range(3):
        for L, e, c in _plain_basis(rng, recipes[a]):
            mol.shells.append(ShellSpec(tuple(mol.coords[a]), L, e, c, atom=a))
    return mol


def _organic(name, seed, n_heavy, n_h, heavy_z, box_a, heavy_recipe, h_recipe):
    rng = np.random.default_rng(seed)
    xyz = _random_positions(rng, n_heavy + n_h, box_a, 1.0) * ANGSTROM_TO_BOHR
    Z = np.concatenate([rng.choice(heavy_z, size=n_heavy), np.ones(n_h, dtype=int)])
    elements = sorted(set(int(z) for z in Z))
    basis = {}
    for z in elements:
        basis[z] = _rank_scaled_basis(rng, h_recipe if z == 1 else heavy_recipe)
    return _attach(Molecule(name, Z.astype(np.int64), xyz), basis)


def cfg1() -> Molecule:
    return _organic("cfg1_organic24", 2, 14, 10, [6, 7, 8], 10.0, _CFG1_HEAVY, _CFG1_H)


def cfg2() -> Molecule:
    return _organic("cfg2_highL60", 3, 40, 20, [6, 7, 8, 16], 15.0, _CFG2_HEAVY, _CFG2_H)


def cfg3(n_molecules: int = 256) -> List[Molecule]:
    rng = np.random.default_rng(4)
    basis = {z: _rank_scaled_basis(rng, _CFG1_H if z == 1 else _CFG1_HEAVY)
             for z in (1, 6, 7, 8)}
    mols = []
    for m in range(n_molecules):
        n = int(rng.integers(3, 31))
        Z = rng.choice([1, 6, 7, 8], size=n, p=[0.40, 0.35, 0.12, 0.13])
        box = 1.6 * n ** (1.0 / 3.0) + 2.0
        xyz = _random_positions(rng, n, box, 1.0) * ANGSTROM_TO_BOHR
        mols.append(_attach(Molecule(f"cfg3_{m}", Z.astype(np.int64), xyz), basis))
    return mols


def _random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def water_cluster(n_waters: int = 400, seed: int = 5, grid=(7, 8, 8),
                  spacing: float = 3.0, jitter: float = 0.25) -> Molecule:
    rng = np.random.default_rng(seed)
    basis = {8: _ranged_basis(rng, _CFG4_O), 1: _ranged_basis(rng, _CFG4_H)}
    sites = np.array([(i, j, k) for i in range(grid[0]) for j in range(grid[1])
                      for k in range(grid[2])], dtype=float) * spacing
    if n_waters > len(sites):
        raise ValueError("more waters than grid sites")
    chosen = np.sort(rng.choice(len(sites), size=n_waters, replace=False))
    Z, xyz = [], []
    for s in chosen:
        centre = sites[s] + rng.uniform(-jitter, jitter, size=3)
        R = _random_rotation(rng)
        for atom, z in zip(_WATER_A, (8, 1, 1)):
            Z.append(z)
            xyz.append(centre + R @ atom)
    mol = Molecule(f"water{n_waters}", np.array(Z), np.array(xyz) * ANGSTROM_TO_BOHR)
    return _attach(mol, basis)


def cfg4() -> Molecule:
    return water_cluster(400, 5)


def fragment(mol: Molecule, atoms: Sequence[int], name: str = "") -> Molecule:
    """The sub-molecule of the listed atoms with their shells (same
    exponents and coefficients), atoms renumbered in the given order."""
    atoms = [int(a) for a in atoms]
    remap = {a: k for k, a in enumerate(atoms)}
    out = Molecule(name or f"{mol.name}_frag", mol.charges[atoms].copy(), mol.coords[atoms].copy())
    for a in atoms:
        for sh in mol.shells:
            if sh.atom == a:
                out.shells.append(ShellSpec(sh.center, sh.L, sh.exponents.copy(), sh.coefficients.copy(),
                                            atom=remap[a]))
    return out


def cfg2_fragment() -> Molecule:
    """Two heavy atoms and one hydrogen of cfg2 (shells up to f, M = 74):
    the f-shell parity case."""
    return fragment(cfg2(), [0, 1, 40], "cfg2_fragment")


def random_density(n_bf: int, n_occ: int, seed: int) -> np.ndarray:
    """D = C C^T with C (n_bf x n_occ) ~ N(0,1)/sqrt(n_bf)."""
    rng = np.random.default_rng(seed)
    C = rng.normal(size=(n_bf, n_occ)) / np.sqrt(n_bf)
    return C @ C.T


def cfg0_density() -> np.ndarray:
    rng = np.random.default_rng(1)
    C = rng.normal(size=(7, 5)) / np.sqrt(7.0)
    return C @ C.T


CONFIGS = {"cfg0": cfg0, "cfg1": cfg1, "cfg2": cfg2, "cfg4": cfg4}
N_OCC = {"cfg0": 5, "cfg1": 45, "cfg2": 130, "cfg4": 2000}
SCHWARZ = {"cfg0": 1e-12, "cfg1": 1e-12, "cfg2": 1e-12, "cfg3": 1e-12, "cfg4": 1e-11}


def density_for(name: str, mol: Molecule) -> np.ndarray:
    if name == "cfg0":
        return cfg0_density()
    return random_density(mol.n_sph, N_OCC[name], seed={"cfg1": 102, "cfg2": 103, "cfg4": 105}[name])
