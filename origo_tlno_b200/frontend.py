"""Molecule input and named-basis front end.

Host-side counterpart of the reference's front end:

* ``read_inp_file`` / ``read_xyz_file`` / ``molecule_spec`` --
  benchmarks/common/molecule_io.cpp:36-165 (``* xyz charge multiplicity``
  block, coordinates in bohr, the same error texts);
* ``parse_basis_kind`` -- core/basis/basis_general.cpp:48-75 (the same names
  and aliases, the same error text);
* ``build_basis_general`` -- core/basis/basis_general.cpp:77-111: one
  contracted shell per basis-set entry on every atom, the nuclear charges
  and the electron count (sum of Z minus the molecular charge).

The reference compiles its basis sets into the library; this front end reads
them from basis-set files in the Gaussian94 format of the Basis Set Exchange
(``load_basis_library``), one library per basis kind, so that any basis the
exchange publishes can be used.  The engine normalises every Cartesian
component of a shell as the reference's make_shell does, so a molecule built
here gives the reference's integrals.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .molecules import Molecule, ShellSpec

ELEMENTS = ("H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn "
            "Ga Ge As Se Br Kr").split()
Z_OF = {s.upper(): i + 1 for i, s in enumerate(ELEMENTS)}


class FrontendError(RuntimeError):
    pass


@dataclass
class MoleculeInput:
    symbols: List[str] = field(default_factory=list)
    coords_bohr: List[Tuple[float, float, float]] = field(default_factory=list)
    charge: int = 0
    multiplicity: int = 1


@dataclass
class MoleculeSpec:
    symbols: List[str]
    coords: List[Tuple[float, float, float]]
    charge: int = 0


def _append_atom_line(mol: MoleculeInput, line: str, path: str, line_number: int) -> None:
    parts = line.split()
    try:
        symbol = parts[0]
        xyz = tuple(float(v) for v in parts[1:4])
        if len(xyz) != 3 or not all(math.isfinite(v) for v in xyz):
            raise ValueError
    except (IndexError, ValueError):
        raise FrontendError(f"bad coordinate line {line_number}: {path}") from None
    mol.symbols.append(symbol)
    mol.coords_bohr.append(xyz)


def read_inp_file(path: str) -> MoleculeInput:
    """The ``* xyz charge multiplicity`` block of an input file (bohr)."""
    try:
        with open(path) as f:
            lines = f.read().splitlines()
    except OSError:
        raise FrontendError(f"Cannot open input file: {path}") from None
    mol = MoleculeInput()
    found = closed = False
    for number, raw in enumerate(lines, start=1):
        text = raw.strip()
        if not text:
            continue
        if not found:
            if text[0] != "*":
                continue
            head = text[1:].split()
            if head and head[0].lower() == "xyz":
                # formatted extraction: a missing or malformed integer reads 0
                # and stops the extraction
                vals = []
                for tok in head[1:3]:
                    m = re.match(r"[+-]?\d+", tok)
                    if not m:
                        break
                    vals.append(int(m.group(0)))
                    if m.end() != len(tok):
                        break
                charge = vals[0] if len(vals) > 0 else 0
                mult = vals[1] if len(vals) > 1 else 0
                if mult < 1:
                    raise FrontendError(f"xyz multiplicity must be at least one: {path}")
                mol.charge, mol.multiplicity = charge, mult
                found = True
            continue
        if text[0] == "*":
            closed = True
            break
        if text[0] in "#!":
            continue
        _append_atom_line(mol, text, path, number)
    if not found:
        raise FrontendError(f"Missing '* xyz charge multiplicity' block in input: {path}")
    if not closed:
        raise FrontendError(f"Unterminated xyz block: {path}")
    if not mol.symbols:
        raise FrontendError(f"Empty xyz block: {path}")
    return mol


def read_xyz_file(path: str, charge: int = 0, multiplicity: int = 1) -> MoleculeInput:
    """An XYZ file whose coordinates are already in bohr."""
    if multiplicity < 1:
        raise FrontendError("XYZ multiplicity must be at least one.")
    try:
        with open(path) as f:
            lines = f.read().splitlines()
    except OSError:
        raise FrontendError(f"cannot open XYZ file: {path}") from None
    if not lines:
        raise FrontendError(f"empty XYZ file: {path}")
    try:
        count = int(lines[0].strip())
    except ValueError:
        raise FrontendError(f"XYZ line 1 must contain the atom count: {path}") from None
    if count < 1:
        raise FrontendError(f"XYZ atom count must be at least one: {path}")
    if len(lines) < 2:
        raise FrontendError(f"XYZ file is missing its comment line: {path}")
    mol = MoleculeInput(charge=charge, multiplicity=multiplicity)
    for atom in range(count):
        if 2 + atom >= len(lines):
            raise FrontendError(f"XYZ file ended after {atom} atoms: {path}")
        _append_atom_line(mol, lines[2 + atom], path, atom + 3)
    return mol


def molecule_spec(inp: MoleculeInput) -> MoleculeSpec:
    return MoleculeSpec(list(inp.symbols), list(inp.coords_bohr), inp.charge)


BASIS_KINDS = {
    "sto-3g": ("STO-3G", "STO3G"),
    "4-31g": ("4-31G", "431G"),
    "6-31g": ("6-31G", "631G"),
    "6-31g(d)": ("6-31G(D)", "631G(D)", "631GD", "6-31G*", "631G*"),
    "6-31g(d,p)": ("6-31G(D,P)", "631G(D,P)", "631GDP", "6-31G(P,D)", "631G(P,D)", "631GPD", "6-31G**", "631G**"),
    "def2-svp": ("DEF2-SVP", "DEF2SVP", "DEF2-DZVP", "DEF2DZVP"),
    "def2-tzvp": ("DEF2-TZVP", "DEF2TZVP"),
}


def parse_basis_kind(name: str) -> str:
    """Canonical basis kind of a name or alias."""
    upper = name.upper()
    for kind, aliases in BASIS_KINDS.items():
        if upper in aliases:
            return kind
    raise FrontendError(f"Unsupported basis set: {name}. Valid: sto-3g, 4-31g, 6-31g, 6-31g(d), 6-31g*, "
                        "6-31g(d,p), 6-31g**, def2-svp, def2-tzvp.")


_L_OF = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4}


def load_basis_library(text: str) -> Dict[str, List[Tuple[int, np.ndarray, np.ndarray]]]:
    """Parses a Gaussian94-format basis-set file (the Basis Set Exchange's
    "gaussian94" output): per element symbol, the contracted shells as
    (L, exponents, raw contraction coefficients) in file order; SP shells are
    split into an S and a P shell."""
    lib: Dict[str, List[Tuple[int, np.ndarray, np.ndarray]]] = {}
    lines = [ln.strip() for ln in text.splitlines()]
    i = 0
    cur: Optional[str] = None
    while i < len(lines):
        ln = lines[i]
        i += 1
        if not ln or ln.startswith("!"):
            continue
        if ln == "****":
            cur = None
            continue
        if cur is None:
            sym = ln.split()[0]
            if sym.upper() not in Z_OF:
                raise FrontendError(f"basis file: unknown element '{sym}'")
            cur = ELEMENTS[Z_OF[sym.upper()] - 1]
            lib.setdefault(cur, [])
            continue
        kind = ln.split()[0].upper()
        nprim = int(ln.split()[1])
        rows = []
        for _ in range(nprim):
            rows.append([float(v.replace("D", "E").replace("d", "e")) for v in lines[i].split()])
            i += 1
        rows = np.array(rows)
        if kind == "SP":
            lib[cur].append((0, rows[:, 0].copy(), rows[:, 1].copy()))
            lib[cur].append((1, rows[:, 0].copy(), rows[:, 2].copy()))
        elif kind in _L_OF:
            lib[cur].append((_L_OF[kind], rows[:, 0].copy(), rows[:, 1].copy()))
        else:
            raise FrontendError(f"basis file: unsupported shell type '{kind}'")
    return lib


def build_basis_general(spec: MoleculeSpec, library: Dict[str, List[Tuple[int, np.ndarray, np.ndarray]]],
                        name: str = "molecule") -> Tuple[Molecule, int]:
    """Contracted shells of every atom from a basis library, the nuclear
    charges and the electron count (the Molecule the engine consumes)."""
    if len(spec.symbols) != len(spec.coords):
        raise FrontendError("Atom and coordinate count mismatch.")
    shells = []
    charges = []
    for a, (sym, xyz) in enumerate(zip(spec.symbols, spec.coords)):
        key = sym.upper()
        if key not in Z_OF:
            raise FrontendError(f"Unsupported element: {sym}")
        canon = ELEMENTS[Z_OF[key] - 1]
        if canon not in library:
            raise FrontendError(f"basis library has no entry for {canon}")
        charges.append(Z_OF[key])
        for L, e, c in library[canon]:
            shells.append(ShellSpec(tuple(float(v) for v in xyz), int(L), np.asarray(e, dtype=float),
                                    np.asarray(c, dtype=float), atom=a))
    mol = Molecule(name, np.array(charges, dtype=np.int32), np.array(spec.coords, dtype=float), shells)
    return mol, int(sum(charges)) - spec.charge
