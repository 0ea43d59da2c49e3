"""XYZ ingestion on the host, without ASE.

The reference takes ASE ``Atoms`` (or dicts / tuples) and leaves file reading
to ``ase.io.read`` in its examples.  ``read_xyz`` reads plain and extended XYZ
files into the structure dicts that ``SOAP.create`` / ``SOAP.derivatives``
accept (``positions``, ``atomic_numbers``, and for extended XYZ with a
``Lattice`` entry, ``cell`` and ``pbc``), so a file can be described without
ASE installed.

Format handled, per frame:
  line 1  number of atoms
  line 2  comment; extended XYZ key=value pairs are read from it:
          ``Lattice="ax ay az bx by bz cx cy cz"`` (cell rows a, b, c) and
          ``pbc="T T F"``; a Lattice without pbc means periodic on all axes
  then    one line per atom: element symbol (or atomic number) and x y z in
          Angstrom; further columns are ignored.
"""
from __future__ import annotations

import shlex
from typing import Dict, List, Optional, Union

import numpy as np

_ELEMENTS = ("H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As "
             "Se Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd "
             "Tb Dy Ho Er Tm Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am "
             "Cm Bk Cf Es Fm Md No Lr Rf Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og").split()
ATOMIC_NUMBERS: Dict[str, int] = {s: z for z, s in enumerate(_ELEMENTS, start=1)}


def atomic_number(token: str) -> int:
    """Atomic number of an element symbol (any case) or of a number string."""
    t = token.strip()
    if t.isdigit():
        return int(t)
    key = t[:1].upper() + t[1:].lower()
    if key not in ATOMIC_NUMBERS:
        raise ValueError(f"unknown element symbol '{token}'")
    return ATOMIC_NUMBERS[key]


def _parse_comment(line: str) -> Dict[str, str]:
    """key=value pairs of an extended XYZ comment line (values may be quoted)."""
    out: Dict[str, str] = {}
    try:
        tokens = shlex.split(line)
    except ValueError:
        return out
    for tok in tokens:
        if "=" in tok:
            k, v = tok.split("=", 1)
            out[k.strip().lower()] = v.strip()
    return out


def _frame(lines: List[str], start: int, path: str) -> tuple:
    try:
        n = int(lines[start].split()[0])
    except (IndexError, ValueError):
        raise ValueError(f"{path}: line {start + 1}: expected an atom count") from None
    if n < 0 or start + 2 + n > len(lines):
        raise ValueError(f"{path}: frame at line {start + 1} declares {n} atoms but the file is shorter")
    meta = _parse_comment(lines[start + 1])
    pos = np.empty((n, 3), dtype=np.float64)
    z = np.empty(n, dtype=np.int64)
    for i in range(n):
        parts = lines[start + 2 + i].split()
        if len(parts) < 4:
            raise ValueError(f"{path}: line {start + 3 + i}: expected 'symbol x y z'")
        z[i] = atomic_number(parts[0])
        pos[i] = [float(parts[1]), float(parts[2]), float(parts[3])]
    system: Dict[str, object] = {"positions": pos, "atomic_numbers": z}
    if "lattice" in meta:
        vals = [float(v) for v in meta["lattice"].split()]
        if len(vals) != 9:
            raise ValueError(f"{path}: Lattice needs 9 numbers, got {len(vals)}")
        system["cell"] = np.array(vals, dtype=np.float64).reshape(3, 3)
        if "pbc" in meta:
            flags = meta["pbc"].split()
            if len(flags) != 3:
                raise ValueError(f"{path}: pbc needs 3 flags")
            system["pbc"] = [f.upper() in ("T", "TRUE", "1") for f in flags]
        else:
            system["pbc"] = [True, True, True]
    return system, start + 2 + n


def read_xyz(path: str, index: Optional[Union[int, slice]] = None) -> Union[Dict[str, object], List[Dict[str, object]]]:
    """Frames of a plain or extended XYZ file as structure dicts.

    ``index`` None or a slice -> list of frames; an int -> that frame (negative
    counts from the end), like ``ase.io.read``'s index argument."""
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    frames: List[Dict[str, object]] = []
    i = 0
    while i < len(lines):
        if not lines[i].strip():
            i += 1
            continue
        system, i = _frame(lines, i, path)
        frames.append(system)
    if index is None:
        return frames
    if isinstance(index, slice):
        return frames[index]
    if not frames:
        raise IndexError(f"{path}: no frames")
    return frames[index]
