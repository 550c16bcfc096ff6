"""Writers and readers for YAMC's own file formats.

* ``parameters.prm``: one ``name = value`` per line, ``#`` comments
  (parameters.f90:266-305, keys at parameters.f90:102-148).
* ``.mol``: ``name x y z sigma epsilon charge mass hard_core`` per atom,
  Angstrom and kcal/mol (Molecule.f90:142-188).
* ``.composition``: number of species, then ``molfile count`` lines
  (composition.f90:84-142).  The reference resolves the molecule file names
  relative to the working directory; the readers here resolve them relative
  to the composition file, so names are written without a directory part.
* moltab binary: per molecule ``x y z theta phi psi`` as little-endian
  fixed-point integers of ``nbytes`` bytes (MoleculeTable.f90:170-319):
  ``xi = nint((x + 0.5) * 256**nbytes)``, ``itheta = nint(theta/2pi * 256**nbytes)``.
* ``energy.dat``: list-directed rows ``frame U_total U_total_ew U_total_lj
  uu_ew uu_lj6 uu_lj12 E_k_coulomb E_k_lj`` (runmc.f90:336-354).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Sequence

import numpy as np

TWO_PI = 2.0 * 3.14159265358979323846


@dataclass
class MolAtom:
    name: str
    x: float
    y: float
    z: float
    sigma: float      # Angstrom
    epsilon: float    # kcal/mol
    charge: float     # e
    mass: float
    hard_core: float  # Angstrom, 0 -> sigma*sqrt(0.4) (Molecule.f90:179)


def write_mol(path: str, atoms: Sequence[MolAtom]) -> None:
    with open(path, "w") as f:
        for a in atoms:
            f.write(f"{a.name:<4s} {a.x!r} {a.y!r} {a.z!r} {a.sigma!r} {a.epsilon!r} "
                    f"{a.charge!r} {a.mass!r} {a.hard_core!r}\n")


def write_composition(path: str, entries: Sequence[tuple]) -> None:
    """entries: (mol_file_name, count) in composition order."""
    with open(path, "w") as f:
        f.write(f"{len(entries)}\n")
        for name, count in entries:
            f.write(f"{os.path.basename(name)} {int(count)}\n")


def write_parameters(path: str, params: Dict[str, object]) -> None:
    with open(path, "w") as f:
        for k, v in params.items():
            if isinstance(v, float):
                f.write(f"{k} = {v!r}\n")
            else:
                f.write(f"{k} = {v}\n")


def _le_bytes(vals: np.ndarray, nbytes: int) -> np.ndarray:
    v = vals.astype(np.int64)
    out = np.zeros((v.size, nbytes), dtype=np.uint8)
    for b in range(nbytes):
        out[:, b] = (v >> (8 * b)) & 0xFF
    return out


def write_moltab(path: str, x, y, z, theta, phi, psi, nbytes_xyz: int = 3, nbytes_ang: int = 3) -> None:
    """MoleculeTable_save_binary (MoleculeTable.f90:170-217); positions in box units."""
    pxyz = float(256 ** nbytes_xyz)
    pang = float(256 ** nbytes_ang)
    rint = lambda a: np.where(a >= 0, np.floor(a + 0.5), np.ceil(a - 0.5))  # Fortran nint
    cols = []
    for a in (x, y, z):
        cols.append(_le_bytes(rint((np.asarray(a, dtype=np.float64) + 0.5) * pxyz), nbytes_xyz))
    for a in (theta, phi, psi):
        cols.append(_le_bytes(rint(np.asarray(a, dtype=np.float64) / TWO_PI * pang), nbytes_ang))
    rec = np.concatenate(cols, axis=1)
    with open(path, "wb") as f:
        f.write(rec.tobytes())


def read_moltab(path: str, nmol: int, nbytes_xyz: int = 3, nbytes_ang: int = 3):
    """MoleculeTable_load_binary (MoleculeTable.f90:240-319)."""
    raw = np.fromfile(path, dtype=np.uint8)
    rec = 3 * nbytes_xyz + 3 * nbytes_ang
    if raw.size < rec * nmol:
        raise ValueError(f"{path}: {raw.size} bytes, need {rec * nmol}")
    raw = raw[: rec * nmol].reshape(nmol, rec).astype(np.int64)
    def col(off, nb):
        v = np.zeros(nmol, dtype=np.int64)
        for b in range(nb):
            v += raw[:, off + b] << (8 * b)
        return v
    pxyz = float(256 ** nbytes_xyz)
    pang = float(256 ** nbytes_ang)
    out = []
    off = 0
    for _ in range(3):
        out.append(col(off, nbytes_xyz) / pxyz - 0.5)
        off += nbytes_xyz
    for _ in range(3):
        out.append(col(off, nbytes_ang) / pang * TWO_PI)
        off += nbytes_ang
    return tuple(out)


def format_energy_row(frame: int, e: Sequence[float]) -> str:
    """gfortran list-directed layout of one energy.dat row (integer width 12,
    reals with 17 significant digits)."""
    parts = [f"{int(frame):12d}"]
    for v in e:
        parts.append(f"{v: .17G}".rjust(25))
    return " ".join(parts) + "     "


def write_energy_rows(path: str, rows: np.ndarray, append: bool = True) -> None:
    with open(path, "a" if append else "w") as f:
        for r in np.asarray(rows).reshape(-1, 9):
            f.write(format_energy_row(int(round(r[0])), r[1:]) + "\n")


def read_energy_dat(path: str) -> np.ndarray:
    rows = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if len(t) >= 9:
                rows.append([float(v) for v in t[:9]])
    return np.array(rows, dtype=np.float64).reshape(-1, 9)


def read_freq_file(path: str, nmol: int):
    """The frequencies file of run_mc (read_freq_file, runmc.f90:70-173): comment ('#') and empty
    lines, then the number of records, then records "first-last move_prob xchange_prob" with
    1-based molecule intervals that must not overlap and must cover every molecule.  Returns
    (move weights, exchange weights), one per molecule; the move weights are yamc_system's
    move_weights.  Raises ValueError where the reference throws ERROR_PARAMETER / ERROR_IO."""
    import numpy as np
    with open(path) as f:
        lines = f.read().splitlines()
    it = iter(lines)
    head = None
    for line in it:
        if line.strip() and "#" not in line:
            head = line
            break
    if head is None:
        raise ValueError(f"read_freq_file: unexpected end of file {path}")
    nrec = int(head.split()[0])
    mv = np.full(nmol, -1.0)
    xc = np.full(nmol, -1.0)
    for _ in range(nrec):
        try:
            rec = next(it)
        except StopIteration:
            raise ValueError(f"read_freq_file: unexpected end of file {path}")
        tok = rec.replace("-", " ").split()
        first, last, mp, xp = int(tok[0]), int(tok[1]), float(tok[2]), float(tok[3])
        if last > nmol:
            raise ValueError(f"read_freq_file: {path} is inconsistent with the composition")
        for j in range(first - 1, last):
            if mv[j] > 0:
                raise ValueError(f"read_freq_file: crossing intervals in {path}")
            mv[j] = mp
            xc[j] = xp
    if np.any(mv < 0):
        raise ValueError(f"read_freq_file: not all frequences defined ({path} is inconsistent with composition?)")
    return mv, xc


def write_rdf(prefix: str, r, g, labels=None) -> list:
    """save_rdfs' files (mcrdf2.f90:371-440): one per species pair t1 <= t2, named
    prefix + "NN_MM.dat" (two-digit 1-based species numbers) or prefix + "label1_label2.dat",
    each line "r g(r)" at the bin centres.  Returns the paths written."""
    nt = g.shape[0]
    paths = []
    for i in range(nt):
        for j in range(i, nt):
            name = f"{labels[i]}_{labels[j]}" if labels else f"{i + 1:02d}_{j + 1:02d}"
            path = f"{prefix}{name}.dat"
            with open(path, "w") as f:
                for rk, gk in zip(r, g[i, j]):
                    f.write(f" {rk:24.16E} {gk:24.16E}\n")
            paths.append(path)
    return paths
