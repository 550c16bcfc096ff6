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


# ---------------------------------------------------------------- trajectory writers
# store_traj_frame (runmc.f90:373-417): MoleculeTable_calcPositionsOrientations (MoleculeTable.f90:707-769)
# turns atom positions into molecule centres and ZYZ angles, MoleculeTable_save_binary writes them;
# frames.dat and boxlength.dat get one row per frame / accepted volume step.

def read_mol_template(path: str):
    """Molecule_read_from_file + Molecule_centrate (Molecule.f90:142-209): the atom coordinates
    of a .mol file (Angstrom) relative to its centre of mass, and the masses."""
    rows = [ln.split() for ln in open(path) if ln.strip()]
    x = np.array([float(r[1]) for r in rows]); y = np.array([float(r[2]) for r in rows])
    z = np.array([float(r[3]) for r in rows]); m = np.array([float(r[7]) for r in rows])
    cx, cy, cz = _center_of_mass(x, y, z, m)
    return x - cx, y - cy, z - cz, m


def _center_of_mass(x, y, z, m):
    """center_of_mass (geometry.f90:170-201), summed in atom order."""
    sx = sy = sz = tm = 0.0
    for i in range(len(m)):
        sx = sx + m[i] * x[i]; sy = sy + m[i] * y[i]; sz = sz + m[i] * z[i]; tm = tm + m[i]
    return sx / tm, sy / tm, sz / tm


def _atan2_two_pi(y, x):
    """atan2_two_pi (geometry.f90:204-215)"""
    r = math.atan2(y, x)
    return r + TWO_PI if r < 0 else r


def _prod_vect(x1, y1, z1, x2, y2, z2):
    return y1 * z2 - z1 * y2, z1 * x2 - x1 * z2, x1 * y2 - y1 * x2


def _inv3(A):
    """matrix3x3_inv (matrix3x3.f90): adjugate over determinant"""
    d = (A[0][0] * A[1][1] * A[2][2] + A[0][1] * A[1][2] * A[2][0] + A[0][2] * A[1][0] * A[2][1]
         - A[0][0] * A[1][2] * A[2][1] - A[0][1] * A[1][0] * A[2][2] - A[0][2] * A[1][1] * A[2][0])
    B = [[A[1][1] * A[2][2] - A[1][2] * A[2][1], -A[0][1] * A[2][2] + A[0][2] * A[2][1], A[0][1] * A[1][2] - A[0][2] * A[1][1]],
         [-A[1][0] * A[2][2] + A[1][2] * A[2][0], A[0][0] * A[2][2] - A[0][2] * A[2][0], -A[0][0] * A[1][2] + A[0][2] * A[1][0]],
         [A[1][0] * A[2][1] - A[1][1] * A[2][0], -A[0][0] * A[2][1] + A[0][1] * A[2][0], A[0][0] * A[1][1] - A[0][1] * A[1][0]]]
    return [[B[i][j] / d for j in range(3)] for i in range(3)]


def xyz_to_angles(tx, ty, tz, xn, yn, zn):
    """xyz_to_angles (geometry.f90:352-451): the ZYZ angles (theta, phi, psi) of the rotation that
    takes the template coordinates (tx, ty, tz) to (xn, yn, zn), both relative to the centre and in
    Angstrom: R = X_new X^-1 from two non-collinear atoms and their cross product
    (rotation_matrix, :334-350), then ZYZRotation_matrix_to_angles (:221-250); one atom on the
    centre gives zeros, two atoms or a linear molecule xyz_to_angles_two_atoms (:461-520)."""
    n = len(tx)
    i1 = next((i for i in range(n) if abs(tx[i]) + abs(ty[i]) + abs(tz[i]) > 1e-8), -1)
    if i1 < 0:
        return 0.0, 0.0, 0.0
    i2, prod = -1, None
    for i in range(i1 + 1, n):
        if abs(tx[i]) + abs(ty[i]) + abs(tz[i]) < 1e-8:
            continue
        p = _prod_vect(tx[i1], ty[i1], tz[i1], tx[i], ty[i], tz[i])
        if abs(p[0]) + abs(p[1]) + abs(p[2]) > 1e-8:
            i2, prod = i, p
            break
    if i2 < 0:
        x, y, z = tx[i1], ty[i1], tz[i1]
        dxz = math.sqrt(x ** 2 + z ** 2)
        alpha = math.atan2(z, -x)
        v = (math.asin(zn[i1] / dxz) - alpha) / PI_
        theta = (v - math.floor(v)) * PI_
        a = x * math.cos(theta) + z * math.sin(theta)
        beta = math.atan2(y, a)
        w = (math.atan2(yn[i1], xn[i1]) - beta) / TWO_PI
        return theta, (w - math.floor(w)) * TWO_PI, 0.0
    X = [[tx[i1], tx[i2], prod[0]], [ty[i1], ty[i2], prod[1]], [tz[i1], tz[i2], prod[2]]]
    pn = _prod_vect(xn[i1], yn[i1], zn[i1], xn[i2], yn[i2], zn[i2])
    Xn = [[xn[i1], xn[i2], pn[0]], [yn[i1], yn[i2], pn[1]], [zn[i1], zn[i2], pn[2]]]
    Xi = _inv3(X)
    R = [[sum(Xn[i][k] * Xi[k][j] for k in range(3)) for j in range(3)] for i in range(3)]
    cos_theta = R[2][2]
    if abs(cos_theta - 1.0) < 1e-8:
        return 0.0, _atan2_two_pi(-R[0][1], R[0][0]), 0.0
    return math.acos(cos_theta), _atan2_two_pi(R[1][2], R[0][2]), _atan2_two_pi(R[2][1], -R[2][0])


PI_ = 3.14159265358979323846


def traj_frame(x, y, z, first_atom, last_atom, species, templates, box_length):
    """MoleculeTable_calcPositionsOrientations (MoleculeTable.f90:707-769): per molecule the centre
    of mass (box units) and the ZYZ angles of its atoms (box units, 1-based inclusive atom ranges)
    against its species' centred template.  Returns (cx, cy, cz, theta, phi, psi)."""
    M = len(first_atom)
    out = [np.zeros(M) for _ in range(6)]
    for m in range(M):
        a, b = int(first_atom[m]) - 1, int(last_atom[m])
        tx, ty, tz, mass = templates[int(species[m])]
        cx, cy, cz = _center_of_mass(x[a:b], y[a:b], z[a:b], mass)
        xn = [(v - cx) * box_length for v in x[a:b]]
        yn = [(v - cy) * box_length for v in y[a:b]]
        zn = [(v - cz) * box_length for v in z[a:b]]
        th, ph, ps = xyz_to_angles(tx, ty, tz, xn, yn, zn)
        for k, v in enumerate((cx, cy, cz, th, ph, ps)):
            out[k][m] = v
    return tuple(out)


def append_moltab(path: str, x, y, z, theta, phi, psi, nbytes_xyz: int = 3, nbytes_ang: int = 3) -> None:
    """MoleculeTable_save_binary appended to a trajectory (store_traj_frame seeks to the end)."""
    tmp = path + ".frame"
    write_moltab(tmp, x, y, z, theta, phi, psi, nbytes_xyz, nbytes_ang)
    with open(tmp, "rb") as f, open(path, "ab") as g:
        g.write(f.read())
    os.remove(tmp)


def format_frames_row(frame: int, box_length: float, n_mv_steps: float, n_mv_accepted: float, n_vol_steps: float,
                      n_vol_accepted: float, n_xchg_steps: float, n_xchg_accepted: float, wall_time: int) -> str:
    """frames.dat row, format (I12,F15.10,F12.0,F12.0,F12.0,F12.0,F12.0,F12.0,I12) (runmc.f90:413-414)."""
    def f0(v):  # F12.0 of a whole count: 11 digits and the point
        return f"{int(math.floor(float(v) + 0.5)):11d}."
    return (f"{int(frame):12d}{float(box_length):15.10f}" + "".join(f0(v) for v in (
        n_mv_steps, n_mv_accepted, n_vol_steps, n_vol_accepted, n_xchg_steps, n_xchg_accepted)) + f"{int(wall_time):12d}")


def format_boxlength_row(frame: int, box_length: float) -> str:
    """boxlength.dat row (store_boxlength, runmc.f90:356-371): the frame and BoxLength."""
    return f" {int(frame):11d} {float(box_length)!r}"


# ---------------------------------------------------------------- force dump (mc_calc_forces)
# store_forces (mc_calc_forces.f90:350-368) writes per atom fx/L, fy/L, fz/L with write_float
# (FloatingPoint.f90): a 24-bit mantissa (sign bit + 23 bits) and an 8-bit exponent (sign bit +
# 7 bits), little-endian, 4 bytes per number.
LN2 = 0.6931471805599453


def _myint(x: float) -> int:
    """myint (FloatingPoint.f90): truncation toward zero above 0, else toward -inf (with 1e-14)"""
    return int(x) if x > 0 else int(x - 1.0 + 1e-14)


def float_bits(a: float, mantisse_width: int = 24, exp_width: int = 8):
    """mantisse_exponent_real + mantisse_exponent_bits (FloatingPoint.f90): (mm, nn)."""
    if abs(a) < float(np.float32(1e-14)):
        m, n = math.copysign(1.0, a), -1000
    elif abs(a) > float(np.float32(1e14)):
        m, n = math.copysign(1.0, a), 1000
    else:
        n = _myint(math.log(abs(a)) / LN2)
        m = a / 2.0 ** n
    m_scale, n_scale = 2 ** (mantisse_width - 1), 2 ** (exp_width - 1)
    sgn_m = 0 if m > 0 else 1
    sgn_n = 0 if n > 0 else 1
    if abs(n) >= n_scale:
        return sgn_m * m_scale, sgn_n * n_scale + n_scale - 1
    return sgn_m * m_scale + int((abs(m) - 1.0) * (m_scale - 1)), sgn_n * n_scale + abs(n)


def float_value(mm: int, nn: int, mantisse_width: int = 24, exp_width: int = 8) -> float:
    """construct_float (FloatingPoint.f90)."""
    m_scale, n_scale = 2 ** (mantisse_width - 1), 2 ** (exp_width - 1)
    mm1, sign_m = (mm - m_scale, -1) if mm >= m_scale else (mm, 1)
    nn1, sign_n = (nn - n_scale, -1) if nn >= n_scale else (nn, 1)
    if nn1 == n_scale - 1:
        return 0.0 if sign_n == -1 else 1e14
    m = mm1 / (m_scale - 1.0) + 1.0
    return sign_m * m * 2.0 ** (sign_n * nn1)


def append_forces(path: str, fx, fy, fz, box_length: float) -> None:
    """store_forces: one frame of per-atom forces (kT per box length, as yamc_forces gives them)
    divided by BoxLength, x, y, z per atom, each as write_float's 3 + 1 little-endian bytes."""
    out = bytearray()
    for i in range(len(fx)):
        for v in (fx[i], fy[i], fz[i]):
            mm, nn = float_bits(float(v) / box_length)
            out += int(mm).to_bytes(3, "little") + int(nn).to_bytes(1, "little")
    with open(path, "ab") as f:
        f.write(bytes(out))


def read_forces(path: str, natom: int):
    """read_float over a force dump: frames x natom x 3."""
    raw = np.fromfile(path, dtype=np.uint8).reshape(-1, 4)
    mm = raw[:, 0].astype(np.int64) | (raw[:, 1].astype(np.int64) << 8) | (raw[:, 2].astype(np.int64) << 16)
    nn = raw[:, 3].astype(np.int64)
    vals = np.array([float_value(int(a), int(b)) for a, b in zip(mm, nn)])
    return vals.reshape(-1, natom, 3)
