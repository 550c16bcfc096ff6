"""Known-answer systems for the Ewald machinery (test helpers)."""
import math
import os

import numpy as np

from yamc_b200.formats import MolAtom, write_composition, write_mol, write_moltab, write_parameters

MADELUNG_NACL = 1.747564594633182  # rock salt, referred to the nearest-neighbour distance


def rocksalt(directory, n=6, d=2.82, alpha=0.473, kmax=11):
    """n^3 alternating Na+/Cl- on a simple cubic lattice of spacing d (A)."""
    os.makedirs(directory, exist_ok=True)
    L = n * d
    write_mol(os.path.join(directory, "Na.mol"), [MolAtom("Na", 0, 0, 0, 2.584, 0.1, 1.0, 1.0, 2.0)])
    write_mol(os.path.join(directory, "Cl.mol"), [MolAtom("Cl", 0, 0, 0, 4.401, 0.1, -1.0, 1.0, 2.0)])
    idx = np.array([(i, j, k) for i in range(n) for j in range(n) for k in range(n)])
    even = idx.sum(1) % 2 == 0
    sites = np.concatenate([idx[even], idx[~even]]).astype(float)
    pos = -0.5 + (sites + 0.25) / n
    write_composition(os.path.join(directory, "system.composition"), [("Na.mol", int(even.sum())), ("Cl.mol", int((~even).sum()))])
    z = np.zeros(len(pos))
    write_moltab(os.path.join(directory, "system.moltab"), pos[:, 0], pos[:, 1], pos[:, 2], z, z, z, 3, 3)
    aL = alpha * L
    write_parameters(os.path.join(directory, "parameters.prm"), {
        "sr": aL / 2.0, "sk": kmax * math.pi / aL, "alphaL": aL, "temp": 298.15, "external_permutivity": 70.0,
        "BoxLength": L, "density": 0.0, "dr_a": 0.1, "d_angle_degree": 5.0, "xlambda_c": 0.0, "xlambda_f": 0.0,
        "pressure_step_multiplier": 0.0, "n_store_energy_interval": 1e9, "input_nbytes_xyz": 3, "input_nbytes_ang": 3})
    return {"parameters": os.path.join(directory, "parameters.prm"),
            "composition": os.path.join(directory, "system.composition"),
            "moltab": os.path.join(directory, "system.moltab"), "N": len(pos), "d": d}


def lj_lattice(directory, n=5, a=3.5, sigma=3.166, eps_kcal=0.1554, alpha=0.5, kmax=12):
    """n^3 uncharged LJ sites on a simple cubic lattice of spacing a (A)."""
    os.makedirs(directory, exist_ok=True)
    L = n * a
    write_mol(os.path.join(directory, "Ar.mol"), [MolAtom("Ar", 0, 0, 0, sigma, eps_kcal, 0.0, 1.0, 2.0)])
    idx = np.array([(i, j, k) for i in range(n) for j in range(n) for k in range(n)], dtype=float)
    pos = -0.5 + (idx + 0.3) / n
    write_composition(os.path.join(directory, "system.composition"), [("Ar.mol", len(pos))])
    z = np.zeros(len(pos))
    write_moltab(os.path.join(directory, "system.moltab"), pos[:, 0], pos[:, 1], pos[:, 2], z, z, z, 3, 3)
    aL = alpha * L
    write_parameters(os.path.join(directory, "parameters.prm"), {
        "sr": aL / 2.0, "sk": kmax * math.pi / aL, "alphaL": aL, "temp": 298.15, "external_permutivity": 70.0,
        "BoxLength": L, "density": 0.0, "dr_a": 0.1, "d_angle_degree": 5.0, "xlambda_c": 0.0, "xlambda_f": 0.0,
        "pressure_step_multiplier": 0.0, "n_store_energy_interval": 1e9, "input_nbytes_xyz": 3, "input_nbytes_ang": 3})
    return {"parameters": os.path.join(directory, "parameters.prm"),
            "composition": os.path.join(directory, "system.composition"),
            "moltab": os.path.join(directory, "system.moltab"), "N": len(pos), "a": a, "sigma": sigma,
            "eps_kcal": eps_kcal}


def lj_lattice_energy_kT(N, a, sigma, eps_kT, R=40.0):
    """Direct lattice sum of 4 eps [(s/r)^12 - (s/r)^6] for a simple cubic crystal (per system),
    lattice vectors up to R lattice constants plus the analytic r^-6 tail beyond."""
    m = int(R) + 1
    g = np.arange(-m, m + 1, dtype=float)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    r2 = (X * X + Y * Y + Z * Z).ravel()
    r2 = r2[(r2 > 0) & (r2 <= R * R)] * a * a
    sr6 = (sigma * sigma / r2) ** 3
    per = 0.5 * np.sum(4 * eps_kT * (sr6 * sr6 - sr6))
    rho = 1.0 / a ** 3
    Rc = R * a
    per += 0.5 * rho * 4 * math.pi * 4 * eps_kT * (sigma ** 12 / (9 * Rc ** 9) - sigma ** 6 / (3 * Rc ** 3))
    return N * per
