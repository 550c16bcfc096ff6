"""Seeded synthetic systems in YAMC's own input formats.

The workloads are SPC/E water with Na+/Cl- (Dang parameters, Lorentz-Berthelot
mixing) in cubic boxes.  Ewald settings are expressed in the reference's own
parameters: ``alphaL = alpha * L``, ``sr = alpha * rc`` (so ``rmax = sr /
alphaL = rc / L``, parameters.f90:387) and ``sk = kmax * pi / alphaL`` so that
``kmax = nint(sk * alphaL / pi)`` (parameters.f90:388) lands on the requested
integer.  Translation amplitude ``dr_a`` and rotation ``d_angle_degree`` feed
the reference's proposal (a ball of radius dr_a, MonteCarloMove.f90:239-250,
and a uniform angle about a random axis, :399-416).

Named workloads (sizes only; data are generated from a seed):

=========  ==============================  =======  ======  ===== ====== ==== ======
name       molecules                        atoms    L (A)   a*L   sr     kmax lambda
=========  ==============================  =======  ======  ===== ====== ==== ======
spce256    256 SPC/E                        768      19.73   6.9055 3.15  7    0
nacl1m     2048 SPC/E + 38 Na + 38 Cl       6220     39.6    11.88  3.6   12   0
nacl4k     4096 SPC/E + 76 Na + 76 Cl       12440    50.0    14.0   3.36  15   0.1
nacl16k    16384 SPC/E + 300 Na + 300 Cl    49752    79.3    17.446 2.64  24   0.1
=========  ==============================  =======  ======  ===== ====== ==== ======

The batched workload draws 96 replicas (water count log-uniform in 216..4096,
NaCl 0..2 M, density 0.0334 +- 2 %/A^3, T uniform in 280..360 K, alpha*L = 5.6,
cutoff min(12 A, L/2), one common integer k-set) -- see :func:`batch_specs`.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from .formats import MolAtom, write_composition, write_mol, write_moltab, write_parameters

PI = 3.14159265358979323846
KJ_PER_KCAL = 4.184


def spce_atoms() -> List[MolAtom]:
    """SPC/E: O-H 1.0 A, H-O-H 109.47 deg, q_O -0.8476, sigma 3.166 A, eps 0.650 kJ/mol.
    H carries no mass (the centre of mass is the O site, as in the reference's SPCE.mol)."""
    th = math.radians(109.47)
    eps = 0.650 / KJ_PER_KCAL
    return [
        MolAtom("O", 0.0, 0.0, 0.0, 3.166, eps, -0.8476, 16.0, 2.0),
        MolAtom("H", 1.0, 0.0, 0.0, 0.0, 0.0, 0.4238, 0.0, 0.0),
        MolAtom("H", math.cos(th), math.sin(th), 0.0, 0.0, 0.0, 0.4238, 0.0, 0.0),
    ]


def na_atoms() -> List[MolAtom]:
    return [MolAtom("Na", 0.0, 0.0, 0.0, 2.584, 0.4184 / KJ_PER_KCAL, 1.0, 1.0, 2.0)]


def cl_atoms() -> List[MolAtom]:
    return [MolAtom("Cl", 0.0, 0.0, 0.0, 4.401, 0.4184 / KJ_PER_KCAL, -1.0, 1.0, 2.0)]


@dataclass
class SystemSpec:
    name: str
    n_water: int
    n_na: int
    n_cl: int
    box: float            # Angstrom
    alpha: float          # 1/Angstrom
    rc: float             # Angstrom
    kmax: int
    temp: float = 298.15
    dr_a: float = 0.15
    d_angle_rad: float = 0.15
    xlambda: float = 0.0
    lattice: str = "jitter"   # "first_sites" (7x7x7 first sites) or "jitter"
    lattice_n: int = 0        # sites per edge for "first_sites"
    external_permutivity: float = 70.0
    n_store_energy_interval: float = 1.0e9
    max_cycle: int = 1000000

    @property
    def nmol(self) -> int:
        return self.n_water + self.n_na + self.n_cl

    @property
    def natom(self) -> int:
        return 3 * self.n_water + self.n_na + self.n_cl

    @property
    def alphaL(self) -> float:
        return self.alpha * self.box

    def params(self, seed: int = 0) -> Dict[str, object]:
        aL = self.alphaL
        return {
            "sr": self.alpha * self.rc,
            "sk": self.kmax * PI / aL,
            "alphaL": aL,
            "temp": float(self.temp),
            "external_permutivity": float(self.external_permutivity),
            "BoxLength": float(self.box),
            "density": 0.0,
            "dr_a": float(self.dr_a),
            "d_angle_degree": math.degrees(self.d_angle_rad),
            "xlambda_c": float(self.xlambda),
            "xlambda_f": float(self.xlambda),
            "pressure": 100000.0,
            "pressure_step_multiplier": 0.0,
            "max_volume_scaling": 1.05,
            "max_cycle": int(self.max_cycle),
            "n_store_traj_interval": 1.0e9,
            "n_store_energy_interval": float(self.n_store_energy_interval),
            "input_nbytes_xyz": 3,
            "input_nbytes_ang": 3,
            "output_nbytes_xyz": 3,
            "output_nbytes_ang": 3,
            "random_seed": int(seed),
        }


WORKLOADS: Dict[str, SystemSpec] = {
    "spce256": SystemSpec("spce256", 256, 0, 0, 19.73, 0.35, 9.0, 7, lattice="first_sites", lattice_n=7),
    "nacl1m": SystemSpec("nacl1m", 2048, 38, 38, 39.6, 0.30, 12.0, 12),
    "nacl4k": SystemSpec("nacl4k", 4096, 76, 76, 50.0, 0.28, 12.0, 15, xlambda=0.1),
    "nacl16k": SystemSpec("nacl16k", 16384, 300, 300, 79.3, 0.22, 12.0, 24, xlambda=0.1),
}


def small_spec(name: str = "tiny", n_water: int = 24, n_na: int = 2, n_cl: int = 2, box: float = 10.0,
               alpha: float = 0.5, rc: float = 4.9, kmax: int = 4, xlambda: float = 0.0,
               dr_a: float = 0.15, d_angle_rad: float = 0.15) -> SystemSpec:
    """A small system the oracle handles in milliseconds (parity tests)."""
    return SystemSpec(name, n_water, n_na, n_cl, box, alpha, rc, kmax, xlambda=xlambda, dr_a=dr_a,
                      d_angle_rad=d_angle_rad)


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices from uniform unit quaternions."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z); R[:, 0, 1] = 2 * (x * y - z * w); R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w); R[:, 1, 1] = 1 - 2 * (x * x + z * z); R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w); R[:, 2, 1] = 2 * (y * z + x * w); R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _zyz_angles(R: np.ndarray):
    """(theta, phi, psi) with R = Rz(phi) Ry(theta) Rz(psi), the moltab convention
    (MoleculeTable.f90:656-673), mapped into [0, 2pi)."""
    theta = np.arccos(np.clip(R[:, 2, 2], -1.0, 1.0))
    phi = np.arctan2(R[:, 1, 2], R[:, 0, 2])
    psi = np.arctan2(R[:, 2, 1], -R[:, 2, 0])
    return theta % (2 * PI), phi % (2 * PI), psi % (2 * PI)


def generate(spec: SystemSpec, seed: int = 1):
    """Molecule centres (box units) and ZYZ angles, in composition order
    (waters, then Na, then Cl)."""
    rng = np.random.default_rng(seed)
    nmol = spec.nmol
    if spec.lattice == "first_sites":
        n = spec.lattice_n
        idx = np.arange(n ** 3)[:nmol]
        ix, iy, iz = idx // (n * n), (idx // n) % n, idx % n
        pos = np.stack([ix, iy, iz], axis=1).astype(np.float64)
        pos = -0.5 + (pos + 0.5) / n
    else:
        n = int(math.ceil(nmol ** (1.0 / 3.0) - 1e-9))
        while n ** 3 < nmol:
            n += 1
        sites = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
        sites = sites[rng.permutation(len(sites))[:nmol]]
        spacing = 1.0 / n
        jitter = rng.uniform(-0.12, 0.12, size=(nmol, 3)) * spacing
        pos = -0.5 + (sites + 0.5) * spacing + jitter
        # species assignment by seeded shuffle: the site list is already shuffled
    pos = (pos + 0.5) % 1.0 - 0.5
    theta, phi, psi = _zyz_angles(_random_rotations(rng, nmol))
    return pos[:, 0], pos[:, 1], pos[:, 2], theta, phi, psi


def write_system(spec: SystemSpec, directory: str, seed: int = 1, rng_seed: int = 12345) -> Dict[str, str]:
    """Write parameters.prm, the .mol files, system.composition and system.moltab."""
    os.makedirs(directory, exist_ok=True)
    entries = []
    if spec.n_water:
        write_mol(os.path.join(directory, "SPCE.mol"), spce_atoms())
        entries.append(("SPCE.mol", spec.n_water))
    if spec.n_na:
        write_mol(os.path.join(directory, "Na_Dang.mol"), na_atoms())
        entries.append(("Na_Dang.mol", spec.n_na))
    if spec.n_cl:
        write_mol(os.path.join(directory, "Cl_Dang.mol"), cl_atoms())
        entries.append(("Cl_Dang.mol", spec.n_cl))
    comp = os.path.join(directory, "system.composition")
    write_composition(comp, entries)
    x, y, z, th, ph, ps = generate(spec, seed)
    moltab = os.path.join(directory, "system.moltab")
    write_moltab(moltab, x, y, z, th, ph, ps, 3, 3)
    prm = os.path.join(directory, "parameters.prm")
    write_parameters(prm, spec.params(rng_seed))
    return {"parameters": prm, "composition": comp, "moltab": moltab, "dir": directory}


def batch_specs(n_replicas: int = 96, seed: int = 7, sk_common: float = 3.2) -> List[SystemSpec]:
    """Ragged replicas: water log-uniform 216..4096, NaCl 0..2 M, density 0.0334 +- 2 %
    molecules/A^3, T uniform in 280..360 K, alpha*L = 5.6, cutoff min(12 A, L/2), and one
    k-set for all replicas fixed by sk_common (kmax = nint(sk*5.6/pi))."""
    rng = np.random.default_rng(seed)
    aL = 5.6
    kmax = int(math.floor(sk_common * aL / PI + 0.5))
    out = []
    for r in range(n_replicas):
        nw = int(round(math.exp(rng.uniform(math.log(216), math.log(4096)))))
        molar = rng.uniform(0.0, 2.0)
        dens = 0.0334 * (1.0 + rng.uniform(-0.02, 0.02))
        # ions per water: c[mol/L] / 55.5 mol/L of water
        nion = int(round(nw * molar / 55.5))
        nmol = nw + 2 * nion
        box = (nmol / dens) ** (1.0 / 3.0)
        rc = min(12.0, box / 2.0)
        alpha = aL / box
        temp = float(rng.uniform(280.0, 360.0))
        out.append(SystemSpec(f"rep{r:03d}", nw, nion, nion, box, alpha, rc, kmax, temp=temp, xlambda=0.1))
    return out
