"""The CPU oracle against the reference's own known answers and invariants.

The oracle is the checker of the GPU engine, so it is pinned first:
parameters.out (the reference's printed derivation), the k-grid counts, the
special functions against independent implementations, the reference's debug
invariants (incremental vs full recompute, MC.f90:1886-1951; rigid geometry,
MC.f90:1957-2049) and physics known answers (NaCl Madelung energy, a direct
Lennard-Jones lattice sum)."""
import ctypes
import json
import math
import os

import numpy as np
import pytest

import pyoracle
from yamc_b200 import rng as grng
from yamc_b200 import systems

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _prm_file(tmp_path, prm):
    p = tmp_path / "parameters.prm"
    p.write_text("".join(f"{k} = {v}\n" for k, v in prm.items()))
    return str(p)


def test_parameters_out_golden(tmp_path):
    g = json.load(open(os.path.join(GOLDEN, "parameters_out.json")))
    p = pyoracle.read_params(_prm_file(tmp_path, g["prm"]))
    assert pyoracle.lib().orc_params_init(ctypes.byref(p), g["nmol"]) == 0
    printed = g["printed"]
    assert p.kmax == int(printed["kmax"])
    for name in ("BoxLength", "rmax", "kT_kcal_mol", "rmax2", "dbjr_a", "dbjr", "xclb", "alpha_over_sqrt_pi",
                 "two_alpha_over_sqrt_pi", "kext", "minus_two_kext", "dr", "d_angle", "log_max_volume_scaling",
                 "pressure_angstr_kT"):
        ref = float(printed[name].replace("D", "E"))
        assert getattr(p, name) == ref, (name, getattr(p, name), ref)
    assert p.alphaL == float(printed["alphaL"])


@pytest.mark.parametrize("kmax,count", [(7, 238), (10, 647), (12, 1068), (15, 2045), (24, 7912)])
def test_fourier_grid_counts(kmax, count):
    assert pyoracle.grid_count(kmax) == count


def test_erfc_luc_accuracy():
    xs = np.linspace(0.0, 6.0, 3001)
    err = max(abs(pyoracle.erfc_luc(x) - math.erfc(x)) for x in xs)
    assert err < 1.5e-7  # Abramowitz & Stegun 7.1.26 bound, the series pieces are tighter
    for x in (0.1, 0.455, 1.0, 2.9, 3.0, 3.5):
        assert abs(pyoracle.erf_luc(x) + pyoracle.erfc_luc(x) - 1.0) < 1e-15


def test_bet6_bet12_against_quadrature():
    from scipy.integrate import quad
    pi15 = math.pi ** 1.5
    for b in (0.3, 0.5, 0.7, 1.3, 2.5, 5.0, 7.9, 8.0, 9.0):
        erfk, b6, b12 = pyoracle.bet6_bet12(b)
        # beta6 = pi^1.5 b^3/2 int_b^inf e^{-t^2}/t^4 dt, beta12 = pi^1.5 b^9/120 int_b^inf e^{-t^2}/t^10 dt
        i6 = quad(lambda t: math.exp(-t * t) / t ** 4, b, math.inf, epsabs=0, epsrel=1e-13)[0]
        i12 = quad(lambda t: math.exp(-t * t) / t ** 10, b, math.inf, epsabs=0, epsrel=1e-13)[0]
        # the reference ends its integration with a three-term asymptotic series at b = 8,
        # good to ~1e-5 (beta6) and ~1e-4 (beta12) there; elsewhere the forms are accurate
        tol = 1e-6 if b < 7.5 else 5e-4
        assert abs(b6 - pi15 * b ** 3 / 2 * i6) <= tol * abs(b6)
        assert abs(b12 - pi15 * b ** 9 / 120 * i12) <= tol * abs(b12)
        assert abs(erfk - math.erfc(b)) < 2e-7


def test_shi_sans_exp():
    from scipy.special import shichi
    for x in (0.05, 0.5, 1.0, 2.0, 4.9, 7.0, 12.0, 17.0, 19.9, 25.0):
        ref = shichi(x)[0] * math.exp(-x)
        assert abs(pyoracle.shi_sans_exp(x) - ref) < 2e-5 * abs(ref)


def test_gfortran_stream_golden():
    g = json.load(open(os.path.join(GOLDEN, "gfortran_rng.json")))
    for seed, vals in g["streams"].items():
        got = grng.gfortran_stream(int(seed), len(vals))
        assert np.array_equal(got, np.array(vals, dtype=np.float32)), seed
    # the stream is a pure function of the seed, and values are REAL(4) multiples of 2**-24
    a = grng.gfortran_stream(99, 1000)
    assert np.array_equal(a, grng.gfortran_stream(99, 1000))
    assert np.all(a * 2.0 ** 24 == np.floor(a * 2.0 ** 24))


def test_incremental_equals_full_recompute(tiny_files):
    """The reference's own debug check (MC.f90:1886-1951): after moves, the
    incrementally updated energies, uu, F and rho match a full recompute."""
    o = pyoracle.Oracle(tiny_files)
    buf = grng.gfortran_stream(7, 200000)
    log, _, _ = o.run_mc(buf, 3000)
    assert (log["flags"] & 1).sum() > 300
    e_inc = o.energies()
    uu, fx, fy, fz = o.uuF()
    rho = o.rho()
    e_full = o.full_sums()
    uu2, fx2, fy2, fz2 = o.uuF()
    assert np.all(np.abs(e_inc - e_full) <= 1e-9 * np.maximum(1.0, np.abs(e_full)))
    assert np.abs(uu - uu2).max() < 1e-9
    assert max(np.abs(fx - fx2).max(), np.abs(fy - fy2).max(), np.abs(fz - fz2).max()) < 1e-8
    assert np.abs(rho - o.rho()).max() < 1e-9


def test_rigid_geometry_kept(tiny_files):
    """check_distances (MC.f90:1957-2049): intra-molecular distances stay those of the .mol file."""
    o = pyoracle.Oracle(tiny_files)
    L = o.params.BoxLength
    x0, y0, z0, *_ = o.atoms()
    o.run_mc(grng.gfortran_stream(3, 200000), 2000)
    x, y, z, q, t, m = o.atoms()
    f, l = o.mols()
    for i in range(o.nmol):
        a, b = f[i] - 1, l[i]
        if b - a < 2:
            continue
        for u in range(a, b):
            for v in range(u + 1, b):
                d0 = ((x0[u] - x0[v]) ** 2 + (y0[u] - y0[v]) ** 2 + (z0[u] - z0[v]) ** 2) * L * L
                d1 = ((x[u] - x[v]) ** 2 + (y[u] - y[v]) ** 2 + (z[u] - z[v]) ** 2) * L * L
                assert abs(d1 - d0) < 1e-6


def test_madelung_rocksalt(tmp_path):
    """Ewald Coulomb energy of a rock-salt crystal = -(N/2) M e^2/(4 pi eps0 d)."""
    from physics import MADELUNG_NACL, rocksalt
    sysd = rocksalt(str(tmp_path / "nacl"))
    o = pyoracle.Oracle(sysd)
    e = o.energies()
    uext = o.params.kext * float(np.sum(o.mu() ** 2))
    e_coul = e[1] - uext  # U_total_ew without the external (surface) term: tin-foil Ewald energy
    ref = -(sysd["N"] / 2) * MADELUNG_NACL * o.params.dbjr_a / sysd["d"]
    assert abs(e_coul - ref) < 2e-6 * abs(ref)


def test_lj_dispersion_ewald_lattice(tmp_path):
    """Dispersion-Ewald LJ energy (real + k-space + tails) of a simple cubic crystal
    equals the direct lattice sum."""
    from physics import lj_lattice, lj_lattice_energy_kT
    sysd = lj_lattice(str(tmp_path / "lj"))
    o = pyoracle.Oracle(sysd)
    e = o.energies()
    eps_kT = sysd["eps_kcal"] / o.params.kT_kcal_mol
    ref = lj_lattice_energy_kT(sysd["N"], sysd["a"], sysd["sigma"], eps_kT)
    assert abs(e[2] - ref) < 1e-6 * abs(ref)
    assert abs(e[1]) < 1e-12  # no charges


def test_run_mc_cycle_structure(tiny_files):
    """run_mc (runmc.f90:178-334): one pressure draw per cycle, then for every move the
    exchange draw, the molecule choice and movemc's own draws; energy rows per cycle."""
    spec_files = dict(tiny_files)
    o = pyoracle.Oracle(spec_files)
    buf = grng.gfortran_stream(11, 100000)
    log, rows, cur = o.run_mc(buf, 3 * o.nmol)
    assert log["cursor"][-1] == cur
    assert np.all(np.diff(log["cursor"]) > 0)
    assert np.all((log["imol"] >= 1) & (log["imol"] <= o.nmol))
