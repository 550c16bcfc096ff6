"""The reference's tutorial run as a statistical pin (helpers of test_tutorial_pin.py).

The reference ships one NPT run of its tutorial: its inputs (parameters.prm, ions100.composition
and the three .mol files) and its outputs (energy.dat every 100 cycles, boxlength.dat at every
accepted volume step, and mcrdf2's RDFs over the run's 100 trajectory frames).  Its initial
configuration and random seed are not shipped, so a run here cannot repeat it move for move;
instead the same inputs are run from seeded lattice starts of the same density and the
reference's numbers are required to lie within the spread of those runs:

    z = |ref - mean(ours)| / (sd(ours) * sqrt(1 + 1/n))

where sd is the run-to-run standard deviation of n independent runs here, which is also the
uncertainty of the reference's single run (the same process, another seed).  Quantities: the
means of U_total, U_total_ew, U_total_lj, uu_ew and E_k_coulomb over the energy.dat rows of a
cycle window, the time average of the box length over the same cycles (boxlength.dat is a
step function of the cycle), and the height and position of the first g(r) peak.

The fixture (golden/tutorial_npt.json) is made by golden/make_tutorial_golden.py from the
reference's files; nothing here reads the reference tree.
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "tutorial_npt.json")))
NMOL = 110
N_WATER, N_NA, N_CL = 100, 5, 5
# energy.dat columns compared (index into a 9-column row) and the names they carry
QUANTITIES = {"U_total": 1, "U_total_ew": 2, "U_total_lj": 3, "uu_ew": 4, "E_k_coulomb": 7}
# RDFs compared: (name in the fixture, species index pair in composition order)
RDF_PAIRS = {"water_water": (0, 0), "water_Na": (0, 1), "water_Cl": (0, 2), "Na_Cl": (1, 2)}


def prm_value(name: str) -> float:
    for line in GOLD["inputs"]["parameters.prm"].splitlines():
        t = line.split("#")[0].replace("=", " ").split()
        if len(t) >= 2 and t[0] == name:
            return float(t[1])
    raise KeyError(name)


def initial_box_length() -> float:
    """Parameters_init with BoxLength = 0: the box from the density in molecules per nm^3
    (parameters.f90:323-352), in Angstrom."""
    return 10.0 * (NMOL / prm_value("density")) ** (1.0 / 3.0)


def write_inputs(directory: str, seed: int) -> dict:
    """The reference's tutorial inputs, verbatim, and a seeded lattice start of our own.

    The reference's genMoleculeTable puts the molecules on a grid with random orientations
    (MoleculeTable_placeMoleculesToGrid); here a jittered simple-cubic lattice with a seeded
    species shuffle and uniform random orientations (systems.generate), written as a moltab
    with the byte widths parameters.prm names."""
    from yamc_b200 import formats, systems
    os.makedirs(directory, exist_ok=True)
    for name, text in GOLD["inputs"].items():
        with open(os.path.join(directory, name), "w") as f:
            f.write(text)
    L = initial_box_length()
    spec = systems.SystemSpec("tutorial", N_WATER, N_NA, N_CL, L, 8.0 / L, L / 2.0, 10)
    x, y, z, th, ph, ps = systems.generate(spec, seed=seed)
    nb_xyz, nb_ang = int(prm_value("input_nbytes_xyz")), int(prm_value("input_nbytes_ang"))
    moltab = os.path.join(directory, "system.moltab")
    formats.write_moltab(moltab, x, y, z, th, ph, ps, nb_xyz, nb_ang)
    return {"parameters": os.path.join(directory, "parameters.prm"),
            "composition": os.path.join(directory, "ions100.composition"), "moltab": moltab, "dir": directory}


def box_per_cycle(cycles, boxes, n_cycles: int, L0: float) -> np.ndarray:
    """The box length during each cycle 1..n_cycles (index 0 unused) from the accepted volume
    steps: a step accepted in cycle c sets the box from cycle c on."""
    out = np.empty(n_cycles + 1)
    cur, j = L0, 0
    order = np.argsort(np.asarray(cycles), kind="stable")
    cycles = np.asarray(cycles)[order]
    boxes = np.asarray(boxes)[order]
    for c in range(1, n_cycles + 1):
        while j < len(cycles) and cycles[j] <= c:
            cur = boxes[j]
            j += 1
        out[c] = cur
    return out


def window_means(rows: np.ndarray, box: np.ndarray, lo: int, hi: int) -> dict:
    """Means over cycles (lo, hi]: the energy rows whose frame falls there, and the box."""
    rows = np.asarray(rows)
    sel = (rows[:, 0] > lo) & (rows[:, 0] <= hi)
    out = {k: float(rows[sel, c].mean()) for k, c in QUANTITIES.items()}
    out["BoxLength"] = float(np.mean(box[lo + 1: hi + 1]))
    return out


def reference_window_means(lo: int, hi: int) -> dict:
    rows = np.asarray(GOLD["energy"])
    b = np.asarray(GOLD["boxlength"])
    box = box_per_cycle(b[:, 0].astype(int), b[:, 1], GOLD["n_cycles"], initial_box_length())
    return window_means(rows, box, lo, hi)


def rdf_peak(g: np.ndarray, rmin_bin: int = 15):
    """(bin, height) of the first maximum: the largest value beyond rmin_bin bins (1.5 A, inside
    every hard core, where g is 0)."""
    i = int(np.argmax(g[rmin_bin:])) + rmin_bin
    return i, float(g[i])


def z_score(ref: float, ours) -> float:
    ours = np.asarray(ours, dtype=np.float64)
    n = ours.size
    sd = float(ours.std(ddof=1))
    return abs(ref - float(ours.mean())) / (sd * np.sqrt(1.0 + 1.0 / n))


def oracle_run(seed: int, n_cycles: int):
    """One oracle NPT run of the tutorial inputs (in a worker process): energy rows, accepted
    volume steps (cycle, box) and the initial box length."""
    import sys
    import tempfile
    root = os.path.dirname(HERE)
    for p in (root, os.path.join(root, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import pyoracle
    from yamc_b200 import rng
    with tempfile.TemporaryDirectory() as d:
        files = write_inputs(d, seed)
        o = pyoracle.Oracle(files, extra=f"random_seed={seed}", fast=True)
        L0 = o.box_length
        buf = rng.gfortran_stream(seed, n_cycles * NMOL * 20)
        _, vlog, rows, _, done = o.run_cycles(buf, n_cycles, max_rows=n_cycles // 100 + 2)
        o.close()
    assert done == n_cycles
    acc = vlog[(vlog["flags"] & 1) == 1]
    return rows, np.asarray(acc["cycle"]), np.asarray(acc["box_new"]), L0
