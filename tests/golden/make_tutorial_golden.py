"""Regenerates tutorial_npt.json: the reference's own NPT tutorial run, as shipped.

The reference ships the inputs and outputs of one run of its tutorial (Tutorial.txt): 100
SPC/E waters + 5 Na + 5 Cl (ions100.composition with SPCE.mol, Na_Dang.mol, Cl_Dang.mol), NPT
at 300 K and 1 bar with a volume cycle on average every pressure_step_multiplier + 1 = 6 cycles
(parameters.prm), 10,000 cycles from a lattice start at 30 molecules/nm^3.  Its outputs are:

* energy.dat -- the 9 columns of store_energy (runmc.f90:336-351) every 100 cycles;
* boxlength.dat -- the box length after every accepted volume step (store_boxlength,
  runmc.f90:353-368);
* RDF_<a>_<b>.dat -- mcrdf2's molecule-centre g(r) (bins of 0.1 A up to 12 A, the tutorial's
  ``mcrdf2 parameters.prm ions100.composition RDF_ 0.1 12 water,Na,Cl``) over the 100
  trajectory frames of the run (one every 100 cycles).

The initial configuration and the random seed of that run are not shipped, so these outputs
pin the reference statistically: the tests run the same inputs from a lattice start of their
own and compare ensemble averages and RDF peaks.  This script copies the input files as text
and the output numbers as they were printed into one JSON fixture, so the tests need nothing
from the reference tree at run time.

Run from the repository root:  python tests/golden/make_tutorial_golden.py [reference_dir]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
INPUTS = ("parameters.prm", "ions100.composition", "SPCE.mol", "Na_Dang.mol", "Cl_Dang.mol")
RDFS = ("water_water", "water_Na", "water_Cl", "Na_Na", "Na_Cl", "Cl_Cl")


def main(ref):
    texts = {f: open(os.path.join(ref, f)).read() for f in INPUTS}
    energy = np.loadtxt(os.path.join(ref, "energy.dat"))
    box = np.loadtxt(os.path.join(ref, "boxlength.dat"))
    rdf = {}
    r_col = None
    for name in RDFS:
        a = np.loadtxt(os.path.join(ref, f"RDF_{name}.dat"))
        r_col = a[:, 0] if r_col is None else r_col
        assert np.allclose(a[:, 0], r_col)
        rdf[name] = [float(v) for v in a[:, 1]]
    dr = float(r_col[1] - r_col[0])
    out = {
        "source": "the reference's shipped tutorial run: inputs " + ", ".join(INPUTS) +
                  "; outputs energy.dat, boxlength.dat, RDF_*.dat",
        "inputs": texts,
        "n_cycles": 10000,
        "energy_columns": ["frame", "U_total", "U_total_ew", "U_total_lj", "uu_ew", "uu_lj6", "uu_lj12",
                           "E_k_coulomb", "E_k_lj"],
        "energy": [[float(v) for v in row] for row in energy],
        "boxlength": [[int(row[0]), float(row[1])] for row in box],
        "rdf_dr": dr,
        "rdf_rmax": 12.0,
        "rdf_species": ["water", "Na", "Cl"],
        "rdf_r": [float(v) for v in r_col],
        "rdf": rdf,
    }
    json.dump(out, open(os.path.join(HERE, "tutorial_npt.json"), "w"), indent=0)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
