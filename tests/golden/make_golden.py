"""Regenerates the golden fixtures of this directory.

* parameters_out.json -- the reference's own known answer: the derived
  parameters it printed to parameters.out for its shipped parameters.prm and
  the 110-molecule ions100.composition (parameters.f90:151-205).  Both files
  are read as text from the reference tree; the values are stored as the
  decimal strings the reference printed.
* gfortran_rng.json -- the first values of the reference's random stream
  (random.f90:25-93) for a few seeds, drawn by calling libgfortran, which pins
  the runtime that the tests and the benchmark use.

Run from the repository root:  python tests/golden/make_golden.py [reference_dir]
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))


def parse_prm(path):
    out = {}
    for line in open(path):
        t = line.replace("=", " ").split()
        if len(t) >= 2 and not t[0].startswith("#"):
            out[t[0]] = t[1]
    return out


def parse_out(path):
    out = {}
    for line in open(path):
        if "=" in line:
            k, v = line.split("=", 1)
            out[k.strip()] = v.strip()
    return out


def main(ref):
    prm = parse_prm(os.path.join(ref, "parameters.prm"))
    printed = parse_out(os.path.join(ref, "parameters.out"))
    comp = open(os.path.join(ref, "ions100.composition")).read().split()
    nmol = sum(int(comp[i]) for i in range(2, len(comp), 2))
    json.dump({"source": "reference parameters.prm + parameters.out, nmol from ions100.composition",
               "nmol": nmol, "prm": prm, "printed": printed},
              open(os.path.join(HERE, "parameters_out.json"), "w"), indent=1)
    from yamc_b200 import rng
    data = {"runtime": rng.runtime_description(), "streams": {}}
    for seed in (0, 1, 12345, 2024):
        data["streams"][str(seed)] = [float(v) for v in rng.gfortran_stream(seed, 16)]
    json.dump(data, open(os.path.join(HERE, "gfortran_rng.json"), "w"), indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
