"""Exchange steps and RDF frames of one workload, for profilers.

    python -m yamc_b200.profile_steps WORKLOAD [XCHG_STEPS] [RDF_FRAMES]

builds the named workload (systems.WORKLOADS) on cuda:0, evaluates XCHG_STEPS exchange steps of
random molecule pairs through yamc_xchange_eval / _commit (rejected, so the state stays; default
4) and adds RDF_FRAMES frames of the engine's configuration to a GPU RDF (default 2), timing
each on the host.  Capture one kernel at a time, e.g.
``ncu --clock-control none -k regex:k_rdf_count -s 1 -c 1`` (``--clock-control none`` leaves the
GPU's clocks as they are).
"""
from __future__ import annotations

import sys
import tempfile
import time

import numpy as np


def main(argv):
    from . import api, systems
    name = argv[0]
    nx = int(argv[1]) if len(argv) > 1 else 4
    nr = int(argv[2]) if len(argv) > 2 else 2
    with tempfile.TemporaryDirectory() as d:
        files = systems.write_system(systems.WORKLOADS[name], d, seed=3)
        eng = api.Engine.from_files(files)
    rng = np.random.default_rng(1)
    tx = []
    for _ in range(nx):
        i1, i2 = (int(v) for v in rng.choice(np.arange(1, eng.nmol + 1), 2, replace=False))
        t0 = time.perf_counter()
        eng.xchange_eval(i1, i2)
        eng.xchange_commit(False)
        tx.append(time.perf_counter() - t0)
    rdf = api.RDF.for_engine(eng)
    tr = []
    for _ in range(nr):
        t0 = time.perf_counter()
        rdf.add_engine(eng)
        tr.append(time.perf_counter() - t0)
    best = lambda t: f"{1e3 * min(t):.3f} ms (best of {len(t)})" if t else "not run"
    print(f"{name}: {eng.natom} atoms, {eng.nmol} molecules: exchange step {best(tx)}, RDF frame {best(tr)}")


if __name__ == "__main__":
    main(sys.argv[1:])
