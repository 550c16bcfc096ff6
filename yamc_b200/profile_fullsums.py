"""Full recomputations and NPT volume steps of one workload, for profilers.

    python -m yamc_b200.profile_fullsums WORKLOAD [REPEATS] [VOLUME_STEPS] [FORCES]

builds the named workload (systems.WORKLOADS) on cuda:0, runs yamc_full_sums once as a
warm-up and then REPEATS more times (default 3), timing each call on the host (the call
synchronises), then VOLUME_STEPS volume steps through yamc_volume_eval/_commit (default 0)
and FORCES calls of the adjoint yamc_forces (default 0).
Capture one kernel of the second call at a time, e.g.
``ncu --clock-control none -k regex:k_realspace_full -s 1 -c 1`` (``--clock-control none`` leaves
the GPU's clocks as they are).
"""
from __future__ import annotations

import sys
import tempfile
import time


def main(argv):
    from . import api, systems
    name = argv[0]
    reps = int(argv[1]) if len(argv) > 1 else 3
    nvol = int(argv[2]) if len(argv) > 2 else 0
    nfor = int(argv[3]) if len(argv) > 3 else 0
    with tempfile.TemporaryDirectory() as d:
        files = systems.write_system(systems.WORKLOADS[name], d, seed=3)
        eng = api.Engine.from_files(files)
    eng.full_sums()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        eng.full_sums()
        ts.append(time.perf_counter() - t0)
    print(f"{name}: {eng.natom} atoms, {eng.nsigned} signed k: full sums {1e3 * min(ts):.3f} ms (best of {reps})")
    L = eng.current_params().BoxLength
    tv = []
    for k in range(nvol):
        t0 = time.perf_counter()
        du, ov = eng.volume_eval(L * (1.0 + 0.001 * (1 if k % 2 else -1)))
        eng.volume_commit(False)
        tv.append(time.perf_counter() - t0)
    if tv:
        print(f"volume step (eval + rejecting commit): {1e3 * min(tv):.3f} ms (best of {nvol})")
    tf = []
    for _ in range(nfor):
        t0 = time.perf_counter()
        eng.forces()
        tf.append(time.perf_counter() - t0)
    if tf:
        print(f"adjoint forces (yamc_forces, with the host's molecular sums): {1e3 * min(tf):.3f} ms (best of {nfor})")


if __name__ == "__main__":
    main(sys.argv[1:])
