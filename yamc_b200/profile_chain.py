"""One chain launch of a chosen shape, for profilers.

    python -m yamc_b200.profile_chain WORKLOAD G THREADS PRECISION LAYOUT [MOVES]

builds the named workload (systems.WORKLOADS) on cuda:0 with PRECISION (0 FP64, 1 mixed),
k-space LAYOUT (1 registers, 2 streamed) and a cluster of G CTAs of THREADS threads, runs a
300-move warm-up launch and then one launch of MOVES moves (default 1000), and prints its
CUDA-event time.  Capture the second launch with
``ncu --clock-control none -k regex:k_chain -s 1 -c 1`` (``--clock-control none`` leaves the
GPU's clocks as they are), on a workload that fits a short capture.
"""
from __future__ import annotations

import sys
import tempfile

import numpy as np


def main(argv):
    import torch
    from . import api, rng as grng, systems
    name, G, B, prec, layout = argv[0], int(argv[1]), int(argv[2]), int(argv[3]), int(argv[4])
    moves = int(argv[5]) if len(argv) > 5 else 1000
    with tempfile.TemporaryDirectory() as d:
        files = systems.write_system(systems.WORKLOADS[name], d, seed=3)
        eng = api.Engine.from_files(files, precision=prec)
    eng.set_kspace_layout(layout)
    eng.set_launch(G, B)
    s = torch.from_numpy(grng.gfortran_stream(5, 40 * (moves + 300) + 100000)).cuda()
    cur, done, st = eng.run_chain_device(s.data_ptr(), s.numel(), 300)
    cur, done, st = eng.run_chain_device(s.data_ptr(), s.numel(), moves, cursor=cur)
    if st != 0 or done != moves:
        raise SystemExit(f"chain stopped: status {st}, {done} moves")
    print(f"{moves} moves in {eng.last_kernel_ms:.3f} ms, launch {eng.launch}")


if __name__ == "__main__":
    main(sys.argv[1:])
