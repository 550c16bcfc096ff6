"""Batched replicas (yamc_batch_*) against the oracle, replica by replica.

A batch of uneven replicas -- water with ions (3 LJ types), water only (1 LJ type) of two
sizes, and a force-biased one -- falls into three kernel-variant groups that run as
concurrent cluster launches inside one CUDA graph.  Every replica must reproduce its own
oracle chain exactly as a single context does: identical molecule choices, overlap flags,
decisions and random-stream cursors, dE components within 1e-10 * max(|dE|, 1 kT) (force-
biased: 1e-10 for the first 500 moves, 1e-8 after, as for single chains), energy totals
within 1e-9 relative.  The autotuner must leave the chains where they were."""
import numpy as np
import pytest

import pyoracle
from yamc_b200 import api, rng as grng, systems

pytestmark = pytest.mark.gpu

DU = ("du_real", "du_k_coul", "du_k_lj", "du_ext")


def _same_chain(glog, olog, biased=False, start=0):
    assert len(glog) == len(olog)
    assert np.array_equal(glog["imol"], olog["imol"])
    assert np.array_equal(glog["flags"], olog["flags"])
    assert np.array_equal(glog["cursor"], olog["cursor"])
    for k in DU:
        tol = np.full(len(glog), 1e-10)
        if biased:
            tol[max(0, 500 - start):] = 1e-8
        ok = np.abs(glog[k] - olog[k]) <= tol * np.maximum(np.abs(olog[k]), 1.0)
        assert ok.all(), (k, int(np.argmin(ok)))


@pytest.fixture(scope="module")
def replica_files(tmp_path_factory):
    specs = [
        (systems.small_spec("ion_a"), 1),
        (systems.small_spec("water_a", n_na=0, n_cl=0), 2),
        (systems.small_spec("ion_b", n_water=26, box=10.4), 5),
        (systems.WORKLOADS["spce256"], 3),
        (systems.small_spec("biased", xlambda=0.1), 2),
    ]
    out = []
    for spec, seed in specs:
        d = str(tmp_path_factory.mktemp(spec.name))
        out.append((systems.write_system(spec, d, seed=seed), spec.xlambda > 0))
    return out


def _inputs(files):
    return api.load_inputs(files["parameters"], files["composition"], files["moltab"])


def test_batch_matches_oracle(replica_files):
    n_moves = 1500
    streams = [grng.gfortran_stream(1000 + 17 * i, 40 * n_moves + 10000) for i in range(len(replica_files))]
    b = api.Batch([_inputs(f) for f, _ in replica_files])
    log, cur, done, st, s = b.run(streams, n_moves, log=True)
    assert s == 0 and (st == 0).all() and (done == n_moves).all()
    for i, (files, biased) in enumerate(replica_files):
        o = pyoracle.Oracle(files)
        olog, _, ocur = o.run_mc(streams[i], n_moves)
        _same_chain(log[i], olog, biased)
        assert cur[i] == ocur
        e, eo = b.replica(i).energies(), o.energies()
        assert np.all(np.abs(e - eo) <= 1e-9 * np.maximum(np.abs(eo), 1.0))
    # a second step continues every chain from its cursor
    log2, cur2, done2, _, s2 = b.run(streams, 300, cursors=cur, log=True)
    assert s2 == 0 and (done2 == 300).all()
    for i, (files, biased) in enumerate(replica_files):
        o = pyoracle.Oracle(files)
        olog, _, ocur = o.run_mc(streams[i], n_moves + 300)
        _same_chain(log2[i], olog[n_moves:], biased, start=n_moves)
        assert cur2[i] == ocur
    b.close()


def test_batch_tune_keeps_state(replica_files):
    import torch
    sel = [replica_files[0], replica_files[2]]
    n_moves = 800
    streams = [grng.gfortran_stream(2000 + i, 40 * n_moves + 10000) for i in range(len(sel))]
    b = api.Batch([_inputs(f) for f, _ in sel])
    d = [torch.from_numpy(s).cuda() for s in streams]
    rate = b.tune([t.data_ptr() for t in d], [t.numel() for t in d], np.zeros(len(sel), dtype=np.int64), 200)
    assert rate > 0
    shape = b.launch
    assert shape["resident_clusters"] > 0
    log, cur, done, st, s = b.run(streams, n_moves, log=True)
    assert s == 0
    for i, (files, _) in enumerate(sel):
        o = pyoracle.Oracle(files)
        olog, _, ocur = o.run_mc(streams[i], n_moves)
        _same_chain(log[i], olog)
        assert cur[i] == ocur
    b.close()


def test_batch_stream_exhausted_resumes(replica_files):
    sel = [replica_files[0], replica_files[1]]
    n_moves = 600
    full = [grng.gfortran_stream(3000 + i, 40 * n_moves + 10000) for i in range(len(sel))]
    short = [full[0][:2000], full[1]]  # replica 0 runs out of random numbers
    b = api.Batch([_inputs(f) for f, _ in sel])
    log, cur, done, st, s = b.run(short, n_moves, log=True)
    assert s == -12 and st[0] == -12 and st[1] == 0 and done[0] < n_moves and done[1] == n_moves
    o = pyoracle.Oracle(sel[0][0])
    olog, _, _ = o.run_mc(full[0], n_moves)
    _same_chain(log[0][: done[0]], olog[: done[0]])
    b.close()
