"""Exchange moves (mc_xchange, MC.f90:1325-1954) and run_mc's exchange steps (runmc.f90:228-259).

Oracle-side tests (no GPU) check the restated exchange against the reference's own invariants:
the incremental state after many exchange steps equals a full recompute, molecules stay rigid,
swapping two molecules of the same species changes nothing and is accepted, and a run cut short
by the random stream resumes exactly.  The GPU tests run yamc_run_mc (exchange steps on the host
and the device's exchange kernels, movemc steps on the chain kernel) and the per-step C ABI against
the oracle on the same random stream: identical step types, molecule pairs, accept bits and
cursors; dE components within 1e-10 * max(|dE|, 1 kT); energies within 1e-9.
"""
import numpy as np
import pytest

import pyoracle
from yamc_b200 import rng as grng

DU = ("du_real", "du_k_coul", "du_k_lj", "du_ext")


def _ion_weights(o):
    w = np.zeros(o.nmol)
    f, l = o.mols()
    w[(l - f) == 0] = 1.0  # one-atom molecules: the ions
    return w


def test_oracle_xchange_invariants(tiny_files):
    o = pyoracle.Oracle(tiny_files)
    o.set_xchange_weights(_ion_weights(o))
    buf = grng.gfortran_stream(7, 400000)
    log, _, _ = o.run_mc(buf, 3000)
    ex = (log["flags"] & 4) != 0
    p = 4.0 / (o.nmol + 4.0)  # Sxch / (Smv + Sxch)
    assert abs(ex.mean() - p) < 5 * np.sqrt(p * (1 - p) / len(log))
    imol2 = log["flags"] >> 8
    f, l = o.mols()
    same_species = ex & (np.abs((log["imol"] - 1) // 2 - (imol2 - 1) // 2) == 0)  # Na-Na (25,26) or Cl-Cl (27,28)
    assert same_species.any()
    for k in DU:  # zero up to the rounding of the incremental per-atom sums
        assert np.all(np.abs(log[k][same_species]) <= 1e-9)
    assert np.all(log["flags"][same_species] & 1)
    e_inc = o.energies()
    e_full = o.full_sums()
    assert np.all(np.abs(e_inc - e_full) <= 1e-9 * np.maximum(np.abs(e_full), 1.0))


def test_oracle_xchange_all_molecules_rigid(tiny_files):
    o = pyoracle.Oracle(tiny_files)
    o.set_xchange_weights(np.full(o.nmol, 0.3))
    x0, y0, z0, *_ = o.atoms()
    f, l = o.mols()
    buf = grng.gfortran_stream(17, 400000)
    log, _, _ = o.run_mc(buf, 3000)
    ex = (log["flags"] & 4) != 0
    assert ex.sum() > 100 and (log["flags"][ex] & 1).any()
    x, y, z, *_ = o.atoms()
    for a, b in zip(f - 1, l - 1):
        for j in range(a + 1, b + 1):
            d0 = np.sqrt((x0[j] - x0[a]) ** 2 + (y0[j] - y0[a]) ** 2 + (z0[j] - z0[a]) ** 2)
            d1 = np.sqrt((x[j] - x[a]) ** 2 + (y[j] - y[a]) ** 2 + (z[j] - z[a]) ** 2)
            assert abs(d1 - d0) < 1e-12
    e_inc = o.energies()
    e_full = o.full_sums()
    assert np.all(np.abs(e_inc - e_full) <= 1e-9 * np.maximum(np.abs(e_full), 1.0))


def test_oracle_xchange_resume(tiny_files):
    buf = grng.gfortran_stream(21, 300000)
    a = pyoracle.Oracle(tiny_files)
    a.set_xchange_weights(np.full(a.nmol, 0.3))
    la, _, _, ca, _ = a.run_cycles(buf, 30)
    b = pyoracle.Oracle(tiny_files)
    b.set_xchange_weights(np.full(b.nmol, 0.3))
    lb1, _, _, cur, d1 = b.run_cycles(buf[: ca // 2], 30, allow_exhausted=True)
    lb2, _, _, cur, d2 = b.run_cycles(buf, 30 - d1, cursor=cur)
    assert cur == ca
    lb = np.concatenate([lb1, lb2])
    assert np.array_equal(la["imol"], lb["imol"]) and np.array_equal(la["flags"], lb["flags"])
    assert np.array_equal(a.energies(), b.energies())


# ---------------------------------------------------------------- GPU


def _compare(files, weights_fn, n_cycles, seed, extra=""):
    from yamc_b200 import api
    buf = grng.gfortran_stream(seed, 60 * n_cycles * 300 + 50000)
    o = pyoracle.Oracle(files, extra=extra)
    w = weights_fn(o)
    o.set_xchange_weights(w)
    olog, ovl, orows, ocur, odone = o.run_cycles(buf, n_cycles, max_rows=n_cycles)
    eng = api.Engine.from_files(files, extra=extra)
    eng.set_xchange_weights(w)
    glog, gvl, grows, gcur, gdone, st = eng.run_mc(buf, n_cycles, max_rows=n_cycles)
    assert st == 0 and gdone == odone == n_cycles
    assert ((olog["flags"] & 4) != 0).sum() > 5
    assert np.array_equal(glog["imol"], olog["imol"]) and np.array_equal(glog["flags"], olog["flags"])
    assert np.array_equal(glog["cursor"], olog["cursor"]) and gcur == ocur
    for k in DU:
        err = np.abs(glog[k] - olog[k]) / np.maximum(np.abs(olog[k]), 1.0)
        assert err.max() <= 1e-10, (k, err.max(), int(np.argmax(err)))
    assert np.array_equal(gvl["flags"], ovl["flags"])
    assert grows.shape == orows.shape
    assert np.all(np.abs(grows - orows) <= 1e-9 * np.maximum(np.abs(orows), 1.0))
    e_g, e_o = eng.energies(), o.energies()
    assert np.all(np.abs(e_g - e_o) <= 1e-9 * np.maximum(np.abs(e_o), 1.0)), (e_g, e_o)
    e_full = eng.full_sums()
    assert np.all(np.abs(e_g - e_full) <= 1e-9 * np.maximum(np.abs(e_full), 1.0))


@pytest.mark.gpu
def test_xchange_ions_matches_oracle(tiny_files):
    _compare(tiny_files, _ion_weights, 25, 51)


@pytest.mark.gpu
def test_xchange_all_molecules_matches_oracle(tiny_files):
    _compare(tiny_files, lambda o: np.full(o.nmol, 0.3), 25, 52)


@pytest.mark.gpu
def test_xchange_with_npt_matches_oracle(tiny_files):
    _compare(tiny_files, lambda o: np.full(o.nmol, 0.3), 30, 53,
             extra="pressure_step_multiplier=2,max_volume_scaling=1.02,n_store_energy_interval=1")


@pytest.mark.gpu
def test_xchange_per_step_api(spce_files):
    """The drop-in for the body of mc_xchange: the oracle's steps drive both."""
    from yamc_b200 import api
    o = pyoracle.Oracle(spce_files)
    eng = api.Engine.from_files(spce_files)
    rng = np.random.default_rng(4)
    buf = grng.gfortran_stream(9, 10000)
    cur = 0
    n_acc = 0
    for _ in range(40):
        i1, i2 = (int(v) for v in rng.choice(np.arange(1, o.nmol + 1), 2, replace=False))
        rec, cur = o.xchange(i1, i2, buf, cur)
        du, ov = eng.xchange_eval(i1, i2)
        assert ov == bool(rec.flags & 2)
        ref = np.array([rec.du_real, rec.du_k_coul, rec.du_k_lj, rec.du_ext])
        assert np.all(np.abs(du - ref) <= 1e-10 * np.maximum(np.abs(ref), 1.0)), (du, ref)
        acc = bool(rec.flags & 1)
        n_acc += acc
        eng.xchange_commit(acc)
        e_g, e_o = eng.energies(), o.energies()
        assert np.all(np.abs(e_g - e_o) <= 1e-9 * np.maximum(np.abs(e_o), 1.0))
    x, y, z = eng.positions()
    xo, yo, zo, *_ = o.atoms()
    assert np.abs(x - xo).max() < 1e-14
    from yamc_b200 import _lib
    with pytest.raises(_lib.YamcError):
        eng.xchange_commit(True)  # nothing pending


@pytest.mark.gpu
def test_batch_replica_refuses_exchange_and_volume_steps(tiny_files):
    """A batch replica is run by the batch's graph (NVT moves): exchange weights, exchange and
    volume steps and run_mc are refused on it."""
    from yamc_b200 import _lib, api
    inp = api.load_inputs(tiny_files["parameters"], tiny_files["composition"], tiny_files["moltab"])
    b = api.Batch([inp, inp])
    rep = b.replica(0)
    with pytest.raises(_lib.YamcError):
        rep.set_xchange_weights(np.full(rep.nmol, 0.3))
    with pytest.raises(_lib.YamcError):
        rep.xchange_eval(1, 2)
    with pytest.raises(_lib.YamcError):
        rep.volume_eval(10.5)
    b.close()


@pytest.mark.gpu
def test_run_mc_without_log_is_the_same_run(tiny_files):
    """run_mc with and without records (without, the chain runs every remaining move of the
    requested cycles in one stretch): the same cursor, rows and energies."""
    from yamc_b200 import api
    buf = grng.gfortran_stream(88, 400000)
    out = []
    for log in (True, False):
        eng = api.Engine.from_files(tiny_files, extra="pressure_step_multiplier=3,max_volume_scaling=1.02,"
                                                      "n_store_energy_interval=1")
        eng.set_xchange_weights(np.full(eng.nmol, 0.2))
        _, vlog, rows, cur, done, st = eng.run_mc(buf, 40, log=log, max_rows=40)
        assert st == 0 and done == 40
        out.append((cur, vlog, rows, eng.energies()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])
    assert np.array_equal(out[0][3], out[1][3])


@pytest.mark.gpu
def test_xchange_ions_nacl1m(nacl_files):
    """Ion exchanges in the 6,220-atom system (the realistic use: swapping Na+ and Cl- positions)."""
    _compare(nacl_files, _ion_weights, 3, 54)
