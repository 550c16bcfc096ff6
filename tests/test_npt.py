"""NPT volume moves (mcvol, MC.f90:701-825) and run_mc with volume cycles (runmc.f90:204-222).

Oracle-side tests (no GPU) check the restated volume step against the reference's own
invariants: the state after many NPT cycles equals a full recompute (MC.f90:1886-1951), rigid
molecules keep their bond lengths in Angstrom through scale_box (MC.f90:1973), a rejected
step puts back positions and energies exactly (mc_restore_state), the acceptance exponent is
-dU - P dV + (nmol+1) ln(V_new/V_old), and a run cut short by the random stream resumes
exactly.  The GPU tests run yamc_run_mc against the oracle on the same random stream:
identical cycle types, molecule choices, accept bits and cursors; per-move dE within
1e-10 * max(|dE|, 1 kT); the volume step's dU within 1e-9 * max(|U|, 1 kT) (two independent
full sums of the whole system); box lengths within 1e-12 relative; energy.dat rows within 1e-9.
"""
import numpy as np
import pytest

import pyoracle
from yamc_b200 import rng as grng

NPT = "pressure_step_multiplier=2,max_volume_scaling=1.02,n_store_energy_interval=1"
DU = ("du_real", "du_k_coul", "du_k_lj", "du_ext")


def _bond_lengths_angstrom(o):
    x, y, z, *_ = o.atoms()
    f, l = o.mols()
    L = o.box_length
    out = []
    for a, b in zip(f - 1, l - 1):
        for j in range(a + 1, b + 1):
            out.append(np.sqrt((x[j] - x[a]) ** 2 + (y[j] - y[a]) ** 2 + (z[j] - z[a]) ** 2) * L)
    return np.array(out)


def test_oracle_npt_invariants(tiny_files):
    o = pyoracle.Oracle(tiny_files, extra=NPT)
    b0 = _bond_lengths_angstrom(o)
    buf = grng.gfortran_stream(99, 300000)
    log, vlog, rows, cur, done = o.run_cycles(buf, 80, max_rows=100)
    assert done == 80 and len(vlog) > 10
    acc = (vlog["flags"] & 1) == 1
    assert acc.any() and (~acc).any()
    assert len(log) == (80 - len(vlog)) * o.nmol
    # the box walks only through accepted steps
    L = vlog["box_old"][0]
    for r in vlog:
        assert r["box_old"] == L
        if r["flags"] & 1:
            L = r["box_new"]
    assert o.box_length == L
    # acceptance exponent (MC.f90:789-795)
    p = o.params
    for r in vlog[(vlog["flags"] & 2) == 0]:
        vo, vn = r["box_old"] ** 3, r["box_new"] ** 3
        arg = -r["du"] - p.pressure_angstr_kT * (vn - vo) + (o.nmol + 1) * np.log(vn / vo)
        assert abs(arg - r["arg"]) <= 1e-12 * max(1.0, abs(arg))
    # rigid bonds in Angstrom (scale_box keeps them; MC.f90:1973 checks 1e-6 A^2)
    assert np.abs(_bond_lengths_angstrom(o) - b0).max() < 1e-12
    # incremental state = full recompute
    e_inc = o.energies()
    e_full = o.full_sums()
    assert np.all(np.abs(e_inc - e_full) <= 1e-9 * np.maximum(np.abs(e_full), 1.0)), (e_inc, e_full)
    assert len(rows) == 80 and np.array_equal(rows[:, 0], np.arange(1, 81))


def test_oracle_rejected_volume_step_restores(tiny_files):
    o = pyoracle.Oracle(tiny_files, extra=NPT + ",pressure=1e9")
    buf = grng.gfortran_stream(5, 20000)
    seen = set()
    cur = 0
    for _ in range(30):
        e0 = o.energies()
        x0 = o.atoms()[0].copy()
        L0 = o.box_length
        rec, cur = o.mcvol(buf, cur)
        acc = bool(rec["flags"] & 1)
        seen.add(acc)
        if not acc:
            assert np.array_equal(o.energies(), e0)
            assert np.array_equal(o.atoms()[0], x0)
            assert o.box_length == L0
    assert seen == {False, True}


def test_oracle_npt_resume(tiny_files):
    """A run cut short by the random stream, resumed from its cursor, is the uninterrupted run."""
    buf = grng.gfortran_stream(123, 200000)
    a = pyoracle.Oracle(tiny_files, extra=NPT)
    la, va, _, ca, _ = a.run_cycles(buf, 40)
    for cut in (3000, 7001, 8500):
        b = pyoracle.Oracle(tiny_files, extra=NPT)
        lb1, vb1, _, cur, d1 = b.run_cycles(buf[:cut], 40, allow_exhausted=True)
        assert d1 < 40
        lb2, vb2, _, cur, d2 = b.run_cycles(buf, 40 - d1, cursor=cur)
        assert d1 + d2 == 40 and cur == ca
        lb, vb = np.concatenate([lb1, lb2]), np.concatenate([vb1, vb2])
        assert np.array_equal(la["imol"], lb["imol"]) and np.array_equal(la["flags"], lb["flags"])
        assert np.array_equal(va["flags"], vb["flags"]) and np.array_equal(va["box_new"], vb["box_new"])
        assert np.array_equal(a.energies(), b.energies())


# ---------------------------------------------------------------- GPU


def _npt_compare(files, n_cycles, seed, extra=NPT):
    from yamc_b200 import api
    buf = grng.gfortran_stream(seed, 40 * n_cycles * 300 + 50000)
    o = pyoracle.Oracle(files, extra=extra)
    olog, ovl, orows, ocur, odone = o.run_cycles(buf, n_cycles, max_rows=n_cycles)
    eng = api.Engine.from_files(files, extra=extra)
    glog, gvl, grows, gcur, gdone, st = eng.run_mc(buf, n_cycles, max_rows=n_cycles)
    assert st == 0 and gdone == odone == n_cycles
    assert len(gvl) == len(ovl) and len(ovl) > 0
    assert np.array_equal(gvl["cycle"], ovl["cycle"]) and np.array_equal(gvl["flags"], ovl["flags"])
    assert np.array_equal(gvl["cursor"], ovl["cursor"])
    assert np.all(np.abs(gvl["box_new"] - ovl["box_new"]) <= 1e-12 * ovl["box_new"])
    u_scale = max(1.0, float(np.abs(o.energies()[0])))
    assert np.all(np.abs(gvl["du"] - ovl["du"]) <= 1e-9 * u_scale), np.abs(gvl["du"] - ovl["du"]).max()
    assert np.array_equal(glog["imol"], olog["imol"]) and np.array_equal(glog["flags"], olog["flags"])
    assert np.array_equal(glog["cursor"], olog["cursor"]) and gcur == ocur
    for k in DU:
        err = np.abs(glog[k] - olog[k]) / np.maximum(np.abs(olog[k]), 1.0)
        assert err.max() <= 1e-10, (k, err.max())
    assert grows.shape == orows.shape
    assert np.all(np.abs(grows - orows) <= 1e-9 * np.maximum(np.abs(orows), 1.0))
    assert abs(eng.current_params().BoxLength - o.box_length) <= 1e-12 * o.box_length
    e_g, e_o = eng.energies(), o.energies()
    assert np.all(np.abs(e_g - e_o) <= 1e-9 * np.maximum(np.abs(e_o), 1.0)), (e_g, e_o)
    return eng, o


@pytest.mark.gpu
def test_npt_run_mc_matches_oracle_tiny(tiny_files):
    eng, o = _npt_compare(tiny_files, 60, 31)
    # the incremental state after the NPT run against the device's own full recompute
    e_inc, e_full = eng.energies(), eng.full_sums()
    assert np.all(np.abs(e_inc - e_full) <= 1e-9 * np.maximum(np.abs(e_full), 1.0))


@pytest.mark.gpu
def test_npt_run_mc_matches_oracle_spce256(spce_files):
    _npt_compare(spce_files, 12, 32, extra="pressure_step_multiplier=1,max_volume_scaling=1.005,"
                                            "n_store_energy_interval=2")


@pytest.mark.gpu
def test_npt_run_mc_matches_oracle_spce256_tutorial_setting(spce_files):
    """The reference tutorial's pressure_step_multiplier (5) over 120 cycles (~28,000 moves)."""
    _npt_compare(spce_files, 120, 34, extra="pressure_step_multiplier=5,max_volume_scaling=1.01,"
                                             "n_store_energy_interval=5")


@pytest.mark.gpu
def test_npt_force_biased(tiny_biased_files):
    _npt_compare(tiny_biased_files, 30, 33)


@pytest.mark.gpu
def test_volume_eval_commit_per_step(tiny_files):
    """The drop-in for the body of mcvol: the host draws, the engine evaluates and commits."""
    from yamc_b200 import api
    buf = grng.gfortran_stream(8, 20000)
    o = pyoracle.Oracle(tiny_files, extra=NPT)
    eng = api.Engine.from_files(tiny_files, extra=NPT)
    cur = 0
    for _ in range(12):
        rec, cur = o.mcvol(buf, cur)
        du, ov = eng.volume_eval(rec["box_new"])
        assert ov == bool(rec["flags"] & 2)
        assert abs(du - rec["du"]) <= 1e-9 * max(1.0, abs(o.energies()[0]))
        eng.volume_commit(bool(rec["flags"] & 1))
        assert abs(eng.current_params().BoxLength - o.box_length) <= 1e-12 * o.box_length
        e_g, e_o = eng.energies(), o.energies()
        assert np.all(np.abs(e_g - e_o) <= 1e-9 * np.maximum(np.abs(e_o), 1.0))


@pytest.mark.gpu
def test_npt_resume_and_nvt_entry_refuses(tiny_files):
    from yamc_b200 import _lib, api
    buf = grng.gfortran_stream(41, 120000)
    a = api.Engine.from_files(tiny_files, extra=NPT)
    la, va, _, ca, _, st = a.run_mc(buf, 30)
    assert st == 0
    b = api.Engine.from_files(tiny_files, extra=NPT)
    lb1, vb1, _, cb, d1, st1 = b.run_mc(buf[: ca // 2], 30)
    assert st1 == _lib.YAMC_ERNG_EXHAUSTED and d1 < 30
    lb2, vb2, _, cb, d2, st2 = b.run_mc(buf, 30 - d1, cursor=cb)
    assert st2 == 0 and cb == ca
    assert np.array_equal(np.concatenate([vb1["flags"], vb2["flags"]]), va["flags"])
    assert np.array_equal(np.concatenate([vb1["box_new"], vb2["box_new"]]), va["box_new"])
    assert np.array_equal(a.energies(), b.energies())
    with pytest.raises(_lib.YamcError):
        a.run_chain(buf, 10)


@pytest.mark.gpu
def test_batch_refuses_npt(tiny_files):
    """Batched replicas run NVT: a replica with volume cycles is refused at creation."""
    from yamc_b200 import _lib, api
    inp = api.load_inputs(tiny_files["parameters"], tiny_files["composition"], tiny_files["moltab"], NPT)
    with pytest.raises(_lib.YamcError):
        api.Batch([inp])


@pytest.mark.gpu
def test_npt_mixed_precision(tiny_files):
    """The mixed form with volume and exchange steps: the volume steps' full sums are FP64, the
    chain's moves mixed; the running energies stay on an FP64 recomputation of the configuration
    and the cycle structure follows the FP64 run up to the first decision the dE error flips."""
    from yamc_b200 import _lib, api
    buf = grng.gfortran_stream(61, 400000)
    runs = {}
    for prec in (_lib.YAMC_FP64, _lib.YAMC_MIXED):
        eng = api.Engine.from_files(tiny_files, extra=NPT, precision=prec)
        eng.set_xchange_weights(np.full(eng.nmol, 0.2))
        log, vlog, rows, cur, done, st = eng.run_mc(buf, 20)
        assert st == 0 and done == 20
        runs[prec] = (log, vlog, eng)
    lf, vf, ef = runs[_lib.YAMC_FP64]
    lm, vm, em = runs[_lib.YAMC_MIXED]
    n = min(len(lf), len(lm))
    same = (lf["imol"][:n] == lm["imol"][:n]) & (lf["flags"][:n] == lm["flags"][:n])
    k = n if same.all() else int(np.argmin(same))
    assert k > 50
    du_f = sum(lf[c][:k] for c in DU)
    du_m = sum(lm[c][:k] for c in DU)
    assert np.abs(du_f - du_m).max() <= 1e-4
    e_inc, e_full = em.energies(), em.full_sums()
    assert abs(e_inc[0] - e_full[0]) <= 1e-3 * max(1.0, abs(e_full[0]))
