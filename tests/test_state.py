"""Exact checkpoints and the non-finite status.

Checkpoint (yamc_save_state / yamc_load_state): the reference restarts a run from its last
trajectory frame with a new seed (mccont.f90:121-171), which continues the ensemble but not the
chain; here a saved state loaded into a fresh context continues the chain bit for bit.  Tests:
an NPT run (volume steps rescale the box-dependent tables with rounding, which the state keeps)
and a mixed-precision run with FP64 rho refreshes (their counters are part of the state) are cut
in two, saved, loaded into a new context, and continued: every record, energy and position equals
the uninterrupted run exactly.  A state is refused by a context of another system.

YAMC_ENAN (error.f90 has no counterpart; the reference would carry the NaN on): non-finite
inputs are refused with the context unchanged (host checks), a full sum with coincident charges
is reported, and a chain whose proposal turns non-finite stops before deciding that move --
injected on the host, as a NaN in the caller's random stream at the move's first translation
draw (MonteCarloMove.f90:242-248) -- with the records, energies and cursor of the moves before
it equal to the oracle's, and continues exactly once the stream is clean.
"""
import ctypes

import numpy as np
import pytest

import pyoracle
from yamc_b200 import _lib, api
from yamc_b200 import rng as grng

DU = ("du_real", "du_k_coul", "du_k_lj", "du_ext")
NPT = "pressure_step_multiplier=2,max_volume_scaling=1.02,n_store_energy_interval=1"


def test_create_refuses_non_finite_input(tiny_files):
    inp = api.load_inputs(tiny_files["parameters"], tiny_files["composition"], tiny_files["moltab"])
    inp.x[5] = np.nan
    lib = _lib.load()
    h = ctypes.c_void_p()
    s = inp.as_struct()
    st = lib.yamc_create(ctypes.byref(s), ctypes.byref(inp.params), 0, ctypes.byref(h))
    assert st == _lib.YAMC_ENAN and not h.value
    assert b"atom 6" in lib.yamc_last_error_detail()


def _records_equal(a, b):
    return a.tobytes() == b.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["npt_fp64", "mixed_refresh"])
def test_checkpoint_continues_bit_for_bit(tiny_files, case):
    extra = NPT if case == "npt_fp64" else "n_store_energy_interval=1"
    prec = _lib.YAMC_FP64 if case == "npt_fp64" else _lib.YAMC_MIXED
    buf = grng.gfortran_stream(4242, 600000)
    a = api.Engine.from_files(tiny_files, extra=extra, precision=prec)
    if case == "mixed_refresh":
        a.set_refresh(37)
    _, _, _, cur1, done, st = a.run_mc(buf, 40, log=False)
    assert st == 0 and done == 40
    state = a.save_state(cur1)
    e_saved = a.energies()
    log_a, vlog_a, rows_a, cur_a, done_a, st_a = a.run_mc(buf, 60, cursor=cur1, max_rows=100)
    assert st_a == 0 and done_a == 60
    if case == "npt_fp64":
        assert len(vlog_a) > 5 and ((vlog_a["flags"] & 1) == 1).any()
    else:
        assert a.refresh_count > 0
    b = api.Engine.from_files(tiny_files, extra=extra, precision=prec)
    if case == "mixed_refresh":
        b.set_refresh(37)
    cur = b.load_state(state)
    assert cur == cur1
    assert np.array_equal(b.energies(), e_saved)
    log_b, vlog_b, rows_b, cur_b, done_b, st_b = b.run_mc(buf, 60, cursor=cur, max_rows=100)
    assert st_b == 0 and done_b == 60 and cur_b == cur_a
    assert _records_equal(log_a, log_b) and _records_equal(vlog_a, vlog_b)
    assert np.array_equal(rows_a, rows_b)
    assert np.array_equal(a.energies(), b.energies())
    for pa, pb in zip(a.positions(), b.positions()):
        assert np.array_equal(pa, pb)
    assert a.current_params().BoxLength == b.current_params().BoxLength
    if case == "mixed_refresh":
        assert a.refresh_count == b.refresh_count
    a.close()
    b.close()


@pytest.mark.gpu
def test_state_refused_by_another_system(tiny_files, spce_files):
    a = api.Engine.from_files(tiny_files)
    b = api.Engine.from_files(spce_files)
    with pytest.raises(_lib.YamcError) as ei:
        b.load_state(a.save_state(0))
    assert ei.value.status == _lib.YAMC_EPARAMETER
    with pytest.raises(_lib.YamcError):
        b.load_state(b"not a state at all, but long enough to hold a header of the state blob")
    a.close()
    b.close()


def _first_translation_draw(olog, nmol, k):
    """Stream position of move k's first translation draw (moves 0-based, none at a cycle
    start): run_mc's exchange draw and molecule draw come first (runmc.f90:232, 258)."""
    assert k % nmol != 0
    return int(olog["cursor"][k - 1]) + 2


@pytest.mark.gpu
@pytest.mark.parametrize("files_name", ["tiny_files", "tiny_biased_files"])
def test_nan_in_stream_stops_chain_before_the_move(files_name, request):
    files = request.getfixturevalue(files_name)
    n, k = 300, 157
    buf = grng.gfortran_stream(777, 200000)
    o = pyoracle.Oracle(files)
    olog, _, ocur = o.run_mc(buf, n)
    pos = _first_translation_draw(olog, o.nmol, k)
    bad = buf.copy()
    bad[pos] = np.nan
    eng = api.Engine.from_files(files)
    glog, _, gcur, done, st = eng.run_chain(bad, n)
    assert st == _lib.YAMC_ENAN and done == k
    assert gcur == int(olog["cursor"][k - 1])
    assert np.array_equal(glog["imol"], olog["imol"][:k]) and np.array_equal(glog["flags"], olog["flags"][:k])
    # the state is that after move k-1: compare with an oracle run of k moves
    o2 = pyoracle.Oracle(files)
    o2.run_mc(buf, k)
    e_g, e_o = eng.energies(), o2.energies()
    assert np.all(np.abs(e_g - e_o) <= 1e-9 * np.maximum(np.abs(e_o), 1.0))
    # the clean stream continues from the cursor exactly as the uninterrupted chain
    glog2, _, gcur2, done2, st2 = eng.run_chain(buf, n - k, cursor=gcur)
    assert st2 == 0 and done2 == n - k and gcur2 == ocur
    assert np.array_equal(glog2["imol"], olog["imol"][k:]) and np.array_equal(glog2["flags"], olog["flags"][k:])
    for key in DU:
        err = np.abs(glog2[key] - olog[key][k:]) / np.maximum(np.abs(olog[key][k:]), 1.0)
        assert err.max() <= 1e-8, key
    eng.close()


@pytest.mark.gpu
def test_non_finite_positions_refused_and_coincident_charges_reported(tiny_files):
    eng = api.Engine.from_files(tiny_files)
    e0 = eng.energies()
    x, y, z = (v.copy() for v in eng.positions())
    xb = x.copy()
    xb[3] = np.inf
    with pytest.raises(_lib.YamcError) as ei:
        eng.set_positions(xb, y, z)
    assert ei.value.status == _lib.YAMC_ENAN
    assert np.array_equal(eng.energies(), e0)
    for p, q in zip(eng.positions(), (x, y, z)):
        assert np.array_equal(p, q)
    # an H atom of molecule 2 on an H atom of molecule 1: H carries no LJ site and no hard core,
    # so nothing keeps the charges apart and the real-space sum is infinite
    xc, yc, zc = x.copy(), y.copy(), z.copy()
    f, l = eng.inputs.first_atom - 1, eng.inputs.last_atom - 1
    h1, h2 = f[0] + 1, f[1] + 1
    assert eng.inputs.sigma[h1] == 0 and eng.inputs.sigma[h2] == 0
    dx, dy, dz = x[h1] - xc[h2], y[h1] - yc[h2], z[h1] - zc[h2]
    for a in range(f[1], l[1] + 1):
        xc[a] += dx; yc[a] += dy; zc[a] += dz
    xc[h2], yc[h2], zc[h2] = x[h1], y[h1], z[h1]  # exactly (a + (b - a) may miss b by an ulp)
    with pytest.raises(_lib.YamcError) as ei:
        eng.set_positions(xc, yc, zc)
    assert ei.value.status == _lib.YAMC_ENAN
    # finite positions again give the original sums
    e1 = eng.set_positions(x, y, z)
    assert np.allclose(e1, e0, rtol=1e-12, atol=1e-9)
    eng.close()
