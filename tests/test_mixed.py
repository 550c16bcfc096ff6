"""The mixed-precision form (YAMC_MIXED) against the FP64 oracle.

Bar: every per-move dE within 1e-4 kT of the FP64 oracle's on the same configuration and
proposal.  Through the per-move C ABI the oracle's decisions drive both engines, so the
comparison covers every move.  A mixed chain driven by the same random stream follows the
oracle's decisions until a move whose acceptance test falls within the dE error of its
threshold; it is compared move by move up to that point.  The mixed forces (force-biased
moves) are checked against the oracle's to 1e-4 of the force scale, and the FP64
refresh of rho(k) every N accepted moves puts the k-space energies back on a full FP64
recomputation.  The mixed-precision configuration itself (16384 SPC/E + 300 Na + 300 Cl,
L = 79.3 A, kmax 24, force-biased) is covered by all three: 240 per-move dE through the C ABI,
a force-biased chain segment up to its first decision split, and refreshes inside the chain."""
import numpy as np
import pytest

import pyoracle
from yamc_b200 import _lib, api, rng as grng

pytestmark = pytest.mark.gpu

DU = ("du_real", "du_k_coul", "du_k_lj", "du_ext")
TOL_KT = 1e-4


def _mixed(files):
    return api.Engine.from_files(files, precision=_lib.YAMC_MIXED)


@pytest.mark.parametrize("which,n_try", [("tiny_files", 80), ("nacl_files", 80), ("tiny_biased_files", 80),
                                         ("nacl16k_files", 240)])
def test_mixed_per_move_de(which, n_try, request):
    files = request.getfixturevalue(which)
    o = pyoracle.Oracle(files)
    eng = _mixed(files)
    rng = np.random.default_rng(11)
    f, l = o.mols()
    L = o.params.BoxLength
    worst = 0.0
    fscale = 0.0
    ferr = 0.0
    n = 0
    for it in range(n_try):
        imol = int(rng.integers(1, o.nmol + 1))
        fo_g, to_g = eng.move_old(imol)
        fo_o, to_o = o.move_old(imol)
        fscale = max(fscale, np.abs(fo_o).max())
        ferr = max(ferr, np.abs(fo_g - fo_o).max())
        x, y, z, *_ = o.atoms()
        a, b = f[imol - 1] - 1, l[imol - 1]
        ang = rng.uniform(-0.15, 0.15)
        c, s = np.cos(ang), np.sin(ang)
        cx, cy = x[a], y[a]
        d = rng.uniform(-0.15, 0.15, 3) / L
        xn = cx + c * (x[a:b] - cx) - s * (y[a:b] - cy) + d[0]
        yn = cy + s * (x[a:b] - cx) + c * (y[a:b] - cy) + d[1]
        zn = z[a:b] + d[2]
        du_g, ov_g, fn_g, tn_g = eng.move_eval(imol, xn, yn, zn)
        du_o, ov_o, fn_o, tn_o = o.move_eval(xn, yn, zn)
        assert ov_g == ov_o
        if ov_o:
            eng.move_commit(False)
            continue
        worst = max(worst, abs(du_g.sum() - du_o.sum()))
        ferr = max(ferr, np.abs(fn_g - fn_o).max())
        n += 1
        acc = du_o.sum() < 0.5
        eng.move_commit(acc)
        if acc:
            o.move_commit()
    assert n > n_try // 2
    assert worst <= TOL_KT, worst
    assert ferr <= 1e-4 * max(fscale, 1.0), (ferr, fscale)
    e_g, e_o = eng.energies(), o.energies()
    assert np.all(np.abs(e_g - e_o) <= 1e-3), (e_g, e_o)


@pytest.mark.parametrize("which,n_moves", [("spce_files", 6000), ("nacl_files", 3000), ("nacl16k_files", 400)])
def test_mixed_chain_follows_oracle(which, n_moves, request):
    files = request.getfixturevalue(which)
    buf = grng.gfortran_stream(2025, 40 * n_moves + 10000)
    o = pyoracle.Oracle(files)
    olog, _, _ = o.run_mc(buf, n_moves)
    eng = _mixed(files)
    glog, _, _, done, st = eng.run_chain(buf, n_moves)
    assert st == 0 and done == n_moves
    same = (glog["imol"] == olog["imol"]) & (glog["flags"] == olog["flags"]) & (glog["cursor"] == olog["cursor"])
    k = n_moves if same.all() else int(np.argmin(same))
    assert k >= min(n_moves, 300), k  # a decision flip needs a draw within ~1e-5 of its threshold
    tot_g = sum(glog[c][:k] for c in DU)
    tot_o = sum(olog[c][:k] for c in DU)
    assert np.abs(tot_g - tot_o).max() <= TOL_KT
    # the running energies against an FP64 recomputation of the mixed chain's own configuration
    e_inc = eng.energies()
    e_full = eng.full_sums()
    assert abs(e_inc[0] - e_full[0]) <= 1e-2, (e_inc, e_full)


def test_mixed_refresh(nacl_files):
    eng = _mixed(nacl_files)
    eng.set_refresh(200)
    buf = grng.gfortran_stream(77, 40 * 3000 + 10000)
    glog, _, _, done, st = eng.run_chain(buf, 3000)
    assert st == 0 and done == 3000
    n_acc = int((glog["flags"] & 1).sum())
    assert eng.refresh_count == n_acc // 200
    e = eng.energies()
    f = eng.full_sums()
    assert abs(e[6] - f[6]) <= 1e-4 and abs(e[7] - f[7]) <= 1e-4  # k-space energies


def test_mixed_refresh_nacl16k(nacl16k_files):
    """FP64 refreshes inside a force-biased mixed chain of the 49,752-atom configuration."""
    eng = _mixed(nacl16k_files)
    eng.set_refresh(40)
    buf = grng.gfortran_stream(78, 60 * 400 + 10000)
    glog, _, _, done, st = eng.run_chain(buf, 400)
    assert st == 0 and done == 400
    n_acc = int((glog["flags"] & 1).sum())
    assert n_acc >= 40 and eng.refresh_count == n_acc // 40
    e = eng.energies()
    f = eng.full_sums()
    assert abs(e[6] - f[6]) <= 1e-3 and abs(e[7] - f[7]) <= 1e-3, (e[6:], f[6:])


def test_mixed_batch(spce_files, tiny_files):
    inputs = [api.load_inputs(f["parameters"], f["composition"], f["moltab"]) for f in (spce_files, tiny_files)]
    b = api.Batch(inputs, precision=_lib.YAMC_MIXED)
    for i in range(2):
        b.replica(i).set_refresh(300)
    n = 2000
    streams = [grng.gfortran_stream(300 + i, 40 * n + 10000) for i in range(2)]
    log, cur, done, st, s = b.run(streams, n, log=True)
    assert s == 0 and (done == n).all()
    for i, files in enumerate((spce_files, tiny_files)):
        o = pyoracle.Oracle(files)
        olog, _, _ = o.run_mc(streams[i], n)
        same = (log[i]["flags"] == olog["flags"]) & (log[i]["cursor"] == olog["cursor"])
        k = n if same.all() else int(np.argmin(same))
        assert k >= 300
        tot_g = sum(log[i][c][:k] for c in DU)
        tot_o = sum(olog[c][:k] for c in DU)
        assert np.abs(tot_g - tot_o).max() <= TOL_KT
        assert b.replica(i).refresh_count >= 1
    b.close()
