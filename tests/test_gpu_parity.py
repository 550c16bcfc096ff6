"""GPU engine against the CPU oracle, through the C ABI, on the same inputs and the
same gfortran random stream.

Tolerances (the contract of the plain FP64 method): per-move dE components
|dE_gpu - dE_ref| <= 1e-10 * max(|dE_ref|, 1 kT); identical molecule choices,
overlap flags, accept/reject decisions and random-stream cursors; energy.dat
totals within 1e-9 relative."""
import numpy as np
import pytest

import pyoracle
from yamc_b200 import _lib, api, rng as grng

pytestmark = pytest.mark.gpu

DU = ("du_real", "du_k_coul", "du_k_lj", "du_ext")


def close_du(a, b, tol=1e-10):
    return np.abs(a - b) <= tol * np.maximum(np.abs(b), 1.0)


def rel_close(a, b, tol):
    return np.all(np.abs(a - b) <= tol * np.maximum(np.abs(b), 1.0))


def compare_logs(glog, olog):
    assert len(glog) == len(olog)
    assert np.array_equal(glog["imol"], olog["imol"])
    bad = np.nonzero(glog["flags"] != olog["flags"])[0]
    assert bad.size == 0, f"first decision mismatch at move {bad[:1]}"
    assert np.array_equal(glog["cursor"], olog["cursor"])
    for k in DU:
        ok = close_du(glog[k], olog[k])
        assert ok.all(), (k, int(np.argmin(ok)), glog[k][~ok][:3], olog[k][~ok][:3])


@pytest.mark.parametrize("which", ["tiny_files", "spce_files", "nacl_files"])
def test_initial_full_sums(which, request):
    files = request.getfixturevalue(which)
    o = pyoracle.Oracle(files)
    eng = api.Engine.from_files(files)
    assert rel_close(eng.energies(), o.energies(), 1e-10)
    assert (eng.nk, eng.ntype) == (o.nk, o.ntype)


LAYOUTS = {"registers": _lib.YAMC_KSPACE_REGISTERS, "streamed": _lib.YAMC_KSPACE_STREAMED}


def _run_pair(files, n_moves, seed=12345, cluster=0, threads=0, layout=_lib.YAMC_KSPACE_AUTO):
    buf = grng.gfortran_stream(seed, 40 * n_moves + 10000)
    o = pyoracle.Oracle(files)
    olog, orows, ocur = o.run_mc(buf, n_moves)
    eng = api.Engine.from_files(files)
    if layout:
        eng.set_kspace_layout(layout)
    if cluster or threads:
        eng.set_launch(cluster, threads)
    glog, grows, gcur, done, st = eng.run_chain(buf, n_moves)
    assert st == 0 and done == n_moves
    return o, olog, ocur, eng, glog, gcur




@pytest.mark.parametrize("layout", ["registers", "streamed"])
@pytest.mark.parametrize("cluster", [1, 2, 4])
def test_chain_matches_oracle_tiny(tiny_files, cluster, layout):
    o, olog, ocur, eng, glog, gcur = _run_pair(tiny_files, 3000, cluster=cluster, layout=LAYOUTS[layout])
    assert eng.launch["entries_per_thread"] == (0 if layout == "streamed" else 1)
    compare_logs(glog, olog)
    assert gcur == ocur
    assert rel_close(eng.energies(), o.energies(), 1e-9)


def test_chain_matches_oracle_spce256_1e5(spce_files):
    """256 SPC/E: the identical accept/reject sequence over 1e5 moves."""
    o, olog, ocur, eng, glog, gcur = _run_pair(spce_files, 100096)
    compare_logs(glog, olog)
    assert rel_close(eng.energies(), o.energies(), 1e-9)
    # the incremental state still equals a full recompute on the device
    assert rel_close(eng.full_sums(), o.full_sums(), 1e-9)


def test_chain_streamed_spce256(spce_files):
    """The k entries streamed from memory every pass instead of held in registers."""
    o, olog, ocur, eng, glog, gcur = _run_pair(spce_files, 20000, layout=_lib.YAMC_KSPACE_STREAMED)
    compare_logs(glog, olog)
    assert rel_close(eng.energies(), o.energies(), 1e-9)
    assert rel_close(eng.full_sums(), o.full_sums(), 1e-9)


@pytest.mark.parametrize("cluster", [1, 3])
def test_chain_streamed_wide(spce_files, cluster):
    """Streamed entries with 384-thread CTAs (11 worker warps)."""
    o, olog, ocur, eng, glog, gcur = _run_pair(spce_files, 5000, cluster=cluster, threads=384,
                                               layout=_lib.YAMC_KSPACE_STREAMED)
    assert eng.launch["threads"] == 384 and eng.launch["entries_per_thread"] == 0
    compare_logs(glog, olog)
    assert rel_close(eng.energies(), o.energies(), 1e-9)


def test_chain_matches_oracle_nacl(nacl_files):
    o, olog, ocur, eng, glog, gcur = _run_pair(nacl_files, 6000)
    compare_logs(glog, olog)
    assert rel_close(eng.energies(), o.energies(), 1e-9)


def test_chain_matches_oracle_nacl1m_1e5(nacl_files):
    """The benchmark's system (2048 SPC/E + 38 Na + 38 Cl): the identical accept/reject sequence
    over 1e5 moves (about a minute of the oracle)."""
    o, olog, ocur, eng, glog, gcur = _run_pair(nacl_files, 100000, seed=2026)
    compare_logs(glog, olog)
    assert gcur == ocur
    assert rel_close(eng.energies(), o.energies(), 1e-9)
    assert rel_close(eng.full_sums(), o.full_sums(), 1e-9)


def compare_biased(glog, olog):
    assert np.array_equal(glog["imol"], olog["imol"]) and np.array_equal(glog["flags"], olog["flags"])
    assert np.array_equal(glog["cursor"], olog["cursor"])
    for k in DU:
        assert close_du(glog[k][:500], olog[k][:500]).all(), k
        assert close_du(glog[k], olog[k], 1e-8).all(), k


@pytest.mark.parametrize("layout", ["registers", "streamed"])
def test_chain_force_biased(tiny_biased_files, layout):
    """Force-biased proposals take the forces into the new positions, so ~1e-12 relative force
    differences (summation order) move the two chains apart slowly (about 1e-10 after ~1500
    moves of this dense 28-molecule box).  The decisions must stay identical; per-move dE meets
    the 1e-10 bound over the first 500 moves and 1e-8 afterwards."""
    o, olog, ocur, eng, glog, gcur = _run_pair(tiny_biased_files, 2000, seed=77, layout=LAYOUTS[layout])
    compare_biased(glog, olog)
    assert rel_close(eng.energies(), o.energies(), 1e-8)


def test_chain_nacl4k_force_biased(nacl4k_files):
    """4096 SPC/E + 76 Na + 76 Cl (12,440 atoms, 7,427 signed k), force-biased moves with
    lambda = 0.1: the k-set is too large for registers, so the entries are streamed."""
    o, olog, ocur, eng, glog, gcur = _run_pair(nacl4k_files, 1000, seed=41)
    assert eng.launch["entries_per_thread"] == 0
    compare_biased(glog, olog)
    assert rel_close(eng.energies(), o.energies(), 1e-8)


def test_chain_nacl16k(nacl16k_files):
    """16384 SPC/E + 300 Na + 300 Cl (49,752 atoms, 29,784 signed k), force-biased."""
    o, olog, ocur, eng, glog, gcur = _run_pair(nacl16k_files, 300, seed=43)
    assert eng.launch["entries_per_thread"] == 0
    compare_biased(glog, olog)
    assert rel_close(eng.energies(), o.energies(), 1e-8)


def test_energy_rows(tiny_files, tmp_path):
    from yamc_b200 import formats, systems
    spec = systems.small_spec()
    spec.n_store_energy_interval = 2.0
    files = systems.write_system(spec, str(tmp_path / "rows"))
    buf = grng.gfortran_stream(5, 200000)
    o = pyoracle.Oracle(files)
    n = 10 * (spec.nmol)
    _, orows, _ = o.run_mc(buf, n, max_rows=20)
    eng = api.Engine.from_files(files)
    _, grows, _, _, _ = eng.run_chain(buf, n, log=False, max_rows=20)
    assert len(orows) == len(grows) == 5
    assert np.array_equal(orows[:, 0], grows[:, 0])
    assert rel_close(grows[:, 1:], orows[:, 1:], 1e-9)
    path = str(tmp_path / "energy.dat")
    formats.write_energy_rows(path, grows, append=False)
    assert np.allclose(formats.read_energy_dat(path), grows, rtol=1e-15, atol=0)


def test_rng_exhausted_resume_is_exact(tiny_files):
    buf = grng.gfortran_stream(9, 200000)
    ref = api.Engine.from_files(tiny_files)
    rlog, _, rcur, rdone, rst = ref.run_chain(buf, 1500)
    assert rst == 0
    eng = api.Engine.from_files(tiny_files)
    cut = int(rlog["cursor"][700]) + 5  # the buffer ends inside move 702
    log1, _, cur1, done1, st1 = eng.run_chain(buf[:cut], 1500)
    assert st1 == -12 and done1 == 701 and cur1 == rlog["cursor"][700]
    log2, _, cur2, done2, st2 = eng.run_chain(buf, 1500 - done1, cursor=cur1)
    assert st2 == 0 and cur2 == rcur
    both = np.concatenate([log1, log2])
    assert np.array_equal(both, rlog)
    assert np.array_equal(eng.energies(), ref.energies())


def test_chain_is_deterministic(spce_files):
    buf = grng.gfortran_stream(4, 200000)
    a = api.Engine.from_files(spce_files)
    b = api.Engine.from_files(spce_files)
    la = a.run_chain(buf, 3000)[0]
    lb = b.run_chain(buf, 3000)[0]
    assert np.array_equal(la, lb)
    assert np.array_equal(a.energies(), b.energies())


@pytest.mark.parametrize("layout", ["registers", "streamed"])
@pytest.mark.parametrize("which", ["tiny_files", "tiny_biased_files"])
def test_per_move_api_matches_oracle(which, layout, request):
    """movemc driven from the host through yamc_move_old / _eval / _commit."""
    files = request.getfixturevalue(which)
    o = pyoracle.Oracle(files)
    eng = api.Engine.from_files(files)
    eng.set_kspace_layout(LAYOUTS[layout])
    rng = np.random.default_rng(3)
    f, l = o.mols()
    L = o.params.BoxLength
    for it in range(60):
        imol = int(rng.integers(1, o.nmol + 1))
        fo_g, to_g = eng.move_old(imol)
        fo_o, to_o = o.move_old(imol)
        assert rel_close(fo_g, fo_o, 1e-9) and rel_close(to_g, to_o, 1e-9)
        x, y, z, *_ = o.atoms()
        a, b = f[imol - 1] - 1, l[imol - 1]
        ang = rng.uniform(-0.2, 0.2)
        c, s = np.cos(ang), np.sin(ang)
        cx, cy, cz = x[a], y[a], z[a]
        d = rng.uniform(-0.2, 0.2, 3) / L
        xn = cx + c * (x[a:b] - cx) - s * (y[a:b] - cy) + d[0]
        yn = cy + s * (x[a:b] - cx) + c * (y[a:b] - cy) + d[1]
        zn = z[a:b] + d[2]
        du_g, ov_g, fn_g, tn_g = eng.move_eval(imol, xn, yn, zn)
        du_o, ov_o, fn_o, tn_o = o.move_eval(xn, yn, zn)
        assert ov_g == ov_o
        if ov_o:
            eng.move_commit(False)
            continue
        assert close_du(du_g, du_o).all(), (du_g, du_o)
        assert rel_close(fn_g, fn_o, 1e-9) and rel_close(tn_g, tn_o, 1e-9)
        acc = (du_o.sum() < 0.5)
        eng.move_commit(acc)
        if acc:
            o.move_commit()
    assert rel_close(eng.energies(), o.energies(), 1e-9)


@pytest.mark.parametrize("zero", [False, True])
def test_weighted_molecule_choice(tiny_files, tmp_path, zero):
    """A frequencies file with move weights only (no exchange): BiasedRandom_choose on uneven
    intervals; with a zero weight the intervals are no longer monotone (end = -1) and the
    device takes the reference's linear scan."""
    from yamc_b200 import formats
    inp = api.load_inputs(tiny_files["parameters"], tiny_files["composition"], tiny_files["moltab"])
    n = inp.nmol
    lines = [f"1-{n - 4} 1.0 0.0", f"{n - 3}-{n} 5.0 0.0"]
    if zero:
        lines = ["1-3 1.0 0.0", "4-4 0.0 0.0", f"5-{n - 4} 1.0 0.0", f"{n - 3}-{n} 5.0 0.0"]
    (tmp_path / "freq").write_text(f"{len(lines)}\n" + "\n".join(lines) + "\n")
    mv, xc = formats.read_freq_file(str(tmp_path / "freq"), n)
    inp.move_weights = mv
    o = pyoracle.Oracle(tiny_files)
    o.set_move_weights(mv)
    buf = grng.gfortran_stream(31, 200000)
    olog, _, ocur = o.run_mc(buf, 3000)
    eng = api.Engine(inp)
    glog, _, gcur, done, st = eng.run_chain(buf, 3000)
    assert st == 0 and done == 3000
    compare_logs(glog, olog)
    assert gcur == ocur
    counts = np.bincount(glog["imol"], minlength=n + 1)[1:]
    assert counts[-4:].mean() > 3 * counts[: n - 4].mean()
    if zero:
        assert counts[3] == 0


@pytest.mark.parametrize("layout", ["registers", "streamed"])
def test_chain_hard_core_per_atom(tmp_path, layout):
    """Two species sharing one LJ type (same sigma, epsilon) with different hard-core diameters:
    the chain kernel takes each atom's own diameter (its per-type table does not apply), and
    overlaps, decisions and dE stay those of the oracle."""
    from yamc_b200 import formats, systems
    spec = systems.small_spec(name="hc", n_water=20, n_na=3, n_cl=3, box=10.0)
    files = systems.write_system(spec, str(tmp_path / "hc"), seed=7)
    d = files["dir"]
    na = systems.na_atoms()[0]
    # Cl becomes Na's LJ twin with the opposite charge and a larger hard core
    formats.write_mol(f"{d}/Cl_Dang.mol", [formats.MolAtom("Cl", 0.0, 0.0, 0.0, na.sigma, na.epsilon, -1.0, 1.0, 2.8)])
    o = pyoracle.Oracle(files)
    assert o.ntype == 2  # O and the shared ion type
    glog, olog = None, None
    eng = api.Engine.from_files(files)
    eng.set_kspace_layout(LAYOUTS[layout])
    buf = grng.gfortran_stream(71, 400000)
    glog, _, gcur, done, st = eng.run_chain(buf, 4000)
    olog, _, ocur = o.run_mc(buf, 4000)
    assert st == 0 and done == 4000 and gcur == ocur
    compare_logs(glog, olog)
    assert ((olog["flags"] & 2) != 0).any()  # the hard core is exercised


def test_fma_peak_measures_the_pipes():
    """yamc_fma_peak: both pipes give a finite positive rate, FP32 at least that of FP64."""
    p64, p32 = api.fma_peak(0, True), api.fma_peak(0, False)
    assert 0.5 < p64 < 500.0 and 0.5 < p32 < 500.0, (p64, p32)
    assert p32 >= p64, (p64, p32)
    with pytest.raises(_lib.YamcError):
        api.fma_peak(-1, True)
