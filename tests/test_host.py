"""Host-side pieces of the product that run without a GPU: the C ABI library
loads and exports every entry point of include/yamc.h, the parameter
derivation matches the reference's parameters.out, the input readers match
the oracle's, and malformed inputs become status codes instead of aborts."""
import ctypes
import json
import os

import numpy as np
import pytest

import pyoracle
from yamc_b200 import _lib, api, formats, systems

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing
    assert set(declared) <= set(_lib.SIGNATURES), set(declared) - set(_lib.SIGNATURES)


def test_params_recalc_matches_parameters_out(tmp_path):
    g = json.load(open(os.path.join(GOLDEN, "parameters_out.json")))
    prm = tmp_path / "parameters.prm"
    prm.write_text("".join(f"{k} = {v}   # comment\n" for k, v in g["prm"].items()) + "# only a comment\n\n")
    p = api.read_parameters(str(prm))
    api.params_init(p, g["nmol"])
    printed = g["printed"]
    assert p.kmax == int(printed["kmax"])
    for name in ("BoxLength", "rmax", "kT_kcal_mol", "rmax2", "dbjr_a", "dbjr", "xclb", "alpha_over_sqrt_pi",
                 "two_alpha_over_sqrt_pi", "kext", "minus_two_kext", "dr", "d_angle", "log_max_volume_scaling",
                 "pressure_angstr_kT"):
        assert getattr(p, name) == float(printed[name].replace("D", "E")), name


def test_params_extra_string(tmp_path):
    prm = tmp_path / "p.prm"
    prm.write_text("sr = 3\nsk = 3\nBoxLength = 20\ntemp = 300\n")
    p = api.read_parameters(str(prm), "sr=4,temp=310.5,xlambda_f=0.25")
    assert (p.sr, p.temp, p.xlambda_f) == (4.0, 310.5, 0.25)
    with pytest.raises(_lib.YamcError):
        api.read_parameters(str(prm), "sr4")


def test_inputs_match_oracle_readers(nacl_files):
    inp = api.load_inputs(nacl_files["parameters"], nacl_files["composition"], nacl_files["moltab"])
    o = pyoracle.Oracle(nacl_files)
    x, y, z, q, t, m = o.atoms()
    assert inp.natom == o.natom == 6220
    assert np.array_equal(inp.x, x) and np.array_equal(inp.y, y) and np.array_equal(inp.z, z)
    assert np.array_equal(inp.charge, q)
    f, l = o.mols()
    assert np.array_equal(inp.first_atom, f) and np.array_equal(inp.last_atom, l)
    assert list(inp.mol_numbers) == [2048, 38, 38]


def test_moltab_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    n = 50
    x, y, z = (rng.uniform(-0.5, 0.5, n) for _ in range(3))
    th, ph, ps = (rng.uniform(0, 6.28, n) for _ in range(3))
    path = str(tmp_path / "t.moltab")
    formats.write_moltab(path, x, y, z, th, ph, ps, 3, 3)
    back = formats.read_moltab(path, n, 3, 3)
    for a, b in zip((x, y, z), back[:3]):
        assert np.abs(a - b).max() <= 0.5 / 256 ** 3 + 1e-15
    formats.write_moltab(path, x, y, z, th, ph, ps, 3, 3)
    assert os.path.getsize(path) == n * 18


def test_malformed_inputs_return_status(tmp_path, tiny_files):
    with pytest.raises(_lib.YamcError) as e:
        api.load_inputs(str(tmp_path / "missing.prm"), tiny_files["composition"], tiny_files["moltab"])
    assert e.value.status == -1
    short = tmp_path / "short.moltab"
    short.write_bytes(open(tiny_files["moltab"], "rb").read()[:50])
    with pytest.raises(_lib.YamcError) as e:
        api.load_inputs(tiny_files["parameters"], tiny_files["composition"], str(short))
    assert e.value.status == -1
    badmol = tmp_path / "bad.composition"
    (tmp_path / "X.mol").write_text("O 0 0 0 3.1 0.1\n")
    badmol.write_text("1\nX.mol 3\n")
    with pytest.raises(_lib.YamcError):
        api.load_inputs(tiny_files["parameters"], str(badmol), tiny_files["moltab"])


def test_workload_sizes():
    s = systems.WORKLOADS
    assert s["spce256"].natom == 768 and s["nacl1m"].natom == 6220
    assert s["nacl4k"].natom == 12440 and s["nacl16k"].natom == 49752
    for w in s.values():
        kmax = int(np.floor(w.params()["sk"] * w.alphaL / np.pi + 0.5))
        assert kmax == w.kmax
    b = systems.batch_specs(96)
    assert len(b) == 96 and min(x.n_water for x in b) >= 216 and max(x.n_water for x in b) <= 4096


def test_freq_file_reader(tmp_path):
    """read_freq_file (runmc.f90:70-173): comments, intervals, coverage and crossing checks."""
    import numpy as np
    import pytest
    from yamc_b200 import formats
    p = tmp_path / "freq.txt"
    p.write_text("# frequencies\n\n3\n1-4 1.0 0.0\n5-5 0.0 0.0\n6-8 2.5 0.0\n")
    mv, xc = formats.read_freq_file(str(p), 8)
    assert np.array_equal(mv, [1, 1, 1, 1, 0, 2.5, 2.5, 2.5]) and np.all(xc == 0)
    p.write_text("2\n1-4 1.0 0.0\n4-8 1.0 0.0\n")
    with pytest.raises(ValueError, match="crossing"):
        formats.read_freq_file(str(p), 8)
    p.write_text("1\n1-6 1.0 0.0\n")
    with pytest.raises(ValueError, match="not all"):
        formats.read_freq_file(str(p), 8)
    p.write_text("1\n1-9 1.0 0.0\n")
    with pytest.raises(ValueError, match="inconsistent"):
        formats.read_freq_file(str(p), 8)
