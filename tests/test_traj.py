"""Trajectory writers (store_traj_frame, runmc.f90:373-417): atom positions -> molecule centres and
ZYZ angles (MoleculeTable_calcPositionsOrientations, MoleculeTable.f90:707-769) -> the moltab
binary.  Round trip through the library's own reader (MoleculeTable_fillAtomicData): a frame of
randomly rotated and displaced molecules, written and read back, gives the same atom positions to
the resolution of the 3-byte fixed-point format; frames.dat and boxlength.dat rows have the
reference's fixed format."""
import os

import numpy as np

from yamc_b200 import api, formats, systems


def _rot(axis, ang):
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K


def test_traj_frame_round_trip(tmp_path):
    files = systems.write_system(systems.small_spec(), str(tmp_path / "sys"), seed=4)
    inp = api.load_inputs(files["parameters"], files["composition"], files["moltab"])
    L = inp.params.BoxLength
    d = os.path.dirname(files["composition"])
    templates = [formats.read_mol_template(os.path.join(d, n)) for n in ("SPCE.mol", "Na_Dang.mol", "Cl_Dang.mol")]
    species = np.repeat(np.arange(3), inp.mol_numbers)
    # rotate every water about its centre of mass and move every molecule a little
    r = np.random.default_rng(2)
    x, y, z = inp.x.copy(), inp.y.copy(), inp.z.copy()
    for m in range(len(inp.first_atom)):
        a, b = inp.first_atom[m] - 1, inp.last_atom[m]
        cx, cy, cz = formats._center_of_mass(x[a:b], y[a:b], z[a:b], inp.mass[a:b])
        R = _rot(r.normal(size=3), r.uniform(0, np.pi))
        rel = np.stack([x[a:b] - cx, y[a:b] - cy, z[a:b] - cz])
        new = R @ rel
        shift = r.uniform(-0.01, 0.01, 3)
        c = (np.array([cx, cy, cz]) + shift + 0.5) % 1.0 - 0.5
        x[a:b], y[a:b], z[a:b] = new[0] + c[0], new[1] + c[1], new[2] + c[2]
    frame = formats.traj_frame(x, y, z, inp.first_atom, inp.last_atom, species, templates, L)
    traj = str(tmp_path / "traj.moltraj")
    formats.append_moltab(traj, *frame)
    formats.append_moltab(traj, *frame)  # a second frame is appended, not overwritten
    assert os.path.getsize(traj) == 2 * len(inp.first_atom) * 18
    # read the first frame back through the library's readers
    one = str(tmp_path / "one.moltab")
    formats.write_moltab(one, *frame)
    back = api.load_inputs(files["parameters"], files["composition"], one)
    err = max(np.abs(back.x - x).max(), np.abs(back.y - y).max(), np.abs(back.z - z).max()) * L
    assert err < 2e-5, err  # Angstrom: 3-byte positions and angles
    th, ph, ps = frame[3:]
    assert np.all((th >= 0) & (th <= np.pi)) and np.all((ph >= 0) & (ph < 2 * np.pi)) and np.all((ps >= 0) & (ps < 2 * np.pi))


def test_frames_and_boxlength_rows():
    row = formats.format_frames_row(7, 39.6012345678, 21240, 12345, 3, 1, 0, 0, 1700000000)
    assert len(row) == 12 + 15 + 6 * 12 + 12
    assert row[:12] == "           7" and row[12:27] == "  39.6012345678"
    assert row[27:39] == "      21240."
    vals = row.replace(".", " ").split()
    assert vals[0] == "7" and vals[-1] == "1700000000"
    b = formats.format_boxlength_row(3, 39.6)
    assert b.split() == ["3", "39.6"]


def test_force_dump_float_format(tmp_path):
    """write_float / read_float (FloatingPoint.f90): known encodings and the round-trip precision
    of a 23-bit mantissa; a frame written with append_forces reads back."""
    assert formats.float_bits(1.0) == (0, 128)            # m = 1, n = 0 (exponent sign bit set for n <= 0)
    assert formats.float_bits(-2.0) == (2 ** 23, 1)       # negative mantissa, n = 1
    assert formats.float_bits(0.0) == (0, 255)            # below 1e-14: the underflow code, read back as 0
    assert formats.float_value(*formats.float_bits(0.0)) == 0.0
    r = np.random.default_rng(1)
    for v in np.concatenate([r.normal(size=200) * 10.0 ** r.integers(-8, 8, 200), [1.0, -1.0, 0.5, 3.0]]):
        back = formats.float_value(*formats.float_bits(float(v)))
        assert abs(back - v) <= 2.0 ** -22 * abs(v), (v, back)
    f = r.normal(size=(5, 3)) * 100
    path = str(tmp_path / "forces.ftraj")
    formats.append_forces(path, f[:, 0], f[:, 1], f[:, 2], 20.0)
    formats.append_forces(path, f[:, 0], f[:, 1], f[:, 2], 20.0)
    back = formats.read_forces(path, 5)
    assert back.shape == (2, 5, 3)
    assert np.all(np.abs(back[1] - f / 20.0) <= 2.0 ** -22 * np.abs(f / 20.0))


import pytest  # noqa: E402


@pytest.mark.gpu
def test_force_dump_of_adjoint_forces(tmp_path, nacl_files):
    """mc_calc_forces' dump, fixed: the adjoint forces of yamc_forces (every pair once, no r = 0
    self pair) written frame by frame with store_forces' format and read back."""
    eng = api.Engine.from_files(nacl_files)
    path = str(tmp_path / "forces.ftraj")
    L = eng.inputs.params.BoxLength
    f, _, _ = eng.forces()
    formats.append_forces(path, f[:, 0], f[:, 1], f[:, 2], L)
    back = formats.read_forces(path, eng.natom)[0]
    assert np.all(np.isfinite(f))
    assert np.all(np.abs(back - f / L) <= 2.0 ** -22 * np.abs(f / L) + 1e-300)
