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
