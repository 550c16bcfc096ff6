"""Radial distribution functions of molecule centres (mcrdf2.f90:110-440) on the GPU.

The oracle restates count_distances and save_rdfs; it is pinned here by a known answer (a simple
cubic lattice: 6, 12 and 8 neighbours at a, a*sqrt(2), a*sqrt(3)).  The GPU counts must equal the
oracle's exactly (integer histograms; the distance arithmetic is rounded like the oracle's) and
g(r) within 1e-12, for frames given as host centres (with and without periodic images beyond
L/2) and for frames taken from an engine's device-resident configuration after a chain run."""
import numpy as np
import pytest

import pyoracle
from yamc_b200 import formats, rng as grng


def _lattice(n, jitter=0.0, seed=0):
    g = (np.arange(n) + 0.5) / n - 0.5
    x, y, z = (v.ravel() for v in np.meshgrid(g, g, g, indexing="ij"))
    if jitter:
        r = np.random.default_rng(seed)
        x, y, z = (v + r.uniform(-jitter, jitter, v.size) / n for v in (x, y, z))
    return x, y, z


def test_oracle_rdf_lattice_known_answer(tmp_path):
    x, y, z = _lattice(4)
    M = x.size
    rdf = pyoracle.RDF(np.ones(M, dtype=np.int32), [M], dr=0.1, rmax=9.99)
    rdf.add_frame(x, y, z, 20.2)  # a = 5.05 A
    c = rdf.cnt4.reshape(1, 1, -1)[0, 0]
    a = 5.05
    for r, k in ((a, 6), (a * np.sqrt(2), 12), (a * np.sqrt(3), 8)):
        assert c[int(r / 0.1)] == k * M
    assert c.sum() == (6 + 12 + 8) * M
    g = rdf.g()
    r_axis = (np.arange(rdf.nbin) + 0.5) * 0.1
    paths = formats.write_rdf(str(tmp_path / "rdf"), r_axis, g)
    assert len(paths) == 1 and paths[0].endswith("rdf01_01.dat")
    back = np.loadtxt(paths[0])
    assert np.allclose(back[:, 1], g[0, 0], rtol=1e-15, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("box,rmax", [(30.0, 12.0), (9.0, 12.0)])  # no images / images up to 1 box away
def test_rdf_frames_match_oracle(box, rmax):
    from yamc_b200 import api
    x, y, z = _lattice(5, jitter=0.3, seed=1)
    M = x.size
    mol_type = np.where(np.arange(M) % 3 == 0, 2, 1).astype(np.int32)
    counts = np.array([(mol_type == 1).sum(), (mol_type == 2).sum()], dtype=np.int32)
    o = pyoracle.RDF(mol_type, counts, dr=0.1, rmax=rmax)
    gpu = api.RDF(mol_type, counts, dr=0.1, rmax=rmax)
    for f in range(3):
        xs, ys, zs = (np.mod(v + 0.07 * f + 0.5, 1.0) - 0.5 for v in (x, y, z))
        o.add_frame(xs, ys, zs, box * (1 + 0.01 * f))
        gpu.add_frame(xs, ys, zs, box * (1 + 0.01 * f))
    r, g, c, nf = gpu.result()
    assert nf == 3
    assert np.array_equal(c, o.cnt4.reshape(c.shape))
    go = o.g()
    assert np.all(np.abs(g - go) <= 1e-12 * np.maximum(np.abs(go), 1.0))
    gpu.close()


@pytest.mark.gpu
def test_rdf_from_engine_matches_oracle(nacl_files):
    from yamc_b200 import api
    eng = api.Engine.from_files(nacl_files)
    rdf = api.RDF.for_engine(eng)
    counts = np.asarray(eng.inputs.mol_numbers, dtype=np.int32)
    mol_type = np.repeat(np.arange(1, counts.size + 1, dtype=np.int32), counts)
    o = pyoracle.RDF(mol_type, counts)
    first, last = eng.inputs.first_atom - 1, eng.inputs.last_atom - 1
    mass = eng.inputs.mass
    buf = grng.gfortran_stream(3, 500000)
    cur = 0
    L = eng.inputs.params.BoxLength
    for f in range(2):
        _, _, cur, done, st = eng.run_chain(buf, 2000, cursor=cur, log=False)
        assert st == 0
        rdf.add_engine(eng)
        x, y, z = eng.positions()
        cx, cy, cz = (np.zeros(eng.nmol) for _ in range(3))
        for m in range(eng.nmol):  # center_of_mass in the oracle's order
            sx = sy = sz = tm = 0.0
            for a in range(first[m], last[m] + 1):
                sx = sx + mass[a] * x[a]; sy = sy + mass[a] * y[a]; sz = sz + mass[a] * z[a]; tm = tm + mass[a]
            cx[m], cy[m], cz[m] = sx / tm, sy / tm, sz / tm
        o.add_frame(cx, cy, cz, L)
    r, g, c, nf = rdf.result()
    assert nf == 2
    assert np.array_equal(c, o.cnt4.reshape(c.shape))
    go = o.g()
    assert np.all(np.abs(g - go) <= 1e-12 * np.maximum(np.abs(go), 1.0))
    # water O-O peak near 2.8 A
    k = int(np.argmax(g[0, 0]))
    assert 2.5 < r[k] < 3.2, r[k]
