"""yamc_realspace_sums_static, the allocation-free entry point, through the C ABI.

Its sums must agree with the engine's own yamc_full_sums (uu_ew, uu_lj6, uu_lj12 of the
8 energy numbers) within the plain method's tolerance, 1e-10 * max(|ref|, 1 kT), on two
calls in a row that share the static scratch: a 6,220-atom system and then a 768-atom one,
so the second call runs over partial sums left behind by the first.  The intra-molecular
parts (sums 3-5) and the per-atom energies and forces are checked against the oracle's full
sum with the same tolerance.  The device arrays are made by torch, which stands for the
caller's own memory pool; the entry point itself allocates nothing: the device's free memory
(cudaMemGetInfo) is the same before and after a call.

The file name sorts last so that pytest runs it after the other tests; it also passes
alone in a fresh process (its first call does the per-device set-up).
"""
import ctypes
import math

import numpy as np
import pytest

from yamc_b200 import _lib, api

TOL = 1e-10


def _close(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)) <= TOL * np.maximum(np.abs(b), 1.0)


def lj_types(sigma, eps):
    """LJTypes_fill + the Lorentz-Berthelot tables (LJTypes.f90:134-308), as the caller
    of the entry point holds them: types by first appearance, sigma below 1e-8 has no LJ."""
    ts, te = [], []
    typ = np.zeros(sigma.size, dtype=np.int32)
    small = float(np.float32(1e-8))
    for i in range(sigma.size):
        if sigma[i] < small:
            continue
        for t in range(len(ts)):
            if abs(sigma[i] - ts[t]) < 1e-8 and abs(eps[i] - te[t]) < 1e-8:
                typ[i] = t + 1
                break
        else:
            ts.append(float(sigma[i]))
            te.append(float(eps[i]))
            typ[i] = len(ts)
    nt = len(ts)
    s6 = np.zeros(max(nt * nt, 1))
    fe = np.zeros(max(nt * nt, 1))
    for i in range(nt):
        for j in range(nt):
            s12, e12 = (ts[i], te[i]) if i == j else ((ts[i] + ts[j]) / 2, math.sqrt(te[i] * te[j]))
            s2 = s12 * s12
            s6[i * nt + j] = s2 * s2 * s2
            fe[i * nt + j] = 4 * e12
    return typ, nt, s6, fe


def molecule_ids(inp):
    mol = np.zeros(inp.natom, dtype=np.int32)
    for m, (f, l) in enumerate(zip(inp.first_atom, inp.last_atom)):
        mol[f - 1:l] = m
    return mol


def static_sums(inp):
    """One call of yamc_realspace_sums_static on device copies of the inputs."""
    import torch
    dev = torch.device("cuda:0")
    d = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a)).to(device=dev, dtype=dt)
    typ, nt, s6, fe = lj_types(inp.sigma, inp.epsilon)
    ins = [d(inp.x, torch.float64), d(inp.y, torch.float64), d(inp.z, torch.float64), d(inp.charge, torch.float64),
           d(molecule_ids(inp), torch.int32), d(typ, torch.int32), d(inp.hard_core, torch.float64)]
    tabs = [d(s6, torch.float64), d(fe, torch.float64)]
    n = inp.natom
    outs = [torch.full((n,), float("nan"), dtype=torch.float64, device=dev) for _ in range(4)]
    sums = torch.full((8,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    free0 = torch.cuda.mem_get_info(dev)[0]
    st = lib.yamc_realspace_sums_static(ctypes.byref(inp.params), n, *[t.data_ptr() for t in ins], nt,
                                        *[t.data_ptr() for t in tabs], *[t.data_ptr() for t in outs],
                                        sums.data_ptr(), stream)
    _lib.check(st, "yamc_realspace_sums_static")
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(dev)[0]
    return sums.cpu().numpy(), [t.cpu().numpy() for t in outs], typ, free1 - free0


@pytest.mark.gpu
def test_static_sums_match_full_sums(spce_files, nacl_files):
    import pyoracle
    for files in (nacl_files, spce_files):  # larger system first: the second call reuses the scratch
        inp = api.load_inputs(files["parameters"], files["composition"], files["moltab"])
        eng = api.Engine(inp)
        e = eng.full_sums()  # the existing entry point
        sums, per_atom, typ, dfree = static_sums(inp)
        sums2, _, _, dfree2 = static_sums(inp)  # after a warm-up call: nothing left allocated either
        assert dfree2 == 0, dfree2
        assert np.array_equal(sums, sums2)
        assert _close(sums[:3], e[3:6]).all(), (sums[:3], e[3:6])
        assert sums[6] == 0.0 and sums[7] == 0.0
        o = pyoracle.Oracle(files)
        assert np.array_equal(typ, o.atoms()[4])
        intra = o.intra_sums()
        assert _close(sums[3:6], intra).all(), (sums[3:6], intra)
        for got, ref in zip(per_atom, o.uuF()):
            ok = _close(got, ref)
            assert ok.all(), (int(np.argmin(ok)), got[~ok][:3], ref[~ok][:3])
        eng.close()


def test_static_sums_rejects_oversize():
    """Sizes above the static scratch are refused before any device work."""
    lib = _lib.load()
    p = _lib.YamcParams()
    st = lib.yamc_realspace_sums_static(ctypes.byref(p), lib_max() + 1, *([None] * 7), 0, None, None,
                                        *([None] * 5), None)
    assert st == _lib.YAMC_ELIMITS
    assert b"262144" in lib.yamc_last_error_detail()


def lib_max():
    import re
    import os
    hdr = open(os.path.join(_lib.HERE, "..", "include", "yamc.h")).read()
    return int(re.search(r"#define YAMC_STATIC_MAX_ATOMS (\d+)", hdr).group(1))
