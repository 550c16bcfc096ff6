"""The adjoint (yamc_forces) against central finite differences of the energy and against the
reference's forces.

Finite differences of rigid-body moves: for a molecule, the energy change of a translation by
+-h (h = 1e-5 A) along each axis and of a rotation by +-theta (1e-5 rad) about each axis
through the centre of mass, each evaluated directly as dE by yamc_move_eval (no difference of
two large totals), give -F and -tau of the molecule.  A step where some pair distance crosses
the cutoff or a boundary of erfc_Luc's pieces (alpha r = 0.455 or 3) is skipped: the energy
jumps there, so no derivative exists.  Bar: |F_fd - F_adj| <= 1e-6 |F_adj| + 1e-9 F_rms
(likewise for tau), on 64 seeded configurations of a small SPC/E + NaCl box, on 64 seeded
configurations of 4096 SPC/E + 76 Na + 76 Cl in a 50 A box (the force-biased configuration:
waters and both ion species sampled in each) and on 256 SPC/E.  Single-atom differences of the
total energy through the torch.autograd wrapper check the per-atom forces, intra-molecular terms
included, with the same bar (the floor scaled to the gradient's rms).

The per-move forces of the force-biased proposal (yamc_move_old, the reference's formula of
movemc Steps 3-4) equal the oracle's to 1e-11 of the force scale, molecule by molecule, at the
start and after a force-biased chain has moved the molecules: the 1e-8 drift of long
force-biased chains comes from summation order, not from a different force.

The reference's own forces (the oracle's movemc Steps 3-4) take the real-space Coulomb force
from the exact erfc derivative while the energy uses erfc_Luc; the adjoint differentiates
erfc_Luc, so the two agree to the accuracy of erfc_Luc's derivative (bar 2e-4 relative to the
force scale) while the k-space and external parts agree exactly."""
import math

import numpy as np
import pytest
import torch

import pyoracle
from yamc_b200 import api, systems
from yamc_b200.autograd import total_energy

pytestmark = pytest.mark.gpu

H_ANG = 1e-5
THETA = 1e-5


def _minimg(d):
    return np.where(d > 0.5, d - 1.0, np.where(d < -0.5, d + 1.0, d))


def _bounds(p):
    a = p.alpha  # alpha * L: box units
    return [p.rmax2, (3.0 / a) ** 2, (0.455 / a) ** 2]


def _crosses(pos, sel, A, B, bounds):
    """Does any pair (molecule atom, other atom) cross a bound between positions A and B?"""
    other = np.ones(len(pos), bool)
    other[sel] = False
    P = pos[other]
    for a in range(len(sel)):
        ra = ((_minimg(A[a] - P)) ** 2).sum(1)
        rb = ((_minimg(B[a] - P)) ** 2).sum(1)
        for b in bounds:
            if np.any((ra - b) * (rb - b) <= 0):
                return True
    return False


def _rot(axis, ang):
    k = np.zeros(3); k[axis] = 1.0
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + math.sin(ang) * K + (1 - math.cos(ang)) * K @ K


def _de(eng, imol, xyz):
    eng.move_old(imol)
    du, ov, _, _ = eng.move_eval(imol, xyz[:, 0], xyz[:, 1], xyz[:, 2])
    eng.move_commit(False)
    return None if ov else float(du[0] + (du[1] + du[2]) + du[3])


def rigid_fd_check(eng, inp, mols, tol=1e-6):
    """Returns (worst force error, worst torque error, checks done), errors relative to the bar."""
    p = inp.params
    L = p.BoxLength
    bounds = _bounds(p)
    x, y, z = eng.positions()
    pos = np.stack([x, y, z], 1)
    _, mf, mt = eng.forces()
    frms = math.sqrt((mf ** 2).sum(1).mean())
    trms = math.sqrt((mt ** 2).sum(1).mean())
    worst_f = worst_t = 0.0
    n = 0
    h = H_ANG / L
    for imol in mols:
        a0, a1 = inp.first_atom[imol - 1] - 1, inp.last_atom[imol - 1]
        sel = np.arange(a0, a1)
        X = pos[sel]
        m = inp.mass[sel]
        com = (m[:, None] * X).sum(0) / m.sum()
        for d in range(3):
            e = np.zeros(3); e[d] = h
            Xp, Xm = X + e, X - e
            if not _crosses(pos, sel, Xp, Xm, bounds):
                dp, dm = _de(eng, imol, Xp), _de(eng, imol, Xm)
                if dp is not None and dm is not None:
                    f_fd = -(dp - dm) / (2 * h)
                    err = abs(f_fd - mf[imol - 1, d]) / (tol * abs(mf[imol - 1, d]) + 1e-9 * frms)
                    worst_f = max(worst_f, err); n += 1
            if len(sel) > 1:
                Rp, Rm = _rot(d, THETA), _rot(d, -THETA)
                Xp, Xm = com + (X - com) @ Rp.T, com + (X - com) @ Rm.T
                if not _crosses(pos, sel, Xp, Xm, bounds):
                    dp, dm = _de(eng, imol, Xp), _de(eng, imol, Xm)
                    if dp is not None and dm is not None:
                        t_fd = -(dp - dm) / (2 * THETA)
                        err = abs(t_fd - mt[imol - 1, d]) / (tol * abs(mt[imol - 1, d]) + 1e-9 * trms)
                        worst_t = max(worst_t, err); n += 1
    return worst_f, worst_t, n


def _inputs(files):
    return api.load_inputs(files["parameters"], files["composition"], files["moltab"])


def test_rigid_fd_64_configurations(tmp_path):
    """64 seeded configurations of 24 SPC/E + 2 Na + 2 Cl: every molecule, every axis."""
    total = 0
    for seed in range(64):
        d = tmp_path / f"c{seed}"
        d.mkdir()
        files = systems.write_system(systems.small_spec(), str(d), seed=100 + seed)
        inp = _inputs(files)
        try:
            eng = api.Engine(inp)
        except Exception:  # a seed whose start has a hard-core overlap
            continue
        wf, wt, n = rigid_fd_check(eng, inp, range(1, inp.nmol + 1))
        assert wf <= 1.0 and wt <= 1.0, (seed, wf, wt)
        total += n
        eng.close()
    assert total > 64 * 100


def test_rigid_fd_64_configurations_nacl4k(tmp_path):
    """64 seeded configurations of 4096 SPC/E + 76 Na + 76 Cl (L = 50 A, kmax 15): in each, two
    waters, one Na and one Cl, every axis."""
    spec = systems.WORKLOADS["nacl4k"]
    total, ions = 0, 0
    for seed in range(64):
        d = tmp_path / f"n{seed}"
        d.mkdir()
        files = systems.write_system(spec, str(d), seed=1000 + seed)
        inp = _inputs(files)
        eng = api.Engine(inp)
        rng = np.random.default_rng(seed)
        nw = spec.n_water
        mols = [int(v) for v in rng.choice(np.arange(1, nw + 1), 2, replace=False)]
        mols += [int(rng.integers(nw + 1, nw + spec.n_na + 1)), int(rng.integers(nw + spec.n_na + 1, inp.nmol + 1))]
        wf, wt, n = rigid_fd_check(eng, inp, mols)
        assert wf <= 1.0 and wt <= 1.0, (seed, mols, wf, wt)
        total += n
        eng.close()
    assert total >= 64 * 10, total


@pytest.mark.parametrize("which,nmols", [("spce_files", 40), ("nacl4k_files", 24)])
def test_rigid_fd_large(which, nmols, request):
    files = request.getfixturevalue(which)
    inp = _inputs(files)
    eng = api.Engine(inp)
    rng = np.random.default_rng(7)
    mols = list(rng.choice(np.arange(1, inp.nmol + 1), nmols, replace=False))
    if which == "nacl4k_files":  # the ions are the last 152 molecules
        mols += list(range(inp.nmol - 3, inp.nmol + 1))
    wf, wt, n = rigid_fd_check(eng, inp, mols)
    assert n >= 4 * nmols
    assert wf <= 1.0 and wt <= 1.0, (wf, wt)


def test_autograd_single_atom_fd(tiny_files):
    """Per-atom gradient through torch.autograd (backward = the adjoint) against central
    differences of the total energy, intra-molecular terms included."""
    inp = _inputs(tiny_files)
    eng = api.Engine(inp)
    p = inp.params
    x, y, z = eng.positions()
    pos0 = np.stack([x, y, z], 1)
    pos = torch.tensor(pos0, dtype=torch.float64, requires_grad=True)
    E = total_energy(eng, pos)
    E.backward()
    grad = pos.grad.numpy()
    grms = math.sqrt((grad ** 2).mean())
    h = H_ANG / p.BoxLength
    bounds = _bounds(p)
    rng = np.random.default_rng(3)
    done = 0
    for i in rng.choice(len(pos0), 20, replace=False):
        for d in range(3):
            e = np.zeros(3); e[d] = h
            A, B = pos0[i] + e, pos0[i] - e
            # every other atom, the own molecule's too
            P = np.delete(pos0, i, axis=0)
            ra = (_minimg(A - P) ** 2).sum(1); rb = (_minimg(B - P) ** 2).sum(1)
            if any(np.any((ra - b) * (rb - b) <= 0) for b in bounds):
                continue
            Pp, Pm = pos0.copy(), pos0.copy()
            Pp[i] += e; Pm[i] -= e
            ep = eng.set_positions(Pp[:, 0], Pp[:, 1], Pp[:, 2])[0]
            em = eng.set_positions(Pm[:, 0], Pm[:, 1], Pm[:, 2])[0]
            g_fd = (ep - em) / (2 * h)
            assert abs(g_fd - grad[i, d]) <= 1e-6 * abs(grad[i, d]) + 1e-9 * grms, (i, d, g_fd, grad[i, d])
            done += 1
    assert done >= 40
    eng.set_positions(pos0[:, 0], pos0[:, 1], pos0[:, 2])


@pytest.mark.parametrize("which", ["tiny_files", "nacl4k_files"])
def test_adjoint_vs_reference_forces(which, request):
    files = request.getfixturevalue(which)
    inp = _inputs(files)
    eng = api.Engine(inp)
    o = pyoracle.Oracle(files)
    _, mf, mt = eng.forces()
    frms = math.sqrt((mf ** 2).sum(1).mean())
    trms = math.sqrt((mt ** 2).sum(1).mean())
    rng = np.random.default_rng(5)
    for imol in rng.choice(np.arange(1, inp.nmol + 1), min(40, inp.nmol), replace=False):
        f, t = o.move_old(int(imol))
        assert np.all(np.abs(f - mf[imol - 1]) <= 2e-4 * frms), (imol, f, mf[imol - 1])
        assert np.all(np.abs(t - mt[imol - 1]) <= 2e-4 * trms), (imol, t, mt[imol - 1])


@pytest.mark.parametrize("which", ["tiny_biased_files", "nacl4k_files"])
def test_move_old_forces_match_oracle(which, request):
    """The force-biased proposal's old-position forces (yamc_move_old) against the oracle's
    movemc Steps 3-4, molecule by molecule: at the start, and after 300 force-biased chain moves
    on the same random stream (the same decisions, so the same configuration to rounding)."""
    from yamc_b200 import rng as grng
    files = request.getfixturevalue(which)
    o = pyoracle.Oracle(files)
    eng = api.Engine.from_files(files, extra="xlambda_f=0.1,xlambda_c=0.1")
    o2 = pyoracle.Oracle(files, extra="xlambda_f=0.1,xlambda_c=0.1")
    buf = grng.gfortran_stream(606, 60000)
    for stage in range(2):
        if stage == 1:
            glog, _, _, done, st = eng.run_chain(buf, 300)
            olog, _, _ = o2.run_mc(buf, 300)
            assert st == 0 and done == 300 and np.array_equal(glog["flags"], olog["flags"])
            o = o2
        rng = np.random.default_rng(21 + stage)
        mols = rng.choice(np.arange(1, o.nmol + 1), min(60, o.nmol), replace=False)
        fs, ts, fg, tg = [], [], [], []
        for imol in mols:
            f_o, t_o = o.move_old(int(imol))
            f_g, t_g = eng.move_old(int(imol))
            eng.move_commit(False)
            fs.append(f_o); ts.append(t_o); fg.append(f_g); tg.append(t_g)
        fs, ts, fg, tg = (np.array(v) for v in (fs, ts, fg, tg))
        frms = math.sqrt((fs ** 2).sum(1).mean())
        trms = math.sqrt((ts ** 2).sum(1).mean())
        assert np.abs(fg - fs).max() <= 1e-11 * frms, (stage, np.abs(fg - fs).max() / frms)
        assert np.abs(tg - ts).max() <= 1e-11 * trms, (stage, np.abs(tg - ts).max() / trms)
    eng.close()
