"""Benchmark: MC trial moves/s of YAMC's movemc path on B200.

Workload (default, the force-biased configuration the metric's target is stated on): 4096
SPC/E + 76 Na+ + 76 Cl- (12,440 atoms), L = 50 A, alpha = 0.28/A, rc = 12 A, kmax = 15 (2,045
half-space / 7,427 signed k), dispersion-Ewald LJ, force-biased moves (lambda = 0.1 for force
and torque, 0.15 A / 0.15 rad), synthetic jittered-lattice starts, gfortran random streams.
One step = one batch graph launch that advances every chain of a GPU by --moves moves: as many
independent chains as the launch shapes keep resident (replicas only: a Markov chain does not
shard), the launch shape picked by the batch autotuner.

  value   moves/s of the mixed-precision form with the random streams already in HBM, CUDA
          events around each launch, L2 flushed (256 MB write) between steps
  config  fp64_batched: the same chains and shape search in FP64 (mixed_over_fp64_batched);
          plain_fp64_one_chain: the FP64 drop-in, one chain alone, the same move set
          (target_ratio = value over it, target 5); the mixed form's dE, force and
          total-energy error against FP64 (precision_errors_vs_fp64)
  e2e     the same through yamc_batch_run with the streams in pinned host memory, host->device
          copy of each step's stream windows and device->host read of every chain's energies
          inside the timed region
  configs the other configurations of the metric, each with its plain FP64 chain, mixed and
          FP64 batches and precision errors: spce256 (256 SPC/E), nacl1m (2048 SPC/E + NaCl,
          unbiased), nacl16k (16384 SPC/E + NaCl, force-biased), batch_ragged_96 (96 ragged
          replicas in one batch), npt_run_mc (NPT run_mc with volume steps), per_move_drop_in
          (host latency of the per-move C ABI: movemc split as a Fortran host calls it)
  cpu_baseline  the oracle (-O3 C restatement of the reference) on one host core, a bounded
          sample of the same workload
  --impl reference  the CPU restatement of the reference (oracle/, -O3) timed on the host
          cores: independent chains, one per core
"""
from __future__ import annotations

import argparse
import contextlib
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MC trial moves/s (SPC/E+NaCl Ewald); mixed vs FP64 GPU at |ΔE err|≤1e-4 kT"


# DRAM bytes per move of the chain kernel in the timed shape, by workload, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum of one launch / its moves; profiles/), used for
# roofline.traffic: nacl1m mixed streamed 2 x 384 threads, 1,000 moves: 1.102 MB; nacl4k mixed
# force-biased streamed 3 x 384 threads, one chain, 400 moves: 2.088 MB
TRAFFIC_PER_MOVE = {"nacl1m": 1102.0, "nacl4k": 5222.0}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float, device) -> float:
    """The largest of every rank's x (the job's time is its slowest rank's); x itself at N = 1."""
    ws, _, _ = dist_env()
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seeds(rank: int, r: int):
    """(initial-configuration seed, random-stream seed) of chain r on rank `rank`: distinct for
    every (rank, chain) of the job, so replicas are independent across GPUs too."""
    return 3 + 1000 * rank + r, 12345 + 100000 * rank + 7 * r


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes_per_move(spec, nk, nsigned, ntype, p_acc):
    """Bytes a move must move at least (the per-move accounting of the design notes):
    real-space neighbours (old + new positions, 3 sites share most neighbours: 1.3x),
    40 B per neighbour atom; rho(k) read; beta tables; k indices; accepted rho write."""
    L = spec.box
    natom = spec.natom
    nnb = natom / L ** 3 * 4.0 / 3.0 * math.pi * spec.rc ** 3
    real = 2 * 1.3 * nnb * 40
    rho = (1 + ntype) * 2 * nsigned * 8
    beta = (1 + ntype * (ntype + 1) / 2) * nk * 8
    kidx = 12 * nk
    commit = p_acc * (1 + ntype) * 2 * nsigned * 8
    return real + rho + beta + kidx + commit


def algorithmic_flops_per_move(spec, nsigned, ntype, forces=False):
    """Floating-point work of a move at least: real-space pairs at the old and the new positions
    (2 n_m N_nb pairs at 60 flop each, sqrt/exp/divide counted as one) and the k-space energy,
    S (2 n_m 14 + 6 (1 + T^2)) flop; a force-biased move adds the k-space forces at both
    positions, S 2 n_m (6 + 6 T).  n_m = mean atoms of a chosen molecule."""
    nnb = spec.natom / spec.box ** 3 * 4.0 / 3.0 * math.pi * spec.rc ** 3
    n_m = spec.natom / spec.nmol
    f = 2 * n_m * nnb * 60 + nsigned * (2 * n_m * 14 + 6 * (1 + ntype * ntype))
    if forces:
        f += nsigned * 2 * n_m * (6 + 6 * ntype)
    return f


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = open(f"/tmp/yamc_clocks_{os.getpid()}.csv", "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.out:
            self.out.close()

    def summary(self):
        path = f"/tmp/yamc_clocks_{os.getpid()}.csv"
        try:
            rows = [l.strip().split(",") for l in open(path) if l.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if "Active" in v and "Not" not in v:
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_baseline(files, seconds=12.0):
    """The oracle's -O3 build on one host core: a bounded sample of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from yamc_b200 import rng as grng
    o = pyoracle.Oracle(files, fast=True)
    buf = grng.gfortran_stream(12345, 2_000_000)
    cur = 0
    done = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        _, _, cur = o.run_mc(buf, 500, cursor=cur)
        done += 500
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "moves/s", "cores": 1, "kind": "port",
            "sample": f"{done} moves of the same workload from its initial configuration, one chain, "
                      f"C restatement of the reference built -O3 (oracle/liboracle_fast.so)"}


def _ref_worker(args):
    files, seed, moves = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from yamc_b200 import rng as grng
    o = pyoracle.Oracle(files, fast=True)
    buf = grng.gfortran_stream(seed, 60 * moves + 10000)
    t0 = time.perf_counter()
    o.run_mc(buf, moves)
    return moves, time.perf_counter() - t0


def run_reference(args, files, spec_name):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    moves = args.ref_moves
    ctx = mp.get_context("spawn")
    # each step: one chain per core, each built (initmc: the full sums) and then timed over its
    # moves alone; the step's rate is the sum of the chains' rates (every core busy throughout)
    vals = []
    with ctx.Pool(cores) as pool:
        for w in range(args.warmup + args.steps):
            res = pool.map(_ref_worker, [(files, 1000 + 97 * c + w, moves) for c in range(cores)])
            if w >= args.warmup:
                vals.append(sum(m / t for m, t in res))
    value = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "moves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * moves * cores / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": spec_name, "moves_per_chain_per_step": moves, "chains": cores},
            "cpu_baseline": {"value": value, "unit": "moves/s", "cores": cores, "kind": "port",
                             "sample": f"{cores} independent chains x {moves} moves per step (each chain's moves "
                                       f"timed after its initmc; the chains' rates summed), C restatement of "
                                       f"the reference (-O3), no Fortran compiler on this image"},
            "e2e": {"value": value, "unit": "moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _files_for(spec, tag, rank, r):
    """Input files of chain r of a workload (distinct seeds for every rank and chain)."""
    from yamc_b200 import systems
    seed, rng_seed = replica_seeds(rank, r)
    return systems.write_system(spec, f"/tmp/yamc_bench_{tag}_r{rank}_{os.getpid()}_{r}", seed=seed, rng_seed=rng_seed)


def _resident_chains(inp, local, precision):
    """The most chains of this system any launch shape keeps resident at once."""
    from yamc_b200 import api
    probe = api.Batch([inp], device=local, precision=precision)
    resident = {}
    for G in range(1, 17):
        try:
            probe.set_launch(G, 0)
        except Exception:
            continue
        resident[G] = probe.launch["resident_clusters"]
    probe.close()
    return min(148, max(resident.values(), default=1)), resident


def single_chain_rate(files, local, precision, moves, per_move, reps=2, extra=""):
    """One chain alone (the plain drop-in: no batching), device-resident stream, CUDA-event time."""
    import torch
    from yamc_b200 import api, rng as grng
    eng = api.Engine.from_files(files, extra=extra, device=local, precision=precision)
    s0 = torch.from_numpy(grng.gfortran_stream(99, per_move * moves * (reps + 1) + 10000)).to(f"cuda:{local}")
    cur, done, st = eng.run_chain_device(s0.data_ptr(), s0.numel(), moves)
    assert st == 0 and done == moves, (st, done)
    ms = []
    for _ in range(reps):
        cur, done, st = eng.run_chain_device(s0.data_ptr(), s0.numel(), moves, cursor=cur)
        assert st == 0 and done == moves, (st, done)
        ms.append(eng.last_kernel_ms)
    out = {"value": moves / (np.mean(ms) / 1e3), "unit": "moves/s", "launch": eng.launch}
    eng.close()
    return out


def precision_errors(files, local, n_chk=1500, n_force=200, seed=4242):
    """The mixed form against FP64 on one system (its dE, force and total-energy errors, stated
    for every result): a mixed and an FP64 chain on the same random stream, compared move
    by move up to their first different decision; the molecular forces of the force-bias path
    (yamc_move_old, movemc Steps 3-4) of both forms on the same configuration; the mixed chain's
    running total energy against an FP64 recomputation of its own configuration."""
    from yamc_b200 import _lib, api, rng as grng
    chk = grng.gfortran_stream(seed, 60 * n_chk + 10000)
    logs, e_tot = {}, {}
    for prec in (_lib.YAMC_FP64, _lib.YAMC_MIXED):
        eng = api.Engine.from_files(files, device=local, precision=prec)
        logs[prec] = eng.run_chain(chk, n_chk)[0]
        if prec == _lib.YAMC_MIXED:
            e_tot = {"incremental": float(eng.energies()[0]), "fp64_full": float(eng.full_sums()[0])}
        eng.close()
    lf, lm = logs[_lib.YAMC_FP64], logs[_lib.YAMC_MIXED]
    same = (lf["imol"] == lm["imol"]) & (lf["flags"] == lm["flags"]) & (lf["cursor"] == lm["cursor"])
    k = n_chk if same.all() else int(np.argmin(same))
    cols = ("du_real", "du_k_coul", "du_k_lj", "du_ext")
    de = np.abs(sum(lm[c][:k] for c in cols) - sum(lf[c][:k] for c in cols)) if k else np.zeros(1)
    ef = api.Engine.from_files(files, device=local, precision=_lib.YAMC_FP64)
    em = api.Engine.from_files(files, device=local, precision=_lib.YAMC_MIXED)
    ferr, fscale, nf = 0.0, 0.0, 0
    for imol in range(1, ef.nmol + 1, max(1, ef.nmol // n_force)):
        f1, _ = ef.move_old(imol)
        ef.move_commit(False)
        f2, _ = em.move_old(imol)
        em.move_commit(False)
        fscale = max(fscale, float(np.abs(f1).max()))
        ferr = max(ferr, float(np.abs(f2 - f1).max()))
        nf += 1
    ef.close()
    em.close()
    return {"de_max_kT": float(de.max()), "de_rms_kT": float(np.sqrt((de ** 2).mean())), "moves_compared": k,
            "bar_kT": 1e-4, "force_max_abs_err": ferr, "force_scale": fscale,
            "force_rel_err": ferr / max(fscale, 1e-300), "molecules_compared": nf,
            "total_energy_err_kT": abs(e_tot["incremental"] - e_tot["fp64_full"]),
            "total_energy_kT": e_tot["fp64_full"], "mixed_chain_moves": n_chk}


def batch_rates(spec, tag, local, rank, moves, steps, warmup, per_move, precisions, chains=0, tune_moves=200):
    """As many independent chains of a workload as one launch shape keeps resident, run as one
    batch (one graph launch per step), for each precision: moves/s over `steps` timed steps
    (CUDA events on the batch stream, L2 flushed between steps)."""
    import torch
    from yamc_b200 import _lib, api, rng as grng
    dev = f"cuda:{local}"
    f0 = _files_for(spec, tag, rank, 0)
    inp0 = api.load_inputs(f0["parameters"], f0["composition"], f0["moltab"])
    R = chains or _resident_chains(inp0, local, _lib.YAMC_MIXED)[0]
    files = [f0] + [_files_for(spec, tag, rank, r) for r in range(1, R)]
    inputs = [inp0] + [api.load_inputs(f["parameters"], f["composition"], f["moltab"]) for f in files[1:]]
    ds = [torch.from_numpy(grng.gfortran_stream(replica_seeds(rank, r)[1], per_move * moves * (steps + warmup + 1)
                                                + 10000)).to(dev) for r in range(R)]
    ptrs, nr = [t.data_ptr() for t in ds], [t.numel() for t in ds]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    out = {"chains": R}
    for prec in precisions:
        b = api.Batch(inputs, device=local, precision=prec)
        cur = np.zeros(R, dtype=np.int64)
        b.tune(ptrs, nr, cur, tune_moves)
        ms = []
        for w in range(warmup + steps):
            done, st, s_all = b.run_device(ptrs, nr, cur, moves)
            assert s_all == 0 and (done == moves).all(), (s_all, done)
            if w >= warmup:
                ms.append(b.last_kernel_ms)
            flush.fill_(1.0)
        torch.cuda.synchronize()
        name = "mixed" if prec == _lib.YAMC_MIXED else "fp64"
        out[name] = {"value": R * moves * steps / (sum(ms) / 1e3), "unit": "moves/s", "launch": b.groups}
        b.close()
    del ds
    return out, files[0]


def ragged_batch_block(local, rank, n_replicas=96, moves=10000):
    """Ragged replicas (water log-uniform 216..4096, NaCl 0..2 M, density 0.0334 +- 2 %, T 280..360 K,
    alpha = 5.6/L, cutoff min(12 A, L/2), one k-set), mixed precision, force-biased (lambda = 0.1),
    all in one batch: one graph launch per kernel-variant group, launch shape from the autotuner,
    `moves` trial moves per replica.  The mixed form's dE, force and total-energy error against
    FP64 on the smallest and the largest replica."""
    import torch
    from yamc_b200 import _lib, api, rng as grng, systems
    dev = f"cuda:{local}"
    specs = systems.batch_specs(n_replicas, seed=7)
    base = f"/tmp/yamc_bench_c4_r{rank}_{os.getpid()}"
    files = [systems.write_system(sp, f"{base}_{i}", seed=11 + i, rng_seed=900 + i) for i, sp in enumerate(specs)]
    inputs = [api.load_inputs(f["parameters"], f["composition"], f["moltab"]) for f in files]
    b = api.Batch(inputs, device=local, precision=_lib.YAMC_MIXED)
    per_move = 40
    ds = [torch.from_numpy(grng.gfortran_stream(5000 + i, per_move * (moves + 400) + 10000)).to(dev)
          for i in range(n_replicas)]
    ptrs, nr = [t.data_ptr() for t in ds], [t.numel() for t in ds]
    cur = np.zeros(n_replicas, dtype=np.int64)
    b.tune(ptrs, nr, cur, 200)
    done, st, s_all = b.run_device(ptrs, nr, cur, 200)  # warm-up
    done, st, s_all = b.run_device(ptrs, nr, cur, moves)
    assert s_all == 0 and (done == moves).all(), (s_all, done)
    ms = b.last_kernel_ms
    launch = b.groups
    b.close()
    # the mixed form against FP64 on the smallest and the largest replica: dE on the same random
    # stream, forces and the running total energy
    natoms = [inp.natom for inp in inputs]
    errs = {}
    for tag, i in (("smallest", int(np.argmin(natoms))), ("largest", int(np.argmax(natoms)))):
        errs[tag] = {"atoms": natoms[i], **precision_errors(files[i], local, n_chk=1000, n_force=100, seed=6000 + i)}
    return {"workload": f"{n_replicas} ragged replicas: water 216..4096 (log-uniform), NaCl 0..2 M, T 280..360 K, "
                        f"alpha = 5.6/L, kmax {specs[0].kmax}; {min(natoms)}..{max(natoms)} atoms",
            "method": "mixed precision, force-biased (lambda = 0.1), one batch", "moves_per_replica": moves,
            "value": n_replicas * moves / (ms / 1e3), "unit": "moves/s", "ms": ms, "launch": launch,
            "precision_errors_vs_fp64": errs}


def npt_block(local, rank, cycles=12):
    """NPT run_mc on nacl1m as the reference's own parameters.prm runs it (a volume step on
    average once every pressure_step_multiplier + 1 = 6 cycles), through yamc_run_mc: move
    cycles as chain-kernel launches, volume steps as a host-built box rescale plus the full
    sums on the device.  Reported: moves/s over the whole run and the mean time of a volume
    step (host clock; both include the volume steps' host work)."""
    from yamc_b200 import api, rng as grng, systems
    base = f"/tmp/yamc_bench_npt_r{rank}_{os.getpid()}"
    files = systems.write_system(systems.WORKLOADS["nacl1m"], base, seed=3)
    extra = "pressure_step_multiplier=5,max_volume_scaling=1.002,pressure=100000"
    eng = api.Engine.from_files(files, extra=extra, device=local)
    buf = grng.gfortran_stream(4242, 40 * 2124 * (cycles + 2) + 100000)
    log, vlog, _, cur, done, st = eng.run_mc(buf, 2)  # warm-up (kernel shape, first launch)
    t0 = time.perf_counter()
    log, vlog, _, cur, done, st = eng.run_mc(buf, cycles, cursor=cur)
    t = time.perf_counter() - t0
    assert st == 0 and done == cycles, (st, done)
    L = eng.current_params().BoxLength
    tv = []
    for k in range(6):
        t1 = time.perf_counter()
        eng.volume_eval(L * (1.0 + 0.0005 * (1 if k % 2 else -1)))
        eng.volume_commit(False)
        tv.append(time.perf_counter() - t1)
    t2 = time.perf_counter()
    eng.full_sums()
    t_full = time.perf_counter() - t2
    eng.close()
    return {"workload": "nacl1m (6220 atoms), NPT: pressure 1 bar, pressure_step_multiplier 5, "
                        "max_volume_scaling 1.002, FP64, unbiased moves",
            "cycles": cycles, "volume_steps": int(len(vlog)), "volume_accepted": int((vlog["flags"] & 1).sum()),
            "moves": int(len(log)), "moves_per_s": len(log) / t, "wall_s": t,
            "volume_step_ms": 1e3 * float(np.median(tv)), "full_sums_ms": 1e3 * t_full,
            "box_length_A": L}


def per_move_block(local, rank, n=300):
    """The per-move drop-in (yamc_move_old + yamc_move_eval + yamc_move_commit, movemc split as a
    Fortran host calls it) on nacl1m, FP64: host-clock latency per move of n moves of random
    waters, each displaced by 1e-3 box units and rejected, called through ctypes with every
    argument built before the timed loop (the median and the parts' medians)."""
    import ctypes
    from yamc_b200 import api, systems
    base = f"/tmp/yamc_bench_pm_r{rank}_{os.getpid()}"
    files = systems.write_system(systems.WORKLOADS["nacl1m"], base, seed=3)
    eng = api.Engine.from_files(files, device=local)
    lib, h = eng.lib, eng.h
    x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in eng.positions())
    rs = np.random.default_rng(0)
    mols = rs.integers(1, 2049, size=n)
    new = [tuple(np.ascontiguousarray(v[3 * (m - 1):3 * m] + (1e-3 if k == 0 else 0.0)) for k, v in enumerate((x, y, z)))
           for m in mols]
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    f, t, du = np.zeros(3), np.zeros(3), np.zeros(4)
    pf, pt, pdu = dp(f), dp(t), dp(du)
    ov = ctypes.c_int32(0)
    pov = ctypes.byref(ov)
    args = [(int(m), dp(a), dp(b), dp(c)) for m, (a, b, c) in zip(mols, new)]
    for m, pa, pb, pc in args[:20]:  # warm-up
        lib.yamc_move_old(h, m, pf, pt); lib.yamc_move_eval(h, m, pa, pb, pc, pdu, pov, pf, pt); lib.yamc_move_commit(h, 0)
    to, te, tc = [], [], []
    clk = time.perf_counter
    for m, pa, pb, pc in args:
        t0 = clk()
        r0 = lib.yamc_move_old(h, m, pf, pt)
        t1 = clk()
        r1 = lib.yamc_move_eval(h, m, pa, pb, pc, pdu, pov, pf, pt)
        t2 = clk()
        r2 = lib.yamc_move_commit(h, 0)
        t3 = clk()
        assert r0 == r1 == r2 == 0, (r0, r1, r2)
        to.append(t1 - t0); te.append(t2 - t1); tc.append(t3 - t2)
    eng.close()
    med = lambda v: 1e6 * float(np.median(v))
    tot = [a + b + c for a, b, c in zip(to, te, tc)]
    return {"workload": "nacl1m (6220 atoms), FP64, one water per move, rejected",
            "calls": "yamc_move_old + yamc_move_eval + yamc_move_commit through ctypes, arguments prebuilt",
            "moves": n, "us_per_move_median": med(tot), "old_us": med(to), "eval_us": med(te), "commit_us": med(tc)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--moves", type=int, default=4000, help="moves per chain per step")
    ap.add_argument("--workload", default="nacl4k")
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--ref-moves", type=int, default=300)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--replicas", type=int, default=0, help="chains per GPU (0 = as many clusters as are resident)")
    ap.add_argument("--no-blocks", action="store_true",
                    help="skip the other configurations (spce256, nacl1m, nacl16k, 96 ragged replicas, NPT)")
    args = ap.parse_args()

    from yamc_b200 import systems
    ws, rank, local = dist_env()
    spec = systems.WORKLOADS[args.workload]
    wdir = f"/tmp/yamc_bench_{args.workload}_r{rank}_{os.getpid()}"
    files = systems.write_system(spec, wdir, seed=replica_seeds(rank, 0)[0], rng_seed=replica_seeds(rank, 0)[1])

    if args.impl == "reference":
        if ws > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=600))
        run_reference(args, files, args.workload)
        if ws > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    from yamc_b200 import _lib, api, rng as grng

    dev = f"cuda:{local}"
    biased = spec.xlambda > 0
    # random numbers per move, an upper bound (about 11 for an unbiased move, 20 for a force-biased one)
    per_move = 40 if biased else 16
    n_stream = per_move * args.moves * (2 * (args.warmup + args.steps) + 2) + 100000
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def l2_flush():
        flush.fill_(1.0)
        torch.cuda.synchronize()

    # ---------------- the plain drop-in: one FP64 chain alone, with the workload's own move set and
    # (force-biased workloads) with unbiased moves; one mixed chain
    single = {"fp64": single_chain_rate(files, local, _lib.YAMC_FP64, max(500, args.moves // 4), per_move),
              "mixed": single_chain_rate(files, local, _lib.YAMC_MIXED, max(500, args.moves // 4), per_move)}
    if biased:
        single["fp64_unbiased_moves"] = single_chain_rate(files, local, _lib.YAMC_FP64, max(500, args.moves // 4), 16,
                                                          extra="xlambda_f=0,xlambda_c=0")

    # ---------------- the mixed form's errors against FP64 (dE, force, total energy)
    de_err = precision_errors(files, local, n_chk=1500 if biased else 4000, seed=4242 + rank)

    # ---------------- the batch: R independent chains of the workload, one graph launch per step
    # R = the most chains any launch shape keeps resident at once (the tuner then picks the shape)
    inp0 = api.load_inputs(files["parameters"], files["composition"], files["moltab"])
    R, resident = _resident_chains(inp0, local, _lib.YAMC_MIXED)
    if args.replicas:
        R = args.replicas
    rep_files = [files] + [systems.write_system(spec, f"{wdir}_{r}", seed=replica_seeds(rank, r)[0],
                                                rng_seed=replica_seeds(rank, r)[1]) for r in range(1, R)]
    rep_inputs = [inp0] + [api.load_inputs(f["parameters"], f["composition"], f["moltab"]) for f in rep_files[1:]]
    streams = [grng.gfortran_stream(replica_seeds(rank, r)[1], n_stream) for r in range(R)]
    d_streams = [torch.from_numpy(x).to(dev) for x in streams]
    d_ptrs = [t.data_ptr() for t in d_streams]
    n_rng = [t.numel() for t in d_streams]

    def timed_batch(precision, clk=None):
        b = api.Batch(rep_inputs, device=local, precision=precision)
        cur = np.zeros(R, dtype=np.int64)
        b.tune(d_ptrs, n_rng, cur, max(200, args.moves // 20))
        for w in range(args.warmup):
            b.run_device(d_ptrs, n_rng, cur, args.moves)
            l2_flush()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ms, counts = [], []
        ctx = clk if clk is not None else contextlib.nullcontext()
        with ctx:
            for s in range(args.steps):
                done, st, s_all = b.run_device(d_ptrs, n_rng, cur, args.moves)
                assert s_all == 0 and (done == args.moves).all(), (s_all, done)
                ms.append(b.last_kernel_ms)
                counts.append(b.last_launches)
                l2_flush()
        torch.cuda.synchronize()
        t = max_over_ranks(sum(ms) / 1e3, dev)
        return b, cur, ms, t, counts

    b64, _, ms64, t64, _ = timed_batch(_lib.YAMC_FP64)
    value_fp64 = ws * R * args.steps * args.moves / t64
    launch_fp64 = b64.groups
    b64.close()
    clk = Clocks(local)
    b, cur, kernel_ms, t_dev, launch_counts = timed_batch(_lib.YAMC_MIXED, clk)
    value = ws * R * args.steps * args.moves / t_dev

    # ---------------- end to end through the C ABI with host buffers
    pinned = [torch.from_numpy(x).pin_memory() for x in streams]
    host = [x.numpy() for x in pinned]
    views = [b.replica(r) for r in range(R)]
    window = per_move * args.moves
    ecur = cur.copy()
    e_moves = 0
    h2d = 0
    for w in range(args.warmup):
        _, ecur, _, _, _ = b.run(host, args.moves, cursors=ecur, limits=ecur + window)
        l2_flush()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e_times = []
    run_slot = 80
    for s in range(args.steps):
        lim = np.minimum(ecur + window, [h.size for h in host])
        h2d = int(4 * (lim - ecur).sum()) + R * run_slot
        t0 = time.perf_counter()
        _, ecur, done, st, s_all = b.run(host, args.moves, cursors=ecur, limits=lim)
        energies = [v.energies() for v in views]
        e_times.append(time.perf_counter() - t0)
        assert s_all == 0 and (done == args.moves).all(), (s_all, done)
        e_moves += int(done.sum())
        l2_flush()
    t_e2e = max_over_ranks(sum(e_times), dev)
    e2e = ws * e_moves / t_e2e
    d2h = R * (run_slot + 8 * 17 + 8 * 2)  # run slot + engine scalars + counters per replica

    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    # ---------------- roofline of the chain kernel
    log, _, _, _, _ = b.run(host, 1000, cursors=ecur, log=True)
    p_acc = float(np.mean(log["flags"] & 1))
    v0 = views[0]
    bpm = algorithmic_bytes_per_move(spec, v0.nk, v0.nsigned, v0.ntype, p_acc)
    ms_launch = float(np.mean(kernel_ms))
    moves_launch = R * args.moves
    achieved = bpm * moves_launch / (ms_launch / 1e3) / 1e9
    peak, which = peaks()
    fpm = algorithmic_flops_per_move(spec, v0.nsigned, v0.ntype, biased)
    fp_achieved = fpm * moves_launch / (ms_launch / 1e3) / 1e12
    p64, p32 = api.fma_peak(local, True), api.fma_peak(local, False)
    launch = b.groups
    b.close()
    del d_streams
    torch.cuda.empty_cache()
    move_set = "force-biased moves (lambda = 0.1)" if biased else "unbiased moves"
    line = {
        "metric": METRIC, "value": value, "unit": "moves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (mixed)", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {spec.n_water} SPC/E + {spec.n_na} Na + {spec.n_cl} Cl, "
                               f"{spec.natom} atoms, L={spec.box} A, alpha={spec.alpha}/A, rc={spec.rc} A, "
                               f"kmax={spec.kmax}, {move_set}",
                   "method": "mixed precision (FP32 phases, k-space terms and pair exp; FP64 rho, sums, "
                             f"Metropolis; FP64 rho refresh every 1e4 accepted moves), {move_set}, "
                             "independent chains batched in one graph launch per step",
                   "fp64_batched": {"value": value_fp64, "unit": "moves/s", "launch": launch_fp64,
                                    "note": "the same chains, workload and shape search in FP64"},
                   "mixed_over_fp64_batched": value / value_fp64,
                   "plain_fp64_one_chain": single["fp64"],
                   "target_ratio": {"value": value / single["fp64"]["value"], "target": 5.0,
                                    "what": "mixed batched moves/s over the plain FP64 drop-in (one chain, the same "
                                            "move set)"},
                   "single_chain": single,
                   "precision_errors_vs_fp64": de_err,
                   "moves_per_step_per_chain": args.moves, "chains_per_gpu": R,
                   "parallelism": "independent replicas (one cluster per chain)",
                   "launch": launch, "l2": "256 MB write between steps", "accept_fraction": p_acc,
                   "resident_clusters_by_cluster_size": resident},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": which,
                     "algorithmic_bytes_per_move": bpm,
                     "fp_pipe": {"algorithmic_flops_per_move": fpm, "achieved_tflops": fp_achieved,
                                 "fp64_fma_peak_tflops": p64, "fp32_fma_peak_tflops": p32,
                                 "frac_of_fp64": fp_achieved / p64, "frac_of_fp32": fp_achieved / p32,
                                 "peak_source": "measured live (yamc_fma_peak)"}},
        "e2e": {"value": e2e, "unit": "moves/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(sum(launch_counts)),
        "clocks": clk.summary(),
    }
    tpm = TRAFFIC_PER_MOVE.get(args.workload)
    if tpm is not None:
        line["roofline"]["traffic"] = tpm * moves_launch
        line["roofline"]["traffic_note"] = "ncu DRAM bytes per move of the timed kernel shape x moves of one launch"
    blocks = {}
    if not args.no_blocks:
        blocks["spce256"] = config_block("spce256", local, rank, moves=10000, steps=3, warmup=2)
        blocks["nacl1m"] = config_block("nacl1m", local, rank, moves=10000, steps=3, warmup=2)
        blocks["nacl16k"] = config_block("nacl16k", local, rank, moves=300, steps=3, warmup=1)
        blocks["batch_ragged_96"] = ragged_batch_block(local, rank, moves=4000)
        blocks["npt_run_mc"] = npt_block(local, rank)
        blocks["per_move_drop_in"] = per_move_block(local, rank)
    line["configs"] = blocks
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(files)
    print(json.dumps(line), flush=True)


def config_block(name, local, rank, moves, steps, warmup):
    """One more configuration of the metric: its plain FP64 chain, the mixed and FP64 batches
    (as many chains as are resident at once) and the mixed form's errors against FP64."""
    from yamc_b200 import _lib, systems
    spec = systems.WORKLOADS[name]
    per_move = 40 if spec.xlambda > 0 else 16
    rates, f0 = batch_rates(spec, name, local, rank, moves, steps, warmup, per_move, (_lib.YAMC_FP64, _lib.YAMC_MIXED))
    one = single_chain_rate(f0, local, _lib.YAMC_FP64, max(200, moves // 4), per_move)
    out = {"workload": f"{name}: {spec.n_water} SPC/E + {spec.n_na} Na + {spec.n_cl} Cl, {spec.natom} atoms, "
                       f"L={spec.box} A, alpha={spec.alpha}/A, rc={spec.rc} A, kmax={spec.kmax}, "
                       + ("force-biased moves (lambda = 0.1)" if spec.xlambda > 0 else "unbiased moves"),
           "plain_fp64_one_chain": one, **rates,
           "mixed_over_fp64_batched": rates["mixed"]["value"] / rates["fp64"]["value"],
           "batched_mixed_over_plain_fp64": rates["mixed"]["value"] / one["value"],
           "moves_per_step_per_chain": moves, "steps": steps,
           "precision_errors_vs_fp64": precision_errors(f0, local, n_chk=400 if spec.natom > 20000 else 1500,
                                                        n_force=60 if spec.natom > 20000 else 200)}
    return out


if __name__ == "__main__":
    main()
