"""Benchmark: MC trial moves/s of YAMC's movemc path on B200.

Workload (default): 2048 SPC/E + 38 Na+ + 38 Cl- (6,220 atoms), L = 39.6 A,
alpha = 0.30/A, rc = 12 A, kmax = 12 (1,068 half-space / 3,796 signed k),
dispersion-Ewald LJ, unbiased moves (0.15 A ball, 0.15 rad), synthetic
jittered-lattice starts, gfortran random streams.  One step = one batch graph
launch that advances every chain of a GPU by --moves moves: as many independent
chains as the launch shapes keep resident (replicas only: a Markov chain does not
shard), the launch shape picked by the batch autotuner.

  value  moves/s of the mixed-precision form with the random streams already in
         HBM, CUDA events around each launch, L2 flushed (256 MB write) between
         steps; config.fp64 the plain FP64 form on the same batch, and the mixed
         form's dE, force and total-energy error against FP64
  e2e    the same through yamc_batch_run with the streams in pinned host memory,
         host->device copy of each step's stream windows and device->host read of
         every chain's energies inside the timed region
  blocks nacl4k_mixed_batch_vs_plain (4096 SPC/E + NaCl, mixed batched force-biased against
         the plain FP64 chain), batch_ragged_96 (96 ragged replicas), npt_run_mc
         (NPT run_mc with volume steps), cpu_baseline (the oracle on one core)
  --impl reference  the CPU restatement of the reference (oracle/, -O3) timed on
         the host cores: independent chains, one per core
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


# DRAM bytes per move of the chain kernel in the timed shape (mixed, streamed, cluster of 2 x 384
# threads) from the ncu capture of one 1,000-move launch on nacl1m (dram__bytes_read.sum +
# dram__bytes_write.sum = 1.094 MB), used for roofline.traffic
TRAFFIC_PER_MOVE = 1094.0


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


def algorithmic_flops_per_move(spec, nsigned, ntype):
    """Floating-point work of an unbiased move at least: real-space pairs at the old and the
    new positions (2 n_m N_nb pairs at 60 flop each, sqrt/exp/divide counted as one) and the
    k-space energy, S (2 n_m 14 + 6 (1 + T^2)) flop; n_m = mean atoms of a chosen molecule."""
    nnb = spec.natom / spec.box ** 3 * 4.0 / 3.0 * math.pi * spec.rc ** 3
    n_m = spec.natom / spec.nmol
    return 2 * n_m * nnb * 60 + nsigned * (2 * n_m * 14 + 6 * (1 + ntype * ntype))


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
    buf = grng.gfortran_stream(seed, 40 * moves + 10000)
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
    vals = []
    with ctx.Pool(cores) as pool:
        for w in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = pool.map(_ref_worker, [(files, 1000 + 97 * c + w, moves) for c in range(cores)])
            dt = time.perf_counter() - t0
            if w >= args.warmup:
                vals.append(sum(m for m, _ in res) / dt)
    value = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "moves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * moves * cores / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": spec_name, "moves_per_chain_per_step": moves, "chains": cores},
            "cpu_baseline": {"value": value, "unit": "moves/s", "cores": cores, "kind": "port",
                             "sample": f"{cores} independent chains x {moves} moves per step, C restatement of "
                                       f"the reference (-O3), no Fortran compiler on this image"},
            "e2e": {"value": value, "unit": "moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def target_block(local, rank, moves=2000, steps=3, warmup=2):
    """The north-star comparison on 4096 SPC/E + 76 Na + 76 Cl (12,440 atoms, L = 50 A,
    alpha = 0.28/A, rc = 12 A, kmax = 15, the configuration of force-biased moves): one plain FP64
    chain (the drop-in) with the configuration's force-biased moves, and one with unbiased moves,
    against a batch of mixed-precision force-biased chains (lambda = 0.1), all resident at once,
    with the mixed chains' dE against FP64 chains on the same random stream."""
    import torch
    from yamc_b200 import _lib, api, rng as grng, systems
    dev = f"cuda:{local}"
    spec_b = systems.WORKLOADS["nacl4k"]                      # force-biased, lambda = 0.1
    spec_p = systems.SystemSpec(**{**spec_b.__dict__, "name": "nacl4k_plain", "xlambda": 0.0})
    base = f"/tmp/yamc_bench_target_r{rank}_{os.getpid()}"
    fp = systems.write_system(spec_p, base + "_plain", seed=5)
    per_move = 40
    # one plain FP64 chain
    eng = api.Engine.from_files(fp, device=local)
    s0 = torch.from_numpy(grng.gfortran_stream(99, per_move * moves * (steps + warmup) + 10000)).to(dev)
    cur = 0
    ms = []
    for w in range(warmup + steps):
        cur, done, st = eng.run_chain_device(s0.data_ptr(), s0.numel(), moves, cursor=cur)
        assert st == 0 and done == moves
        if w >= warmup:
            ms.append(eng.last_kernel_ms)
    plain = moves * steps / (sum(ms) / 1e3)
    plain_launch = eng.launch
    eng.close()
    del s0
    # dE of mixed vs FP64 force-biased chains on the same stream
    fb = systems.write_system(spec_b, base + "_b0", seed=5)
    # one plain FP64 chain with the configuration's own move set (force-biased, lambda = 0.1)
    eng = api.Engine.from_files(fb, device=local)
    s1 = torch.from_numpy(grng.gfortran_stream(98, 60 * moves * (steps + warmup) + 10000)).to(dev)
    cur = 0
    ms = []
    for w in range(warmup + steps):
        cur, done, st = eng.run_chain_device(s1.data_ptr(), s1.numel(), moves, cursor=cur)
        assert st == 0 and done == moves
        if w >= warmup:
            ms.append(eng.last_kernel_ms)
    plain_fb = moves * steps / (sum(ms) / 1e3)
    plain_fb_launch = eng.launch
    eng.close()
    del s1
    n_chk = 1500
    chk = grng.gfortran_stream(4243, 60 * n_chk + 10000)
    logs = {}
    for prec in (_lib.YAMC_FP64, _lib.YAMC_MIXED):
        e = api.Engine.from_files(fb, device=local, precision=prec)
        logs[prec] = e.run_chain(chk, n_chk)[0]
        e.close()
    lf, lm = logs[_lib.YAMC_FP64], logs[_lib.YAMC_MIXED]
    same = (lf["imol"] == lm["imol"]) & (lf["flags"] == lm["flags"]) & (lf["cursor"] == lm["cursor"])
    k = n_chk if same.all() else int(np.argmin(same))
    cols = ("du_real", "du_k_coul", "du_k_lj", "du_ext")
    de = np.abs(sum(lm[c][:k] for c in cols) - sum(lf[c][:k] for c in cols)) if k else np.zeros(1)
    # the mixed force-biased batch: as many chains as one shape keeps resident
    inp0 = api.load_inputs(fb["parameters"], fb["composition"], fb["moltab"])
    probe = api.Batch([inp0], device=local, precision=_lib.YAMC_MIXED)
    R = 1
    for G in range(1, 17):
        try:
            probe.set_launch(G, 0)
        except Exception:
            continue
        R = max(R, probe.launch["resident_clusters"])
    probe.close()
    R = min(R, 148)
    files = [fb] + [systems.write_system(spec_b, f"{base}_b{r}", seed=5 + 13 * r, rng_seed=777 + r) for r in range(1, R)]
    b = api.Batch([api.load_inputs(f["parameters"], f["composition"], f["moltab"]) for f in files], device=local,
                  precision=_lib.YAMC_MIXED)
    ds = [torch.from_numpy(grng.gfortran_stream(1000 + r, per_move * moves * (steps + warmup + 1) + 10000)).to(dev)
          for r in range(R)]
    ptrs, nr = [t.data_ptr() for t in ds], [t.numel() for t in ds]
    curs = np.zeros(R, dtype=np.int64)
    b.tune(ptrs, nr, curs, 200)
    ms = []
    for w in range(warmup + steps):
        done, st, s_all = b.run_device(ptrs, nr, curs, moves)
        assert s_all == 0 and (done == moves).all(), (s_all, done)
        if w >= warmup:
            ms.append(b.last_kernel_ms)
    batched = R * moves * steps / (sum(ms) / 1e3)
    out = {"workload": "nacl4k: 4096 SPC/E + 76 Na + 76 Cl, 12440 atoms, L=50 A, alpha=0.28/A, rc=12 A, kmax=15",
           "plain_fp64_one_chain": {"value": plain, "unit": "moves/s", "launch": plain_launch,
                                    "moves": "unbiased"},
           "plain_fp64_one_chain_force_biased": {"value": plain_fb, "unit": "moves/s", "launch": plain_fb_launch,
                                                 "moves": "force-biased, lambda = 0.1 (the configuration's move set)"},
           "mixed_batched_force_biased": {"value": batched, "unit": "moves/s", "chains": R, "launch": b.launch,
                                          "lambda": 0.1},
           # the target's ratio, the same move set on both sides; and against the unbiased plain chain
           "ratio": batched / plain_fb,
           "ratio_vs_unbiased_plain": batched / plain,
           "de_error_mixed_vs_fp64_force_biased": {"max_kT": float(de.max()), "moves_compared": k},
           "moves_per_step_per_chain": moves, "steps": steps}
    b.close()
    return out


def ragged_batch_block(local, rank, n_replicas=96, moves=10000):
    """Ragged replicas (water log-uniform 216..4096, NaCl 0..2 M, density 0.0334 +- 2 %, T 280..360 K,
    alpha = 5.6/L, cutoff min(12 A, L/2), one k-set), mixed precision, force-biased (lambda = 0.1),
    all in one batch: one graph launch per kernel-variant group, launch shape from the autotuner,
    `moves` trial moves per replica.  dE of the mixed form against FP64 on two replicas."""
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
    # mixed against FP64 on the smallest and the largest replica, same random stream
    de = []
    natoms = [inp.natom for inp in inputs]
    for i in (int(np.argmin(natoms)), int(np.argmax(natoms))):
        chk = grng.gfortran_stream(6000 + i, 60 * 1000 + 10000)
        logs = []
        for prec in (_lib.YAMC_FP64, _lib.YAMC_MIXED):
            e = api.Engine(inputs[i], device=local, precision=prec)
            logs.append(e.run_chain(chk, 1000)[0])
            e.close()
        lf, lm = logs
        same = (lf["imol"] == lm["imol"]) & (lf["flags"] == lm["flags"]) & (lf["cursor"] == lm["cursor"])
        k = 1000 if same.all() else int(np.argmin(same))
        cols = ("du_real", "du_k_coul", "du_k_lj", "du_ext")
        if k:
            de.append(float(np.abs(sum(lm[c][:k] for c in cols) - sum(lf[c][:k] for c in cols)).max()))
    return {"workload": f"{n_replicas} ragged replicas: water 216..4096 (log-uniform), NaCl 0..2 M, T 280..360 K, "
                        f"alpha = 5.6/L, kmax {specs[0].kmax}; {min(natoms)}..{max(natoms)} atoms",
            "method": "mixed precision, force-biased (lambda = 0.1), one batch", "moves_per_replica": moves,
            "value": n_replicas * moves / (ms / 1e3), "unit": "moves/s", "ms": ms, "launch": launch,
            "de_error_vs_fp64_max_kT": max(de) if de else None}


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--moves", type=int, default=20000, help="moves per step")
    ap.add_argument("--workload", default="nacl1m")
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--ref-moves", type=int, default=1500)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--replicas", type=int, default=0, help="chains per GPU (0 = as many clusters as are resident)")
    ap.add_argument("--no-target", action="store_true", help="skip the 4096-water mixed/batched/force-biased block")
    ap.add_argument("--no-ragged", action="store_true", help="skip the 96 ragged replicas block")
    ap.add_argument("--no-npt", action="store_true", help="skip the NPT run_mc block")
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
    n_steps = args.warmup + args.steps
    per_move = 16  # upper bound of random numbers per unbiased move (about 11 on average)
    n_stream = per_move * args.moves * (2 * n_steps + 2) + 100000
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def l2_flush():
        flush.fill_(1.0)
        torch.cuda.synchronize()

    # ---------------- one chain alone: the latency of the move, FP64 and mixed (beside the batch)
    def single_chain(precision):
        eng = api.Engine.from_files(files, device=local, precision=precision)
        s0 = grng.gfortran_stream(replica_seeds(rank, 0)[1], per_move * args.moves * 3 + 100000)
        d_s0 = torch.from_numpy(s0).to(dev)
        c0, _, _ = eng.run_chain_device(d_s0.data_ptr(), d_s0.numel(), args.moves)
        ms = []
        for _ in range(2):
            l2_flush()
            c0, done, st = eng.run_chain_device(d_s0.data_ptr(), d_s0.numel(), args.moves, cursor=c0)
            assert st == 0 and done == args.moves
            ms.append(eng.last_kernel_ms)
        out = {"moves_per_s": args.moves / (np.mean(ms) / 1e3), "launch": eng.launch}
        eng.close()
        return out

    single = {"fp64": single_chain(_lib.YAMC_FP64), "mixed": single_chain(_lib.YAMC_MIXED)}

    # ---------------- dE of the mixed form against the FP64 form, move by move on the same stream
    # (both chains take the same decisions until a draw falls within the dE error of its
    # threshold; the comparison runs up to there)
    n_chk = 4000
    chk = grng.gfortran_stream(4242 + rank, 40 * n_chk + 10000)
    logs = {}
    e_tot = {}
    for prec in (_lib.YAMC_FP64, _lib.YAMC_MIXED):
        eng = api.Engine.from_files(files, device=local, precision=prec)
        logs[prec] = eng.run_chain(chk, n_chk)[0]
        if prec == _lib.YAMC_MIXED:
            # the mixed chain's running total energy against an FP64 recomputation of its own configuration
            e_tot = {"incremental": float(eng.energies()[0]), "fp64_full": float(eng.full_sums()[0])}
        eng.close()
    lf, lm = logs[_lib.YAMC_FP64], logs[_lib.YAMC_MIXED]
    same = (lf["imol"] == lm["imol"]) & (lf["flags"] == lm["flags"]) & (lf["cursor"] == lm["cursor"])
    k_same = n_chk if same.all() else int(np.argmin(same))
    cols = ("du_real", "du_k_coul", "du_k_lj", "du_ext")
    de = np.abs(sum(lm[c][:k_same] for c in cols) - sum(lf[c][:k_same] for c in cols))
    # molecular forces of the force-bias path (movemc Steps 3-4) in both forms, same configuration
    ef = api.Engine.from_files(files, device=local, precision=_lib.YAMC_FP64)
    em = api.Engine.from_files(files, device=local, precision=_lib.YAMC_MIXED)
    ferr, fscale, nf = 0.0, 0.0, 0
    for imol in range(1, ef.nmol + 1, max(1, ef.nmol // 200)):
        f1, t1 = ef.move_old(imol)
        f2, t2 = em.move_old(imol)
        fscale = max(fscale, float(np.abs(f1).max()))
        ferr = max(ferr, float(np.abs(f2 - f1).max()))
        nf += 1
    ef.close()
    em.close()
    de_err = {"max_kT": float(de.max()) if k_same else None, "rms_kT": float(np.sqrt((de ** 2).mean())) if k_same else None,
              "moves_compared": k_same, "bar_kT": 1e-4,
              "force_max_abs_err": ferr, "force_scale": fscale, "molecules_compared": nf,
              "total_energy_err_kT": abs(e_tot["incremental"] - e_tot["fp64_full"]),
              "total_energy_kT": e_tot["fp64_full"]}

    # ---------------- the batch: R independent chains of the workload, one graph launch per step
    # R = the most chains any launch shape keeps resident at once (the tuner then picks the shape)
    probe = api.Batch([api.load_inputs(files["parameters"], files["composition"], files["moltab"])], device=local)
    R = args.replicas
    resident = {}
    for G in range(1, 17):
        try:
            probe.set_launch(G, 0)
        except Exception:
            continue
        resident[G] = probe.launch["resident_clusters"]
    if not R:
        R = min(148, max(resident.values(), default=1))
    probe.close()
    R = max(R, 1)
    rep_files = [files] + [systems.write_system(spec, f"{wdir}_{r}", seed=replica_seeds(rank, r)[0],
                                                rng_seed=replica_seeds(rank, r)[1]) for r in range(1, R)]
    rep_inputs = [api.load_inputs(f["parameters"], f["composition"], f["moltab"]) for f in rep_files]
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
    launch_fp64 = b64.launch
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
    log, _, _, _, _ = b.run(host, 2000, cursors=ecur, log=True)
    p_acc = float(np.mean(log["flags"] & 1))
    v0 = views[0]
    bpm = algorithmic_bytes_per_move(spec, v0.nk, v0.nsigned, v0.ntype, p_acc)
    ms_launch = float(np.mean(kernel_ms))
    moves_launch = R * args.moves
    achieved = bpm * moves_launch / (ms_launch / 1e3) / 1e9
    peak, which = peaks()
    fpm = algorithmic_flops_per_move(spec, v0.nsigned, v0.ntype)
    fp_achieved = fpm * moves_launch / (ms_launch / 1e3) / 1e12
    p64, p32 = api.fma_peak(local, True), api.fma_peak(local, False)
    launch = b.launch
    line = {
        "metric": METRIC, "value": value, "unit": "moves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (mixed)", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {spec.n_water} SPC/E + {spec.n_na} Na + {spec.n_cl} Cl, "
                               f"{spec.natom} atoms, L={spec.box} A, alpha={spec.alpha}/A, rc={spec.rc} A, "
                               f"kmax={spec.kmax}",
                   "method": "mixed precision (FP32 phases, k-space terms and pair exp; FP64 rho, sums, "
                             "Metropolis; FP64 rho refresh every 1e4 accepted moves), unbiased moves",
                   "fp64": {"value": value_fp64, "unit": "moves/s", "launch": launch_fp64},
                   "mixed_over_fp64": value / value_fp64,
                   "de_error_vs_fp64": de_err,
                   "moves_per_step_per_chain": args.moves, "chains_per_gpu": R,
                   "parallelism": "independent replicas (one cluster per chain)",
                   "launch": launch, "l2": "256 MB write between steps", "accept_fraction": p_acc,
                   "single_chain": single, "resident_clusters_by_cluster_size": resident},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": TRAFFIC_PER_MOVE * moves_launch, "peak_source": which,
                     "algorithmic_bytes_per_move": bpm,
                     "fp_pipe": {"algorithmic_flops_per_move": fpm, "achieved_tflops": fp_achieved,
                                 "fp64_fma_peak_tflops": p64, "fp32_fma_peak_tflops": p32,
                                 "frac_of_fp64": fp_achieved / p64, "frac_of_fp32": fp_achieved / p32,
                                 "peak_source": "measured live (yamc_fma_peak)"}},
        "e2e": {"value": e2e, "unit": "moves/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(sum(launch_counts)),
        "clocks": clk.summary(),
    }
    if not args.no_target:
        line["nacl4k_mixed_batch_vs_plain"] = target_block(local, rank)
    if not args.no_ragged:
        line["batch_ragged_96"] = ragged_batch_block(local, rank)
    if not args.no_npt:
        line["npt_run_mc"] = npt_block(local, rank)
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(files)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
