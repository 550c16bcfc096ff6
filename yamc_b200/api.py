"""Host-side mirror of the reference's MC interface over the C ABI.

``Engine`` stands where the reference's MC module is: ``initmc`` (construction),
``mc_total_energy`` / ``mc_calc_total_sums`` (``energies`` / ``full_sums``), the
body of ``movemc`` split like the C ABI (``move_old`` / ``move_eval`` /
``move_commit``) and the device-resident ``run_mc`` loop (``run_chain``).
All arithmetic happens in libyamc_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from ._lib import MOVE_RECORD_DTYPE, YamcParams, YamcSystem, check

ENERGY_COLUMNS = ("U_total", "U_total_ew", "U_total_lj", "uu_ew", "uu_lj6", "uu_lj12", "E_k_coulomb", "E_k_lj")


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def read_parameters(path: str, extra: str = "") -> YamcParams:
    """Parameters_read (defaults + parameters.prm + "k=v,..." overrides)."""
    lib = _lib.load()
    p = YamcParams()
    check(lib.yamc_params_read(path.encode(), extra.encode(), ctypes.byref(p)), "yamc_params_read")
    return p


def params_init(p: YamcParams, nmol: int) -> YamcParams:
    lib = _lib.load()
    check(lib.yamc_params_init(ctypes.byref(p), int(nmol)), "yamc_params_init")
    return p


@dataclass
class Inputs:
    """A system as the reference host holds it after MoleculeTable_fillAtomicData."""
    params: YamcParams
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    charge: np.ndarray
    sigma: np.ndarray
    epsilon: np.ndarray
    hard_core: np.ndarray
    mass: np.ndarray
    first_atom: np.ndarray
    last_atom: np.ndarray
    mol_numbers: np.ndarray
    move_weights: Optional[np.ndarray] = None

    @property
    def natom(self) -> int:
        return int(self.x.size)

    @property
    def nmol(self) -> int:
        return int(self.first_atom.size)

    def as_struct(self) -> YamcSystem:
        s = YamcSystem()
        s.natom = self.natom
        s.nmol = self.nmol
        s.x, s.y, s.z = _dptr(self.x), _dptr(self.y), _dptr(self.z)
        s.charge, s.sigma, s.epsilon = _dptr(self.charge), _dptr(self.sigma), _dptr(self.epsilon)
        s.hard_core_angstr, s.mass = _dptr(self.hard_core), _dptr(self.mass)
        s.first_atom, s.last_atom = _iptr(self.first_atom), _iptr(self.last_atom)
        s.n_species = int(self.mol_numbers.size)
        s.mol_numbers = _iptr(self.mol_numbers)
        s.move_weights = _dptr(self.move_weights) if self.move_weights is not None else None
        return s


def load_inputs(parameters: str, composition: str, moltab: str, extra: str = "") -> Inputs:
    """The reference readers (composition, .mol, moltab, fillAtomicData) in the library."""
    lib = _lib.load()
    h = ctypes.c_void_p()
    check(lib.yamc_inputs_load(parameters.encode(), composition.encode(), moltab.encode(), extra.encode(),
                               ctypes.byref(h)), "yamc_inputs_load")
    try:
        s = YamcSystem()
        p = YamcParams()
        check(lib.yamc_inputs_get(h, ctypes.byref(s), ctypes.byref(p)), "yamc_inputs_get")
        n, m = s.natom, s.nmol
        cp = lambda ptr, k: np.ctypeslib.as_array(ptr, shape=(k,)).copy()
        return Inputs(p, cp(s.x, n), cp(s.y, n), cp(s.z, n), cp(s.charge, n), cp(s.sigma, n), cp(s.epsilon, n),
                      cp(s.hard_core_angstr, n), cp(s.mass, n), cp(s.first_atom, m).astype(np.int32),
                      cp(s.last_atom, m).astype(np.int32), cp(s.mol_numbers, s.n_species).astype(np.int32))
    finally:
        lib.yamc_inputs_free(h)


def fma_peak(device: int = 0, fp64: bool = True) -> float:
    """Measured FP64 (or FP32) FMA throughput of ``device`` in TFLOP/s (yamc_fma_peak)."""
    t = ctypes.c_double()
    check(_lib.load().yamc_fma_peak(int(device), 1 if fp64 else 0, ctypes.byref(t)), "yamc_fma_peak")
    return t.value


class Engine:
    """initmc + movemc + run_mc of one system on one GPU."""

    def __init__(self, inputs: Inputs, device: int = 0, precision: int = _lib.YAMC_FP64):
        self.lib = _lib.load()
        self.inputs = inputs
        p = YamcParams()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(inputs.params), ctypes.sizeof(YamcParams))
        p.precision = precision
        self.params = p
        self._sys = inputs.as_struct()
        h = ctypes.c_void_p()
        check(self.lib.yamc_create(ctypes.byref(self._sys), ctypes.byref(p), int(device), ctypes.byref(h)), "yamc_create")
        self.h = h
        sz = np.zeros(5, dtype=np.int32)
        check(self.lib.yamc_sizes(self.h, _iptr(sz)), "yamc_sizes")
        self.natom, self.nmol, self.nk, self.nsigned, self.ntype = (int(v) for v in sz)

    @classmethod
    def from_files(cls, files: dict, extra: str = "", device: int = 0, precision: int = _lib.YAMC_FP64) -> "Engine":
        return cls(load_inputs(files["parameters"], files["composition"], files["moltab"], extra), device, precision)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.yamc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- energies ---------------------------------------------------------------------------
    def energies(self) -> np.ndarray:
        e = np.zeros(8)
        check(self.lib.yamc_energies(self.h, _dptr(e)), "yamc_energies")
        return e

    def full_sums(self) -> np.ndarray:
        e = np.zeros(8)
        check(self.lib.yamc_full_sums(self.h, _dptr(e)), "yamc_full_sums")
        return e

    def positions(self):
        x, y, z = (np.zeros(self.natom) for _ in range(3))
        check(self.lib.yamc_get_positions(self.h, _dptr(x), _dptr(y), _dptr(z)), "yamc_get_positions")
        return x, y, z

    def set_positions(self, x, y, z) -> np.ndarray:
        """New atom positions (box units); full recompute; returns the 8 energy numbers."""
        x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
        e = np.zeros(8)
        check(self.lib.yamc_set_positions(self.h, _dptr(x), _dptr(y), _dptr(z), _dptr(e)), "yamc_set_positions")
        return e

    def forces(self):
        """Adjoint forces: (per-atom forces [natom, 3], molecular forces [nmol, 3], torques [nmol, 3])."""
        fx, fy, fz = (np.zeros(self.natom) for _ in range(3))
        mf, mt = np.zeros((self.nmol, 3)), np.zeros((self.nmol, 3))
        check(self.lib.yamc_forces(self.h, _dptr(fx), _dptr(fy), _dptr(fz), _dptr(mf), _dptr(mt)), "yamc_forces")
        return np.stack([fx, fy, fz], axis=1), mf, mt

    # -- per-move drop-in -------------------------------------------------------------------
    def move_old(self, imol: int):
        f, t = np.zeros(3), np.zeros(3)
        check(self.lib.yamc_move_old(self.h, int(imol), _dptr(f), _dptr(t)), "yamc_move_old")
        return f, t

    def move_eval(self, imol: int, xn, yn, zn):
        xn, yn, zn = (np.ascontiguousarray(v, dtype=np.float64) for v in (xn, yn, zn))
        du, f, t = np.zeros(4), np.zeros(3), np.zeros(3)
        ov = ctypes.c_int32(0)
        check(self.lib.yamc_move_eval(self.h, int(imol), _dptr(xn), _dptr(yn), _dptr(zn), _dptr(du), ctypes.byref(ov),
                                      _dptr(f), _dptr(t)), "yamc_move_eval")
        return du, bool(ov.value), f, t

    def move_commit(self, accepted: bool) -> None:
        check(self.lib.yamc_move_commit(self.h, 1 if accepted else 0), "yamc_move_commit")

    # -- device-resident run_mc -------------------------------------------------------------
    def run_chain(self, rng: np.ndarray, n_moves: int, cursor: int = 0, log: bool = True, max_rows: int = 0):
        """Runs n_moves movemc calls on the device.  Returns (log, rows, cursor, moves_done, status)."""
        rng = np.ascontiguousarray(rng, dtype=np.float32)
        cur = ctypes.c_int64(int(cursor))
        done = ctypes.c_int64(0)
        nrow = ctypes.c_int32(0)
        rec = np.zeros(n_moves if log else 0, dtype=MOVE_RECORD_DTYPE)
        rows = np.zeros((max(max_rows, 0), 9))
        st = self.lib.yamc_run_chain(self.h, rng.ctypes.data, rng.size, ctypes.byref(cur), int(n_moves), ctypes.byref(done),
                                     rec.ctypes.data if log else None, rows.ctypes.data if max_rows else None,
                                     int(max_rows), ctypes.byref(nrow))
        if st not in (_lib.YAMC_OK, _lib.YAMC_ERNG_EXHAUSTED, _lib.YAMC_ENAN):
            check(st, "yamc_run_chain")
        return rec[: done.value], rows[: nrow.value], cur.value, done.value, st

    def run_mc(self, rng: np.ndarray, n_cycles: int, cursor: int = 0, log: bool = True, max_rows: int = 0):
        """run_mc by cycles, NPT volume steps included (pressure_step_multiplier > 0).
        Returns (move log, volume log, rows, cursor, cycles_done, status)."""
        rng = np.ascontiguousarray(rng, dtype=np.float32)
        cur = ctypes.c_int64(int(cursor))
        done, nlog, nvlog = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        nrow = ctypes.c_int32(0)
        max_log = int(n_cycles) * self.nmol if log else 0
        rec = np.zeros(max(max_log, 1), dtype=MOVE_RECORD_DTYPE)
        vrec = np.zeros(max(int(n_cycles), 1), dtype=_lib.VOLUME_RECORD_DTYPE)
        rows = np.zeros((max(max_rows, 1), 9))
        st = self.lib.yamc_run_mc(self.h, rng.ctypes.data, rng.size, ctypes.byref(cur), int(n_cycles), ctypes.byref(done),
                                  rec.ctypes.data if log else None, max_log, ctypes.byref(nlog), vrec.ctypes.data,
                                  int(n_cycles), ctypes.byref(nvlog), rows.ctypes.data if max_rows else None,
                                  int(max_rows), ctypes.byref(nrow))
        if st not in (_lib.YAMC_OK, _lib.YAMC_ERNG_EXHAUSTED, _lib.YAMC_ENAN):
            check(st, "yamc_run_mc")
        return rec[: nlog.value], vrec[: nvlog.value], rows[: nrow.value], cur.value, done.value, st

    def volume_eval(self, new_box_length: float):
        """mcvol up to the acceptance test for a given new box length: (dU, overlap)."""
        du = ctypes.c_double(0)
        ov = ctypes.c_int32(0)
        check(self.lib.yamc_volume_eval(self.h, float(new_box_length), ctypes.byref(du), ctypes.byref(ov)),
              "yamc_volume_eval")
        return du.value, bool(ov.value)

    def volume_commit(self, accepted: bool) -> None:
        check(self.lib.yamc_volume_commit(self.h, int(bool(accepted))), "yamc_volume_commit")

    def set_xchange_weights(self, weights) -> None:
        """Exchange weights per molecule (the third column of a frequencies file)."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        if w.size != self.nmol:
            raise ValueError("one exchange weight per molecule")
        check(self.lib.yamc_set_xchange_weights(self.h, _dptr(w)), "yamc_set_xchange_weights")

    def xchange_eval(self, imol1: int, imol2: int):
        """mc_xchange up to the acceptance test: (du[4], overlap)."""
        du = np.zeros(4)
        ov = ctypes.c_int32(0)
        check(self.lib.yamc_xchange_eval(self.h, int(imol1), int(imol2), _dptr(du), ctypes.byref(ov)),
              "yamc_xchange_eval")
        return du, bool(ov.value)

    def xchange_commit(self, accepted: bool) -> None:
        check(self.lib.yamc_xchange_commit(self.h, int(bool(accepted))), "yamc_xchange_commit")

    def save_state(self, cursor: int = 0) -> bytes:
        """The context's exact state and the caller's stream cursor (yamc_save_state)."""
        n = ctypes.c_int64(0)
        check(self.lib.yamc_state_size(self.h, ctypes.byref(n)), "yamc_state_size")
        buf = ctypes.create_string_buffer(n.value)
        check(self.lib.yamc_save_state(self.h, int(cursor), buf, n.value), "yamc_save_state")
        return buf.raw

    def load_state(self, state: bytes) -> int:
        """Puts a saved state into this context (same system); returns the saved cursor."""
        cur = ctypes.c_int64(0)
        buf = ctypes.create_string_buffer(bytes(state), len(state))
        check(self.lib.yamc_load_state(self.h, buf, len(state), ctypes.byref(cur)), "yamc_load_state")
        return cur.value

    def current_params(self) -> "_lib.YamcParams":
        """The parameters as they stand now (BoxLength follows accepted volume steps)."""
        p = _lib.YamcParams()
        check(self.lib.yamc_get_params(self.h, ctypes.byref(p)), "yamc_get_params")
        return p

    def run_chain_device(self, d_rng_ptr: int, n_rng: int, n_moves: int, cursor: int = 0, d_log_ptr: int = 0):
        cur = ctypes.c_int64(int(cursor))
        done = ctypes.c_int64(0)
        nrow = ctypes.c_int32(0)
        st = self.lib.yamc_run_chain_device(self.h, ctypes.c_void_p(d_rng_ptr), int(n_rng), ctypes.byref(cur), int(n_moves),
                                            ctypes.byref(done), ctypes.c_void_p(d_log_ptr) if d_log_ptr else None, None, 0,
                                            ctypes.byref(nrow))
        if st not in (_lib.YAMC_OK, _lib.YAMC_ERNG_EXHAUSTED):
            check(st, "yamc_run_chain_device")
        return cur.value, done.value, st

    # -- launch control ---------------------------------------------------------------------
    def set_launch(self, cluster_blocks: int = 0, threads: int = 0) -> None:
        check(self.lib.yamc_set_launch(self.h, int(cluster_blocks), int(threads)), "yamc_set_launch")

    def set_refresh(self, accepted_moves: int) -> None:
        """Mixed form: FP64 recomputation of rho(k) every `accepted_moves` accepted moves."""
        check(self.lib.yamc_set_refresh(self.h, int(accepted_moves)), "yamc_set_refresh")

    @property
    def refresh_count(self) -> int:
        v = ctypes.c_int64(0)
        check(self.lib.yamc_refresh_count(self.h, ctypes.byref(v)), "yamc_refresh_count")
        return v.value

    def set_kspace_layout(self, layout: int) -> None:
        """_lib.YAMC_KSPACE_AUTO / _REGISTERS / _STREAMED"""
        check(self.lib.yamc_set_kspace_layout(self.h, int(layout)), "yamc_set_kspace_layout")

    @property
    def launch(self):
        out = np.zeros(4, dtype=np.int32)
        check(self.lib.yamc_get_launch(self.h, _iptr(out)), "yamc_get_launch")
        return {"cluster_blocks": int(out[0]), "threads": int(out[1]), "entries_per_thread": int(out[2]),
                "smem_bytes": int(out[3])}

    PHASES = ("choose", "speculate", "propose", "tables", "kspace", "pair_filter", "pairs", "reduce",
              "old_pass", "metropolis", "commit", "kspace_next")

    def phase_cycles(self, mode: int = 2) -> dict:
        out = np.zeros(len(self.PHASES), dtype=np.int64)
        check(self.lib.yamc_phase_cycles(self.h, int(mode), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                         out.size), "yamc_phase_cycles")
        return dict(zip(self.PHASES, (int(v) for v in out)))

    @property
    def last_kernel_ms(self) -> float:
        v = ctypes.c_double(0)
        check(self.lib.yamc_last_kernel_ms(self.h, ctypes.byref(v)), "yamc_last_kernel_ms")
        return v.value


class Batch:
    """Independent replicas advanced together (yamc_batch_*): one persistent cluster launch per
    kernel variant, the step replayed as a CUDA graph.  Each replica is its own system with its
    own random stream; ``replica(i)`` gives it as an Engine-like view."""

    def __init__(self, inputs: list, device: int = 0, precision: int = _lib.YAMC_FP64):
        self.lib = _lib.load()
        self.inputs = list(inputs)
        n = len(self.inputs)
        self._systems = (YamcSystem * n)()
        self._params = (YamcParams * n)()
        for i, inp in enumerate(self.inputs):
            self._systems[i] = inp.as_struct()
            ctypes.memmove(ctypes.byref(self._params[i]), ctypes.byref(inp.params), ctypes.sizeof(YamcParams))
            self._params[i].precision = precision
        h = ctypes.c_void_p()
        check(self.lib.yamc_batch_create(n, self._systems, self._params, int(device), ctypes.byref(h)), "yamc_batch_create")
        self.h = h
        self.n = n
        self._views = {}

    def close(self) -> None:
        if getattr(self, "h", None):
            self._views.clear()
            self.lib.yamc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def replica(self, i: int) -> "_ReplicaView":
        if i not in self._views:
            c = ctypes.c_void_p()
            check(self.lib.yamc_batch_replica(self.h, int(i), ctypes.byref(c)), "yamc_batch_replica")
            self._views[i] = _ReplicaView(self, c, self.inputs[i])
        return self._views[i]

    @staticmethod
    def _ptrs(addrs, sizes):
        p = (ctypes.c_void_p * len(addrs))(*[int(a) for a in addrs])
        n = np.ascontiguousarray(sizes, dtype=np.int64)
        return p, n

    def run(self, streams, n_moves: int, cursors=None, log: bool = False, limits=None):
        """n_moves moves of every replica, replica i reading host stream streams[i] (float32)
        from cursors[i] up to limits[i] (default: its end).  Returns (log[n, n_moves] or None,
        cursors, moves_done, status per replica, overall status)."""
        streams = [np.ascontiguousarray(s, dtype=np.float32) for s in streams]
        sizes = [s.size for s in streams] if limits is None else [min(int(l), s.size) for l, s in zip(limits, streams)]
        ptrs, n = self._ptrs([s.ctypes.data for s in streams], sizes)
        cur = np.zeros(self.n, dtype=np.int64) if cursors is None else np.array(cursors, dtype=np.int64)
        done = np.zeros(self.n, dtype=np.int64)
        st = np.zeros(self.n, dtype=np.int32)
        rec = np.zeros(self.n * n_moves if log else 0, dtype=MOVE_RECORD_DTYPE)
        s = self.lib.yamc_batch_run(self.h, ptrs, n.ctypes.data, cur.ctypes.data, int(n_moves),
                                    done.ctypes.data, st.ctypes.data, rec.ctypes.data if log else None)
        if s not in (_lib.YAMC_OK, _lib.YAMC_ERNG_EXHAUSTED):
            check(s, "yamc_batch_run")
        return (rec.reshape(self.n, n_moves) if log else None), cur, done, st, s

    def run_device(self, d_ptrs, n_rng, cursors: np.ndarray, n_moves: int, d_log_ptr: int = 0):
        """n_moves moves of every replica from device streams d_ptrs[i] of n_rng[i] floats;
        cursors (int64 array) updated in place.  Returns (moves_done, status, overall)."""
        ptrs, n = self._ptrs(d_ptrs, n_rng)
        done = np.zeros(self.n, dtype=np.int64)
        st = np.zeros(self.n, dtype=np.int32)
        s = self.lib.yamc_batch_run_device(self.h, ptrs, n.ctypes.data, cursors.ctypes.data, int(n_moves),
                                           done.ctypes.data, st.ctypes.data,
                                           ctypes.c_void_p(d_log_ptr) if d_log_ptr else None)
        if s not in (_lib.YAMC_OK, _lib.YAMC_ERNG_EXHAUSTED):
            check(s, "yamc_batch_run_device")
        return done, st, s

    def tune(self, d_ptrs, n_rng, cursors, n_moves: int) -> float:
        """Autotune the launch shape on n_moves moves per replica (state restored)."""
        ptrs, n = self._ptrs(d_ptrs, n_rng)
        best = ctypes.c_double(0)
        cur = np.ascontiguousarray(cursors, dtype=np.int64)
        check(self.lib.yamc_batch_tune(self.h, ptrs, n.ctypes.data, cur.ctypes.data, int(n_moves),
                                       ctypes.byref(best)), "yamc_batch_tune")
        return best.value

    def set_launch(self, cluster_blocks: int = 0, threads: int = 0) -> None:
        check(self.lib.yamc_batch_set_launch(self.h, int(cluster_blocks), int(threads)), "yamc_batch_set_launch")

    def set_kspace_layout(self, layout: int) -> None:
        check(self.lib.yamc_batch_set_kspace_layout(self.h, int(layout)), "yamc_batch_set_kspace_layout")

    @property
    def launch(self):
        out = np.zeros(5, dtype=np.int32)
        check(self.lib.yamc_batch_get_launch(self.h, _iptr(out)), "yamc_batch_get_launch")
        return {"cluster_blocks": int(out[0]), "threads": int(out[1]), "entries_per_thread": int(out[2]),
                "smem_bytes": int(out[3]), "resident_clusters": int(out[4])}

    @property
    def groups(self):
        """Launch shape of every group (kernel variant x size class) of the batch."""
        n = ctypes.c_int32(0)
        check(self.lib.yamc_batch_groups(self.h, ctypes.byref(n)), "yamc_batch_groups")
        out = []
        for g in range(n.value):
            v = np.zeros(7, dtype=np.int32)
            check(self.lib.yamc_batch_group_launch(self.h, g, _iptr(v)), "yamc_batch_group_launch")
            out.append({"cluster_blocks": int(v[0]), "threads": int(v[1]), "entries_per_thread": int(v[2]),
                        "smem_bytes": int(v[3]), "resident_clusters": int(v[4]), "replicas": int(v[5]),
                        "mixed": bool(v[6])})
        return out

    @property
    def last_kernel_ms(self) -> float:
        v = ctypes.c_double(0)
        check(self.lib.yamc_batch_last_kernel_ms(self.h, ctypes.byref(v)), "yamc_batch_last_kernel_ms")
        return v.value

    @property
    def last_launches(self) -> int:
        v = ctypes.c_int32(0)
        check(self.lib.yamc_batch_last_launches(self.h, ctypes.byref(v)), "yamc_batch_last_launches")
        return v.value


class _ReplicaView(Engine):
    """A replica of a Batch seen through the per-context calls; the batch owns it."""

    def __init__(self, batch: Batch, handle: ctypes.c_void_p, inputs: Inputs):
        self.lib = batch.lib
        self.inputs = inputs
        self.params = inputs.params
        self._batch = batch
        self.h = handle
        sz = np.zeros(5, dtype=np.int32)
        check(self.lib.yamc_sizes(self.h, _iptr(sz)), "yamc_sizes")
        self.natom, self.nmol, self.nk, self.nsigned, self.ntype = (int(v) for v in sz)

    def close(self) -> None:  # owned by the batch
        self.h = None


class RDF:
    """Molecule-centre radial distribution functions on the GPU (mcrdf2.f90:110-440): frames from
    host centres (a trajectory frame) or from an Engine's device-resident configuration."""

    def __init__(self, mol_type, mol_numbers, dr: float = 0.1, rmax: float = 12.0, device: int = 0):
        self.lib = _lib.load()
        self.mol_type = np.ascontiguousarray(mol_type, dtype=np.int32)
        self.mol_numbers = np.ascontiguousarray(mol_numbers, dtype=np.int32)
        self.ntypes = int(self.mol_numbers.size)
        self.dr, self.rmax = float(dr), float(rmax)
        self.h = ctypes.c_void_p()
        check(self.lib.yamc_rdf_create(self.mol_type.size, _iptr(self.mol_type), self.ntypes, _iptr(self.mol_numbers),
                                       self.dr, self.rmax, int(device), ctypes.byref(self.h)), "yamc_rdf_create")
        nb = ctypes.c_int32(0)
        check(self.lib.yamc_rdf_nbin(self.h, ctypes.byref(nb)), "yamc_rdf_nbin")
        self.nbin = nb.value

    @classmethod
    def for_engine(cls, eng: "Engine", dr: float = 0.1, rmax: float = 12.0, device: int = 0) -> "RDF":
        """Species per molecule in composition order from the engine's inputs."""
        counts = np.asarray(eng.inputs.mol_numbers, dtype=np.int32)
        mol_type = np.repeat(np.arange(1, counts.size + 1, dtype=np.int32), counts)
        return cls(mol_type, counts, dr, rmax, device)

    def add_frame(self, x, y, z, box_length: float) -> None:
        x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
        check(self.lib.yamc_rdf_add_frame(self.h, _dptr(x), _dptr(y), _dptr(z), float(box_length)), "yamc_rdf_add_frame")

    def add_engine(self, eng: "Engine") -> None:
        check(self.lib.yamc_rdf_add_ctx(self.h, eng.h), "yamc_rdf_add_ctx")

    def result(self):
        """(r, g[ntypes, ntypes, nbin], counts[ntypes, ntypes, nbin], n_frames); r = bin centres."""
        g = np.zeros(self.ntypes * self.ntypes * self.nbin)
        c = np.zeros_like(g)
        nf = ctypes.c_int32(0)
        check(self.lib.yamc_rdf_result(self.h, _dptr(g), _dptr(c), ctypes.byref(nf)), "yamc_rdf_result")
        r = (np.arange(self.nbin) + 0.5) * self.dr
        shape = (self.ntypes, self.ntypes, self.nbin)
        return r, g.reshape(shape), c.reshape(shape), nf.value

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.yamc_rdf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
