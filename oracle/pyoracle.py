"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Imported only by tests/, ``__graft_entry__.smoke()`` and the cpu_baseline leg
of bench.py, as the checker.  The oracle is a plain-C restatement of the
reference Fortran (see yamc_oracle.h for what is and is not pinned).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")


def build(force: bool = False) -> None:
    libs = [os.path.join(BUILD, "liboracle.so"), os.path.join(BUILD, "liboracle_fast.so")]
    src = [os.path.join(HERE, "yamc_oracle.c"), os.path.join(HERE, "yamc_oracle.h")]
    newest = max(os.path.getmtime(p) for p in src)
    if force or not all(os.path.exists(l) and os.path.getmtime(l) >= newest for l in libs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


class Params(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "sr", "sk", "alphaL", "temp", "external_permutivity", "BoxLength", "density",
        "dr_a", "d_angle_degree", "xlambda_c", "xlambda_f", "pressure",
        "pressure_step_multiplier", "max_volume_scaling",
        "n_store_traj_interval", "n_store_energy_interval")] + [
        ("max_cycle", ctypes.c_int32), ("rnd_seed", ctypes.c_int32),
        ("input_nbytes_xyz", ctypes.c_int32), ("input_nbytes_ang", ctypes.c_int32),
        ("output_nbytes_xyz", ctypes.c_int32), ("output_nbytes_ang", ctypes.c_int32)] + [
        (n, ctypes.c_double) for n in (
        "alpha", "rmax", "rmax2", "kT_kcal_mol", "dbjr_a", "dbjr", "xclb",
        "alpha_over_sqrt_pi", "two_alpha_over_sqrt_pi", "kext", "minus_two_kext",
        "dr", "d_angle", "log_max_volume_scaling", "pressure_angstr_kT")] + [
        ("kmax", ctypes.c_int32), ("are_read", ctypes.c_int32), ("freq_file", ctypes.c_char * 256)]


class MoveRec(ctypes.Structure):
    _fields_ = [("imol", ctypes.c_int32), ("flags", ctypes.c_int32), ("cursor", ctypes.c_int64),
                ("du_real", ctypes.c_double), ("du_k_coul", ctypes.c_double),
                ("du_k_lj", ctypes.c_double), ("du_ext", ctypes.c_double),
                ("f_old", ctypes.c_double * 3), ("t_old", ctypes.c_double * 3),
                ("f_new", ctypes.c_double * 3), ("t_new", ctypes.c_double * 3)]


MOVE_DTYPE = np.dtype([("imol", np.int32), ("flags", np.int32), ("cursor", np.int64),
                       ("du_real", np.float64), ("du_k_coul", np.float64), ("du_k_lj", np.float64),
                       ("du_ext", np.float64), ("f_old", np.float64, 3), ("t_old", np.float64, 3),
                       ("f_new", np.float64, 3), ("t_new", np.float64, 3)])
assert MOVE_DTYPE.itemsize == ctypes.sizeof(MoveRec)

# orc_vol_rec: one mcvol step
VOL_DTYPE = np.dtype([("cycle", np.int64), ("flags", np.int32), ("pad", np.int32), ("cursor", np.int64),
                      ("box_old", np.float64), ("box_new", np.float64), ("du", np.float64), ("arg", np.float64)])

_libs = {}


def lib(fast: bool = False):
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name not in _libs:
        build()
        L = ctypes.CDLL(os.path.join(BUILD, name))
        P = ctypes.POINTER
        dp = P(ctypes.c_double)
        L.orc_params_defaults.argtypes = [P(Params)]
        L.orc_params_read.argtypes = [P(Params), ctypes.c_char_p]
        L.orc_params_read_string.argtypes = [P(Params), ctypes.c_char_p]
        L.orc_params_init.argtypes = [P(Params), ctypes.c_int32]
        L.orc_params_recalc.argtypes = [P(Params), ctypes.c_double]
        for f in ("orc_erfc_luc", "orc_erf_luc", "orc_shi_sans_exp"):
            getattr(L, f).argtypes = [ctypes.c_double]
            getattr(L, f).restype = ctypes.c_double
        L.orc_erfc_bet6_bet12.argtypes = [ctypes.c_double] * 3 + [dp] * 3
        L.orc_grid_count.argtypes = [ctypes.c_int32]
        L.orc_grid_count.restype = ctypes.c_int32
        L.orc_create.argtypes = [P(Params), ctypes.c_char_p, ctypes.c_char_p, P(ctypes.c_int32)]
        L.orc_create.restype = ctypes.c_void_p
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        for f in ("orc_natom", "orc_nmol", "orc_nk", "orc_ntype"):
            getattr(L, f).argtypes = [ctypes.c_void_p]
            getattr(L, f).restype = ctypes.c_int32
        L.orc_get_params.argtypes = [ctypes.c_void_p, P(Params)]
        L.orc_get_atoms.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 6
        L.orc_get_mols.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_energies.argtypes = [ctypes.c_void_p, dp]
        L.orc_full_sums.argtypes = [ctypes.c_void_p, dp]
        L.orc_full_sums.restype = ctypes.c_int32
        L.orc_get_uuF.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4
        L.orc_get_rho.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_intra_sums.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_mu.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.orc_mu.restype = ctypes.c_double
        L.orc_run_mc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, P(ctypes.c_int64),
                                 ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                 P(ctypes.c_int32)]
        L.orc_run_mc.restype = ctypes.c_int32
        L.orc_movemc.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64,
                                 P(ctypes.c_int64), P(MoveRec)]
        L.orc_movemc.restype = ctypes.c_int32
        L.orc_run_cycles.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, P(ctypes.c_int64),
                                     ctypes.c_int64, P(ctypes.c_int64), ctypes.c_void_p, ctypes.c_int64,
                                     P(ctypes.c_int64), ctypes.c_void_p, ctypes.c_int64, P(ctypes.c_int64),
                                     ctypes.c_void_p, ctypes.c_int32, P(ctypes.c_int32)]
        L.orc_run_cycles.restype = ctypes.c_int32
        L.orc_mcvol.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, P(ctypes.c_int64), ctypes.c_void_p]
        L.orc_mcvol.restype = ctypes.c_int32
        L.orc_set_xchange_weights.argtypes = [ctypes.c_void_p, dp, ctypes.c_int32]
        L.orc_set_xchange_weights.restype = ctypes.c_int32
        L.orc_xchange.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64,
                                  P(ctypes.c_int64), P(MoveRec)]
        L.orc_xchange.restype = ctypes.c_int32
        L.orc_rdf_count.argtypes = [ctypes.c_int32] + [ctypes.c_void_p] * 4 + [ctypes.c_int32] + [ctypes.c_double] * 3 + \
            [ctypes.c_void_p] * 2
        L.orc_rdf_normalize.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_void_p]
        L.orc_box_length.argtypes = [ctypes.c_void_p]
        L.orc_box_length.restype = ctypes.c_double
        L.orc_move_old.argtypes = [ctypes.c_void_p, ctypes.c_int32, dp, dp]
        L.orc_move_old.restype = ctypes.c_int32
        L.orc_move_eval.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, P(ctypes.c_int32), dp, dp]
        L.orc_move_eval.restype = ctypes.c_int32
        L.orc_move_commit.argtypes = [ctypes.c_void_p]
        L.orc_move_commit.restype = ctypes.c_int32
        L.orc_set_move_weights.argtypes = [ctypes.c_void_p, dp, ctypes.c_int32]
        L.orc_set_move_weights.restype = ctypes.c_int32
        L.orc_force_kspace_atom.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, dp]
        _libs[name] = L
    return _libs[name]


def read_params(path: str, extra: str = "", fast: bool = False) -> Params:
    L = lib(fast)
    p = Params()
    L.orc_params_defaults(ctypes.byref(p))
    if L.orc_params_read(ctypes.byref(p), path.encode()) != 0:
        raise IOError(path)
    if extra:
        if L.orc_params_read_string(ctypes.byref(p), extra.encode()) != 0:
            raise ValueError(extra)
    return p


class Oracle:
    """initmc + run_mc state of the reference for one system."""

    def __init__(self, files: dict, extra: str = "", fast: bool = False):
        self.L = lib(fast)
        self.params_in = read_params(files["parameters"], extra, fast)
        st = ctypes.c_int32(0)
        self.h = self.L.orc_create(ctypes.byref(self.params_in), files["composition"].encode(),
                                   files["moltab"].encode(), ctypes.byref(st))
        if not self.h:
            raise RuntimeError(f"orc_create failed: {st.value}")
        self.status = st.value
        if st.value < 0:
            self.L.orc_destroy(self.h)
            self.h = None
            raise RuntimeError(f"orc_create failed: {st.value}")
        self.natom = self.L.orc_natom(self.h)
        self.nmol = self.L.orc_nmol(self.h)
        self.nk = self.L.orc_nk(self.h)
        self.ntype = self.L.orc_ntype(self.h)
        self.params = Params()
        self.L.orc_get_params(self.h, ctypes.byref(self.params))

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def energies(self) -> np.ndarray:
        e = np.zeros(8)
        self.L.orc_energies(self.h, e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return e

    def full_sums(self) -> np.ndarray:
        e = np.zeros(8)
        ov = self.L.orc_full_sums(self.h, e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if ov:
            raise RuntimeError("overlap in the configuration")
        return e

    def atoms(self):
        n = self.natom
        x, y, z, q = (np.zeros(n) for _ in range(4))
        t = np.zeros(n, dtype=np.int32)
        m = np.zeros(n, dtype=np.int32)
        self.L.orc_get_atoms(self.h, x.ctypes.data, y.ctypes.data, z.ctypes.data, q.ctypes.data,
                             t.ctypes.data, m.ctypes.data)
        return x, y, z, q, t, m

    def set_move_weights(self, w) -> None:
        """init_freq with a frequencies file: BiasedRandom_init on the molecules' move weights."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        if self.L.orc_set_move_weights(self.h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), w.size) != 0:
            raise ValueError("one weight per molecule")

    def set_xchange_weights(self, w) -> None:
        """init_freq's exchange weights: xchange_freq and xchange_probability = Sxch/(Smv+Sxch)."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        if self.L.orc_set_xchange_weights(self.h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), w.size) != 0:
            raise ValueError("one weight per molecule")

    def xchange(self, imol1: int, imol2: int, rng: np.ndarray, cursor: int = 0):
        """One mc_xchange with its acceptance draw from rng: (record, cursor)."""
        rng = np.ascontiguousarray(rng, dtype=np.float32)
        rec = MoveRec()
        cur = ctypes.c_int64(cursor)
        r = self.L.orc_xchange(self.h, imol1, imol2, rng.ctypes.data, rng.size, ctypes.byref(cur), ctypes.byref(rec))
        if r != 0:
            raise RuntimeError(f"orc_xchange returned {r}")
        return rec, cur.value

    def mols(self):
        f = np.zeros(self.nmol, dtype=np.int32)
        l = np.zeros(self.nmol, dtype=np.int32)
        self.L.orc_get_mols(self.h, f.ctypes.data, l.ctypes.data)
        return f, l

    def uuF(self):
        n = self.natom
        a = [np.zeros(n) for _ in range(4)]
        self.L.orc_get_uuF(self.h, *[v.ctypes.data for v in a])
        return a

    def intra_sums(self) -> np.ndarray:
        """uu_ew_intra, uu_lj6_intra, uu_lj12_intra of the last full real-space sum."""
        out = np.zeros(3)
        self.L.orc_intra_sums(self.h, out.ctypes.data)
        return out

    def rho(self) -> np.ndarray:
        out = np.zeros((1 + self.ntype, 8, self.nk))
        self.L.orc_get_rho(self.h, out.ctypes.data)
        return out

    def mu(self) -> np.ndarray:
        return np.array([self.L.orc_mu(self.h, c) for c in range(3)])

    def run_mc(self, rng: np.ndarray, n_moves: int, cursor: int = 0, max_rows: int = 0):
        rng = np.ascontiguousarray(rng, dtype=np.float32)
        log = np.zeros(n_moves, dtype=MOVE_DTYPE)
        rows = np.zeros((max(max_rows, 1), 9))
        nrows = ctypes.c_int32(0)
        cur = ctypes.c_int64(cursor)
        r = self.L.orc_run_mc(self.h, rng.ctypes.data, rng.size, ctypes.byref(cur), n_moves,
                              log.ctypes.data, rows.ctypes.data, max_rows, ctypes.byref(nrows))
        if r != 0:
            raise RuntimeError(f"orc_run_mc returned {r}")
        return log, rows[: nrows.value], cur.value

    def run_cycles(self, rng: np.ndarray, n_cycles: int, cursor: int = 0, max_rows: int = 0,
                   allow_exhausted: bool = False):
        """run_mc by cycles, NPT volume steps included: (move log, volume log, energy rows,
        cursor, cycles done)."""
        rng = np.ascontiguousarray(rng, dtype=np.float32)
        max_log = n_cycles * self.nmol
        log = np.zeros(max(max_log, 1), dtype=MOVE_DTYPE)
        vlog = np.zeros(max(n_cycles, 1), dtype=VOL_DTYPE)
        rows = np.zeros((max(max_rows, 1), 9))
        nrows = ctypes.c_int32(0)
        nlog = ctypes.c_int64(0)
        nv = ctypes.c_int64(0)
        done = ctypes.c_int64(0)
        cur = ctypes.c_int64(cursor)
        r = self.L.orc_run_cycles(self.h, rng.ctypes.data, rng.size, ctypes.byref(cur), n_cycles, ctypes.byref(done),
                                  log.ctypes.data, max_log, ctypes.byref(nlog), vlog.ctypes.data, n_cycles,
                                  ctypes.byref(nv), rows.ctypes.data, max_rows, ctypes.byref(nrows))
        if r != 0 and not (allow_exhausted and r == -6):
            raise RuntimeError(f"orc_run_cycles returned {r}")
        return log[: nlog.value], vlog[: nv.value], rows[: nrows.value], cur.value, done.value

    def mcvol(self, rng: np.ndarray, cursor: int = 0):
        rng = np.ascontiguousarray(rng, dtype=np.float32)
        rec = np.zeros(1, dtype=VOL_DTYPE)
        cur = ctypes.c_int64(cursor)
        r = self.L.orc_mcvol(self.h, rng.ctypes.data, rng.size, ctypes.byref(cur), rec.ctypes.data)
        if r != 0:
            raise RuntimeError(f"orc_mcvol returned {r}")
        return rec[0], cur.value

    @property
    def box_length(self) -> float:
        return self.L.orc_box_length(self.h)

    def movemc(self, imol: int, rng: np.ndarray, cursor: int = 0):
        rng = np.ascontiguousarray(rng, dtype=np.float32)
        rec = MoveRec()
        cur = ctypes.c_int64(cursor)
        r = self.L.orc_movemc(self.h, imol, rng.ctypes.data, rng.size, ctypes.byref(cur), ctypes.byref(rec))
        if r != 0:
            raise RuntimeError(f"orc_movemc returned {r}")
        return rec, cur.value


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _oracle_move_old(self, imol: int):
    f, t = np.zeros(3), np.zeros(3)
    if self.L.orc_move_old(self.h, int(imol), _dp(f), _dp(t)) != 0:
        raise RuntimeError("orc_move_old")
    return f, t


def _oracle_move_eval(self, xn, yn, zn):
    xn, yn, zn = (np.ascontiguousarray(v, dtype=np.float64) for v in (xn, yn, zn))
    du, f, t = np.zeros(4), np.zeros(3), np.zeros(3)
    ov = ctypes.c_int32(0)
    self.L.orc_move_eval(self.h, _dp(xn), _dp(yn), _dp(zn), _dp(du), ctypes.byref(ov), _dp(f), _dp(t))
    return du, bool(ov.value), f, t


def _oracle_move_commit(self):
    self.L.orc_move_commit(self.h)


Oracle.move_old = _oracle_move_old
Oracle.move_eval = _oracle_move_eval
Oracle.move_commit = _oracle_move_commit


def erfc_luc(x: float) -> float:
    return lib().orc_erfc_luc(x)


def erf_luc(x: float) -> float:
    return lib().orc_erf_luc(x)


def shi_sans_exp(x: float) -> float:
    return lib().orc_shi_sans_exp(x)


def bet6_bet12(x: float):
    e = ctypes.c_double(); b6 = ctypes.c_double(); b12 = ctypes.c_double()
    lib().orc_erfc_bet6_bet12(x, x * x, np.exp(-x * x), ctypes.byref(e), ctypes.byref(b6), ctypes.byref(b12))
    return e.value, b6.value, b12.value


def grid_count(kmax: int) -> int:
    return lib().orc_grid_count(kmax)


class RDF:
    """mcrdf2's molecule-centre RDFs (count_distances + save_rdfs, mcrdf2.f90:110-440)."""

    def __init__(self, mol_type, mol_numbers, dr: float = 0.1, rmax: float = 12.0):
        self.L = lib()
        self.type = np.ascontiguousarray(mol_type, dtype=np.int32)
        self.mol_numbers = np.ascontiguousarray(mol_numbers, dtype=np.int32)
        self.nt = int(self.mol_numbers.size)
        self.dr, self.rmax = float(dr), float(rmax)
        self.nbin = int((rmax - 1e-10) / dr) + 2
        self.cnt4 = np.zeros(self.nt * self.nt * self.nbin)
        self.n_total = np.zeros(self.nt * self.nt)
        self.n_frame = 0
        self.sum_inv_vol = 0.0

    def add_frame(self, x, y, z, box_length: float) -> None:
        x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
        self.L.orc_rdf_count(x.size, x.ctypes.data, y.ctypes.data, z.ctypes.data, self.type.ctypes.data, self.nt,
                             box_length, self.dr, self.rmax, self.cnt4.ctypes.data, self.n_total.ctypes.data)
        self.n_frame += 1
        self.sum_inv_vol += 1.0 / box_length ** 3

    def g(self) -> np.ndarray:
        out = np.zeros_like(self.cnt4)
        self.L.orc_rdf_normalize(self.nt, self.mol_numbers.ctypes.data, self.dr, self.rmax, self.cnt4.ctypes.data,
                                 self.n_total.ctypes.data, self.n_frame, self.sum_inv_vol / self.n_frame,
                                 out.ctypes.data)
        return out.reshape(self.nt, self.nt, self.nbin)
