"""The reference's random stream: gfortran ``random_number`` into REAL(4).

YAMC seeds with ``random_seed(put=[seed]*n)`` (random.f90:25-54) and draws
``random_number`` into a REAL(4) variable (random.f90:65-93).  The stream is
whatever the linked libgfortran produces; here it is produced by calling the
libgfortran shipped inside the numpy wheel (GFORTRAN_8 symbol version) through
ctypes, so the buffer is bit-for-bit the sequence a gfortran build linked
against that runtime would draw.  The redraw of values outside
``[1e-14, 1-1e-14]`` is applied by the consumer (device or host), not here,
so the buffer is the raw ``random_number`` output.
"""
from __future__ import annotations

import ctypes
import glob
import os
from typing import Optional

import numpy as np

_lib = None
_lib_path: Optional[str] = None


class _Dtype(ctypes.Structure):
    _fields_ = [("elem_len", ctypes.c_size_t), ("version", ctypes.c_int),
                ("rank", ctypes.c_byte), ("type", ctypes.c_byte), ("attribute", ctypes.c_short)]


class _Dim(ctypes.Structure):
    _fields_ = [("stride", ctypes.c_ssize_t), ("lbound", ctypes.c_ssize_t), ("ubound", ctypes.c_ssize_t)]


class _Desc(ctypes.Structure):
    """gfortran rank-1 array descriptor (libgfortran >= 8 layout)."""
    _fields_ = [("base", ctypes.c_void_p), ("offset", ctypes.c_size_t), ("dtype", _Dtype),
                ("span", ctypes.c_ssize_t), ("dim", _Dim * 1)]


def _desc(ptr: int, n: int, elem_len: int, type_code: int) -> _Desc:
    d = _Desc()
    d.base = ptr
    d.offset = ctypes.c_size_t(-1).value  # lbound 1, stride 1
    d.dtype.elem_len = elem_len
    d.dtype.version = 0
    d.dtype.rank = 1
    d.dtype.type = type_code  # 1 = integer, 3 = real
    d.dtype.attribute = 0
    d.span = elem_len
    d.dim[0].stride = 1
    d.dim[0].lbound = 1
    d.dim[0].ubound = n
    return d


def libgfortran_path() -> str:
    import numpy
    cands = sorted(glob.glob(os.path.join(os.path.dirname(numpy.__file__) + ".libs", "libgfortran*.so*")))
    if not cands:
        cands = sorted(glob.glob("/usr/lib*/**/libgfortran.so.5*", recursive=True))
    if not cands:
        raise RuntimeError("libgfortran runtime not found; the gfortran random stream cannot be produced")
    return cands[0]


def _load():
    global _lib, _lib_path
    if _lib is None:
        _lib_path = libgfortran_path()
        _lib = ctypes.CDLL(_lib_path)
    return _lib


def seed_size() -> int:
    lib = _load()
    n = ctypes.c_int(0)
    lib._gfortran_random_seed_i4(ctypes.byref(n), None, None)
    return n.value


class GfortranStream:
    """``randomize(seed)`` then successive ``random_number`` REAL(4) draws."""

    def __init__(self, seed: int):
        self.seed = int(seed)
        self.reseed()

    def reseed(self) -> None:
        lib = _load()
        n = seed_size()
        arr = (ctypes.c_int * n)(*([self.seed] * n))
        d = _desc(ctypes.cast(arr, ctypes.c_void_p).value, n, 4, 1)
        lib._gfortran_random_seed_i4(None, ctypes.byref(d), None)
        self.drawn = 0

    def draw(self, n: int) -> np.ndarray:
        """The next n REAL(4) values (arandom_r4 on a contiguous array)."""
        lib = _load()
        buf = np.empty(int(n), dtype=np.float32)
        if n > 0:
            d = _desc(buf.ctypes.data, int(n), 4, 3)
            lib._gfortran_arandom_r4(ctypes.byref(d))
        self.drawn += int(n)
        return buf


def gfortran_stream(seed: int, n: int) -> np.ndarray:
    """n raw ``random_number`` values after ``randomize(seed)``."""
    return GfortranStream(seed).draw(n)


def runtime_description() -> str:
    _load()
    return f"libgfortran {os.path.basename(_lib_path)} (seed size {seed_size()})"
