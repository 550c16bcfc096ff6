"""The random stream the engine consumes is the stream the reference draws.

The reference draws one REAL(4) at a time: ``call random_number(MRandom_current_random_number)``
on a scalar (random.f90:65-93), which gfortran compiles to the scalar entry
``_gfortran_random_r4``.  ``yamc_b200.rng`` fills whole buffers with the array entry
``_gfortran_arandom_r4``, so the buffers are the reference's draws only if the two entries
walk the same generator state.  These tests call both entries of the same libgfortran (the
runtime whose stream the golden fixture and the GPU tests use) and require bit-identical
values, for several seeds, long runs, and array and scalar draws interleaved.
"""
import ctypes

import numpy as np
import pytest

from yamc_b200 import rng


def _scalar_draws(n: int) -> np.ndarray:
    lib = rng._load()
    f = ctypes.c_float()
    out = np.empty(n, dtype=np.float32)
    for i in range(n):
        lib._gfortran_random_r4(ctypes.byref(f))
        out[i] = f.value
    return out


@pytest.mark.parametrize("seed", [0, 1, 12345, 2024, 987654321, -7])
def test_scalar_random_r4_equals_array_fill(seed):
    n = 20000
    rng.GfortranStream(seed)  # randomize(seed): random_seed(put=[seed]*n)
    scalar = _scalar_draws(n)
    array = rng.gfortran_stream(seed, n)
    assert scalar.view(np.uint32).tolist() == array.view(np.uint32).tolist()


def test_interleaved_scalar_and_array_draws_are_one_stream():
    seed = 31337
    full = rng.gfortran_stream(seed, 5000)
    s = rng.GfortranStream(seed)
    parts, k = [], 0
    sizes = [1, 7, 64, 3, 1000, 1, 250, 2000, 5, 1669]
    for i, m in enumerate(sizes):
        parts.append(_scalar_draws(m) if i % 2 else s.draw(m))
        k += m
    assert k == full.size
    assert np.concatenate(parts).view(np.uint32).tolist() == full.view(np.uint32).tolist()


def test_stream_matches_golden_prefix():
    import json
    import os
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "gfortran_rng.json")))
    for seed, vals in gold["streams"].items():
        rng.GfortranStream(int(seed))
        got = _scalar_draws(len(vals))
        assert np.array_equal(got, np.asarray(vals, dtype=np.float32)), seed
