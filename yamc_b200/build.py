"""Build recipe of the engine library (nvcc, sm_100a).

``python -m yamc_b200.build`` compiles ``csrc/`` into ``yamc_b200/libyamc_b200.so``
in-tree, so the shared object travels with the source tree; ``--checked`` builds the
bounds-checked variant ``yamc_b200/libyamc_b200_checked.so`` (``-DYAMC_CHECKED``: every index the
chain kernel computes is checked, an out-of-bounds one is recorded and replaced by 0, and the call
returns YAMC_EBOUNDS).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libyamc_b200.so")
LIB_CHECKED = os.path.join(HERE, "libyamc_b200_checked.so")
# (source, object, extra flags): the chain kernel's variants are compiled once per LJ type count
UNITS = [("yamc_chain_inst.cu", f"yamc_chain_nt{n}.o", [f"-DYAMC_NT={n}"]) for n in (1, 2, 3, 4)] + [
    (src, src.rsplit(".", 1)[0] + ".o", []) for src in
    ("yamc_engine.cu", "yamc_static.cu", "yamc_peaks.cu", "yamc_host.cpp", "yamc_inputs.cpp")]
SOURCES = sorted({u[0] for u in UNITS})
HEADERS = ["yamc_chain.cuh", "yamc_device.cuh", "yamc_internal.h", os.path.join("..", "..", "include", "yamc.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-v",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def stale(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    """Compile every unit to an object in parallel (the chain kernel's variants once per LJ type
    count), then link the shared library (the bounds-checked variant when checked)."""
    lib = LIB_CHECKED if checked else LIB
    if not force and not stale(lib):
        return lib
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(HERE, "_build", "checked") if checked else os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    defs = ["-DYAMC_CHECKED=1"] if checked else []

    def compile_one(unit):
        src, objname, extra = unit
        obj = os.path.join(objdir, objname)
        cmd = [nvcc(), *NVCC_FLAGS, *defs, *extra, "-c", "-o", obj, os.path.join(CSRC, src)]
        res = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
        return obj, cmd, res

    with ThreadPoolExecutor(max_workers=max(1, min(len(UNITS), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, UNITS))
    log = ""
    failed = False
    for obj, cmd, res in results:
        log += " ".join(cmd) + "\n" + res.stdout + res.stderr
        failed = failed or res.returncode != 0
    if not failed:
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib + ".tmp",
               *[obj for obj, _, _ in results], "-lcudart"]
        res = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
        log += " ".join(cmd) + "\n" + res.stdout + res.stderr
        failed = res.returncode != 0
    with open(os.path.join(HERE, "build_checked.log" if checked else "build.log"), "w") as f:
        f.write(log)
    if failed:
        sys.stderr.write(log)
        raise RuntimeError("nvcc failed (see yamc_b200/build.log)")
    if verbose:
        sys.stderr.write(log)
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))
