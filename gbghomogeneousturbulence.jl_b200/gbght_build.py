"""Build the in-tree CUDA library libgbght.so for sm_100a (B200) with nvcc.

The engine's kernel instantiations are split across translation units by precision and grid
size, and compiled in parallel. Usage: python gbght_build.py [--force] [--verbose] [--hostcheck]
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgbght.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-O2", "-Xptxas", "-O3"]
SIZES = [8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512]
PRECISIONS = ["double", "float"]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh")))


def _digest() -> str:
    h = hashlib.sha256()
    for p in _sources() + [os.path.abspath(__file__), os.path.join(HERE, "..", "include", "gbght.h")]:
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()


def _units():
    """(name, defines) of every translation unit: one per (precision, N, dealiasing) for the engine,
    and the C ABI with the engine factory."""
    units = [("capi", ["-DGBGHT_UNIT_CAPI"], "gbght_capi.cu"),
             ("noalloc", [], "gbght_noalloc.cu"),
             ("factory", ["-DGBGHT_UNIT_FACTORY"], "gbght_engine.cu")]
    for t in PRECISIONS:
        for n in SIZES:
            units.append((f"eng_{t}_{n}", [f"-DGBGHT_UNIT_T={t}", f"-DGBGHT_UNIT_N={n}"], "gbght_engine.cu"))
            units.append((f"eng_{t}_{n}_houli", [f"-DGBGHT_UNIT_T={t}", f"-DGBGHT_UNIT_N={n}", "-DGBGHT_UNIT_D=1"],
                          "gbght_engine.cu"))
    return units


def _unit_digest(unit) -> str:
    """The inputs of one translation unit: every header, its own source, the flags and defines."""
    name, defs, src = unit
    h = hashlib.sha256()
    for p in [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cuh")] + \
             [os.path.join(CSRC, src), os.path.join(HERE, "..", "include", "gbght.h")]:
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(ARCH + FLAGS + defs).encode())
    return h.hexdigest()


def _compile(unit, verbose, force=False):
    """Compile one unit, unless its object is current (a stamp of the unit's inputs)."""
    name, defs, src = unit
    obj = os.path.join(BUILD, name + ".o")
    stamp = obj + ".sha256"
    digest = _unit_digest(unit)
    if not force and os.path.exists(obj) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == digest:
                return obj
    cmd = [NVCC] + ARCH + FLAGS + defs + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {name}:\n{r.stdout}\n{r.stderr}")
    with open(stamp, "w") as f:
        f.write(digest)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    stamp = OUT + ".sha256"
    digest = _digest()
    if not force and os.path.exists(OUT) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == digest:
                return OUT
    os.makedirs(BUILD, exist_ok=True)
    units = _units()
    jobs = max(1, min(len(units), os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda u: _compile(u, verbose, force), units))
    tmp = OUT + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, OUT)
    with open(stamp, "w") as f:
        f.write(digest)
    return OUT


HOSTCHECK = os.path.join(BUILD, "hostcheck", "libgbght_hostcheck.so")


def build_hostcheck(force: bool = False) -> str:
    """Compile the same kernel bodies and C ABI with the host C++ compiler (-DGBGHT_EMU): every
    launch runs block by block on one CPU thread. This build is test infrastructure for checking
    the kernels' index arithmetic against the oracle on a machine without a GPU; nothing in the
    package loads it."""
    stamp = HOSTCHECK + ".sha256"
    digest = _digest()
    if not force and os.path.exists(HOSTCHECK) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == digest:
                return HOSTCHECK
    os.makedirs(os.path.dirname(HOSTCHECK), exist_ok=True)
    tmp = HOSTCHECK + ".tmp"
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-DGBGHT_EMU", "-x", "c++", "-fPIC", "-shared",
           "-ffp-contract=off", os.path.join(CSRC, "gbght_engine.cu"), os.path.join(CSRC, "gbght_capi.cu"),
           "-o", tmp]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host-check build failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, HOSTCHECK)
    with open(stamp, "w") as f:
        f.write(digest)
    return HOSTCHECK


if __name__ == "__main__":
    if "--hostcheck" in sys.argv:
        print(build_hostcheck(force="--force" in sys.argv))
        sys.exit(0)
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
