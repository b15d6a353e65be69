"""Build libbafqmc_b200.so in-tree with nvcc for sm_100a.

    python -m bafqmc_b200.build [--force]

Each source compiles to its own object (in parallel) and nvcc links the
shared library.  Staleness is decided by content: a SHA-256 over the nvcc
flags and every source and header is stored beside the library
(libbafqmc_b200.so.sha256); a library whose digest differs, or that has no
digest, is rebuilt, whatever the files' modification times.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libbafqmc_b200.so"
STAMP = PKG / "libbafqmc_b200.so.sha256"
OBJDIR = PKG.parent / "_build"
SOURCES = ["sweep_kernels.cu", "pole_kernels.cu", "proposer.cu", "capi.cu"]
HEADERS = ["cplx.cuh", "linalg.cuh", "linalg_big.cuh", "tc.cuh", "sweep.cuh", "kernels.h", "net.h", "conv_tc.cuh"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def digest() -> str:
    h = hashlib.sha256()
    h.update(" ".join(NVCC_FLAGS).encode())
    for f in [CSRC / s for s in SOURCES + HEADERS] + [PKG.parent / "include" / "bafqmc_b200.h"]:
        h.update(f.name.encode())
        h.update(f.read_bytes())
    return h.hexdigest()


def up_to_date() -> bool:
    return LIB.exists() and STAMP.exists() and STAMP.read_text().strip() == digest()


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    OBJDIR.mkdir(exist_ok=True)
    nvcc = _nvcc()

    def compile_one(src: str) -> Path:
        obj = OBJDIR / (Path(src).stem + ".o")
        cmd = [nvcc, *NVCC_FLAGS, "-c", "-o", str(obj), str(CSRC / src)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True, cwd=str(CSRC))
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp), *map(str, objs)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    STAMP.write_text(digest() + "\n")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
