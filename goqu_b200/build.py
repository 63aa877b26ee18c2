"""In-tree build of the engine (libgqb200.so, sm_100a) and of the host
emulator library the scheduler tests use (libgqb200_emu.so)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ENGINE = os.path.join(HERE, "libgqb200.so")
EMULATOR = os.path.join(HERE, "libgqb200_emu.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "-Xcompiler", "-Wno-unknown-pragmas",
    "-shared",
]

ENGINE_SOURCES = ["engine.cu", "noalloc.cu", "qaoa.cu", "schedule.cpp", "jit.cpp", "jit_gen.cpp", "params.cpp"]
EMULATOR_SOURCES = ["emulate.cpp", "schedule.cpp", "jit_gen.cpp", "params.cpp"]
HEADERS = ["tile_core.cuh", "kernels.cuh", "counts.cuh", "verify.cuh", "schedule.hpp", "jit.hpp", "params.hpp", os.path.join("..", "..", "include", "gqb200.h")]
# tile_core.cuh as a C++ string literal, compiled into the engine for the
# run-time specialised pass kernels (generated; not committed).
TILE_CORE_INC = os.path.join(CSRC, "tile_core_src.inc")


def write_tile_core_inc():
    with open(os.path.join(CSRC, "tile_core.cuh")) as f:
        text = f.read()
    assert ")GQSRC\"" not in text
    body = 'R"GQSRC(' + text + ')GQSRC"\n'
    if os.path.exists(TILE_CORE_INC):
        with open(TILE_CORE_INC) as f:
            if f.read() == body:
                return
    with open(TILE_CORE_INC, "w") as f:
        f.write(body)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(os.path.join(CSRC, s)) > t for s in sources + HEADERS)


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build_engine(force=False, verbose=False):
    write_tile_core_inc()
    if not force and not _stale(ENGINE, ENGINE_SOURCES):
        return ENGINE
    cmd = [nvcc()] + NVCC_FLAGS + [os.path.join(CSRC, s) for s in ENGINE_SOURCES] + ["-o", ENGINE, "-ldl"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return ENGINE


def build_emulator(force=False):
    write_tile_core_inc()
    if not force and not _stale(EMULATOR, EMULATOR_SOURCES):
        return EMULATOR
    inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-Wno-unknown-pragmas", "-I", inc, "-x", "c++"]
    cmd += [os.path.join(CSRC, s) for s in EMULATOR_SOURCES] + ["-o", EMULATOR, "-ldl"]
    subprocess.run(cmd, check=True)
    return EMULATOR


def build_all(force=False):
    build_engine(force)
    build_emulator(force)


if __name__ == "__main__":
    build_all(force=True)
