"""Builds oracle/_ref/libcpufem.so, the C++/OpenMP restatement used as the CPU
baseline (test / benchmark infrastructure; never loaded by the product)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIB = OUT / "libcpufem.so"
SRC = HERE / "cpu_fem.cpp"


def build() -> Path:
    OUT.mkdir(exist_ok=True)
    if LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
                    "-o", str(tmp), str(SRC)], check=True)
    os.replace(tmp, LIB)
    return LIB


def load() -> C.CDLL:
    lib = C.CDLL(str(build()))
    P = C.POINTER
    lib.cpu_fem_solve.restype = C.c_int
    lib.cpu_fem_solve.argtypes = [C.c_int, C.c_int, P(C.c_double), P(C.c_int), C.c_int, P(C.c_double),
                                  C.c_double, C.c_double, C.c_double, P(C.c_uint8), P(C.c_double),
                                  P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double),
                                  C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                  P(C.c_double)]
    lib.cpu_fem_threads.restype = C.c_int
    return lib


if __name__ == "__main__":
    print(build())
