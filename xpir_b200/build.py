"""Builds the engine's shared library in-tree with nvcc for sm_100a.

    python -m xpir_b200.build        # -> xpir_b200/libxpir_b200.so

The library is self-contained (static CUDA runtime) and exports only the C ABI declared
in include/xpir_b200.h.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libxpir_b200.so"
PIR_LIB = PKG / "libxpir_b200_pir.so"  # the libpir-shaped C++ API (host code over the C ABI)
PIR_SOURCES = ["host/pir_reply_generator.cpp"]
SOURCES = ["params.cpp", "sm100_host.cu", "import.cu", "reply.cu", "capi.cu", "batch.cu", "server.cu", "extract.cu", "querygen.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the engine is CUDA-only and cannot be built without it")


def build(force: bool = False, extra: list[str] | None = None, verbose: bool = False) -> Path:
    srcs = [CSRC / s for s in SOURCES]
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "xpir_b200.h"]
    if not force and LIB.exists():
        newest = max(p.stat().st_mtime for p in srcs + headers)
        if LIB.stat().st_mtime >= newest and not extra:
            return LIB
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--use_fast_math", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-shared", "-cudart", "static", "-ccbin", "g++",
           "-I", str(ROOT / "include"), "-o", str(LIB), *map(str, srcs)]
    if extra:
        cmd[1:1] = extra
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr)
    return LIB


def build_pir(force: bool = False) -> Path:
    """The C++ API of include/xpir_b200_pir.hpp: host code only, linked against the engine
    library next to it (rpath $ORIGIN)."""
    srcs = [PKG / s for s in PIR_SOURCES]
    headers = [ROOT / "include" / "xpir_b200_pir.hpp", ROOT / "include" / "xpir_b200.h"]
    if not force and PIR_LIB.exists() and PIR_LIB.stat().st_mtime >= max(p.stat().st_mtime for p in srcs + headers):
        return PIR_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-I", str(ROOT / "include"), "-o", str(PIR_LIB),
           *map(str, srcs), "-L", str(PKG), "-l:libxpir_b200.so", "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"g++ failed:\n{res.stdout}\n{res.stderr}")
    return PIR_LIB


def build_xpir(xpir_ref: str) -> Path:
    """XPIR's pir library with the B200 engine plugged in (xpir_b200/xpir/Makefile):
    XPIR's sources from `xpir_ref` with libpir.cpp and PIRReplyGeneratorFactory.cpp
    replaced by the B200 ones, archived as xpir_b200/xpir/_build/libpir_b200.a, and XPIR's
    own server and client linked with it (xpir_b200/xpir/_build/pir_server, pir_client)."""
    res = subprocess.run(["make", "-s", "-j8", "-C", str(PKG / "xpir"), "all", "apps", f"XPIR_REF={xpir_ref}"],
                         capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"building the XPIR binding failed:\n{res.stdout}\n{res.stderr}")
    return PKG / "xpir" / "_build" / "libpir_b200.a"


if __name__ == "__main__":
    verbose = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else None
    print(build(force=True, extra=extra, verbose=verbose or bool(extra)))
    print(build_pir(force=True))
