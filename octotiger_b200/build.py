"""Builds libotfmm.so (sm_100a) in-tree with nvcc.

    python -m octotiger_b200.build            # build if sources changed
    python -m octotiger_b200.build --force -v # rebuild, print ptxas resource usage
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libotfmm.so"
SOURCES = [CSRC / "otfmm.cu"]
DEPS = SOURCES + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "otfmm.h", Path(__file__)]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _digest() -> str:
    h = hashlib.sha256()
    for p in DEPS:
        h.update(p.read_bytes())
    return h.hexdigest()


PASS_LIB = PKG / "libotfmm_adapter_pass.so"
PASS_SRC = CSRC / "adapter_pass.cpp"
PASS_DEPS = [PASS_SRC, CSRC / "octotiger_standins.hpp", ROOT / "include" / "otfmm_octotiger.hpp",
             ROOT / "include" / "otfmm.h"]


def build_adapter_pass(force: bool = False) -> Path:
    """libotfmm_adapter_pass.so: the adapter driven like node_server::compute_fmm
    (host C++, linked against libotfmm.so)."""
    if not force and PASS_LIB.exists() and all(PASS_LIB.stat().st_mtime >= p.stat().st_mtime
                                                for p in PASS_DEPS + [LIB]):
        return PASS_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", "-I", str(ROOT / "include"), "-I", str(CSRC),
           str(PASS_SRC), "-L", str(PKG), "-lotfmm", "-Wl,-rpath,$ORIGIN", "-o", str(PASS_LIB) + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("g++ failed building libotfmm_adapter_pass.so")
    os.replace(str(PASS_LIB) + ".tmp", PASS_LIB)
    return PASS_LIB


def build(force: bool = False, verbose: bool = False) -> Path:
    stamp = PKG / ".libotfmm.sha256"
    dig = _digest()
    if not force and LIB.exists() and stamp.exists() and stamp.read_text().strip() == dig:
        build_adapter_pass()
        return LIB
    cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "--expt-relaxed-constexpr", "--default-stream", "per-thread", "-I", str(ROOT / "include"), "-o",
           str(LIB) + ".tmp", *map(str, SOURCES)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libotfmm.so")
    if verbose:
        sys.stdout.write(res.stdout + res.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    stamp.write_text(dig)
    build_adapter_pass(force=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose))
