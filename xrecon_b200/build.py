"""Build recipe for libxrecon_b200.so (sm_100a only).

The library is compiled in-tree with plain nvcc, so the built .so travels
with the source tree; there is no JIT cache and no CPU fallback.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
# XRECON_B200_BOUNDS=1 selects a separate build with the kernels' index
# checks compiled in (XR_DEBUG_BOUNDS: an index outside its buffer sets bit 2
# of the device error word and is clamped); it is slower and only for tests.
BOUNDS = os.environ.get("XRECON_B200_BOUNDS", "0") not in ("", "0")
LIB = PKG / ("libxrecon_b200_bounds.so" if BOUNDS else "libxrecon_b200.so")
SOURCES = [PKG / "csrc" / "xr_abi.cu"]
DEPS = SOURCES + sorted((PKG / "csrc").glob("*.cuh")) + sorted((PKG / "csrc").glob("*.hpp")) + \
    [ROOT / "include" / "xrecon_b200.h"]
NVCC = os.environ.get("NVCC", str(Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "bin" / "nvcc"))
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared", f"-I{ROOT / 'include'}",
         "-lpthread"] + (["-DXR_DEBUG_BOUNDS"] if BOUNDS else [])


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(d.stat().st_mtime > t for d in DEPS if d.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return LIB
    cmd = [NVCC] + FLAGS + ["-o", str(LIB)] + [str(s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed ({proc.returncode}):\n{proc.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
