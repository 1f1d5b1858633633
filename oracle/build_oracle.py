"""Build recipe for the test oracle (test infrastructure only).

* ``oracle/lib/libxr_oracle.so`` -- the FP64 C restatement ``dd_oracle.c``.
* ``oracle/_ref/libxrecon_ref_helical.so`` -- the reference's own helical
  CUDA operators (XRecon ``src/kernels/helical_arc3d.cu``, which needs only
  the reference ``include/`` directory) compiled in place with the
  reference's nvcc flags (setup.py:16) for sm_100a, together with
  ``ref_helical_shim.cu``; it only serves tests/golden/make_golden_helical.py,
  which records the reference's helical outputs on a GPU.
* ``oracle/_ref/libxrecon_ref_cpu.so`` -- the reference's own CPU operators
  (XRecon ``src/cpu/{forward2d,backward2d,system_matrix2d,system_matrix3d,
  forward3d,backward3d}.cpp``) compiled in place from the reference sources together with
  ``ref_shim.cpp``.  Built only where the reference tree is present; the
  resulting .so travels with the repository snapshot (it is git-ignored).

The reference's own build system is not used: its CPU path is six C++ files
that only need the reference ``include/`` directory and the CUDA headers for
the ``__host__ __device__`` qualifiers of ``include/types.h``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_DIR = HERE / "lib"
REF_DIR = HERE / "_ref"
ORACLE_SO = LIB_DIR / "libxr_oracle.so"
REF_SO = REF_DIR / "libxrecon_ref_cpu.so"
REF_HELICAL_SO = REF_DIR / "libxrecon_ref_helical.so"
# Root of the XRecon reference tree, from the environment; unset: the
# reference libraries are not built (prebuilt ones are used when present).
def reference_root() -> Path | None:
    r = os.environ.get("XRECON_REFERENCE_ROOT")
    return Path(r) if r else None
REF_CPU_SOURCES = ["forward2d.cpp", "backward2d.cpp", "system_matrix2d.cpp", "system_matrix3d.cpp",
                   "forward3d.cpp", "backward3d.cpp"]
CUDA_INCLUDE = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stderr}")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build_oracle(force: bool = False) -> Path:
    src = HERE / "dd_oracle.c"
    LIB_DIR.mkdir(exist_ok=True)
    if force or _stale(ORACLE_SO, [src]):
        _run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(ORACLE_SO), str(src), "-lm"])
    return ORACLE_SO


def build_ref(force: bool = False) -> Path | None:
    """Compile the reference CPU operators; returns None when the reference
    tree is absent (the prebuilt .so, if shipped, is then used as is)."""
    root = reference_root()
    cpu_dir = root / "src" / "cpu" if root else None
    if cpu_dir is None or not cpu_dir.is_dir():
        return REF_SO if REF_SO.exists() else None
    srcs = [cpu_dir / s for s in REF_CPU_SOURCES] + [HERE / "ref_shim.cpp"]
    REF_DIR.mkdir(exist_ok=True)
    # where the reference tree was found, for the tests that import its
    # Python package next to this one (skipped where the tree is absent)
    (REF_DIR / "reference_root.txt").write_text(str(root) + "\n")
    if force or _stale(REF_SO, srcs):
        # -O3 matches the reference's own C++ flags (setup.py:15).
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread",
              f"-I{root / 'include'}", f"-I{CUDA_INCLUDE}",
              "-o", str(REF_SO)] + [str(s) for s in srcs])
    return REF_SO


def build_ref_helical(force: bool = False) -> Path | None:
    """Compile the reference's helical CUDA launchers with the shim; returns
    None when the reference tree is absent (a prebuilt .so is used as is)."""
    root = reference_root()
    if root is None:
        return REF_HELICAL_SO if REF_HELICAL_SO.exists() else None
    src = root / "src" / "kernels" / "helical_arc3d.cu"
    if not src.is_file():
        return REF_HELICAL_SO if REF_HELICAL_SO.exists() else None
    shim = HERE / "ref_helical_shim.cu"
    REF_DIR.mkdir(exist_ok=True)
    if force or _stale(REF_HELICAL_SO, [src, shim]):
        nvcc = str(Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "bin" / "nvcc")
        _run([nvcc, "-O3", "--use_fast_math", "-lineinfo", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
              "-Xcompiler", "-fPIC", "-shared", f"-I{root / 'include'}", "-o", str(REF_HELICAL_SO),
              str(src), str(shim)])
    return REF_HELICAL_SO


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
    print(build_ref_helical(force="--force" in sys.argv))
