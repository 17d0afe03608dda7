"""Build recipe of the native library (nvcc, sm_100a, in-tree).

``python -m sap_warp_b200.build`` compiles every ``csrc/*.cu`` into
``sap_warp_b200/libsapb.so``.  The library is built in the source tree so it
travels with the repository to the machine that runs it.  Each source is
compiled to a relocatable-free object in parallel (one nvcc per source), then
the objects are linked into the shared library.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR / "csrc"
INCLUDE = PKG_DIR.parent / "include"
LIB_NAME = "libsapb.so"
LIB_PATH = PKG_DIR / LIB_NAME

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMPILE_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libsapb.so")
    return cand


# The units that take longest to compile start first.
_HEAVY = ("sapb_solve_ngeneric", "sapb_solve_nwide", "sapb_blocked_nb", "sapb_mlp", "sapb_solve_n35")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"), key=lambda p: (not p.stem.startswith(_HEAVY), p.name))


def needs_build() -> bool:
    if not LIB_PATH.exists():
        return True
    lib_mtime = LIB_PATH.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > lib_mtime for p in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")


def build_library(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile the CUDA sources into the in-tree shared library."""
    if not force and not needs_build():
        return LIB_PATH
    nvcc = _nvcc()
    srcs = sources()
    jobs = jobs or min(len(srcs), max(os.cpu_count() or 1, 1))
    with tempfile.TemporaryDirectory(prefix="sapb_build_") as tmpdir:
        objs = [Path(tmpdir) / (s.stem + ".o") for s in srcs]
        cmds = [[nvcc, *ARCH_FLAGS, *COMPILE_FLAGS, "-I", str(INCLUDE), "-c", "-o", str(o), str(s)]
                for s, o in zip(srcs, objs)]
        with ThreadPoolExecutor(max_workers=jobs) as ex:
            for f in [ex.submit(_run, c, verbose) for c in cmds]:
                f.result()
        tmp = LIB_PATH.with_suffix(".so.tmp")
        _run([nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *map(str, objs)], verbose)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
