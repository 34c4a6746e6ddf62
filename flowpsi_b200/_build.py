"""Build of the native library ``libfpsi.so`` (sm_100a CUDA + host C++).

The library is compiled in-tree with nvcc so that the shared object travels
with the source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libfpsi.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def build(force: bool = False, verbose: bool = False) -> Path:
    deps = sources() + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [
        PKG.parent / "include" / "fpsi.h"
    ]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [
        nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared",
        "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
        "-I", str(PKG.parent / "include"),
        "-o", str(LIB) + ".tmp", *[str(s) for s in sources()],
        "-lcudart",
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    if verbose:
        print(r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    import sys

    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
