"""Build of the oracle (test infrastructure, the checker).

* ``oracle/liboracle.so``: the C++ restatement in ``oracle/oracle.cpp``,
  built with OpenMP so the CPU-baseline leg can use every host core.
* ``oracle/_ref/libfpsiref.so``: the reference's own face functions, compiled
  from their source where it lies (flowPsi ``src/fluxInviscid.loci`` and
  ``include/bcTools.h``) with a small Loci-type shim (``oracle/ref_shim.h``).
  The line ranges are cut out at build time into ``oracle/_ref/`` (git
  ignored); nothing of the reference is stored in the repository.  Only
  possible where the reference tree is present; the shared object then
  travels with the working tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
REF_LIB = REF_DIR / "libfpsiref.so"


def reference_tree(path: str | os.PathLike | None = None) -> Path | None:
    """The flowPsi source tree to cut the face functions from: the caller's
    path, else the FLOWPSI_REFERENCE environment variable, else none."""
    p = path if path is not None else os.environ.get("FLOWPSI_REFERENCE")
    return Path(p) if p else None


# (file, first line, last line, what) -- ranges of plain C++ in the reference
REF_RANGES = [
    ("src/fluxInviscid.loci", 157, 256, "hllc_flux"),
    ("src/fluxInviscid.loci", 869, 1014, "roeCT_flux"),
    ("src/fluxInviscid.loci", 1018, 1168, "RoeJacobian, roeCT_jacobian"),
    ("include/bcTools.h", 25, 81, "cv_inflow, cv_outflow"),
]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build_oracle(force: bool = False) -> Path:
    deps = [HERE / "oracle.cpp", HERE / "oracle.h", HERE.parent / "include" / "fpsi.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
           "-o", str(LIB) + ".tmp", str(HERE / "oracle.cpp")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


def build_ref(force: bool = False, reference: str | os.PathLike | None = None) -> Path | None:
    """Compile the reference face functions from the flowPsi tree at
    `reference` (or FLOWPSI_REFERENCE); without a tree the library built
    before is kept, else None."""
    shim = HERE / "ref_shim.h"
    glue = HERE / "ref_glue.inc"
    REFERENCE = reference_tree(reference)
    if REFERENCE is None:
        return REF_LIB if REF_LIB.exists() else None
    srcs = [REFERENCE / f for f, *_ in REF_RANGES]
    if not all(s.exists() for s in srcs):
        return REF_LIB if REF_LIB.exists() else None
    if not force and not _stale(REF_LIB, srcs + [shim, glue, Path(__file__)]):
        return REF_LIB
    REF_DIR.mkdir(exist_ok=True)
    parts = ['#include "ref_shim.h"', "namespace flowPsi {"]
    for f, a, b, what in REF_RANGES:
        lines = (REFERENCE / f).read_text().splitlines()[a - 1:b]
        parts.append(f"// ---- {f}:{a}-{b} ({what})")
        parts.append(f'#line {a} "{REFERENCE / f}"')
        parts.extend(lines)
    parts.append("}  // namespace flowPsi")
    parts.append('#include "ref_glue.inc"')
    cut = REF_DIR / "ref_functions.cpp"
    cut.write_text("\n".join(parts) + "\n")
    cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-I", str(HERE),
           "-o", str(REF_LIB) + ".tmp", str(cut)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference face-function build failed:\n" + r.stderr)
    os.replace(str(REF_LIB) + ".tmp", REF_LIB)
    return REF_LIB


def build(force: bool = False, reference: str | os.PathLike | None = None) -> None:
    build_oracle(force)
    build_ref(force, reference)


if __name__ == "__main__":
    # python oracle/build.py [--force] [path of the flowPsi source tree]
    args = [a for a in sys.argv[1:] if a != "--force"]
    build(force="--force" in sys.argv, reference=args[0] if args else None)
    print(LIB, REF_LIB if REF_LIB.exists() else "(no reference tree)")
