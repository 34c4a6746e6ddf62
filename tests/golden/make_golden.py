"""Generate the golden face-function vectors in tests/golden/face_functions.npz.

The outputs come from flowPsi's own hllc_flux, roeCT_flux, roeCT_jacobian,
cv_inflow and cv_outflow, compiled from the reference source by
oracle/build.py (oracle/_ref/libfpsiref.so).  Inputs are seeded log-normal
face states, including states near rest, sonic and supersonic normal speeds
and strong pressure jumps (which switch the preconditioning off).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import RefFunctions  # noqa: E402
from oracle.build import build_ref  # noqa: E402
from tests.helpers import face_states  # noqa: E402


def main():
    if build_ref() is None:
        raise SystemExit("reference tree not present: cannot generate golden vectors")
    R = RefFunctions()
    out = {}
    sets = {
        "mild": face_states(96, seed=11, jump=0.05, speed=50.0),
        "strong": face_states(96, seed=12, jump=0.5, speed=400.0),
        "rest": face_states(32, seed=13, jump=0.01, speed=1e-3),
    }
    for name, (qL, qR, an, area) in sets.items():
        out[f"{name}_qL"], out[f"{name}_qR"] = qL, qR
        out[f"{name}_an"], out[f"{name}_area"] = an, area
        for eta in (1.0, 0.3):
            tag = f"{name}_eta{eta:g}"
            out[f"{tag}_hllc"] = R.flux("hllc", qL, qR, an, area, eta=eta)
            out[f"{tag}_roe"] = R.flux("roe", qL, qR, an, area, eta=eta)
            out[f"{tag}_fjp"] = R.jacobian(qL, qR, an, area, +1, eta=eta)
            out[f"{tag}_fjm"] = R.jacobian(qL, qR, an, area, -1, eta=eta)
        q0 = np.tile(np.array([1e5, 300.0, 150.0, 0.0, 0.0]), (qL.shape[0], 1))
        out[f"{name}_q0"] = q0
        out[f"{name}_cv_in"] = R.cv_state(0, qL, q0, an)
        out[f"{name}_cv_out"] = R.cv_state(1, qL, q0, an)
    dst = Path(__file__).resolve().parent / "face_functions.npz"
    np.savez_compressed(dst, **out)
    print(dst, sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()
