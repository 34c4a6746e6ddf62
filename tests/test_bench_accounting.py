"""Host logic of bench.py's roofline accounting: the colour launch
sequence of the symmetric sweeps and the algorithmic bytes of the explicit
and compact Jacobian layouts. CPU only."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import bench  # noqa: E402


def test_launch_sequence_skips_repeated_colours():
    seq = bench.sgs_launch_sequence(4, 8)
    assert len(seq) == 49
    assert seq[:8] == [0, 1, 2, 3, 2, 1, 0, 1]
    assert all(a != b for a, b in zip(seq, seq[1:]))
    assert bench.sgs_launch_sequence(1, 5) == [0]


def test_compact_slots_save_ten_values_per_face_side():
    colour = np.array([0, 0, 1, 1, 1])
    nint = np.array([4, 3, 4, 2, 0])
    for tb, tx in ((4, 4), (4, 8), (8, 8)):
        ex = bench.sgs_colour_bytes(colour, nint, tb, tx)
        cp = bench.sgs_colour_bytes(colour, nint, tb, tx, slot=15)
        np.testing.assert_array_equal(ex - cp, np.bincount(colour, weights=10.0 * tb * nint))
        # per cell LU + B + x write, per face side slot + index + neighbour x
        assert ex[0] == 2 * (30 * tb + 5 * tx) + 7 * (25 * tb + 4 + 5 * tx)


def test_compact_assembly_and_jacobian_bytes():
    nc, nfi, nbf, tb, tx = 1000, 2000, 100, 4, 4
    nf = nfi + nbf
    kw = dict(nc=nc, nfi=nfi, nbf=nbf, sweeps=8, tb=tb, tx=tx)
    ex = {k: bench.kernel_bytes(k, **kw) for k in ("face_jacobian", "assemble_lu")}
    cp = {k: bench.kernel_bytes(k, compact=True, **kw) for k in ("face_jacobian", "assemble_lu")}
    assert ex["face_jacobian"] - cp["face_jacobian"] == (2 * nfi + nbf) * 25 * tb - nf * 24 * tb
    assert ex["assemble_lu"] - cp["assemble_lu"] == ((2 * nfi + nbf) + 2 * nfi) * 10 * tb
