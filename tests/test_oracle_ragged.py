"""The prism grid (five faces per cell, triangles and quads) in the oracle:
geometry closes and a uniform stream is a steady state.  CPU only."""
import math

import numpy as np
import pytest

from flowpsi_b200 import cases
from flowpsi_b200.solver import GeneratedMesh, bc, default_params
from oracle import Oracle


@pytest.mark.parametrize("side", [(0,) * 6, (-1,) * 6, (0, 0, -1, -1, 0, 0)])
def test_prism_geometry_closes(side):
    U0 = 0.5 * math.sqrt(1.4 * cases.RTILDE * 300.0)
    mesh = GeneratedMesh("prism", n=(3, 4, 2), bc_side=side,
                         bcs=[bc("farfield", T=300.0, pg=1e5, u=(U0, 0.0, 0.0))])
    a = mesh.arrays()
    o = Oracle(mesh, default_params(precision="fp64"))
    g = o.geometry()
    assert a.ncells == 48
    assert np.allclose(g["vol"], 1.0 / 48, rtol=1e-13)
    faces = np.bincount(a.cl, minlength=a.ncells) + np.bincount(a.cr[a.cr >= 0], minlength=a.ncells)
    assert np.all(faces == 5)
    nodes = np.diff(np.asarray(a.face_off))
    assert set(nodes.tolist()) == {3, 4}
    # outward area vectors of every cell sum to zero
    A = g["area_vec"]  # area-weighted normals
    S = np.zeros((a.ncells, 3))
    np.add.at(S, a.cl, A)
    inner = a.cr >= 0
    np.add.at(S, a.cr[inner], -A[inner])
    assert np.abs(S).max() <= 1e-14


def test_uniform_stream_is_steady_on_prisms():
    U0 = 0.5 * math.sqrt(1.4 * cases.RTILDE * 300.0)
    u0 = (U0, 0.3 * U0, -0.2 * U0)
    mesh = GeneratedMesh("prism", n=(4, 3, 3), bc_side=(0,) * 6,
                         bcs=[bc("farfield", T=300.0, pg=1e5, u=u0)])
    o = Oracle(mesh, default_params(flux="roe", precision="fp64"))
    nc = o.ncells
    o.set_state(np.full(nc, 300.0), np.full(nc, 1e5), np.tile(u0, (nc, 1)))
    src, _ = o.residual()
    rho = 1e5 / (cases.RTILDE * 300.0)
    scale = rho * U0 * (1.0 / 3) ** 2 * (1e5 / rho + U0 * U0)
    assert np.abs(src).max() <= 1e-11 * scale
