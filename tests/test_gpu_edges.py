"""Edge cases of the C ABI on the device: malformed meshes and parameters
are refused with FPSI_E_INVALID, a one-cell and a two-cell grid run the whole
step and match the oracle, zero relaxation sweeps leave the block Jacobi
start, and bad line input is refused.  GPU only; tolerances as in
test_gpu_parity."""
import ctypes as C
import math

import numpy as np
import pytest

from flowpsi_b200 import FlowPsi, FpsiError, cases
from flowpsi_b200 import _native as N
from flowpsi_b200.solver import bc, default_params
from oracle import Oracle

pytestmark = pytest.mark.gpu

U0 = 0.5 * math.sqrt(1.4 * cases.RTILDE * 300.0)


class RawMesh:
    """an fpsi_mesh over numpy arrays (kept alive with the struct)"""

    def __init__(self, xyz, faces, cl, cr, bcs):
        self.xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1)
        self.off = np.zeros(len(faces) + 1, np.int64)
        self.off[1:] = np.cumsum([len(f) for f in faces])
        self.nodes = np.ascontiguousarray(np.concatenate([np.asarray(f) for f in faces])
                                          if faces else np.zeros(0), np.int32)
        self.cl = np.ascontiguousarray(cl, np.int32)
        self.cr = np.ascontiguousarray(cr, np.int32)
        self.bcs = (N.BCSpec * max(len(bcs), 1))(*bcs)
        m = N.Mesh()
        m.nnodes = len(self.xyz) // 3
        m.ncells = int(max(self.cl.max(initial=-1), self.cr.max(initial=-1)) + 1)
        m.nfaces = len(faces)
        m.xyz = self.xyz.ctypes.data_as(C.POINTER(C.c_double))
        m.face_off = self.off.ctypes.data_as(C.POINTER(C.c_int64))
        m.face_nodes = self.nodes.ctypes.data_as(C.POINTER(C.c_int32))
        m.cl = self.cl.ctypes.data_as(C.POINTER(C.c_int32))
        m.cr = self.cr.ctypes.data_as(C.POINTER(C.c_int32))
        m.pshift = None
        m.nbc = len(bcs)
        m.bcs = self.bcs
        self.m = m

    def arrays(self):
        return type("A", (), {"ncells": self.m.ncells, "cl": self.cl, "cr": self.cr})


def hex_row(ncell):
    """ncell unit hexes along x, every outer face a farfield boundary"""
    nx = ncell + 1
    xyz = [(i, j, k) for k in range(2) for j in range(2) for i in range(nx)]
    v = lambda i, j, k: i + nx * (j + 2 * k)  # noqa: E731
    faces, cl, cr = [], [], []
    for c in range(ncell):
        i = c
        if i == 0:
            faces.append([v(0, 0, 0), v(0, 0, 1), v(0, 1, 1), v(0, 1, 0)]), cl.append(c), cr.append(-1)
        if i + 1 < ncell:
            faces.append([v(i + 1, 0, 0), v(i + 1, 1, 0), v(i + 1, 1, 1), v(i + 1, 0, 1)])
            cl.append(c), cr.append(c + 1)
        else:
            faces.append([v(i + 1, 0, 0), v(i + 1, 1, 0), v(i + 1, 1, 1), v(i + 1, 0, 1)])
            cl.append(c), cr.append(-1)
        faces.append([v(i, 0, 0), v(i + 1, 0, 0), v(i + 1, 0, 1), v(i, 0, 1)]), cl.append(c), cr.append(-1)
        faces.append([v(i, 1, 0), v(i, 1, 1), v(i + 1, 1, 1), v(i + 1, 1, 0)]), cl.append(c), cr.append(-1)
        faces.append([v(i, 0, 0), v(i, 1, 0), v(i + 1, 1, 0), v(i + 1, 0, 0)]), cl.append(c), cr.append(-1)
        faces.append([v(i, 0, 1), v(i + 1, 0, 1), v(i + 1, 1, 1), v(i, 1, 1)]), cl.append(c), cr.append(-1)
    ff = bc("farfield", T=300.0, pg=1e5, u=(U0, 0.0, 0.0))
    return RawMesh(np.array(xyz, float), faces, cl, cr, [ff])


def _code(fn):
    with pytest.raises(FpsiError) as e:
        fn()
    return e.value.code


def test_malformed_meshes_are_refused(need_gpu):
    p = default_params(precision="fp64")
    good = hex_row(2)
    FlowPsi(good.m, p).close()
    bad_cl = hex_row(2)
    bad_cl.cl[0] = 7  # beyond ncells
    assert _code(lambda: FlowPsi(bad_cl.m, p)) == -1
    same = hex_row(2)
    i = int(np.nonzero(same.cr >= 0)[0][0])
    same.cr[i] = same.cl[i]  # a face between a cell and itself
    assert _code(lambda: FlowPsi(same.m, p)) == -1
    nobc = hex_row(2)
    nobc.m.nbc = 0  # boundary faces name a missing condition
    assert _code(lambda: FlowPsi(nobc.m, p)) == -1
    twonode = hex_row(1)
    twonode.off[1] = twonode.off[0] + 2  # a face of two nodes
    assert _code(lambda: FlowPsi(twonode.m, p)) == -1
    empty = hex_row(1)
    empty.m.ncells, empty.m.nfaces = 0, 0
    assert _code(lambda: FlowPsi(empty.m, p)) == -1


@pytest.mark.parametrize("field,value", [("flux", 5), ("limiter", -1), ("precision", 5),
                                         ("gauss_seidel_iter", -1), ("solver", 3),
                                         ("viscous", 3), ("turbulence", 2)])
def test_bad_parameters_are_refused(need_gpu, field, value):
    p = default_params(precision="fp64")
    setattr(p, field, value)
    mesh = hex_row(2)  # the struct points into its arrays: keep them alive
    assert _code(lambda: FlowPsi(mesh.m, p)) == -1


def test_sa_needs_the_turbulent_regime(need_gpu):
    p = default_params(precision="fp64", viscous=1, turbulence=1)
    mesh = hex_row(2)
    assert _code(lambda: FlowPsi(mesh.m, p)) == -1


@pytest.mark.parametrize("ncell", [1, 2])
def test_tiny_grids_run_the_whole_step(need_gpu, ncell):
    mesh = hex_row(ncell)
    p = default_params(flux="roe", precision="fp64", solver="sgs", gauss_seidel_iter=3,
                       cflmax=10.0)
    g = FlowPsi(mesh.m, p)
    o = Oracle(mesh.m, p)
    T = 300.0 * (1 + 0.01 * np.arange(ncell))
    pg = np.full(ncell, 1e5)
    u = np.tile([U0, 1.0, -2.0], (ncell, 1))
    g.set_state(T, pg, u)
    o.set_state(T, pg, u)
    for _ in range(3):
        g.newton_step()
        o.newton_step(colour=g.colours())
    for a, b in zip(g.get_state(), o.get_state()):
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()


def test_zero_sweeps_leave_the_jacobi_start(need_gpu):
    case = cases.farfield_cube(6, precision="fp64")
    case.params.gauss_seidel_iter = 0
    g = FlowPsi(case.mesh, case.params)
    g.keep_blocks(True)
    o = Oracle(case.mesh, case.params)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    g.set_state(T, p, u)
    o.set_state(T, p, u)
    g.residual()
    o.residual()
    g.assemble()
    o.assemble()
    dg = g.linear_solve()
    do = o.linear_solve(colour=g.colours())
    blk = o.blocks()
    xj = np.linalg.solve(blk["fluid_D"], blk["fluid_B"][:, :, None])[:, :, 0]
    assert np.abs(dg - do).max() <= 1e-10 * np.abs(do).max()
    assert np.abs(dg - xj).max() <= 1e-10 * np.abs(xj).max()


def test_bad_lines_are_refused(need_gpu):
    case = cases.boundary_layer_block(4, 6, 3, dy0=1e-3, growth=1.2, precision="fp64")
    g = FlowPsi(case.mesh, case.params)
    lines = case.mesh.lines_along(1)
    repeated = [l.copy() for l in lines]
    repeated[1][0] = repeated[0][0]
    assert _code(lambda: g.set_lines(repeated)) == -1
    jumped = [l.copy() for l in lines]
    jumped[0] = jumped[0][::2]  # consecutive cells without a shared face
    assert _code(lambda: g.set_lines(jumped)) == -1
    g.set_lines(lines)  # still usable
    g.set_state(*case.initial_state(g.geometry()["cellcenter"]))
    g.newton_step()
