"""Line SGS (fluidLinearSolver 'lsgs') on the GPU against the oracle's
restatement of linearSolverLSGS.loci, through the C ABI.  GPU only.

The GPU sweeps the lines colour by colour; the oracle is given the same
lines and colours.  Tolerances: FP64 1e-8 of max|dq| (block conditioning as
in the SGS tests); with FP32 blocks the GPU result must lie as close to the
FP64 solution as the oracle's FP32 result does (x2).
"""
import numpy as np
import pytest

from flowpsi_b200 import FlowPsi, cases
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _bl(prec):
    return cases.boundary_layer_block(8, 12, 4, dy0=1e-4, growth=1.3, precision=prec)


def _cube(prec):
    c = cases.farfield_cube(6, precision=prec)
    c.params.solver = 1  # lsgs
    c.lines = c.mesh.lines_along(1)
    return c


CASES = {"bl_wall_normal": _bl, "cube_y_lines": _cube}


def _setup(case, lines=True):
    g = FlowPsi(case.mesh, case.params)
    if lines:
        g.set_lines(case.lines)
    o = Oracle(case.mesh, case.params)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    g.set_state(T, p, u)
    o.set_state(T, p, u)
    return g, o


@pytest.mark.parametrize("prec", ["fp64", "ref", "mixed"])
@pytest.mark.parametrize("name", list(CASES))
def test_lsgs_matches_oracle(need_gpu, name, prec):
    case = CASES[name](prec)
    g, o = _setup(case)
    lines, colours = g.line_list()
    assert sum(len(l) for l in lines) == g.ncells
    g.residual()
    o.residual()
    g.assemble()
    o.assemble()
    dg, ig = g.linear_solve(info=True)
    do, io = o.lsgs_solve(lines, colours)
    if prec == "fp64":
        assert ig["iterations"] == io["iterations"]
        for k in range(5):
            assert np.abs(dg[:, k] - do[:, k]).max() <= 1e-8 * np.abs(do[:, k]).max(), k
    else:
        c64 = CASES[name]("fp64")
        o64 = Oracle(c64.mesh, c64.params)
        o64.set_state(*o.get_state())
        o64.residual()
        o64.assemble()
        d64, _ = o64.lsgs_solve(lines, colours)
        for k in range(5):
            e_orc = np.abs(do[:, k] - d64[:, k]).max()
            e_gpu = np.abs(dg[:, k] - d64[:, k]).max()
            assert e_gpu <= 2.0 * e_orc + 1e-6 * np.abs(d64[:, k]).max(), k
    nb, nr = g.linear_residual()
    assert nr < nb


def test_lsgs_converges_like_a_direct_solve(need_gpu):
    case = _bl("fp64")
    p = case.params
    p.lsgs_max_iter, p.lsgs_rel_tol, p.lsgs_abs_tol = 300, 1e-13, 0.0
    g, _ = _setup(case)
    g.residual()
    g.assemble()
    dq, info = g.linear_solve(info=True)
    nb, nr = g.linear_residual()
    assert nr < 1e-9 * nb, (nr, nb, info)


def test_default_lines_are_connected(need_gpu):
    case = _bl("ref")
    g, _ = _setup(case, lines=False)
    lines, colours = g.line_list()
    a = case.mesh.arrays()
    inner = a.cr >= 0
    pairs = set(zip(a.cl[inner].tolist(), a.cr[inner].tolist()))
    for L in lines:
        for x, y in zip(L[:-1], L[1:]):
            assert (x, y) in pairs or (y, x) in pairs
    # near the wall (dy << dx, dz) the strongest couplings are wall-normal
    assert max(len(L) for L in lines) >= 4


def test_lsgs_newton_step_matches_oracle(need_gpu):
    case = _bl("fp64")
    g, o = _setup(case)
    lines, colours = g.line_list()
    for _ in range(2):
        g.newton_step()
        o.residual()
        o.assemble()
        o.lsgs_solve(lines, colours)
        o.update()
    for a, b in zip(g.get_state(), o.get_state()):
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_single_cell_lines_match_oracle(need_gpu, prec):
    """The reference's own line set.  Its connection pass
    (linearSolverLSGS.loci:642-664) runs over equation numbers after unique()
    has removed every duplicate (:626-631), so it never links two cells and
    every line is one cell: LSGS is then the relaxed block iteration over
    single cells.  fpsi_set_lines expresses that set; the GPU result must
    match the oracle's restatement on the same lines and colours."""
    case = _bl(prec)
    g = FlowPsi(case.mesh, case.params)
    o = Oracle(case.mesh, case.params)
    g.set_lines([np.array([c], np.int32) for c in range(g.ncells)])
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    g.set_state(T, p, u)
    o.set_state(T, p, u)
    lines, colours = g.line_list()
    assert len(lines) == g.ncells and all(len(l) == 1 for l in lines)
    g.residual()
    o.residual()
    g.assemble()
    o.assemble()
    dg, ig = g.linear_solve(info=True)
    do, io = o.lsgs_solve(lines, colours)
    if prec == "fp64":
        assert ig["iterations"] == io["iterations"]
        for k in range(5):
            assert np.abs(dg[:, k] - do[:, k]).max() <= 1e-8 * np.abs(do[:, k]).max(), k
    else:
        c64 = _bl("fp64")
        o64 = Oracle(c64.mesh, c64.params)
        o64.set_state(*o.get_state())
        o64.residual()
        o64.assemble()
        d64, _ = o64.lsgs_solve(lines, colours)
        for k in range(5):
            e_orc = np.abs(do[:, k] - d64[:, k]).max()
            e_gpu = np.abs(dg[:, k] - d64[:, k]).max()
            assert e_gpu <= 2.0 * e_orc + 1e-6 * np.abs(d64[:, k]).max(), k
