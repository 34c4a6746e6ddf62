"""Spalart-Allmaras nu~ transport on the GPU against the oracle's restatement
(turbulence/SA/SA_turb.loci, solverScalarTransport.loci,
linearSolverSGS.loci:333-470), through the C ABI.  GPU only.

Tolerances: the wall distance and the eddy viscosity 1e-13 relative; the
scalar right-hand side 1e-9 of its largest entry (it is a difference of
convective fluxes that cancel to 1e-6 of their size in smooth flow); the
off-diagonal coefficients 1e-12; the diagonal 1e-9 (it holds rho V / dtau,
and dtau follows the mean flow's residual, itself a cancelling sum); the
solve 1e-10; states after Newton steps 1e-9.
"""
import numpy as np
import pytest

from flowpsi_b200 import FlowPsi, cases
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _case(prec="fp64", solver="sgs", n=(6, 10, 4)):
    return cases.boundary_layer_block(*n, dy0=1e-4, growth=1.3, viscous=2, precision=prec,
                                      solver=solver, sa=True)


def _pair(case):
    g = FlowPsi(case.mesh, case.params)
    o = Oracle(case.mesh, case.params)
    if case.params.solver == 1:
        g.set_lines(case.lines)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    g.set_state(T, p, u)
    o.set_state(T, p, u)
    rng = np.random.default_rng(3)
    nut = case.nut0 * (0.5 + rng.random(g.ncells))
    g.set_nutilde(nut)
    o.set_nutilde(nut)
    return g, o


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_wall_distance_matches(need_gpu):
    case = _case()
    g, o = _pair(case)
    assert _rel(g.wall_distance(), o.wall_distance()) <= 1e-13


def test_wall_distance_in_a_box_of_walls(need_gpu):
    """five no-slip walls and a stretched grid: the k-d tree search against
    the oracle's exhaustive search"""
    from flowpsi_b200.solver import GeneratedMesh, bc, default_params
    mesh = GeneratedMesh("bl", n=(7, 6, 5), L=(1.0, 1.0, 0.5), dy0=0.05, growth=1.2,
                         bc_side=(1, 1, 1, 0, 1, 1), bcs=[bc("farfield"), bc("viscousWall")])
    p = default_params(viscous=2, turbulence=1, precision="fp64")
    g = FlowPsi(mesh, p)
    o = Oracle(mesh, p)
    dg, do = g.wall_distance(), o.wall_distance()
    assert dg.max() < 1.0
    assert _rel(dg, do) <= 1e-13


def test_eddy_viscosity_and_sa_residual_match(need_gpu):
    case = _case()
    g, o = _pair(case)
    g.residual()
    o.residual()
    assert _rel(g.eddy_viscosity(), o.eddy_viscosity()) <= 1e-13
    bg, bo = g.sa_residual(), o.sa_residual()
    assert _rel(bg, bo) <= 1e-9
    sg, so = g.sa_system(), o.sa_system()
    assert _rel(sg["D"], so["D"]) <= 1e-9
    for k in ("fjp", "fjm"):
        assert _rel(sg[k], so[k]) <= 1e-12, k


@pytest.mark.parametrize("prec", ["fp64", "ref", "mixed"])
def test_sa_solve_and_update_match(need_gpu, prec):
    case = _case(prec)
    g, o = _pair(case)
    g.residual()
    o.residual()
    g.sa_residual()
    o.sa_residual()
    dg = g.sa_solve()
    do = o.sa_solve(g.colours())
    assert _rel(dg, do) <= 1e-10
    g.sa_update()
    o.sa_update()
    assert _rel(g.nutilde(), o.nutilde()) <= 1e-10


def test_newton_steps_with_sa_match(need_gpu):
    case = _case("fp64")
    g, o = _pair(case)
    col = g.colours()
    for _ in range(3):
        g.newton_step()
        o.newton_step(col)
    for a, b in zip(g.get_state(), o.get_state()):
        assert _rel(a, b) <= 1e-9
    assert _rel(g.nutilde(), o.nutilde()) <= 1e-9


def test_line_sgs_steps_with_sa_match(need_gpu):
    case = _case("fp64", solver="lsgs")
    g, o = _pair(case)
    lines, lcol = g.line_list()
    col = g.colours()
    for _ in range(2):
        g.newton_step()
        o.residual()
        o.sa_residual()
        o.sa_solve(col)
        o.assemble()
        o.lsgs_solve(lines, lcol)
        o.update()
        o.sa_update()
    for a, b in zip(g.get_state(), o.get_state()):
        assert _rel(a, b) <= 1e-9
    assert _rel(g.nutilde(), o.nutilde()) <= 1e-9


def test_run_with_sa_keeps_nutilde_positive(need_gpu):
    case = _case("mixed", n=(16, 24, 8))
    g, _ = _pair(case)
    hist = g.run(30)
    nut = g.nutilde()
    assert nut.min() > 0 and np.isfinite(nut).all()
    assert hist[-1]["rtrms"] < hist[0]["rtrms"]
