"""Viscous face flux, thin-layer viscous Jacobians and the adiabatic no-slip
wall on the GPU against the oracle (fluxViscous.loci:112-448,
bcViscousWall.loci:148-240), laminar and turbulent (frozen SA eddy
viscosity).  GPU only; tolerances as in test_gpu_parity."""
import numpy as np
import pytest

from flowpsi_b200 import FlowPsi, cases
from oracle import Oracle
from tests.helpers import block_rel

pytestmark = pytest.mark.gpu


def _case(visc, prec, solver="sgs"):
    return cases.boundary_layer_block(6, 10, 4, dy0=1e-4, growth=1.3, viscous=visc,
                                      precision=prec, solver=solver)


def _pair(case):
    g = FlowPsi(case.mesh, case.params)
    o = Oracle(case.mesh, case.params)
    if case.tmu is not None:
        g.set_eddy_viscosity(case.tmu)
        o.set_eddy_viscosity(case.tmu)
    if case.params.solver == 1:
        g.set_lines(case.lines)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    g.set_state(T, p, u)
    o.set_state(T, p, u)
    return g, o


@pytest.mark.parametrize("flux", [None, 3, 4])
@pytest.mark.parametrize("visc", [1, 2])
def test_viscous_residual_matches_oracle(need_gpu, visc, flux):
    """flux None: the case's Roe flux; 3 and 4: the low-dissipation KEC and
    SSF fluxes with the viscous terms (fluxLowDiss.loci:320-640)"""
    case = _case(visc, "fp64")
    if flux is not None:
        case.params.flux = flux
    g, o = _pair(case)
    sg, ng = g.residual()
    so, no = o.residual()
    # flux scale: the inviscid fluxes dominate; measure against max |F| per cell
    scale = np.abs(so).max(axis=0, keepdims=True) + 1e-300
    fscale = 1e5 * o.geometry()["area"].max() * 400.0
    assert np.abs(sg - so).max() <= 1e-11 * fscale
    for k in ("rtrms", "etrms", "mtrms"):
        assert abs(ng[k] - no[k]) <= 1e-8 * abs(no[k])
    np.testing.assert_allclose(g.dtau(), o.dtau(), rtol=1e-10)
    _ = scale


@pytest.mark.parametrize("prec", ["fp64", "ref"])
@pytest.mark.parametrize("visc", [1, 2])
def test_viscous_blocks_match_oracle(need_gpu, visc, prec):
    g, o = _pair(_case(visc, prec))
    g.residual()
    o.residual()
    g.assemble()
    o.assemble()
    bg, bo = g.blocks(), o.blocks()
    tol = 1e-11 if prec == "fp64" else 1e-6
    for k in ("fjp", "fjm"):
        inner = np.abs(bo[k]).reshape(len(bo[k]), -1).max(1) > 0
        assert block_rel(bg[k][inner], bo[k][inner]) < tol, k


@pytest.mark.parametrize("solver", ["sgs", "lsgs"])
def test_viscous_newton_steps_match_oracle(need_gpu, solver):
    case = _case(2, "fp64", solver=solver)
    g, o = _pair(case)
    if solver == "sgs":
        col = g.colours()
        for _ in range(2):
            g.newton_step()
            o.newton_step(colour=col)
    else:
        lines, colours = g.line_list()
        for _ in range(2):
            g.newton_step()
            o.residual()
            o.assemble()
            o.lsgs_solve(lines, colours)
            o.update()
    for a, b in zip(g.get_state(), o.get_state()):
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()
