"""Ragged cells: the prism grid (every hex split into two triangular prisms,
five faces per cell, triangles and quads mixed) through the whole device
path against the oracle.  GPU only.  Tolerances are those of
test_gpu_parity (stated there); the viscous and SA steps those of
test_gpu_sa."""
import math

import numpy as np
import pytest

from flowpsi_b200 import FlowPsi, cases
from flowpsi_b200.solver import GeneratedMesh, bc, default_params
from oracle import Oracle
from tests.helpers import block_rel
from tests.test_gpu_parity import cell_scale

pytestmark = pytest.mark.gpu

RT, GAMMA = cases.RTILDE, cases.GAMMA


def prism_case(n=(5, 4, 3), prec="fp64", flux="roe", limiter="venkatakrishnan",
               periodic=False, viscous=0, sa=False, solver="sgs", seed=0):
    """farfield (or periodic) prism box at M=0.5 with 1% noise; with a viscous
    regime the y-min side is an adiabatic no-slip wall"""
    T0, p0, M = 300.0, 1e5, 0.5
    U0 = M * math.sqrt(GAMMA * RT * T0)
    ff = bc("farfield", T=T0, pg=p0, u=(U0, 0.1 * U0, 0.0), nu_t=3e-5 if sa else 0.0)
    wall = bc("viscousWall", T=T0, pg=p0)
    if periodic:
        side = (-1,) * 6
    elif viscous:
        side = (0, 0, 1, 0, 0, 0)
    else:
        side = (0,) * 6
    mesh = GeneratedMesh("prism", n=n, bc_side=side, bcs=[ff, wall])
    params = default_params(flux=flux, limiter=limiter, solver=solver, gauss_seidel_iter=6,
                            cflmax=20.0, precision=prec, viscous=viscous,
                            turbulence=1 if sa else 0)

    def init(cc):
        nc = cc.shape[0]
        r = cases.normal
        T = T0 * (1 + 0.01 * r(seed, 0, nc))
        p = p0 * (1 + 0.01 * r(seed, 1, nc))
        u = np.empty((nc, 3))
        u[:, 0] = U0 * (1 + 0.01 * r(seed, 2, nc))
        u[:, 1] = 0.1 * U0 + 0.01 * U0 * r(seed, 3, nc)
        u[:, 2] = 0.01 * U0 * r(seed, 4, nc)
        return T, p, u

    c = cases.Case("prism_box", mesh, params, 10, init)
    c.nut0 = np.full(2 * n[0] * n[1] * n[2], 3e-5) if sa else None
    return c


def _pair(case):
    g = FlowPsi(case.mesh, case.params)
    o = Oracle(case.mesh, case.params)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    g.set_state(T, p, u)
    o.set_state(T, p, u)
    if case.nut0 is not None:
        g.set_nutilde(case.nut0)
        o.set_nutilde(case.nut0)
    return g, o


FLUXES = [("roe", "venkatakrishnan"), ("hllc", "barth"), ("hlle", "none")]


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("flux,limiter", FLUXES)
def test_prism_residual_matches_oracle(need_gpu, flux, limiter, periodic):
    case = prism_case(flux=flux, limiter=limiter, periodic=periodic)
    g, o = _pair(case)
    G, O = g.geometry(), o.geometry()
    np.testing.assert_allclose(G["vol"], O["vol"], rtol=1e-13)
    T, p, u = o.get_state()
    sg, ng = g.residual()
    so, no = o.residual()
    assert np.max(np.abs(sg - so) / cell_scale(o, T, p, u)) < 1e-12
    for k in ("rtrms", "etrms", "mtrms"):
        assert abs(ng[k] - no[k]) <= 1e-9 * abs(no[k]) + 1e-300, k
    gg, lg = g.reconstruction()
    go, lo = o.reconstruction()
    assert np.abs(gg - go).max() <= 1e-10 * np.abs(go).max()
    assert np.abs(lg - lo).max() < 1e-9
    np.testing.assert_allclose(g.dtau(), o.dtau(), rtol=1e-10)


@pytest.mark.parametrize("prec", ["fp64", "ref"])
def test_prism_blocks_and_solve_match_oracle(need_gpu, prec):
    case = prism_case(prec=prec)
    g, o = _pair(case)
    g.residual()
    o.residual()
    g.assemble()
    o.assemble()
    bg, bo = g.blocks(), o.blocks()
    tol = 1e-11 if prec == "fp64" else 1e-6
    for k in ("fjp", "fjm"):
        inner = np.abs(bo[k]).reshape(len(bo[k]), -1).max(1) > 0
        assert block_rel(bg[k][inner], bo[k][inner]) < tol, k
    if prec == "fp64":
        dg = g.linear_solve()
        do = o.linear_solve(colour=g.colours())
        for k in range(5):
            assert np.abs(dg[:, k] - do[:, k]).max() <= 1e-8 * np.abs(do[:, k]).max(), k


def test_prism_newton_steps_match_oracle(need_gpu):
    case = prism_case()
    g, o = _pair(case)
    col = g.colours()
    for _ in range(3):
        g.newton_step()
        o.newton_step(colour=col)
    for a, b in zip(g.get_state(), o.get_state()):
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()


def test_prism_line_sgs_matches_oracle(need_gpu):
    case = prism_case(solver="lsgs", n=(4, 6, 3))
    g, o = _pair(case)
    lines, lcol = g.line_list()
    g.residual()
    o.residual()
    g.assemble()
    o.assemble()
    dg, ig = g.linear_solve(info=True)
    do, io = o.lsgs_solve(lines, lcol)
    assert ig["iterations"] == io["iterations"]
    for k in range(5):
        assert np.abs(dg[:, k] - do[:, k]).max() <= 1e-8 * np.abs(do[:, k]).max(), k


@pytest.mark.parametrize("sa", [False, True])
def test_prism_viscous_steps_match_oracle(need_gpu, sa):
    """laminar, or turbulent with the SA transport, next to a no-slip wall"""
    case = prism_case(viscous=2 if sa else 1, sa=sa)
    g, o = _pair(case)
    col = g.colours()
    for _ in range(2):
        g.newton_step()
        o.newton_step(colour=col)
    for a, b in zip(g.get_state(), o.get_state()):
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()
    if sa:
        nb = o.nutilde()
        assert np.abs(g.nutilde() - nb).max() <= 1e-9 * np.abs(nb).max()
