"""Spalart-Allmaras nu~ transport in the oracle (turbulence/SA/SA_turb.loci,
solverScalarTransport.loci): properties that hold without a GPU.  CPU only."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from flowpsi_b200 import cases
from oracle import Oracle


def _bl(n=(6, 10, 4), solver="sgs"):
    c = cases.boundary_layer_block(*n, dy0=1e-4, growth=1.3, viscous=2, precision="fp64",
                                   solver=solver, sa=True)
    o = Oracle(c.mesh, c.params)
    o.set_state(*c.initial_state(o.geometry()["cellcenter"]))
    o.set_nutilde(c.nut0)
    return c, o


def test_wall_distance_is_the_height_above_the_wall():
    """flat wall at y = 0: the distance to the nearest wall face's plane is
    the cell centre's y (solverTurbulence.loci:133-137)"""
    c, o = _bl()
    y = o.geometry()["cellcenter"][:, 1]
    assert np.array_equal(o.wall_distance(), np.abs(y))


def test_no_walls_gives_a_large_distance():
    c = cases.farfield_cube(4)
    c.params.viscous, c.params.turbulence = 2, 1
    o = Oracle(c.mesh, c.params)
    assert np.all(o.wall_distance() == 1e30)


def test_eddy_viscosity_definition():
    """tmu = rho nu~ f_v1, chi = rho nu~ / mu (SA_turb.loci:91-107)"""
    c, o = _bl()
    rng = np.random.default_rng(1)
    nut = c.nut0 * (0.5 + rng.random(o.ncells))
    o.set_nutilde(nut)
    o.residual()
    T, p, _ = o.get_state()
    rho = p / (cases.RTILDE * T)
    mu = cases.sutherland_mu(T)
    assert np.allclose(o.eddy_viscosity(), cases.sa_eddy_viscosity(nut, rho, mu), rtol=1e-13)


def test_uniform_freestream_has_no_sa_source():
    """uniform flow, uniform nu~ equal to the inflow value, no walls: the
    convective fluxes cancel against the continuity term and every model
    term vanishes"""
    c = cases.farfield_cube(5)
    p = c.params
    p.viscous, p.turbulence = 2, 1
    o = Oracle(c.mesh, p)
    nc = o.ncells
    U0 = 0.5 * np.sqrt(1.4 * cases.RTILDE * 300.0)
    o.set_state(np.full(nc, 300.0), np.full(nc, 1e5), np.tile([U0, 0.0, 0.0], (nc, 1)))
    o.set_nutilde(np.full(nc, 5e-9))
    o.residual()
    src = o.sa_residual()
    scale = 5e-9 * 1.16 * U0 * (1.0 / 5) ** 2  # rho nu~ U A of one face
    assert np.abs(src).max() <= 1e-9 * scale


def test_scalar_sgs_converges_to_the_direct_solution():
    c, o = _bl()
    o.residual()
    B = o.sa_residual()
    S = o.sa_system()
    a = c.mesh.arrays()
    inner = a.cr >= 0
    cl, cr = a.cl[inner].astype(np.int64), a.cr[inner].astype(np.int64)
    nc = o.ncells
    # row cl couples to cr with U = fjm, row cr to cl with L = -fjp
    rows = np.concatenate([np.arange(nc), cl, cr])
    cols = np.concatenate([np.arange(nc), cr, cl])
    vals = np.concatenate([S["D"], S["fjm"][inner], -S["fjp"][inner]])
    A = sp.csr_matrix((vals, (rows, cols)), shape=(nc, nc))
    x = spla.spsolve(A.tocsc(), B)
    p = c.params
    p.gauss_seidel_iter = 200
    o.set_params(p)
    o.residual()
    o.sa_residual()
    dq = o.sa_solve()
    assert np.abs(dq - x).max() <= 1e-9 * np.abs(x).max()


@pytest.mark.parametrize("solver", ["sgs", "lsgs"])
def test_newton_steps_keep_nutilde_positive_and_reduce_the_residual(solver):
    c, o = _bl(solver=solver)
    hist, nmin = [], []
    colour = None
    for _ in range(12):
        if solver == "sgs":
            r = o.newton_step(colour)
        else:
            _, r = o.residual()
            o.sa_residual()
            o.sa_solve()
            o.assemble()
            o.lsgs_solve(c.lines)
            o.update()
            o.sa_update()
        hist.append(r["rtrms"])
        nmin.append(o.nutilde().min())
    assert min(nmin) > 0
    assert hist[-1] < 0.5 * hist[0]


def test_update_is_relaxed_and_positive():
    """X_next = max(X + min(1, urelax X/|dq|) dq, 1e-15)
    (solverScalarTransport.loci:397-405)"""
    c, o = _bl()
    nut0 = o.nutilde()
    o.residual()
    o.sa_residual()
    dq = o.sa_solve()
    o.sa_update()
    ts = np.minimum(1.0, c.params.urelax * nut0 / (np.abs(dq) + 1e-15))
    assert np.allclose(o.nutilde(), np.maximum(nut0 + ts * dq, 1e-15), rtol=1e-15, atol=0)
