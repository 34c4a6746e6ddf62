"""Mesh-level checks of the oracle (CPU): geometry closure, free-stream
preservation, exact gradients of linear fields, SGS convergence and Newton
residual decrease."""
import numpy as np
import pytest

from flowpsi_b200 import GeneratedMesh, bc, cases, default_params
from oracle import Oracle


def _closure(orc, mesh):
    a = mesh.arrays()
    g = orc.geometry()
    s = np.zeros((orc.ncells, 3))
    np.add.at(s, a.cl, g["area_vec"])
    inner = a.cr >= 0
    np.add.at(s, a.cr[inner], -g["area_vec"][inner])
    return np.abs(s).max() / g["area"].max()


@pytest.mark.parametrize("kind", ["hex", "kuhn", "bl"])
def test_geometry_closed_and_volume(kind):
    if kind == "hex":
        m = GeneratedMesh("hex", n=(5, 4, 3), L=(2.0, 1.0, 0.5), bc_side=(0,) * 6,
                          bcs=[bc("farfield")])
        vol = 1.0
    elif kind == "kuhn":
        m = GeneratedMesh("kuhn", n=(5, 4, 6), L=(1.0, 2.0, 3.0), jitter=0.1, seed=5)
        vol = 6.0
    else:
        m = GeneratedMesh("bl", n=(4, 6, 3), L=(1.0, 1.0, 1.0), dy0=1e-3, growth=1.3,
                          bc_side=(0, 0, 0, 0, -1, -1), bcs=[bc("farfield")])
        vol = sum(1e-3 * 1.3 ** j for j in range(6))
    o = Oracle(m, default_params(solver="sgs"))
    assert _closure(o, m) < 1e-12
    assert abs(o.geometry()["vol"].sum() - vol) < 1e-12 * vol


def test_freestream_preserved():
    case = cases.farfield_cube(6)
    o = Oracle(case.mesh, case.params)
    b = case.mesh.arrays().bcs[0]
    nc = o.ncells
    o.set_state(np.full(nc, b.T), np.full(nc, b.pg), np.tile(list(b.u), (nc, 1)))
    src, r = o.residual()
    assert np.abs(src).max() < 1e-9 * 1e5 * o.geometry()["area"].max()


def test_periodic_uniform_state_zero_residual():
    case = cases.taylor_green_tets(5)
    o = Oracle(case.mesh, case.params)
    nc = o.ncells
    o.set_state(np.full(nc, 300.0), np.full(nc, 1e5), np.tile([30.0, -20.0, 10.0], (nc, 1)))
    src, _ = o.residual()
    # energy flux scale rho*(|u|+a)*e0*area ~ 1e7 here: round-off only
    rho, a = 1e5 / (287.05 * 300.0), 347.0
    scale = rho * (40.0 + a) * (287.05 * 300.0 / 0.4) * o.geometry()["area"].max()
    assert np.abs(src).max() < 1e-14 * scale


def test_linear_field_gradient_exact():
    case = cases.taylor_green_tets(6)
    p = default_params(solver="sgs", limiter="none")
    o = Oracle(case.mesh, p)
    cc = o.geometry()["cellcenter"]
    # periodic box: use a field linear inside the box interior only and check
    # cells whose neighbours do not wrap
    L = 2 * np.pi
    T = 300.0 + 3.0 * cc[:, 0] - 2.0 * cc[:, 1] + 1.0 * cc[:, 2]
    o.set_state(T, np.full(len(T), 1e5), np.zeros((len(T), 3)))
    o.residual()
    g, phi = o.reconstruction()
    inner = np.all((cc > 0.25 * L) & (cc < 0.75 * L), axis=1)
    np.testing.assert_allclose(g[inner, 0:3], np.tile([3.0, -2.0, 1.0], (inner.sum(), 1)),
                               rtol=0, atol=1e-9)
    assert np.all(phi == 1.0)


@pytest.mark.parametrize("precision", ["fp64", "ref", "mixed"])
def test_sgs_reduces_linear_residual(precision):
    case = cases.farfield_cube(6, precision=precision)
    o = Oracle(case.mesh, case.params)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    o.set_state(T, p, u)
    o.residual()
    o.assemble()
    res = []
    for sweeps in (0, 1, 3, 6):
        prm = case.params
        prm.gauss_seidel_iter = sweeps
        o.set_params(prm)
        o.assemble()
        o.linear_solve()
        res.append(o.linear_residual()[1])
    assert res[1] < res[0] and res[3] < res[2] < res[1]


def test_multicolour_and_sequential_agree_at_convergence():
    case = cases.farfield_cube(5, precision="fp64")
    o = Oracle(case.mesh, case.params)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    o.set_state(T, p, u)
    o.residual()
    prm = case.params
    prm.gauss_seidel_iter = 60
    o.set_params(prm)
    o.assemble()
    seq = o.linear_solve()
    # red/black-like colouring of the structured hex grid
    idx = np.arange(o.ncells)
    i, j, k = idx % 5, (idx // 5) % 5, idx // 25
    colour = ((i + j + k) % 2).astype(np.int32)
    mc = o.linear_solve(colour=colour)
    assert np.abs(seq - mc).max() < 1e-8 * np.abs(seq).max()


def test_newton_decreases_residual():
    case = cases.farfield_cube(8)
    o = Oracle(case.mesh, case.params)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    o.set_state(T, p, u)
    r = [o.newton_step()["rtrms"] for _ in range(8)]
    assert r[-1] < 0.1 * r[0]


@pytest.mark.parametrize("prec", ["fp64", "ref"])
def test_lsgs_converges_to_the_linear_solution(prec):
    """line SGS with tight tolerances reaches the solution that many SGS
    sweeps reach (same blocks)"""
    case = cases.boundary_layer_block(6, 10, 4, dy0=1e-4, growth=1.3, precision=prec)
    p = case.params
    p.lsgs_max_iter, p.lsgs_rel_tol, p.lsgs_abs_tol, p.gauss_seidel_iter = 400, 1e-14, 0.0, 400
    o = Oracle(case.mesh, p)
    T, pr, u = case.initial_state(o.geometry()["cellcenter"])
    o.set_state(T, pr, u)
    o.residual()
    o.assemble()
    dl, info = o.lsgs_solve(case.lines)
    nb, nr = o.linear_residual()
    assert nr < (1e-9 if prec == "fp64" else 1e-4) * nb
    ds = o.linear_solve()
    assert np.abs(dl - ds).max() < (1e-8 if prec == "fp64" else 1e-3) * np.abs(ds).max()


def test_lsgs_relaxation_and_stopping_rules():
    """the default controls (w=0.25, rel 0.1, max 10) stop early and never
    exceed the iteration cap; a longer line sweep lowers the residual"""
    case = cases.boundary_layer_block(6, 10, 4, dy0=1e-4, growth=1.3, precision="fp64")
    o = Oracle(case.mesh, case.params)
    T, pr, u = case.initial_state(o.geometry()["cellcenter"])
    o.set_state(T, pr, u)
    o.residual()
    o.assemble()
    _, info = o.lsgs_solve(case.lines)
    assert 1 <= info["iterations"] <= 10
    assert info["resid"] < 0.1 * info["resid0"] or info["iterations"] == 10
    r_default = o.linear_residual()[1]
    single = [np.array([c], np.int32) for c in range(o.ncells)]
    o.lsgs_solve(single)
    assert r_default <= o.linear_residual()[1] * 1.0001


def test_viscous_linear_shear_has_no_net_force_inside():
    """a linear velocity field at constant T has constant stress: the viscous
    fluxes of a closed interior cell cancel (face gradients are exact for
    linear fields), so laminar and inviscid residuals agree there"""
    res = {}
    for visc in (0, 1):
        case = cases.boundary_layer_block(6, 8, 4, dy0=1e-3, growth=1.2, viscous=visc,
                                          solver="sgs", precision="fp64")
        p = case.params
        p.limiter = 2  # none: unlimited gradients keep the linear field exact
        o = Oracle(case.mesh, p)
        cc = o.geometry()["cellcenter"]
        nc = o.ncells
        u = np.zeros((nc, 3))
        u[:, 0] = 50.0 + 2.0e3 * cc[:, 1]  # z is periodic: no z dependence
        o.set_state(np.full(nc, 300.0), np.full(nc, 2e4), u)
        res[visc] = o.residual()[0]
    # two cells away from the walls: the boundary states (which differ
    # between the two regimes) reach one cell further through the gradients
    idx = np.arange(nc)
    i, j = idx % 6, (idx // 6) % 8
    inner = (i >= 2) & (i <= 3) & (j >= 2) & (j <= 5)
    mu = float(cases.sutherland_mu(300.0))
    scale = mu * 2.0e3 * o.geometry()["area"].max()
    d = np.abs(res[1][inner, 1:4] - res[0][inner, 1:4]).max()
    assert d < 1e-10 * scale, (d, scale)


def test_bdf2_oracle_properties():
    """The oracle's BDF2 step (solverTimestep.loci:397-428): a uniform state
    on a periodic grid is an exact solution (rhs zero, state kept), and on
    the Taylor-Green state the Newton iterations of one step converge."""
    from flowpsi_b200 import cases
    from oracle import Oracle

    c = cases.taylor_green_tets(3, precision="fp64")
    c.params.time_accurate, c.params.newton_iters, c.params.dtmax = 1, 12, 0.005
    o = Oracle(c.mesh, c.params)
    nc = o.ncells
    T, p, u = np.full(nc, 300.0), np.full(nc, 1e5), np.tile([30.0, -10.0, 5.0], (nc, 1))
    o.set_state(T, p, u)
    h = o.time_step()
    assert max(x["rtrms"] for x in h) < 1e-9
    for a, b in zip(o.get_state(), (T, p, u)):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-9)
    o.set_state(*c.initial_state(o.geometry()["cellcenter"]))
    h = o.time_step()
    assert h[-1]["rtrms"] < 1e-3 * h[0]["rtrms"]


def test_fsgs_reaches_the_sgs_steady_state():
    """FSGS (zero start, breadth-first order, linearSolverFSGS.loci) and SGS
    (Jacobi start, cell order) relax the same systems, so the steady state
    they converge to is the same"""
    from flowpsi_b200 import cases
    from oracle import Oracle

    out = []
    for solver in (0, 2):
        c = cases.farfield_cube(6, precision="fp64")
        c.params.solver = solver
        o = Oracle(c.mesh, c.params)
        o.set_state(*c.initial_state(o.geometry()["cellcenter"]))
        r0 = None
        for _ in range(200):
            r = o.newton_step()
            r0 = r0 or r["rtrms"]
            if r["rtrms"] < 1e-11 * r0:
                break
        assert r["rtrms"] < 1e-10 * r0
        out.append(o.get_state())
    for a, b in zip(*out):
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()


def _kec_case(flux=3, **lds):
    case = cases.taylor_green_tets(5, precision="fp64")
    case.params.flux = flux  # 3 KEC, 4 SSF
    for k, v in lds.items():
        setattr(case.params, k, v)
    return case


@pytest.mark.parametrize("flux", [3, 4])
def test_kec_preserves_uniform_flow(flux):
    """uniform flow on the jittered periodic tet grid: alpha_diss is 0 (no
    divergence), the upwind part sees equal states and the central kinetic-
    energy-consistent flux (fluxLowDiss.loci:258-298) of equal states is the
    analytic flux, so the residual is round-off"""
    case = _kec_case(flux)
    o = Oracle(case.mesh, case.params)
    nc = o.ncells
    o.set_state(np.full(nc, 300.0), np.full(nc, 1e5), np.tile([30.0, -20.0, 10.0], (nc, 1)))
    src, _ = o.residual()
    rho, a = 1e5 / (287.05 * 300.0), 347.0
    scale = rho * (40.0 + a) * (287.05 * 300.0 / 0.4) * o.geometry()["area"].max()
    assert np.abs(src).max() < 1e-14 * scale


@pytest.mark.parametrize("flux", [3, 4])
def test_kec_with_full_upwinding_is_hllc(flux):
    """LDS_useUpwind = 1 makes alpha_diss = 1 on every cell, so alpha = 1,
    the Thornber factor Ma = 1 and the central parts (and SSF's filter) have
    zero area: both low-dissipation fluxes are hllc_flux of the face states
    (fluxLowDiss.loci:371-399, 492-512)"""
    c_kec = _kec_case(flux, lds_use_upwind=1.0)
    c_hllc = cases.taylor_green_tets(5, precision="fp64")
    c_hllc.params.flux = 0
    a, b = Oracle(c_kec.mesh, c_kec.params), Oracle(c_hllc.mesh, c_hllc.params)
    st = c_kec.initial_state(a.geometry()["cellcenter"])
    a.set_state(*st)
    b.set_state(*st)
    sa, _ = a.residual()
    sb, _ = b.residual()
    assert np.array_equal(sa, sb)


def test_kec_differs_from_hllc_and_steps():
    """on the Taylor-Green state (M = 0.1, smooth) alpha_diss and the
    geometric switch stay small, so the KEC residual is mostly the central
    flux and differs from HLLC's; an implicit step with it (the Jacobians
    stay the Roe ones, inviscidFlux.h:92-107) lowers the residual"""
    case = _kec_case()
    o = Oracle(case.mesh, case.params)
    st = case.initial_state(o.geometry()["cellcenter"])
    o.set_state(*st)
    c_hllc = cases.taylor_green_tets(5, precision="fp64")
    c_hllc.params.flux = 0
    h = Oracle(c_hllc.mesh, c_hllc.params)
    h.set_state(*st)
    sk, _ = o.residual()
    sh, _ = h.residual()
    assert np.abs(sk - sh).max() > 1e-6 * np.abs(sh).max()
    r0 = o.newton_step()
    r1 = o.newton_step()
    assert np.isfinite(r1["rtrms"]) and r1["rtrms"] < r0["rtrms"]


def test_ssf_differs_from_kec():
    """the skew-symmetric scheme's extrapolated states and MILES filter
    (fluxLowDiss.loci:556-640) change the residual of the Taylor-Green state"""
    a, b = _kec_case(3), _kec_case(4)
    oa, ob = Oracle(a.mesh, a.params), Oracle(b.mesh, b.params)
    st = a.initial_state(oa.geometry()["cellcenter"])
    oa.set_state(*st)
    ob.set_state(*st)
    sa, _ = oa.residual()
    sb, _ = ob.residual()
    assert np.abs(sa - sb).max() > 1e-8 * np.abs(sa).max()
    r0 = ob.newton_step()
    r1 = ob.newton_step()
    assert np.isfinite(r1["rtrms"]) and r1["rtrms"] < r0["rtrms"]
