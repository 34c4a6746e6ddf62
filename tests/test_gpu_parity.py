"""Parity of the CUDA path with the oracle, through the C ABI.  GPU only.

Tolerances (stated per quantity):
  * face fluxes and the residual 'src': 1e-12 of the flux scale (the
    magnitude of the flux terms; see tests.helpers.flux_scale);
  * FP32 (real_fj) Jacobian blocks: 1e-6 of the block's largest entry; FP64
    blocks 1e-11 (the device contracts multiply-adds, the oracle does not);
    fluid_D the same, relative to the summed magnitude of its face blocks;
  * gradients 1e-10 of the field's largest gradient, limiter values 1e-9;
  * relaxation result dq with the same colouring: 1e-8 of max|dq| (FP64;
    diagonal blocks reach condition numbers ~1e6); with FP32 blocks the GPU
    result must lie as close to the FP64 solution as the oracle's FP32
    result does (x2);
  * Newton states after 3 steps: 1e-10 relative (FP64); with FP32 blocks
    (REF, and MIXED with its FP32 sweeps and iterate) as close to the FP64
    trajectory as the oracle's FP32 states are (x2, plus 1e-7 relative).
"""
from pathlib import Path

import numpy as np
import pytest

from flowpsi_b200 import (FlowPsi, FpsiError, cases, inviscid_riemann_flux, roe_jacobian)
from flowpsi_b200 import _native as N
from oracle import Oracle, OracleFunctions
from tests.helpers import block_rel, face_states, flux_scale, rel_to_scale

pytestmark = pytest.mark.gpu

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "face_functions.npz")
RT, GAMMA = 8314.4621 / 28.96, 1.4


# --------------------------------------------------------------------------
# face functions
# --------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["mild", "strong", "rest"])
@pytest.mark.parametrize("eta", [1.0, 0.3])
def test_face_functions_golden(need_gpu, name, eta):
    qL, qR, an, area = (GOLD[f"{name}_{k}"] for k in ("qL", "qR", "an", "area"))
    sc = flux_scale(qL, qR, an, area)
    for kind in ("hllc", "roe"):
        got = inviscid_riemann_flux(kind, qL, qR, an, area, eta=eta)
        assert rel_to_scale(got, GOLD[f"{name}_eta{eta:g}_{kind}"], sc) < 1e-12
    for d, key in ((1, "fjp"), (-1, "fjm")):
        got = roe_jacobian(qL, qR, an, area, d, eta=eta)
        assert block_rel(got, GOLD[f"{name}_eta{eta:g}_{key}"]) < 1e-6


def test_face_functions_vs_oracle(need_gpu):
    qL, qR, an, area = face_states(20000, 21, jump=0.4, speed=300.0)
    O = OracleFunctions()
    sc = flux_scale(qL, qR, an, area)
    for kind in ("hllc", "roe", "hlle"):
        assert rel_to_scale(inviscid_riemann_flux(kind, qL, qR, an, area),
                            O.flux(kind, qL, qR, an, area), sc) < 1e-12
    for d in (1, -1):
        a = roe_jacobian(qL, qR, an, area, d, as_double=True)
        b = O.jacobian(qL, qR, an, area, d, as_double=True)
        assert block_rel(a, b) < 1e-11  # FP64 blocks: FMA contraction on the device


# --------------------------------------------------------------------------
# mesh level
# --------------------------------------------------------------------------
def _kec(case, flux=3):
    """the same case with a low-dissipation flux: 3 KEC (fluxLowDiss.loci:320-431),
    4 SSF (fluxLowDiss.loci:436-640)"""
    case.params.flux = flux
    return case


CASES = {
    "farfield_hex": lambda prec: cases.farfield_cube(8, precision=prec),
    "tgv_tets": lambda prec: cases.taylor_green_tets(5, precision=prec),
    "shock_hex": lambda prec: cases.oblique_shock_cube(8, precision=prec),
    "farfield_hllc": lambda prec: cases.farfield_cube(6, precision=prec, flux="hllc",
                                                      limiter="barth"),
    "outflow_p": lambda prec: cases.outflow_duct(6, precision=prec),
    "outflow_pmean": lambda prec: cases.outflow_duct(6, precision=prec, mean=True),
    "isentropic_in": lambda prec: cases.outflow_duct(6, precision=prec, inflow="isentropic"),
    "fixedmass_in": lambda prec: cases.outflow_duct(6, precision=prec, inflow="fixedMass"),
    "fixedmass_out": lambda prec: cases.outflow_duct(6, precision=prec, outflow="fixedMassOutflow"),
    "inflow_in": lambda prec: cases.outflow_duct(6, precision=prec, inflow="inflow"),
    "inflow_leaving": lambda prec: cases.outflow_duct(6, precision=prec, inflow="inflow", u_sign=-1.0),
    "kec_tgv_tets": lambda prec: _kec(cases.taylor_green_tets(5, precision=prec)),
    "kec_farfield_hex": lambda prec: _kec(cases.farfield_cube(6, precision=prec)),
    "kec_shock_hex": lambda prec: _kec(cases.oblique_shock_cube(8, precision=prec)),
    "ssf_tgv_tets": lambda prec: _kec(cases.taylor_green_tets(5, precision=prec), 4),
    "ssf_shock_hex": lambda prec: _kec(cases.oblique_shock_cube(8, precision=prec), 4),
}


def _pair(case):
    g = FlowPsi(case.mesh, case.params)
    o = Oracle(case.mesh, case.params)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    g.set_state(T, p, u)
    o.set_state(T, p, u)
    return g, o


def cell_scale(o, T, p, u):
    """per cell: flux-term magnitude times the cell's total face area"""
    a = o._mesh.arrays()
    area = o.geometry()["area"]
    asum = np.zeros(o.ncells)
    np.add.at(asum, a.cl, area)
    inner = a.cr >= 0
    np.add.at(asum, a.cr[inner], area[inner])
    rho = p / (RT * T)
    c = np.sqrt(GAMMA * RT * T)
    s = np.linalg.norm(u, axis=1) + c
    e0 = RT * T / (GAMMA - 1) + 0.5 * (u * u).sum(1)
    out = np.empty((o.ncells, 5))
    out[:, 0] = rho * s
    out[:, 1:4] = (rho * s * np.abs(u).max(1) + np.abs(p))[:, None]
    out[:, 4] = rho * s * e0 + np.abs(p) * s
    return out * asum[:, None]


@pytest.mark.parametrize("name", list(CASES))
def test_geometry_matches_oracle(need_gpu, name):
    g, o = _pair(CASES[name]("ref"))
    G, O = g.geometry(), o.geometry()
    np.testing.assert_allclose(G["vol"], O["vol"], rtol=1e-13)
    np.testing.assert_allclose(G["cellcenter"], O["cellcenter"], rtol=0,
                               atol=1e-13 * np.abs(O["cellcenter"]).max())
    np.testing.assert_allclose(G["area"], O["area"], rtol=1e-13)
    np.testing.assert_allclose(G["facecenter"], O["facecenter"], rtol=0,
                               atol=1e-13 * np.abs(O["facecenter"]).max())


@pytest.mark.parametrize("name", list(CASES))
def test_residual_matches_oracle(need_gpu, name):
    case = CASES[name]("ref")
    g, o = _pair(case)
    T, p, u = o.get_state()
    sg, ng = g.residual()
    so, no = o.residual()
    assert np.max(np.abs(sg - so) / cell_scale(o, T, p, u)) < 1e-12
    for k in ("rtrms", "etrms", "mtrms", "rtmax", "etmax", "mtmax"):
        assert abs(ng[k] - no[k]) <= 1e-9 * abs(no[k]) + 1e-300, k
    gg, lg = g.reconstruction()
    go, lo = o.reconstruction()
    for v in range(5):
        sl = slice(3 * v, 3 * v + 3)
        assert np.abs(gg[:, sl] - go[:, sl]).max() <= 1e-10 * np.abs(go[:, sl]).max() + 1e-300
    assert np.abs(lg - lo).max() < 1e-9
    np.testing.assert_allclose(g.dtau(), o.dtau(), rtol=1e-10)


# The total-pressure and fixed-mass inflows take one-sided differences of
# their boundary flux with steps of 1e-5 of the state (bcIsentropic.loci:
# 219-239, bcFixedMass.loci:199-224): a difference of the flux in its last
# digits is divided by 1e-5.  The isentropic state is closed-form, so device
# and oracle (whose pow and sqrt differ by an ulp) agree to ~1e-16/1e-5 of
# the block scale; the fixed-mass state comes from a fixed-point iteration
# that stops within 1e-9 of T, so the two agree to ~1e-9/1e-5.  These
# tolerances hold for those faces' blocks and for the diagonal blocks that
# sum them.
FD_TOL = {"isentropic_in": 1e-8, "fixedmass_in": 1e-3}


@pytest.mark.parametrize("prec", ["fp64", "ref", "mixed"])
@pytest.mark.parametrize("name", ["farfield_hex", "tgv_tets", "shock_hex", "isentropic_in",
                                  "fixedmass_in", "fixedmass_out", "inflow_in", "inflow_leaving"])
def test_blocks_match_oracle(need_gpu, name, prec):
    g, o = _pair(CASES[name](prec))
    g.residual()
    o.residual()
    g.assemble()
    o.assemble()
    bg, bo = g.blocks(), o.blocks()
    tol = 1e-11 if prec == "fp64" else 1e-6
    a = o._mesh.arrays()
    fd = np.zeros(a.nfaces, bool)
    if name in FD_TOL:  # the inflow is condition 0 of the duct
        fd = np.asarray(a.cr) == -1
    for k in ("fjp", "fjm"):
        assert bg[k].dtype == bo[k].dtype
        inner = (np.abs(bo[k]).reshape(len(bo[k]), -1).max(1) > 0) & ~fd
        assert block_rel(bg[k][inner], bo[k][inner]) < tol, k
    if fd.any():
        assert block_rel(bg["fjp"][fd], bo["fjp"][fd]) < FD_TOL[name]
        tol = max(tol, FD_TOL[name])
    # fluid_D sums the cell's face blocks (srcJ, solverLinearSystem.loci:106-121)
    # with cancellation; its error is measured against the size of the summands
    mx = lambda b: np.abs(b.astype(np.float64)).reshape(len(b), -1).max(1)  # noqa: E731
    scale = mx(bo["fluid_D"])
    np.add.at(scale, a.cl, mx(bo["fjp"]))
    inner = a.cr >= 0
    np.add.at(scale, a.cr[inner], mx(bo["fjm"])[inner])
    d = np.abs(bg["fluid_D"].astype(np.float64) - bo["fluid_D"]).reshape(len(scale), -1).max(1)
    assert np.max(d / scale) < tol
    np.testing.assert_allclose(bg["fluid_B"], bo["fluid_B"], rtol=tol,
                               atol=tol * np.abs(bo["fluid_B"]).max())


@pytest.mark.parametrize("prec", ["fp64", "ref", "mixed"])
@pytest.mark.parametrize("name", ["farfield_hex", "tgv_tets"])
def test_multicolour_sgs_matches_oracle(need_gpu, name, prec):
    g, o = _pair(CASES[name](prec))
    g.residual()
    o.residual()
    g.assemble()
    o.assemble()
    col = g.colours()
    dg = g.linear_solve()
    do = o.linear_solve(colour=col)
    if prec == "fp64":
        # diagonal blocks reach condition numbers ~1e6 at M=0.1: 1e-8
        for k in range(5):
            assert np.abs(dg[:, k] - do[:, k]).max() <= 1e-8 * np.abs(do[:, k]).max(), k
    else:
        # FP32 blocks: the GPU result must be as close to the FP64 solution of
        # the same system as the oracle's own FP32 result is
        c64 = CASES[name]("fp64")
        o64 = Oracle(c64.mesh, c64.params)
        o64.set_state(*o.get_state())
        o64.residual()
        o64.assemble()
        d64 = o64.linear_solve(colour=col)
        for k in range(5):
            e_orc = np.abs(do[:, k] - d64[:, k]).max()
            e_gpu = np.abs(dg[:, k] - d64[:, k]).max()
            assert e_gpu <= 2.0 * e_orc + 1e-6 * np.abs(d64[:, k]).max(), k
    nb, nr = g.linear_residual()
    assert nr < nb


def test_sgs_converges_on_gpu(need_gpu):
    case = CASES["farfield_hex"]("fp64")
    g, _ = _pair(case)
    g.residual()
    res = []
    for sweeps in (1, 4, 16):
        p = case.params
        p.gauss_seidel_iter = sweeps
        g.set_params(p)
        g.assemble()
        g.linear_solve()
        res.append(g.linear_residual()[1])
    assert res[2] < res[1] < res[0]


@pytest.mark.parametrize("prec", ["fp64", "ref", "mixed"])
@pytest.mark.parametrize("name", ["farfield_hex", "tgv_tets", "shock_hex", "outflow_pmean",
                                  "isentropic_in", "fixedmass_in", "fixedmass_out", "inflow_in",
                                  "inflow_leaving"])
def test_newton_steps_match_oracle(need_gpu, name, prec):
    case = CASES[name](prec)
    g, o = _pair(case)
    col = g.colours()
    if prec != "fp64":
        c64 = CASES[name]("fp64")
        o64 = Oracle(c64.mesh, c64.params)
        o64.set_state(*o.get_state())
    for _ in range(3):
        rg = g.newton_step()
        ro = o.newton_step(colour=col)
        if prec == "fp64":
            assert abs(rg["rtrms"] - ro["rtrms"]) <= 1e-8 * ro["rtrms"]
        else:
            o64.newton_step(colour=col)
            # the norms of the first step come from the same state
            assert abs(rg["rtrms"] - ro["rtrms"]) <= 1e-3 * ro["rtrms"]
    Tg, pg_, ug = g.get_state()
    To, po, uo = o.get_state()
    if prec == "fp64":
        np.testing.assert_allclose(Tg, To, rtol=1e-10)
        np.testing.assert_allclose(pg_, po, rtol=1e-10)
        assert np.abs(ug - uo).max() <= 1e-10 * np.abs(uo).max()
    else:
        # FP32 blocks: the GPU state must be as close to the FP64 trajectory
        # as the oracle's own FP32 state is (x2, plus 1e-7 relative)
        T6, p6, u6 = o64.get_state()
        for a, b, c in ((Tg, To, T6), (pg_, po, p6), (ug, uo, u6)):
            e_orc = np.abs(b - c).max()
            e_gpu = np.abs(a - c).max()
            assert e_gpu <= 2.0 * e_orc + 1e-7 * np.abs(c).max()


def test_run_is_deterministic_and_equals_steps(need_gpu):
    case = CASES["tgv_tets"]("mixed")
    g, o = _pair(case)
    T0, p0, u0 = g.get_state()
    h1 = g.run(3)
    s1 = g.get_state()
    g.set_state(T0, p0, u0)
    h2 = [g.newton_step() for _ in range(3)]
    s2 = g.get_state()
    for a, b in zip(s1, s2):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(h1, h2):
        assert a["rtrms"] == b["rtrms"] and a["etrms"] == b["etrms"]


def _bl_sa(prec, solver):
    return cases.boundary_layer_block(6, 10, 4, dy0=1e-4, growth=1.3, viscous=2, precision=prec,
                                      solver=solver, sa=True)


@pytest.mark.parametrize("name,prec,flux", [("tgv_tets", "mixed", None), ("farfield_hex", "fp64", None),
                                            ("shock_hex", "ref", None), ("tgv_tets", "mixed", 3),
                                            ("bl_sa_sgs", "mixed", None), ("bl_sa_lsgs", "mixed", None),
                                            ("bl_sa_lsgs", "fp64", None)])
def test_step_graphs_replay_the_launched_steps(need_gpu, name, prec, flux):
    """fpsi_run replays a captured graph of its second step for the rest:
    history and state (and nu~ with the SA model) equal those of launching
    every step, bit for bit"""
    case = _bl_sa(prec, name[6:]) if name.startswith("bl_sa") else CASES[name](prec)
    out = []
    for graphs in (1, 0):
        p = N.Params.from_buffer_copy(case.params)
        p.step_graphs = graphs
        if flux is not None:
            p.flux = flux
        g = FlowPsi(case.mesh, p)
        if p.solver == 1:
            g.set_lines(case.lines)
        g.set_state(*case.initial_state(g.geometry()["cellcenter"]))
        if name.startswith("bl_sa"):
            g.set_nutilde(case.nut0)
        h = g.run(6)
        h += g.run(3)
        out.append((h, g.get_state(), g.nutilde() if name.startswith("bl_sa") else None))
        g.close()
    for a, b in zip(out[0][1], out[1][1]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(out[0][0], out[1][0]):
        assert a == b
    if out[0][2] is not None:
        np.testing.assert_array_equal(out[0][2], out[1][2])


def test_nan_state_is_reported(need_gpu):
    case = CASES["farfield_hex"]("ref")
    g, o = _pair(case)
    T, p, u = g.get_state()
    T[3] = np.nan
    g.set_state(T, p, u)
    with pytest.raises(FpsiError) as e:
        g.residual()
    assert e.value.code == -6  # FPSI_E_NAN, as solverResidual.loci:203-208 aborts


def test_run_stops_at_the_nan_step(need_gpu):
    """fpsi_run ends at the first step whose residual norms are NaN, with the
    state of that step, as solverResidual.loci:203-208 aborts"""
    case = CASES["farfield_hex"]("mixed")
    g, _ = _pair(case)
    g.run(2)
    T, p, u = g.get_state()
    good = (T.copy(), p.copy(), u.copy())
    T[3] = np.nan
    g.set_state(T, p, u)
    with pytest.raises(FpsiError) as e:
        g.run(6)
    assert e.value.code == -6
    assert "step 0 of 6" in str(e.value)
    assert all(np.isnan(h["rtrms"]) for h in e.value.history)
    T2, p2, u2 = g.get_state()
    # the queued steps after the NaN residual left the state alone
    np.testing.assert_array_equal(T2, T)
    np.testing.assert_array_equal(p2, p)
    np.testing.assert_array_equal(u2, u)
    # a valid state runs again, with no stale error left behind
    g.set_state(*good)
    h = g.run(2)
    assert all(np.isfinite(x["rtrms"]) for x in h)


@pytest.mark.parametrize("mean", [False, True])
def test_outflow_that_became_inflow_is_flagged(need_gpu, mean):
    """bcOutflow.loci:238-243: a face of an outflow whose flow enters sets
    OUTFLOW_BECAME_INFLOW in the residual's bcErrorCode (flowPsiIO.h:212)"""
    case = cases.outflow_duct(6, precision="fp64", mean=mean)
    g, o = _pair(case)
    _, ng = g.residual()
    assert ng["bcErrorCode"] == 0
    T, p, u = g.get_state()
    u[:, 0] = -np.abs(u[:, 0])
    g.set_state(T, p, u)
    o.set_state(T, p, u)
    sg, ng = g.residual()
    so, no = o.residual()
    assert ng["bcErrorCode"] == no["bcErrorCode"] == 1
    assert np.max(np.abs(sg - so) / cell_scale(o, T, p, u)) < 1e-12
    # the bit belongs to that residual only
    u[:, 0] = np.abs(u[:, 0])
    g.set_state(T, p, u)
    assert g.residual()[1]["bcErrorCode"] == 0


def test_call_order_enforced(need_gpu):
    case = CASES["farfield_hex"]("ref")
    g, _ = _pair(case)
    with pytest.raises(FpsiError) as e:
        g.assemble()
    assert e.value.code == -8
    with pytest.raises(FpsiError):
        g.linear_solve()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_fsgs_matches_oracle(need_gpu, prec):
    """fluidLinearSolver 'fsgs' (linearSolverFSGS.loci:1601-1700): symmetric
    sweeps from a zero start.  The oracle sweeps in the GPU's colour order;
    FP64 1e-8 of max|dq| after one solve and 1e-10 of the state after three
    steps, FP32 as close to the FP64 solution as the oracle's own."""
    def mk(p):
        c = cases.farfield_cube(8, precision=p)
        c.params.solver = 2
        return c

    case = mk(prec)
    g, o = _pair(case)
    col = g.colours()
    g.residual()
    o.residual()
    g.assemble()
    o.assemble()
    dg = g.linear_solve()
    do = o.linear_solve(colour=col)
    if prec == "fp64":
        for k in range(5):
            assert np.abs(dg[:, k] - do[:, k]).max() <= 1e-8 * np.abs(do[:, k]).max(), k
        for _ in range(3):
            g.newton_step()
            o.newton_step(colour=col)
        for a, b in zip(g.get_state(), o.get_state()):
            assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()
    else:
        c64 = mk("fp64")
        o64 = Oracle(c64.mesh, c64.params)
        o64.set_state(*o.get_state())
        o64.residual()
        o64.assemble()
        d64 = o64.linear_solve(colour=col)
        for k in range(5):
            e_orc = np.abs(do[:, k] - d64[:, k]).max()
            e_gpu = np.abs(dg[:, k] - d64[:, k]).max()
            assert e_gpu <= 2.0 * e_orc + 1e-6 * np.abs(d64[:, k]).max(), k
