"""Time-accurate BDF2 stepping (timeStepAccurate, timeStepSchemeBDF2) on the
GPU against the oracle's restatement, through the C ABI.  GPU only.

One time step is params.newton_iters Newton iterations on the state of the
new level with the residual rhs = src - 1.5 (Q(n+1) - Q(n)) V/dt +
0.5 (Q(n) - Q(n-1)) V/dt (solverTimestep.loci:397-428), diagonal blocks
-srcJ + 1.5 V/dtau dQ/dq (solverLinearSystem.loci:376-435) and the update
clipped at 0.75 of T and p (solverNewton.loci:163-182); the first step takes
Q(n-1) = Q(n) = the initial state (solverTimestep.loci:157-166).  The oracle
relaxes in the GPU's colour order.  Tolerances: FP64 rhs norms 1e-8 relative
per iteration and states 1e-10 relative after two steps; FP32 blocks (REF,
MIXED) as close to the FP64 trajectory as the oracle's own FP32 run (x2,
plus 1e-7 relative).
"""
import numpy as np
import pytest

from flowpsi_b200 import FlowPsi, FpsiError, cases
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _case(prec):
    c = cases.taylor_green_tets(5, precision=prec)
    c.params.time_accurate = 1
    c.params.newton_iters = 3
    c.params.dtmax = 0.005
    return c


@pytest.mark.parametrize("prec", ["fp64", "ref", "mixed"])
def test_bdf2_steps_match_oracle(need_gpu, prec):
    case = _case(prec)
    g = FlowPsi(case.mesh, case.params)
    o = Oracle(case.mesh, case.params)
    T, p, u = case.initial_state(o.geometry()["cellcenter"])
    g.set_state(T, p, u)
    o.set_state(T, p, u)
    col = g.colours()
    hg = [g.time_step() for _ in range(2)]
    ho = [o.time_step(colour=col) for _ in range(2)]
    assert len(hg[0]) == 3
    sg, so = g.get_state(), o.get_state()
    if prec == "fp64":
        for a_step, b_step in zip(hg, ho):
            for a, b in zip(a_step, b_step):
                for key in ("rtrms", "etrms", "mtrms"):
                    assert abs(a[key] - b[key]) <= 1e-8 * b[key], (key, a[key], b[key])
        for a, b in zip(sg, so):
            assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()
    else:
        c64 = _case("fp64")
        o64 = Oracle(c64.mesh, c64.params)
        o64.set_state(T, p, u)
        for _ in range(2):
            o64.time_step(colour=col)
        for a, b, c in zip(sg, so, o64.get_state()):
            e_orc = np.abs(b - c).max()
            e_gpu = np.abs(a - c).max()
            assert e_gpu <= 2.0 * e_orc + 1e-7 * np.abs(c).max(), (e_gpu, e_orc)
    # the Newton iterations of a step lower its rhs
    for h in hg:
        assert h[-1]["rtrms"] < h[0]["rtrms"]
    # the state moved in time
    assert np.abs(sg[2] - u).max() > 0


def test_time_step_needs_time_accurate_mode(need_gpu):
    case = cases.taylor_green_tets(5, precision="fp64")
    g = FlowPsi(case.mesh, case.params)
    g.set_state(*case.initial_state(g.geometry()["cellcenter"]))
    with pytest.raises(FpsiError) as e:
        g.time_step()
    assert e.value.code == -8
