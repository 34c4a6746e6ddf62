"""The device path against the reference's own uniform-outcome quick tests
(quickTest/inviscid/{inflow,isentropic,fixedMass,superSonic}; fixture made by
tests/golden/make_quicktest_uniform.py): converged in FP64 and in MIXED, the
duct's state equals the reference's extracted P, T, u within the test's
relative tolerance, and the oracle's converged state within 1e-8 (the
converged-state tolerance; the fixed-mass state is a fixed-point iteration
that stops within 1e-9 of T on either side).  GPU only."""
import numpy as np
import pytest

from flowpsi_b200 import FlowPsi, cases
from tests.test_oracle_quicktest import GOLD, converge_oracle

pytestmark = pytest.mark.gpu


def converge_device(spec, precision, drop=1e-13, chunk=20, max_steps=600):
    c = cases.quicktest_duct(spec, precision=precision)
    g = FlowPsi(c.mesh, c.params)
    g.set_state(*c.initial_state(g.geometry()["cellcenter"]))
    r0, done = None, 0
    while done < max_steps:
        h = g.run(chunk)
        r0 = r0 or h[0]["rtrms"]
        done += chunk
        if h[-1]["rtrms"] < drop * r0:
            break
    st = g.get_state()
    g.close()
    return st, h[-1]["rtrms"] / r0


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(GOLD))
def test_device_reaches_the_reference_quicktest_state(need_gpu, name, prec):
    spec = GOLD[name]
    (T, p, u), drop = converge_device(spec, prec)
    assert drop < 1e-12
    e, tol = spec["expect"], spec["tol"][1]
    for got, want in ((p, e["P"]), (T, e["T"]), (u[:, 0], e["u"])):
        assert np.abs(got - want).max() <= tol * abs(want), (name, got.min(), got.max(), want)
    (To, po, uo), _ = converge_oracle(spec)
    for got, want in ((T, To), (p, po), (u, uo)):
        assert np.abs(got - want).max() <= 1e-8 * np.abs(want).max()
