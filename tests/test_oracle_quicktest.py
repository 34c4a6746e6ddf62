"""The oracle against the reference's own uniform-outcome quick tests
(quickTest/inviscid/{inflow,isentropic,fixedMass,superSonic}; fixture made by
tests/golden/make_quicktest_uniform.py).  Each drives a unit-section duct
from an inflow condition (bcInflow.loci:270-309 and 376-431,
bcIsentropic.loci, bcFixedMass.loci) to an outflow condition
(bcOutflow.loci:127-165 and 174-273), stepped as the test is (its dtmax as
the pseudo-time step, its urelax); the converged state is uniform and fixed
by the two conditions, so it is compared with the reference's extracted P,
T, u at the test's own relative tolerance."""
import json
from pathlib import Path

import numpy as np
import pytest

from flowpsi_b200 import cases
from oracle import Oracle

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "quicktest_uniform.json").read_text())


def converge_oracle(spec, drop=1e-13, max_steps=600):
    c = cases.quicktest_duct(spec)
    o = Oracle(c.mesh, c.params)
    o.set_state(*c.initial_state(o.geometry()["cellcenter"]))
    r0 = None
    for _ in range(max_steps):
        r = o.newton_step()
        r0 = r0 or r["rtrms"]
        if r["rtrms"] < drop * r0:
            break
    return o.get_state(), r["rtrms"] / r0


@pytest.mark.parametrize("name", list(GOLD))
def test_oracle_reaches_the_reference_quicktest_state(name):
    spec = GOLD[name]
    (T, p, u), drop = converge_oracle(spec)
    assert drop < 1e-12
    e, tol = spec["expect"], spec["tol"][1]
    for got, want in ((p, e["P"]), (T, e["T"]), (u[:, 0], e["u"])):
        assert np.abs(got - want).max() <= tol * abs(want), (name, got.min(), got.max(), want)
    assert np.abs(u[:, 1:]).max() <= 1e-9 * e["u"]
