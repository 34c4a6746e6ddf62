"""fpsi_newton_step_ex: the steady step with a chosen starting iterate, a
linear tolerance and the rejection rule, through the C ABI.  GPU only.

The rule under test: the learned start only chooses where the relaxation
begins; a step started elsewhere than the reference's D^-1 B
(linearSolverSGS.loci:57-69) whose FP64 density residual does not drop is
undone and redone from D^-1 B.  A deliberately bad model (weights set from
the host) must therefore leave exactly the state of the reference's step.
"""
import numpy as np
import pytest

from flowpsi_b200 import FlowPsi, cases
from flowpsi_b200.learned import LearnedStart

pytestmark = pytest.mark.gpu


def _solver(prec="mixed", n=6):
    case = cases.farfield_tets(n, precision=prec)
    s = FlowPsi(case.mesh, case.params)
    s.keep_blocks(True)
    s.set_state(*case.initial_state(s.geometry()["cellcenter"]))
    return case, s


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_jacobi_start_equals_newton_step(need_gpu, prec):
    case, a = _solver(prec)
    _, b = _solver(prec)
    for _ in range(3):
        ra = a.newton_step()
        rb = b.newton_step_ex(start="jacobi", reject=False)
        assert ra["rtrms"] == rb["rtrms"]
        assert rb["start"] == "jacobi" and not rb["rejected"]
        assert rb["sweeps"] == case.params.gauss_seidel_iter
    for x, y in zip(a.get_state(), b.get_state()):
        np.testing.assert_array_equal(x, y)
    # the residual of the new state is the next step's starting residual
    r = b.newton_step_ex(start="jacobi", reject=False)
    assert r["rtrms"] == rb["after"]["rtrms"]


def test_untrained_model_gives_the_reference_step(need_gpu):
    """an untrained network outputs zero: the learned start is D^-1 B itself"""
    _, a = _solver("mixed")
    _, b = _solver("mixed")
    m = LearnedStart(seed=3)
    for _ in range(3):
        a.newton_step()
        r = b.newton_step_ex(start="learned", model=m, reject=True)
        assert r["start"] in ("learned", "jacobi")
    for x, y in zip(a.get_state(), b.get_state()):
        np.testing.assert_array_equal(x, y)
    m.close()


def test_bad_model_is_rejected(need_gpu):
    """a model whose start is far off: the step is undone and the
    reference's step is taken, bit for bit"""
    _, a = _solver("mixed")
    _, b = _solver("mixed")
    m = LearnedStart(seed=3)
    w = m.get_params()
    w[-5:] = 50.0  # head bias: d = 50 in every component, x0 = x_J + 50 xs
    m.set_params(w)
    a.newton_step()
    b.newton_step_ex(start="jacobi", reject=False)
    ra = a.newton_step()
    rb = b.newton_step_ex(start="learned", model=m, reject=True)
    assert rb["rejected"] and rb["start"] == "jacobi"
    assert ra["rtrms"] == rb["rtrms"]
    for x, y in zip(a.get_state(), b.get_state()):
        np.testing.assert_array_equal(x, y)
    # without the rule the bad start is kept and the residual rises
    _, c = _solver("mixed")
    c.newton_step_ex(start="jacobi", reject=False)
    rc = c.newton_step_ex(start="learned", model=m, reject=False)
    assert not rc["rejected"] and rc["after"]["rtrms"] > rc["rtrms"]
    m.close()


@pytest.mark.parametrize("start", ["zero", "jacobi"])
def test_linear_tolerance(need_gpu, start):
    """sweeps until ||B - A x|| <= 1e-3 ||B||; from zero the first measured
    residual is ||B|| itself"""
    _, s = _solver("fp64")
    r = s.newton_step_ex(start=start, reject=False, lin_rtol=1e-3, max_sweeps=100,
                         check_every=1)
    assert 0 < r["sweeps"] < 100
    assert r["lin_resid"] < r["lin_resid0"]
    if start == "zero":
        assert r["lin_resid"] <= 1e-3 * r["lin_resid0"] * (1 + 1e-12)
