"""The oracle's face functions against flowPsi's own: the committed golden
vectors (always) and the compiled reference functions (when built here).
CPU only."""
from pathlib import Path

import numpy as np
import pytest

from oracle import OracleFunctions, RefFunctions, ref_available
from tests.helpers import face_states, flux_scale, rel_to_scale

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "face_functions.npz")
SETS = ["mild", "strong", "rest"]
# FP64 flux agreement, relative to the flux scale (see helpers.flux_scale)
FLUX_TOL = 1e-14


def _data(name):
    return (GOLD[f"{name}_qL"], GOLD[f"{name}_qR"], GOLD[f"{name}_an"], GOLD[f"{name}_area"])


@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("eta", [1.0, 0.3])
@pytest.mark.parametrize("kind", ["hllc", "roe"])
def test_flux_golden(name, eta, kind):
    qL, qR, an, area = _data(name)
    got = OracleFunctions().flux(kind, qL, qR, an, area, eta=eta)
    ref = GOLD[f"{name}_eta{eta:g}_{kind}"]
    assert rel_to_scale(got, ref, flux_scale(qL, qR, an, area)) < FLUX_TOL


@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("eta", [1.0, 0.3])
@pytest.mark.parametrize("d", [1, -1])
def test_jacobian_golden_bitwise(name, eta, d):
    # real_fj blocks: the oracle reproduces the reference's float entries exactly
    qL, qR, an, area = _data(name)
    got = OracleFunctions().jacobian(qL, qR, an, area, d, eta=eta)
    ref = GOLD[f"{name}_eta{eta:g}_{'fjp' if d > 0 else 'fjm'}"]
    assert got.dtype == np.float32
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("outflow", [0, 1])
def test_cv_states_golden(name, outflow):
    qL, qR, an, area = _data(name)
    got = OracleFunctions().cv_state(outflow, qL, GOLD[f"{name}_q0"], an)
    ref = GOLD[f"{name}_cv_{'out' if outflow else 'in'}"]
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=0)


@pytest.mark.skipif(not ref_available(), reason="reference functions not built here")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_vs_compiled_reference(seed):
    qL, qR, an, area = face_states(4000, seed, jump=0.4, speed=300.0)
    O, R = OracleFunctions(), RefFunctions()
    sc = flux_scale(qL, qR, an, area)
    for kind in ("hllc", "roe"):
        for eta in (1.0, 0.5):
            assert rel_to_scale(O.flux(kind, qL, qR, an, area, eta=eta),
                                R.flux(kind, qL, qR, an, area, eta=eta), sc) < FLUX_TOL
    for d in (1, -1):
        np.testing.assert_array_equal(O.jacobian(qL, qR, an, area, d), R.jacobian(qL, qR, an, area, d))


def test_hlle_properties():
    """HLLE has no reference counterpart: check consistency F(q,q) = analytic
    flux, upwinding for supersonic states and conservation F(L,R,n) = -F(R,L,-n)."""
    O = OracleFunctions()
    qL, qR, an, area = face_states(500, 7, jump=0.3, speed=150.0)
    same = O.flux("hlle", qL, qL, an, area)
    roe_same = O.flux("roe", qL, qL, an, area)  # Roe reduces to the analytic flux too
    sc = flux_scale(qL, qL, an, area)
    assert rel_to_scale(same, roe_same, sc) < 1e-14
    f1 = O.flux("hlle", qL, qR, an, area)
    f2 = O.flux("hlle", qR, qL, -an, area)
    assert rel_to_scale(f1, -f2, flux_scale(qL, qR, an, area)) < 1e-14
    # supersonic along +n: HLLE equals the left analytic flux
    qs = qL.copy()
    qs[:, 2:5] = an * 2000.0
    qs2 = qR.copy()
    qs2[:, 2:5] = an * 2000.0
    up = O.flux("hlle", qs, qs2, an, area)
    left = O.flux("roe", qs, qs, an, area)
    assert rel_to_scale(up, left, flux_scale(qs, qs2, an, area)) < 1e-14
