"""The C ABI library: loads, exports every declared symbol, host-only entry
points work without a GPU.  CPU only (no compute calls)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from flowpsi_b200 import _native as N
from flowpsi_b200 import default_params, GeneratedMesh, bc
from tests.conftest import gpu_available

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        syms |= set(re.findall(r"\b(fpsi_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(str(N.LIB_PATH))
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_reference_defaults():
    p = default_params()
    assert p.gamma == 1.4
    assert abs(p.Rtilde - 8314.4621 / 28.96) < 1e-12
    assert p.Pambient == 0.0
    assert p.flux == N.FLUX["hllc"]            # inviscidFlux.h:82-90
    assert p.limiter == N.LIMITER["venkatakrishnan"] and p.Kl == 1.0
    assert p.urelax == 0.2 and p.dtmax == 1.0
    assert p.solver == N.SOLVER["lsgs"]        # solverNewton.loci:223-228
    assert p.gauss_seidel_iter == 6            # linearSolverSGS.loci:39-41
    assert (p.lsgs_relaxation, p.lsgs_abs_tol, p.lsgs_rel_tol, p.lsgs_max_iter) == (0.25, 1e-10, 0.1, 10)
    assert p.step_graphs == 1                  # fpsi_run replays a captured step graph


def test_strerror():
    L = N.lib()
    for code, name in N.ERRORS.items():
        assert L.fpsi_strerror(code)
    assert L.fpsi_strerror(0) == b"ok"


def test_mesh_generate_counts():
    m = GeneratedMesh("hex", n=(4, 5, 6), bc_side=(0,) * 6, bcs=[bc("farfield")])
    a = m.arrays()
    assert a.ncells == 120
    nfi = 3 * 5 * 6 + 4 * 4 * 6 + 4 * 5 * 5
    nfb = 2 * (5 * 6 + 4 * 6 + 4 * 5)
    assert a.nfaces == nfi + nfb
    assert np.all(a.cl >= 0)
    inner = a.cr >= 0
    assert np.all(a.cl[inner] < a.cr[inner])
    k = GeneratedMesh("kuhn", n=(4, 4, 4), L=(1, 1, 1), jitter=0.1, seed=3)
    assert k.m.ncells == 6 * 64 and k.m.nfaces == 12 * 64
    ka = k.arrays()
    assert np.all(ka.cr >= 0) and np.all(ka.cl < ka.cr)


def test_invalid_mesh_rejected():
    s = N.MeshSpec()
    s.kind = 0
    s.nx = s.ny = s.nz = 1
    p = C.POINTER(N.Mesh)()
    assert N.lib().fpsi_mesh_generate(C.byref(s), C.byref(p)) == -1


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_no_cpu_fallback_without_device():
    from flowpsi_b200 import FlowPsi, FpsiError
    m = GeneratedMesh("hex", n=(4, 4, 4), bc_side=(0,) * 6, bcs=[bc("farfield")])
    with pytest.raises(FpsiError) as e:
        FlowPsi(m, default_params(solver="sgs"))
    assert e.value.code == -2  # FPSI_E_CUDA
    qL = np.ones((1, 5))
    rc = N.lib().fpsi_face_flux(1, 1, N.dptr(qL), N.dptr(qL), N.dptr(np.ones(3)),
                                N.dptr(np.ones(1)), 0.0, 287.0, 1.4, 0.0, 1.0, N.dptr(np.empty(5)))
    assert rc == -2


def test_bounded_kuhn_mesh_closes():
    """Kuhn tets with bounded sides: face counts, and the oracle's geometry
    fills the box and closes every cell (sum of outward area vectors 0)"""
    from oracle import Oracle

    m = GeneratedMesh("kuhn", n=(3, 4, 5), L=(1.0, 2.0, 3.0), jitter=0.1, seed=2,
                      bc_side=(0,) * 6, bcs=[bc("farfield")])
    a = m.arrays()
    assert a.ncells == 6 * 60
    nb = int((a.cr < 0).sum())
    assert nb == 2 * 2 * (3 * 4 + 4 * 5 + 3 * 5)  # two triangles per boundary quad
    assert 4 * a.ncells == 2 * (a.nfaces - nb) + nb
    assert np.all(a.cl < np.where(a.cr >= 0, a.cr, a.ncells))
    o = Oracle(m, default_params(solver="sgs"))
    g = o.geometry()
    assert abs(g["vol"].sum() - 6.0) < 1e-12 and g["vol"].min() > 0
    s = np.zeros((a.ncells, 3))
    np.add.at(s, a.cl, g["area_vec"])
    inner = a.cr >= 0
    np.add.at(s, a.cr[inner], -g["area_vec"][inner])
    assert np.abs(s).max() < 1e-13
    # boundary faces lie on the sides and point out of the box
    fc, an = g["facecenter"][~inner], g["area_vec"][~inner]
    L = np.array([1.0, 2.0, 3.0])
    on_side = (np.abs(fc) < 1e-12) | (np.abs(fc - L) < 1e-12)
    assert np.all(on_side.sum(1) == 1)
    out = np.where(np.abs(fc) < 1e-12, -1.0, 1.0)
    assert np.all((an * out * on_side).sum(1) > 0)
