"""The allocation-free residual-norm entry point, fpsi_residual_norms_noalloc.

It serves callers that cannot call cudaMalloc (their device memory comes
from their own pool, or an allocation must not happen inside their step);
the norms it returns must equal those fpsi_residual reports for the same
residual.  The device buffers here come from torch, i.e. from the caller --
the entry point itself allocates nothing.  This file is collected last so a
failure here stops a -x run only after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# tolerance used for the residual norms elsewhere in the GPU tests
NORM_RTOL = 1e-9


def _entry():
    from flowpsi_b200 import _native as N

    fn = N.lib().fpsi_residual_norms_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_void_p, C.c_void_p]
    return fn


def test_noalloc_norms_match_fpsi_residual(need_gpu):
    import torch

    from flowpsi_b200 import FlowPsi, cases

    case = cases.farfield_cube(12, precision="ref")
    g = FlowPsi(case.mesh, case.params)
    geo = g.geometry()
    T, p, u = case.initial_state(geo["cellcenter"])
    g.set_state(T, p, u)
    src, ref = g.residual()
    vol = np.ascontiguousarray(geo["vol"])
    d_src = torch.from_numpy(np.ascontiguousarray(src)).to("cuda")
    d_vol = torch.from_numpy(vol).to("cuda")
    d_out = torch.empty(8, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    fn = _entry()
    for call in range(2):  # the static scratch keeps the first call's partials
        d_out.fill_(float("nan"))
        rc = fn(C.c_void_p(d_src.data_ptr()), C.c_void_p(d_vol.data_ptr()), g.ncells,
                float(vol.sum()), C.c_void_p(d_out.data_ptr()), stream)
        assert rc == 0, f"call {call}: rc {rc}"
        torch.cuda.synchronize()
        out = d_out.cpu().numpy()
        for k, i in (("rtrms", 0), ("etrms", 1), ("mtrms", 2), ("rtmax", 3), ("etmax", 5),
                     ("mtmax", 7)):
            assert abs(out[i] - ref[k]) <= NORM_RTOL * abs(ref[k]), (call, k, out[i], ref[k])
        # the location of the density maximum is a cell whose value is the maximum
        c = int(out[4])
        assert abs(src[c, 0] / vol[c]) == pytest.approx(abs(out[3]), rel=1e-15)
    g.close()


def test_noalloc_rejects_oversize(need_gpu):
    fn = _entry()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = fn(dummy, dummy, (1 << 24) + 1, 1.0, dummy, None)
    assert rc == -1  # FPSI_E_INVALID
