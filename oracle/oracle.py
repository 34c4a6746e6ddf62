"""ctypes wrapper of the oracle (``liboracle.so``) and of the reference's own
face functions compiled into ``oracle/_ref/libfpsiref.so``.

TEST INFRASTRUCTURE: used by tests/, the smoke check and bench.py's CPU
baseline only.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from flowpsi_b200 import _native as N

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libfpsiref.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_vp = C.c_void_p

_SIGS = {
    "orc_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(N.Mesh), C.POINTER(N.Params)]),
    "orc_destroy": (None, [C.c_void_p]),
    "orc_set_params": (C.c_int, [C.c_void_p, C.POINTER(N.Params)]),
    "orc_get_geometry": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "orc_set_state": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "orc_set_eddy_viscosity": (C.c_int, [C.c_void_p, _dp]),
    "orc_get_state": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "orc_residual": (C.c_int, [C.c_void_p, _dp, C.POINTER(N.Resid)]),
    "orc_get_reconstruction": (C.c_int, [C.c_void_p, _dp, _dp]),
    "orc_get_dtau": (C.c_int, [C.c_void_p, _dp]),
    "orc_assemble": (C.c_int, [C.c_void_p]),
    "orc_get_blocks": (C.c_int, [C.c_void_p, _vp, _vp, _vp, _vp]),
    "orc_linear_solve": (C.c_int, [C.c_void_p, _ip, _dp, _dp, C.POINTER(N.LsInfo)]),
    "orc_linear_residual": (C.c_int, [C.c_void_p, _dp, _dp]),
    "orc_lsgs_solve": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int64), _ip, _ip, _dp, _dp,
                                 C.POINTER(N.LsInfo)]),
    "orc_update": (C.c_int, [C.c_void_p, _dp]),
    "orc_newton_step": (C.c_int, [C.c_void_p, _ip, C.POINTER(N.StepInfo)]),
    "orc_time_step": (C.c_int, [C.c_void_p, _ip, C.POINTER(N.Resid)]),
    "orc_set_threads": (C.c_int, [C.c_int]),
    "orc_set_nutilde": (C.c_int, [C.c_void_p, _dp]),
    "orc_get_nutilde": (C.c_int, [C.c_void_p, _dp]),
    "orc_get_eddy_viscosity": (C.c_int, [C.c_void_p, _dp]),
    "orc_get_wall_distance": (C.c_int, [C.c_void_p, _dp]),
    "orc_sa_residual": (C.c_int, [C.c_void_p, _dp]),
    "orc_sa_get_system": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "orc_sa_solve": (C.c_int, [C.c_void_p, _ip, _dp]),
    "orc_sa_update": (C.c_int, [C.c_void_p]),
    "orc_face_flux": (C.c_int, [C.c_int32, C.c_int64, _dp, _dp, _dp, _dp, C.c_double,
                                C.c_double, C.c_double, C.c_double, C.c_double, _dp]),
    "orc_face_jacobian": (C.c_int, [C.c_int64, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                    _vp]),
    "orc_cv_state": (C.c_int, [C.c_int32, C.c_int64, _dp, _dp, _dp, C.c_double, C.c_double,
                               C.c_double, C.c_double, C.c_double, _dp]),
}
_REF_SIGS = {
    "ref_face_flux": (C.c_int, [C.c_int32, C.c_int64, _dp, _dp, _dp, _dp, C.c_double,
                                C.c_double, C.c_double, C.c_double, C.c_double, _dp]),
    "ref_face_jacobian": (C.c_int, [C.c_int64, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_double, C.c_int32, _vp]),
    "ref_cv_state": (C.c_int, [C.c_int32, C.c_int64, _dp, _dp, _dp, C.c_double, C.c_double,
                               C.c_double, C.c_double, C.c_double, _dp]),
}

_lib = None
_ref = None


def _load(path: Path, sigs: dict):
    if not path.exists():
        raise RuntimeError(f"{path} missing: run `python oracle/build.py`")
    L = C.CDLL(str(path))
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def olib():
    global _lib
    if _lib is None:
        _lib = _load(LIB, _SIGS)
    return _lib


def ref_available() -> bool:
    return REF_LIB.exists()


def rlib():
    global _ref
    if _ref is None:
        _ref = _load(REF_LIB, _REF_SIGS)
    return _ref


def _chk(rc, where):
    if rc != 0:
        raise RuntimeError(f"{where}: {N.ERRORS.get(rc, rc)}")


def _d(a):
    return None if a is None else np.ascontiguousarray(a, np.float64).ctypes.data_as(_dp)


class _FaceFns:
    """Batched face functions with the fpsi_face_flux packing."""

    _flux = _jac = _cv = None

    def flux(self, kind, qL, qR, an, area, pamb=0.0, Rt=8314.4621 / 28.96, gamma=1.4, us_n=0.0,
             eta=1.0):
        kind = N.FLUX[kind] if isinstance(kind, str) else kind
        qL, qR, an, area = (np.ascontiguousarray(v, np.float64) for v in (qL, qR, an, area))
        out = np.empty((area.size, 5))
        _chk(self._flux(kind, area.size, _d(qL), _d(qR), _d(an), _d(area), pamb, Rt, gamma, us_n,
                        eta, out.ctypes.data_as(_dp)), "flux")
        return out

    def cv_state(self, outflow, qi, q0, an, us_n=0.0, pamb=0.0, gamma=1.4,
                 Rt=8314.4621 / 28.96, beta=1.0):
        qi, q0, an = (np.ascontiguousarray(v, np.float64) for v in (qi, q0, an))
        n = qi.shape[0]
        out = np.empty((n, 5))
        _chk(self._cv(int(outflow), n, _d(qi), _d(q0), _d(an), us_n, pamb, gamma, Rt, beta,
                      out.ctypes.data_as(_dp)), "cv_state")
        return out


class OracleFunctions(_FaceFns):
    def __init__(self):
        L = olib()
        self._flux, self._cv = L.orc_face_flux, L.orc_cv_state
        self._jacfn = L.orc_face_jacobian

    def jacobian(self, qL, qR, an, area, direction, pamb=0.0, Rt=8314.4621 / 28.96, gamma=1.4,
                 us_n=0.0, eta=1.0, as_double=False):
        qL, qR, an, area = (np.ascontiguousarray(v, np.float64) for v in (qL, qR, an, area))
        out = np.empty((area.size, 5, 5), np.float64 if as_double else np.float32)
        _chk(self._jacfn(area.size, _d(qL), _d(qR), _d(an), _d(area), pamb, Rt, gamma, us_n, eta,
                         direction, int(as_double), C.c_void_p(out.ctypes.data)), "jacobian")
        return out


class RefFunctions(_FaceFns):
    """The reference's hllc_flux / roeCT_flux / roeCT_jacobian / cv_* compiled
    from their source (oracle/build.py)."""

    def __init__(self):
        L = rlib()
        self._flux, self._cv = L.ref_face_flux, L.ref_cv_state
        self._jacfn = L.ref_face_jacobian

    def jacobian(self, qL, qR, an, area, direction, pamb=0.0, Rt=8314.4621 / 28.96, gamma=1.4,
                 us_n=0.0, eta=1.0):
        qL, qR, an, area = (np.ascontiguousarray(v, np.float64) for v in (qL, qR, an, area))
        out = np.empty((area.size, 5, 5), np.float32)
        _chk(self._jacfn(area.size, _d(qL), _d(qR), _d(an), _d(area), pamb, Rt, gamma, us_n, eta,
                         direction, C.c_void_p(out.ctypes.data)), "jacobian")
        return out


def set_threads(n: int) -> int:
    return olib().orc_set_threads(n)


class Oracle:
    """Mesh-level oracle with the same methods as flowpsi_b200.FlowPsi."""

    def __init__(self, mesh, params: N.Params):
        self._mesh = mesh
        self.params = params
        mp = mesh.ptr if hasattr(mesh, "ptr") else C.pointer(mesh)
        h = C.c_void_p()
        _chk(olib().orc_create(C.byref(h), mp, C.byref(params)), "orc_create")
        self._h = h
        m = mp.contents
        self.ncells, self.nfaces = m.ncells, m.nfaces

    def __del__(self):
        if getattr(self, "_h", None):
            olib().orc_destroy(self._h)
            self._h = None

    def set_params(self, params):
        _chk(olib().orc_set_params(self._h, C.byref(params)), "orc_set_params")
        self.params = params

    @property
    def block_dtype(self):
        return np.float64 if self.params.precision == N.PRECISION["fp64"] else np.float32

    def geometry(self):
        nc, nf = self.ncells, self.nfaces
        vol, cc = np.empty(nc), np.empty(nc * 3)
        an, ar, fc = np.empty(nf * 3), np.empty(nf), np.empty(nf * 3)
        _chk(olib().orc_get_geometry(self._h, _d(vol), cc.ctypes.data_as(_dp),
                                     an.ctypes.data_as(_dp), ar.ctypes.data_as(_dp),
                                     fc.ctypes.data_as(_dp)), "orc_get_geometry")
        return {"vol": vol, "cellcenter": cc.reshape(nc, 3), "area_vec": an.reshape(nf, 3),
                "area": ar, "facecenter": fc.reshape(nf, 3)}

    def set_state(self, T, pg, u):
        T, pg, u = (np.ascontiguousarray(v, np.float64).reshape(-1) for v in (T, pg, u))
        _chk(olib().orc_set_state(self._h, _d(T), _d(pg), _d(u)), "orc_set_state")

    def set_eddy_viscosity(self, tmu):
        t = np.ascontiguousarray(tmu, np.float64)
        _chk(olib().orc_set_eddy_viscosity(self._h, _d(t)), "orc_set_eddy_viscosity")

    def get_state(self):
        nc = self.ncells
        T, pg, u = np.empty(nc), np.empty(nc), np.empty(nc * 3)
        _chk(olib().orc_get_state(self._h, T.ctypes.data_as(_dp), pg.ctypes.data_as(_dp),
                                  u.ctypes.data_as(_dp)), "orc_get_state")
        return T, pg, u.reshape(nc, 3)

    def residual(self):
        src = np.empty(self.ncells * 5)
        r = N.Resid()
        _chk(olib().orc_residual(self._h, src.ctypes.data_as(_dp), C.byref(r)), "orc_residual")
        return src.reshape(-1, 5), r.as_dict()

    def reconstruction(self):
        g, l = np.empty(self.ncells * 15), np.empty(self.ncells * 5)
        _chk(olib().orc_get_reconstruction(self._h, g.ctypes.data_as(_dp),
                                           l.ctypes.data_as(_dp)), "orc_get_reconstruction")
        return g.reshape(-1, 15), l.reshape(-1, 5)

    def dtau(self):
        d = np.empty(self.ncells)
        _chk(olib().orc_get_dtau(self._h, d.ctypes.data_as(_dp)), "orc_get_dtau")
        return d

    def assemble(self):
        _chk(olib().orc_assemble(self._h), "orc_assemble")

    def blocks(self):
        dt = self.block_dtype
        nc, nf = self.ncells, self.nfaces
        D, fjp, fjm, B = (np.empty((nc, 5, 5), dt), np.empty((nf, 5, 5), dt),
                          np.empty((nf, 5, 5), dt), np.empty((nc, 5), dt))
        _chk(olib().orc_get_blocks(self._h, C.c_void_p(D.ctypes.data), C.c_void_p(fjp.ctypes.data),
                                   C.c_void_p(fjm.ctypes.data), C.c_void_p(B.ctypes.data)),
             "orc_get_blocks")
        return {"fluid_D": D, "fjp": fjp, "fjm": fjm, "fluid_B": B}

    def linear_solve(self, colour=None, x0=None):
        dq = np.empty(self.ncells * 5)
        col = None if colour is None else np.ascontiguousarray(colour, np.int32)
        info = N.LsInfo()
        _chk(olib().orc_linear_solve(self._h, None if col is None else col.ctypes.data_as(_ip),
                                     _d(None if x0 is None else np.asarray(x0).reshape(-1)),
                                     dq.ctypes.data_as(_dp), C.byref(info)), "orc_linear_solve")
        return dq.reshape(-1, 5)

    def lsgs_solve(self, lines, colours=None, x0=None):
        """line SGS over the given lines (list of caller cell arrays); with
        colours (one per line) the lines are swept colour by colour"""
        off = np.zeros(len(lines) + 1, np.int64)
        off[1:] = np.cumsum([len(l) for l in lines])
        cells = np.ascontiguousarray(np.concatenate(lines).astype(np.int32))
        col = None if colours is None else np.ascontiguousarray(colours, np.int32)
        dq = np.empty(self.ncells * 5)
        info = N.LsInfo()
        _chk(olib().orc_lsgs_solve(self._h, len(lines), off.ctypes.data_as(C.POINTER(C.c_int64)),
                                   cells.ctypes.data_as(_ip),
                                   None if col is None else col.ctypes.data_as(_ip),
                                   _d(None if x0 is None else np.asarray(x0).reshape(-1)),
                                   dq.ctypes.data_as(_dp), C.byref(info)), "orc_lsgs_solve")
        return dq.reshape(-1, 5), {"iterations": info.iterations, "resid0": info.resid0,
                                   "resid": info.resid}

    def linear_residual(self):
        nb, nr = C.c_double(), C.c_double()
        _chk(olib().orc_linear_residual(self._h, C.byref(nb), C.byref(nr)), "orc_linear_residual")
        return nb.value, nr.value

    def update(self):
        a = C.c_double()
        _chk(olib().orc_update(self._h, C.byref(a)), "orc_update")
        return a.value

    def newton_step(self, colour=None):
        col = None if colour is None else np.ascontiguousarray(colour, np.int32)
        si = N.StepInfo()
        _chk(olib().orc_newton_step(self._h, None if col is None else col.ctypes.data_as(_ip),
                                    C.byref(si)), "orc_newton_step")
        d = si.resid.as_dict()
        d["min_alpha"] = si.min_alpha
        return d

    def time_step(self, colour=None):
        """one BDF2 time step: newton_iters Newton iterations, then the
        time levels move on; norms of each iteration"""
        col = None if colour is None else np.ascontiguousarray(colour, np.int32)
        nit = self.params.newton_iters
        arr = (N.Resid * max(nit, 1))()
        _chk(olib().orc_time_step(self._h, None if col is None else col.ctypes.data_as(_ip), arr),
             "orc_time_step")
        return [arr[i].as_dict() for i in range(nit)]

    # -- Spalart-Allmaras nu~ (turbulence/SA/SA_turb.loci) -------------------
    def set_nutilde(self, nut):
        _chk(olib().orc_set_nutilde(self._h, _d(np.ascontiguousarray(nut, np.float64))),
             "orc_set_nutilde")

    def _cellvec(self, fn, name):
        v = np.empty(self.ncells)
        _chk(fn(self._h, v.ctypes.data_as(_dp)), name)
        return v

    def nutilde(self):
        return self._cellvec(olib().orc_get_nutilde, "orc_get_nutilde")

    def eddy_viscosity(self):
        return self._cellvec(olib().orc_get_eddy_viscosity, "orc_get_eddy_viscosity")

    def wall_distance(self):
        return self._cellvec(olib().orc_get_wall_distance, "orc_get_wall_distance")

    def sa_residual(self):
        return self._cellvec(olib().orc_sa_residual, "orc_sa_residual")

    def sa_system(self):
        D, fjp, fjm = np.empty(self.ncells), np.empty(self.nfaces), np.empty(self.nfaces)
        _chk(olib().orc_sa_get_system(self._h, D.ctypes.data_as(_dp), fjp.ctypes.data_as(_dp),
                                      fjm.ctypes.data_as(_dp)), "orc_sa_get_system")
        return {"D": D, "fjp": fjp, "fjm": fjm}

    def sa_solve(self, colour=None):
        col = None if colour is None else np.ascontiguousarray(colour, np.int32)
        dq = np.empty(self.ncells)
        _chk(olib().orc_sa_solve(self._h, None if col is None else col.ctypes.data_as(_ip),
                                 dq.ctypes.data_as(_dp)), "orc_sa_solve")
        return dq

    def sa_update(self):
        _chk(olib().orc_sa_update(self._h), "orc_sa_update")
