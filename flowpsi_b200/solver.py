"""Host-side mirror of flowPsi's hot-path rules over the device library.

Each method corresponds to the Loci rule(s) it replaces (reference file:line
in the docstring) and keeps the reference's names, argument meaning and
error behaviour (a NaN residual raises, as solverResidual.loci:203-208
aborts).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


def default_params(**kw) -> N.Params:
    """Reference defaults (solverEoS.loci:27-47, solverTimestep.loci:281-287,
    linearSolverSGS.loci:39-41, linearSolverLSGS.loci:96-108,
    solverNewton.loci:222-228), overridden by keyword (strings accepted for
    flux, limiter, fluidLinearSolver/solver and precision)."""
    p = N.Params()
    N.lib().fpsi_default_params(C.byref(p))
    alias = {"fluidLinearSolver": "solver", "inviscidFlux": "flux"}
    for k, v in kw.items():
        k = alias.get(k, k)
        if k == "flux" and isinstance(v, str):
            v = N.FLUX[v]
        elif k == "limiter" and isinstance(v, str):
            v = N.LIMITER[v]
        elif k == "solver" and isinstance(v, str):
            v = N.SOLVER[v]
        elif k == "precision" and isinstance(v, str):
            v = N.PRECISION[v]
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def bc(kind: str, T: float = 300.0, pg: float = 1e5, u=(0.0, 0.0, 0.0),
       nu_t: float = 0.0, mass_flux: float = 0.0, mdot: float = 0.0,
       mass_relax: float = 1.0) -> N.BCSpec:
    """boundary condition; nu_t: SA nu~ entering through it (<= 0: 5e-9);
    for the total-pressure and fixed-mass conditions T is the total
    temperature T0, pg the total gauge pressure p0 - Pambient
    (isentropicInflow), mass_flux (or mdot over the condition's area) the
    prescribed mass flux"""
    b = N.BCSpec()
    b.kind = N.BC[kind]
    b.T, b.pg, b.nu_t = T, pg, nu_t
    b.mass_flux, b.mdot, b.mass_relax = mass_flux, mdot, mass_relax
    for i in range(3):
        b.u[i] = u[i]
    return b


@dataclass
class MeshArrays:
    """numpy views of a generated mesh (caller/Loci numbering)."""
    ncells: int
    nfaces: int
    xyz: np.ndarray
    face_off: np.ndarray
    face_nodes: np.ndarray
    cl: np.ndarray
    cr: np.ndarray
    pshift: np.ndarray | None
    bcs: list = field(default_factory=list)


class GeneratedMesh:
    """A synthetic grid owned by the library (fpsi_mesh_generate)."""

    def __init__(self, kind: str, n=(8, 8, 8), L=(1.0, 1.0, 1.0), jitter=0.0, seed=0,
                 bc_side=(-1, -1, -1, -1, -1, -1), bcs=(), dy0=1e-3, growth=1.1):
        s = N.MeshSpec()
        s.kind = {"hex": 0, "kuhn": 1, "bl": 2, "prism": 3}[kind]
        s.nx, s.ny, s.nz = n
        s.Lx, s.Ly, s.Lz = L
        s.jitter = jitter
        s.seed = seed
        s.dy0, s.growth = dy0, growth
        for i in range(6):
            s.bc_side[i] = bc_side[i]
        s.nbc = len(bcs)
        for i, b in enumerate(bcs):
            s.bcs[i] = b
        p = C.POINTER(N.Mesh)()
        N.check(N.lib().fpsi_mesh_generate(C.byref(s), C.byref(p)), "fpsi_mesh_generate")
        self._p = p
        self.spec = s

    @property
    def ptr(self):
        return self._p

    @property
    def m(self) -> N.Mesh:
        return self._p.contents

    def arrays(self) -> MeshArrays:
        m = self.m
        nf = m.nfaces
        nfn = np.ctypeslib.as_array(m.face_off, shape=(nf + 1,))[-1]
        pshift = (np.ctypeslib.as_array(m.pshift, shape=(nf * 3,)) if bool(m.pshift) else None)
        return MeshArrays(
            ncells=m.ncells, nfaces=nf,
            xyz=np.ctypeslib.as_array(m.xyz, shape=(m.nnodes * 3,)),
            face_off=np.ctypeslib.as_array(m.face_off, shape=(nf + 1,)),
            face_nodes=np.ctypeslib.as_array(m.face_nodes, shape=(int(nfn),)),
            cl=np.ctypeslib.as_array(m.cl, shape=(nf,)),
            cr=np.ctypeslib.as_array(m.cr, shape=(nf,)),
            pshift=pshift,
            bcs=[m.bcs[i] for i in range(m.nbc)],
        )

    def lines_along(self, axis: int = 1) -> list[np.ndarray]:
        """Cell lines of a structured hex grid (kinds hex and bl) along one
        axis; axis 1 gives the wall-normal lines of the boundary-layer block."""
        s = self.spec
        if s.kind == 1:
            raise ValueError("split-tet grids have no structured lines")
        n = (s.nx, s.ny, s.nz)
        idx = np.arange(n[0] * n[1] * n[2], dtype=np.int32).reshape(n[2], n[1], n[0])
        a = {0: 2, 1: 1, 2: 0}[axis]  # array axis of the grid direction
        cols = np.moveaxis(idx, a, -1).reshape(-1, n[axis])
        return [c.copy() for c in cols]

    def __del__(self):
        # at interpreter exit the module globals may already be gone
        if getattr(self, "_p", None) and N is not None and N.lib is not None:
            N.lib().fpsi_mesh_free(self._p)
            self._p = None


class FlowPsi:
    """One steady implicit solver instance on the GPU (fpsi_ctx)."""

    def __init__(self, mesh: GeneratedMesh | N.Mesh, params: N.Params | None = None):
        self._mesh = mesh  # keep the arrays alive
        self.params = params if params is not None else default_params()
        mp = mesh.ptr if isinstance(mesh, GeneratedMesh) else C.pointer(mesh)
        ctx = C.c_void_p()
        N.check(N.lib().fpsi_create(C.byref(ctx), mp, C.byref(self.params)), "fpsi_create")
        self._ctx = ctx
        nc, nf, ncol, nb = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int64()
        N.lib().fpsi_info(ctx, C.byref(nc), C.byref(nf), C.byref(ncol), C.byref(nb))
        self.ncells, self.nfaces, self.ncolours = nc.value, nf.value, ncol.value
        self.device_bytes = nb.value

    def close(self):
        if getattr(self, "_ctx", None):
            N.lib().fpsi_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- parameters / geometry --------------------------------------------
    def set_params(self, params: N.Params) -> None:
        N.check(N.lib().fpsi_set_params(self._ctx, C.byref(params)), "fpsi_set_params")
        self.params = params

    @property
    def block_dtype(self):
        return np.float64 if self.params.precision == N.PRECISION["fp64"] else np.float32

    def geometry(self) -> dict:
        nc, nf = self.ncells, self.nfaces
        vol, cc = np.empty(nc), np.empty(nc * 3)
        an, ar, fc = np.empty(nf * 3), np.empty(nf), np.empty(nf * 3)
        N.check(N.lib().fpsi_get_geometry(self._ctx, N.dptr(vol), N.dptr(cc), N.dptr(an),
                                          N.dptr(ar), N.dptr(fc)), "fpsi_get_geometry")
        return {"vol": vol, "cellcenter": cc.reshape(nc, 3), "area_vec": an.reshape(nf, 3),
                "area": ar, "facecenter": fc.reshape(nf, 3)}

    def set_lines(self, lines) -> None:
        """lines of the line solver (list of caller cell-index arrays)"""
        off = np.zeros(len(lines) + 1, np.int64)
        off[1:] = np.cumsum([len(l) for l in lines])
        cells = np.ascontiguousarray(np.concatenate(lines).astype(np.int32)) if lines else \
            np.zeros(0, np.int32)
        N.check(N.lib().fpsi_set_lines(self._ctx, len(lines),
                                       off.ctypes.data_as(C.POINTER(C.c_int64)), N.iptr(cells)),
                "fpsi_set_lines")

    def lines(self):
        """(line of each cell, position on the line, colour of each line)"""
        nl = C.c_int64()
        N.check(N.lib().fpsi_get_lines(self._ctx, None, None, None, C.byref(nl)), "fpsi_get_lines")
        lo, po = np.empty(self.ncells, np.int32), np.empty(self.ncells, np.int32)
        lc = np.empty(max(nl.value, 1), np.int32)
        N.check(N.lib().fpsi_get_lines(self._ctx, N.iptr(lo), N.iptr(po), N.iptr(lc), C.byref(nl)),
                "fpsi_get_lines")
        return lo, po, lc[:nl.value]

    def line_list(self):
        """the lines as lists of caller cells in line order, and their colours"""
        lo, po, lc = self.lines()
        order = np.lexsort((po, lo))
        bounds = np.searchsorted(lo[order], np.arange(len(lc) + 1))
        return [order[bounds[i]:bounds[i + 1]].astype(np.int32) for i in range(len(lc))], lc

    def colours(self) -> np.ndarray:
        c = np.empty(self.ncells, np.int32)
        N.check(N.lib().fpsi_get_colours(self._ctx, N.iptr(c)), "fpsi_get_colours")
        return c

    # -- state -------------------------------------------------------------
    def set_state(self, T, pg, u) -> None:
        T = np.ascontiguousarray(T, np.float64)
        pg = np.ascontiguousarray(pg, np.float64)
        u = np.ascontiguousarray(u, np.float64).reshape(-1)
        assert T.size == self.ncells and pg.size == self.ncells and u.size == 3 * self.ncells
        N.check(N.lib().fpsi_set_state(self._ctx, N.dptr(T), N.dptr(pg), N.dptr(u)),
                "fpsi_set_state")

    def set_eddy_viscosity(self, tmu) -> None:
        """eddy viscosity per cell for flowRegime turbulent (caller order)"""
        t = np.ascontiguousarray(tmu, np.float64)
        assert t.size == self.ncells
        N.check(N.lib().fpsi_set_eddy_viscosity(self._ctx, N.dptr(t)), "fpsi_set_eddy_viscosity")

    # -- Spalart-Allmaras nu~ (turbulence/SA/SA_turb.loci) -------------------
    def set_nutilde(self, nut) -> None:
        """the SA working variable nu~ per cell (caller order)"""
        v = np.ascontiguousarray(nut, np.float64)
        assert v.size == self.ncells
        N.check(N.lib().fpsi_set_nutilde(self._ctx, N.dptr(v)), "fpsi_set_nutilde")

    def _cells(self, fn, name):
        v = np.empty(self.ncells)
        N.check(fn(self._ctx, N.dptr(v)), name)
        return v

    def nutilde(self) -> np.ndarray:
        return self._cells(N.lib().fpsi_get_nutilde, "fpsi_get_nutilde")

    def eddy_viscosity(self) -> np.ndarray:
        return self._cells(N.lib().fpsi_get_eddy_viscosity, "fpsi_get_eddy_viscosity")

    def wall_distance(self) -> np.ndarray:
        """dist_noslip (solverTurbulence.loci:133-137)"""
        return self._cells(N.lib().fpsi_get_wall_distance, "fpsi_get_wall_distance")

    def sa_residual(self) -> np.ndarray:
        """nuTilde_src, the scalar right-hand side (after residual())"""
        return self._cells(N.lib().fpsi_sa_residual, "fpsi_sa_residual")

    def sa_system(self) -> dict:
        D, fjp, fjm = np.empty(self.ncells), np.empty(self.nfaces), np.empty(self.nfaces)
        N.check(N.lib().fpsi_sa_get_system(self._ctx, N.dptr(D), N.dptr(fjp), N.dptr(fjm)),
                "fpsi_sa_get_system")
        return {"D": D, "fjp": fjp, "fjm": fjm}

    def sa_solve(self) -> np.ndarray:
        return self._cells(N.lib().fpsi_sa_solve, "fpsi_sa_solve")

    def sa_update(self) -> None:
        N.check(N.lib().fpsi_sa_update(self._ctx), "fpsi_sa_update")

    def get_state(self, out=None):
        """(T, pg, u) in caller order; `out` = caller arrays (float64,
        contiguous; e.g. pinned host memory) to fill instead of new ones"""
        nc = self.ncells
        if out is None:
            T, pg, u = np.empty(nc), np.empty(nc), np.empty(nc * 3)
        else:
            T, pg, u = out
            for a, n in ((T, nc), (pg, nc), (u, 3 * nc)):
                assert a.dtype == np.float64 and a.flags.c_contiguous and a.size == n
        N.check(N.lib().fpsi_get_state(self._ctx, N.dptr(T), N.dptr(pg), N.dptr(u)),
                "fpsi_get_state")
        return T, pg, u.reshape(nc, 3)

    # -- rules ---------------------------------------------------------------
    def residual(self, want_src: bool = True):
        """'src' store and 'residual' norms (fluxInviscid.loci:1253-1268,
        solverResidual.loci:74-112)."""
        src = np.empty(self.ncells * 5) if want_src else None
        r = N.Resid()
        N.check(N.lib().fpsi_residual(self._ctx, N.dptr(src), C.byref(r)), "fpsi_residual")
        return (src.reshape(-1, 5) if want_src else None), r.as_dict()

    def reconstruction(self):
        g, l = np.empty(self.ncells * 15), np.empty(self.ncells * 5)
        N.check(N.lib().fpsi_get_reconstruction(self._ctx, N.dptr(g), N.dptr(l)),
                "fpsi_get_reconstruction")
        return g.reshape(-1, 15), l.reshape(-1, 5)

    def dtau(self) -> np.ndarray:
        """local pseudo time step, solverTimestep.loci:302-329"""
        d = np.empty(self.ncells)
        N.check(N.lib().fpsi_get_dtau(self._ctx, N.dptr(d)), "fpsi_get_dtau")
        return d

    def assemble(self) -> None:
        """fjp/fjm, srcJ, fluid_D, fluid_B and the LU of fluid_D
        (fluxInviscid.loci:1190-1221, solverLinearSystem.loci:45-224,
        linearSolverSGS.loci:43-50)."""
        N.check(N.lib().fpsi_assemble(self._ctx), "fpsi_assemble")

    def blocks(self) -> dict:
        dt = self.block_dtype
        nc, nf = self.ncells, self.nfaces
        D, fjp, fjm, B = (np.empty((nc, 5, 5), dt), np.empty((nf, 5, 5), dt),
                          np.empty((nf, 5, 5), dt), np.empty((nc, 5), dt))
        N.check(N.lib().fpsi_get_blocks(self._ctx, N.vptr(D), N.vptr(fjp), N.vptr(fjm),
                                        N.vptr(B)), "fpsi_get_blocks")
        return {"fluid_D": D, "fjp": fjp, "fjm": fjm, "fluid_B": B}

    def linear_solve(self, x0: np.ndarray | None = None, info: bool = False):
        """SGSBlockedSSolve(fluid) or LSGSBlockedSSolve(fluid,fluid_B) ->
        dfluid (linearSolverSGS.loci:57-329, linearSolverLSGS.loci:1692-1954,
        solverNewton.loci:252-269); x0 None = the reference's start."""
        dq = np.empty(self.ncells * 5)
        x0p = None if x0 is None else np.ascontiguousarray(x0, np.float64).reshape(-1)
        li = N.LsInfo()
        N.check(N.lib().fpsi_linear_solve(self._ctx, N.dptr(x0p), N.dptr(dq), C.byref(li)),
                "fpsi_linear_solve")
        if info:
            return dq.reshape(-1, 5), {"iterations": li.iterations, "resid0": li.resid0,
                                       "resid": li.resid}
        return dq.reshape(-1, 5)

    def set_iterate(self, x0) -> None:
        """start the next sweeps from x0 (caller order, nc x 5)"""
        x = np.ascontiguousarray(x0, np.float64).reshape(-1)
        N.check(N.lib().fpsi_set_iterate(self._ctx, N.dptr(x)), "fpsi_set_iterate")

    def get_iterate(self) -> np.ndarray:
        x = np.empty(self.ncells * 5)
        N.check(N.lib().fpsi_get_iterate(self._ctx, N.dptr(x)), "fpsi_get_iterate")
        return x.reshape(-1, 5)

    def sweeps(self, n: int) -> None:
        """n more symmetric sweeps from the current device iterate"""
        N.check(N.lib().fpsi_linear_sweeps(self._ctx, n), "fpsi_linear_sweeps")

    def sweeps_to_tolerance(self, rtol: float, max_sweeps: int = 200) -> int:
        """symmetric sweeps from the current iterate until ||B - A x|| <=
        rtol ||B|| (the relative linear tolerance); returns the count"""
        for k in range(max_sweeps + 1):
            nb, nr = self.linear_residual()
            if nr <= rtol * nb:
                return k
            if k < max_sweeps:
                self.sweeps(1)
        return max_sweeps + 1

    def linear_residual(self):
        nb, nr = C.c_double(), C.c_double()
        N.check(N.lib().fpsi_linear_residual(self._ctx, C.byref(nb), C.byref(nr)),
                "fpsi_linear_residual")
        return nb.value, nr.value

    def update(self) -> float:
        """clipped Newton update, solverNewton.loci:62-78"""
        a = C.c_double()
        N.check(N.lib().fpsi_update(self._ctx, C.byref(a)), "fpsi_update")
        return a.value

    def newton_step(self) -> dict:
        si = N.StepInfo()
        N.check(N.lib().fpsi_newton_step(self._ctx, C.byref(si)), "fpsi_newton_step")
        d = si.resid.as_dict()
        d["min_alpha"] = si.min_alpha
        return d

    def newton_step_ex(self, start: str = "jacobi", model=None, reject: bool = True,
                       lin_rtol: float = 0.0, max_sweeps: int = 200,
                       check_every: int = 2) -> dict:
        """One steady step (fpsi_newton_step_ex) from a chosen starting
        iterate: 'jacobi' (the reference's D^-1 B, linearSolverSGS.loci:57-69),
        'zero' or 'learned' (model: a learned.LearnedStart).  With reject, a
        step that did not start from D^-1 B and does not lower the FP64
        density residual is undone and redone from D^-1 B.  lin_rtol > 0
        sweeps to ||B - A x|| <= lin_rtol ||B|| instead of
        gauss_seidel_iter sweeps.  Returns the starting norms, the norms of
        the new state ('after'), the sweeps, the start kept and whether the
        first attempt was rejected."""
        o = N.StepOpts()
        o.start = N.START[start]
        o.reject = 1 if reject else 0
        o.lin_rtol, o.max_sweeps, o.check_every = lin_rtol, max_sweeps, check_every
        si = N.StepInfo()
        h = None if model is None else model._h
        N.check(N.lib().fpsi_newton_step_ex(self._ctx, h, C.byref(o), C.byref(si)),
                "fpsi_newton_step_ex")
        d = si.resid.as_dict()
        d.update(min_alpha=si.min_alpha, after=si.resid_after.as_dict(), sweeps=si.ls.iterations,
                 lin_resid0=si.ls.resid0, lin_resid=si.ls.resid,
                 start={v: k for k, v in N.START.items()}[si.start_used],
                 rejected=bool(si.rejected))
        return d

    def run(self, nsteps: int) -> list[dict]:
        """nsteps implicit steps on the device.  A NaN residual stops the run
        at that step (solverResidual.loci:203-208) and raises FpsiError with
        the norm history so far as its ``history``."""
        arr = (N.Resid * max(nsteps, 1))()
        rc = N.lib().fpsi_run(self._ctx, nsteps, arr)
        hist = [arr[i].as_dict() for i in range(nsteps)]
        if rc != N.FPSI_OK:
            e = N.FpsiError(rc, "fpsi_run")
            e.history = hist
            raise e
        return hist

    def time_step(self) -> list[dict]:
        """One BDF2 time step of size dtmax (params.time_accurate = 1):
        params.newton_iters Newton iterations, then the time levels shift
        (solverTimestep.loci:397-428, solverNewton.loci:163-198).  Returns
        the norms of each iteration's rhs."""
        nit = self.params.newton_iters
        arr = (N.Resid * max(nit, 1))()
        rc = N.lib().fpsi_time_step(self._ctx, arr)
        hist = [arr[i].as_dict() for i in range(nit)]
        if rc != N.FPSI_OK:
            e = N.FpsiError(rc, "fpsi_time_step")
            e.history = hist
            raise e
        return hist

    def run_timed(self, nsteps: int):
        """(norm history, device milliseconds) of nsteps steps, timed with
        CUDA events on the library's stream"""
        arr = (N.Resid * max(nsteps, 1))()
        ms = C.c_double()
        rc = N.lib().fpsi_run_timed(self._ctx, nsteps, arr, C.byref(ms))
        hist = [arr[i].as_dict() for i in range(nsteps)]
        if rc != N.FPSI_OK:
            e = N.FpsiError(rc, "fpsi_run_timed")
            e.history = hist
            raise e
        return hist, ms.value

    def kernel_times(self, nsteps: int = 1) -> dict:
        """{kernel: (total ms, launches)} over nsteps steps"""
        cap = 64
        names = C.create_string_buffer(32 * cap)
        ms = np.zeros(cap)
        lc = np.zeros(cap, np.int64)
        cnt = C.c_int32()
        N.check(N.lib().fpsi_kernel_times(self._ctx, nsteps, cap, names, N.dptr(ms),
                                          lc.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(cnt)),
                "fpsi_kernel_times")
        raw = names.raw
        out = {}
        for k in range(cnt.value):
            nm = raw[32 * k:32 * k + 32].split(b"\0")[0].decode()
            out[nm] = (float(ms[k]), int(lc[k]))
        return out

    def keep_blocks(self, keep: bool) -> None:
        N.check(N.lib().fpsi_keep_blocks(self._ctx, 1 if keep else 0), "fpsi_keep_blocks")


# -- inviscidFlux.h entry points on batches ---------------------------------
def inviscid_riemann_flux(kind, qL, qR, an, area, pambient=0.0, Rt=8314.4621 / 28.96,
                          gamma=1.4, us_n=0.0, eta=1.0) -> np.ndarray:
    """Batched inviscidRiemannFlux / roeCT_flux / HLLE; states packed
    [pg, T, u, v, w] per face."""
    kind = N.FLUX[kind] if isinstance(kind, str) else kind
    qL = np.ascontiguousarray(qL, np.float64)
    qR = np.ascontiguousarray(qR, np.float64)
    an = np.ascontiguousarray(an, np.float64)
    area = np.ascontiguousarray(area, np.float64)
    n = area.size
    out = np.empty((n, 5))
    N.check(N.lib().fpsi_face_flux(kind, n, N.dptr(qL), N.dptr(qR), N.dptr(an), N.dptr(area),
                                   pambient, Rt, gamma, us_n, eta, N.dptr(out)), "fpsi_face_flux")
    return out


def roe_jacobian(qL, qR, an, area, direction, pambient=0.0, Rt=8314.4621 / 28.96, gamma=1.4,
                 us_n=0.0, eta=1.0, as_double=False) -> np.ndarray:
    """Batched roeCT_jacobian (fjp for direction=+1, fjm for -1)."""
    qL = np.ascontiguousarray(qL, np.float64)
    qR = np.ascontiguousarray(qR, np.float64)
    an = np.ascontiguousarray(an, np.float64)
    area = np.ascontiguousarray(area, np.float64)
    n = area.size
    out = np.empty((n, 5, 5), np.float64 if as_double else np.float32)
    N.check(N.lib().fpsi_face_jacobian(n, N.dptr(qL), N.dptr(qR), N.dptr(an), N.dptr(area),
                                       pambient, Rt, gamma, us_n, eta, direction,
                                       1 if as_double else 0, N.vptr(out)),
            "fpsi_face_jacobian")
    return out
