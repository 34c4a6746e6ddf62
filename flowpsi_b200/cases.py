"""Synthetic workloads: grids, initial conditions and options.

All random numbers come from a counter-based generator (SplitMix64 followed
by Box-Muller) evaluated on the host, so every run, CPU or GPU, sees the same
inputs for the same seed.

* ``farfield_cube``: inviscid Euler, n^3 hex cube [0,1]^3, farfield on all
  sides at M=0.5 along +x, p=1e5 Pa, T=300 K; initial state the freestream
  with 1% Gaussian noise in rho, u, v, w and p; Roe flux, MUSCL with the
  Venkatakrishnan limiter, 5 SGS sweeps per step, CFL 50 (32^3: the
  CPU-runnable case).
* ``taylor_green_tets``: n^3 hexes split into 6 Kuhn tetrahedra on the
  periodic box [0,2pi]^3, nodes jittered by +-10% of the spacing; Taylor-Green
  vortex at M=0.1 (initial form of examples/taylor/ic_module/
  taylorGreenIC.loci:26-31: constant density, pressure from the analytic
  field); Roe + MUSCL + Venkatakrishnan, 8 multi-colour SGS sweeps (128^3:
  12.58M cells, 25.2M faces).
* ``outflow_duct``: hex duct from a farfield inflow to an outflow held at
  a back pressure ('p' or 'pMean'), periodic sides.
* ``farfield_tets``: the split-tet grid of ``taylor_green_tets`` with
  farfield sides and the freestream-plus-noise start of ``farfield_cube``:
  the steady case on which the 1e-8 residual drop is timed.
* ``oblique_shock_cube``: n^3 hex cube, Mach-2 flow with a Rankine-Hugoniot
  jump across a plane tilted 30 degrees, 0.5% noise, supersonic inflow /
  outflow, HLLE + Barth.
"""
from __future__ import annotations

import math

import numpy as np

from .solver import GeneratedMesh, bc, default_params

RTILDE = 8314.4621 / 28.96
GAMMA = 1.4

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
    return x ^ (x >> np.uint64(31))


def uniform(seed: int, stream: int, n: int) -> np.ndarray:
    """n doubles in (0,1) from counter (seed, stream, i)."""
    with np.errstate(over="ignore"):
        base = np.uint64((seed * 0x100000001B3 + stream * 0x9E3779B1) & 0xFFFFFFFFFFFFFFFF)
        i = np.arange(n, dtype=np.uint64)
        r = splitmix64((base + i * np.uint64(0x632BE59BD9B4E019)) & _M64)
    return ((r >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)


def normal(seed: int, stream: int, n: int) -> np.ndarray:
    u1 = uniform(seed, 2 * stream, n)
    u2 = uniform(seed, 2 * stream + 1, n)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


class Case:
    def __init__(self, name, mesh, params, steps, init):
        self.name = name
        self.mesh = mesh
        self.params = params
        self.steps = steps
        self._init = init

    def initial_state(self, cellcenter: np.ndarray):
        """(T, pg, u[nc,3]) at the given cell centroids (caller order)."""
        return self._init(cellcenter)


def farfield_cube(n: int = 32, seed: int = 0, sweeps: int = 5, flux: str = "roe",
                  limiter: str = "venkatakrishnan", precision: str = "ref") -> Case:
    T0, p0, M = 300.0, 1e5, 0.5
    a0 = math.sqrt(GAMMA * RTILDE * T0)
    U0 = M * a0
    ff = bc("farfield", T=T0, pg=p0, u=(U0, 0.0, 0.0))
    mesh = GeneratedMesh("hex", n=(n, n, n), L=(1.0, 1.0, 1.0), bc_side=(0,) * 6, bcs=[ff])
    params = default_params(flux=flux, limiter=limiter, Kl=1.0, solver="sgs",
                            gauss_seidel_iter=sweeps, cflmax=50.0, precision=precision)

    def init(cc):
        nc = cc.shape[0]
        rho0 = p0 / (RTILDE * T0)
        rho = rho0 * (1.0 + 0.01 * normal(seed, 0, nc))
        p = p0 * (1.0 + 0.01 * normal(seed, 1, nc))
        u = np.empty((nc, 3))
        u[:, 0] = U0 + 0.01 * U0 * normal(seed, 2, nc)
        u[:, 1] = 0.01 * U0 * normal(seed, 3, nc)
        u[:, 2] = 0.01 * U0 * normal(seed, 4, nc)
        T = p / (RTILDE * rho)
        return T, p, u

    return Case(f"farfield_cube_{n}", mesh, params, 20, init)


def outflow_duct(n: int = 16, seed: int = 0, sweeps: int = 5, mean: bool = False,
                 back_pressure: float = 1.02e5, flux: str = "roe",
                 limiter: str = "venkatakrishnan", precision: str = "ref",
                 inflow: str = "farfield", outflow: str = "outflow", u_sign: float = 1.0) -> Case:
    """Subsonic duct: n^3 hex cube [0,1]^3, inflow at x-min, outflow at
    x-max, periodic in y and z; initial state the freestream (M=0.5 along
    +x, p=1e5 Pa, T=300 K) with 1% noise (farfield_cube).  inflow:
    'farfield' or 'inflow' (the subsonic inflow condition) at the
    freestream, 'isentropic' at its total pressure and
    temperature (bcIsentropic.loci), or 'fixedMass' at its mass flux and
    total temperature (bcFixedMass.loci).  outflow: 'outflow' at a back
    pressure (bcOutflow.loci:174-273; with mean=True the pMean form, where
    the area-weighted mean of the boundary pressure is held instead), or
    'fixedMassOutflow' at 1.01 times the freestream mass flux, massRelax 0.5
    (bcFixedMassOutflow.loci).  u_sign = -1 starts the flow along -x, so
    that it leaves through the inflow condition."""
    T0, p0, M = 300.0, 1e5, 0.5
    U0 = M * math.sqrt(GAMMA * RTILDE * T0)
    ff = bc("farfield", T=T0, pg=p0, u=(U0, 0.0, 0.0))
    if inflow == "isentropic":  # total conditions of the freestream
        f = 1.0 + 0.5 * (GAMMA - 1.0) * M * M
        ff = bc("isentropicInflow", T=T0 * f, pg=p0 * f ** (GAMMA / (GAMMA - 1.0)))
    elif inflow == "inflow":  # subsonic inflow at the freestream (bcInflow.loci:376-431)
        ff = bc("inflow", T=T0, pg=p0, u=(U0, 0.0, 0.0))
    elif inflow == "fixedMass":  # the freestream's mass flux at its total temperature
        f = 1.0 + 0.5 * (GAMMA - 1.0) * M * M
        ff = bc("fixedMass", T=T0 * f, mass_flux=p0 / (RTILDE * T0) * U0)
    if outflow == "fixedMassOutflow":
        out = bc("fixedMassOutflow", T=T0, mass_flux=1.01 * p0 / (RTILDE * T0) * U0,
                 mass_relax=0.5)
    else:
        out = bc("outflowMean" if mean else "outflow", T=T0, pg=back_pressure)
    mesh = GeneratedMesh("hex", n=(n, n, n), L=(1.0, 1.0, 1.0), bc_side=(0, 1, -1, -1, -1, -1),
                         bcs=[ff, out])
    params = default_params(flux=flux, limiter=limiter, Kl=1.0, solver="sgs",
                            gauss_seidel_iter=sweeps, cflmax=50.0, precision=precision)

    def init(cc):
        nc = cc.shape[0]
        rho0 = p0 / (RTILDE * T0)
        rho = rho0 * (1.0 + 0.01 * normal(seed, 0, nc))
        p = p0 * (1.0 + 0.01 * normal(seed, 1, nc))
        u = np.empty((nc, 3))
        u[:, 0] = u_sign * U0 + 0.01 * U0 * normal(seed, 2, nc)
        u[:, 1] = 0.01 * U0 * normal(seed, 3, nc)
        u[:, 2] = 0.01 * U0 * normal(seed, 4, nc)
        T = p / (RTILDE * rho)
        return T, p, u

    return Case(f"outflow_duct_{n}", mesh, params, 100, init)


def quicktest_duct(spec: dict, n=(12, 3, 3), precision: str = "fp64", sweeps: int = 5) -> Case:
    """The duct of the reference's uniform-outcome quick tests
    (quickTest/inviscid/{inflow,isentropic,fixedMass,superSonic}.vars): unit
    cross-section, the test's inflow condition at x-min and its outflow
    condition at x-max, periodic in y and z (the tests' symmetry sides carry
    no flux across them either), started from the test's initial state and
    stepped as the test is: pseudo-time step dtmax (cflmax unset), its
    urelax, no limiter.  spec is one entry of
    tests/golden/quicktest_uniform.json.  Inviscid, Roe: only the converged
    state, which the two conditions fix, is compared."""
    i, o = spec["inflow"], spec["outflow"]
    if i["kind"] in ("inflow", "supersonicInflow"):
        inb = bc(i["kind"], T=i["T"], pg=i["p"], u=(i["u"], 0.0, 0.0))
    elif i["kind"] == "isentropicInflow":
        inb = bc("isentropicInflow", T=i["T0"], pg=i["p0"])
    else:
        inb = bc("fixedMass", T=i["T0"], mdot=i["mdot"])
    ic = spec["init"]
    if o["kind"] == "outflow":
        out = bc("outflow", T=ic["T"], pg=o["p"])
    else:
        out = bc("supersonicOutflow")
    mesh = GeneratedMesh("hex", n=tuple(n), L=(1.0, 1.0, 1.0), bc_side=(0, 1, -1, -1, -1, -1),
                         bcs=[inb, out])
    params = default_params(flux="roe", limiter="none", solver="sgs", gauss_seidel_iter=sweeps,
                            cflmax=0.0, dtmax=spec["dtmax"], urelax=spec["urelax"],
                            precision=precision)
    u0 = ic["u"] if "u" in ic else ic["M"] * math.sqrt(GAMMA * RTILDE * ic["T"])

    def init(cc):
        nc = cc.shape[0]
        u = np.zeros((nc, 3))
        u[:, 0] = u0
        return np.full(nc, ic["T"]), np.full(nc, ic["p"]), u

    return Case(f"quicktest_duct_{i['kind']}", mesh, params, spec["stop_iter"], init)


def taylor_green_tets(n: int = 128, seed: int = 0, sweeps: int = 8, jitter: float = 0.1,
                      amplitude: float = 1.0, precision: str = "mixed", flux: str = "roe",
                      limiter: str = "venkatakrishnan") -> Case:
    L = 2.0 * math.pi
    mesh = GeneratedMesh("kuhn", n=(n, n, n), L=(L, L, L), jitter=jitter, seed=seed)
    params = default_params(flux=flux, limiter=limiter, Kl=1.0, solver="sgs",
                            gauss_seidel_iter=sweeps, cflmax=50.0, precision=precision)
    T0, p0, M = 300.0, 1e5, 0.1
    rho0 = p0 / (RTILDE * T0)
    U0 = amplitude * M * math.sqrt(GAMMA * RTILDE * T0)

    def init(cc):
        x, y, z = cc[:, 0], cc[:, 1], cc[:, 2]
        u = np.empty((cc.shape[0], 3))
        u[:, 0] = U0 * np.sin(x) * np.cos(y) * np.cos(z)
        u[:, 1] = -U0 * np.cos(x) * np.sin(y) * np.cos(z)
        u[:, 2] = 0.0
        p = p0 + rho0 * U0 * U0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
        T = p / (rho0 * RTILDE)
        return T, p, u

    return Case(f"taylor_green_tets_{n}", mesh, params, 200, init)


def farfield_tets(n: int = 128, seed: int = 0, sweeps: int = 8, jitter: float = 0.1,
                  precision: str = "mixed", flux: str = "roe",
                  limiter: str = "venkatakrishnan", L: float = 2.0 * math.pi) -> Case:
    """Steady case on the Taylor-Green split-tet grid: n^3 hexes of the box
    [0,L]^3 split into 6 Kuhn tetrahedra, nodes jittered by +-10% of the
    spacing (the sides stay plane), farfield on all six sides at M=0.5
    along +x, p=1e5 Pa, T=300 K; initial state the freestream with 1%
    Gaussian noise in rho, u, v, w and p (as farfield_cube).  Roe + MUSCL +
    Venkatakrishnan, 8 SGS sweeps, CFL 50.  The noise leaves through the
    farfield sides, so the residual falls to machine level."""
    T0, p0, M = 300.0, 1e5, 0.5
    U0 = M * math.sqrt(GAMMA * RTILDE * T0)
    ff = bc("farfield", T=T0, pg=p0, u=(U0, 0.0, 0.0))
    mesh = GeneratedMesh("kuhn", n=(n, n, n), L=(L, L, L), jitter=jitter, seed=seed,
                         bc_side=(0,) * 6, bcs=[ff])
    params = default_params(flux=flux, limiter=limiter, Kl=1.0, solver="sgs",
                            gauss_seidel_iter=sweeps, cflmax=50.0, precision=precision)

    def init(cc):
        nc = cc.shape[0]
        rho0 = p0 / (RTILDE * T0)
        rho = rho0 * (1.0 + 0.01 * normal(seed, 0, nc))
        p = p0 * (1.0 + 0.01 * normal(seed, 1, nc))
        u = np.empty((nc, 3))
        u[:, 0] = U0 + 0.01 * U0 * normal(seed, 2, nc)
        u[:, 1] = 0.01 * U0 * normal(seed, 3, nc)
        u[:, 2] = 0.01 * U0 * normal(seed, 4, nc)
        T = p / (RTILDE * rho)
        return T, p, u

    return Case(f"farfield_tets_{n}", mesh, params, 400, init)


MU_A = (1.458e-6, 1.5, 110.4)  # Sutherland, fluxViscous.loci:58-80
SA_CV1 = 7.1                    # SA_param.h:34


def sutherland_mu(T):
    return MU_A[0] * np.power(T, MU_A[1]) / (T + MU_A[2])


def sa_eddy_viscosity(nu_tilde, rho, mu):
    """Spalart-Allmaras eddy viscosity tmu = rho nu~ fv1, chi = rho nu~ / mu,
    fv1 = chi^3 / (chi^3 + cv1^3) (SA_turb.loci:91-107)"""
    chi3 = (rho * nu_tilde / mu) ** 3
    return nu_tilde * chi3 / (chi3 + SA_CV1 ** 3) * rho


def boundary_layer_block(nx: int = 256, ny: int = 128, nz: int = 64, dy0: float = 1e-6,
                         growth: float = 1.15, seed: int = 0,
                         precision: str = "mixed", solver: str = "lsgs", viscous: int = 0,
                         Re: float = 1e6, Lx: float = 1.0, Lz: float = 0.25,
                         sa: bool = False) -> Case:
    """Flat-plate block: x streamwise, y wall-normal (first spacing dy0,
    geometric growth), z spanwise periodic; wall at y = 0 (slip wall when
    inviscid, adiabatic no-slip wall otherwise), farfield at the top, inflow
    and outflow sides.  M=0.3, T=300 K; viscous cases set the freestream
    density so that Re = rho U / mu(T) per unit length, inviscid ones use
    p = 1e5 Pa.  viscous: 0 inviscid, 1 laminar, 2 turbulent with the
    Spalart-Allmaras eddy viscosity of a frozen nu~ = 3 nu_inf field
    (case.tmu), or with sa=True the Spalart-Allmaras transport of nu~ from
    nu~ = 3 nu_inf (case.nut0; inflow boundaries carry the same value).  The
    wall-normal columns are the LSGS lines (case.lines)."""
    T0, M = 300.0, 0.3
    U0 = M * math.sqrt(GAMMA * RTILDE * T0)
    mu0 = float(sutherland_mu(T0))
    if viscous:
        rho0 = Re * mu0 / U0
        p0 = rho0 * RTILDE * T0
    else:
        p0 = 1e5
        rho0 = p0 / (RTILDE * T0)
    nut_inf = 3.0 * mu0 / rho0
    ff = bc("farfield", T=T0, pg=p0, u=(U0, 0.0, 0.0), nu_t=nut_inf if sa else 0.0)
    wl = bc("viscousWall" if viscous else "reflecting", T=T0, pg=p0)
    mesh = GeneratedMesh("bl", n=(nx, ny, nz), L=(Lx, 1.0, Lz), dy0=dy0, growth=growth,
                         bc_side=(0, 0, 1, 0, -1, -1), bcs=[ff, wl])
    if sa and viscous != 2:
        raise ValueError("the SA model needs viscous=2")
    params = default_params(flux="roe", limiter="venkatakrishnan", solver=solver,
                            gauss_seidel_iter=8, cflmax=50.0, precision=precision,
                            viscous=viscous, turbulence=1 if sa else 0)

    def init(cc):
        nc = cc.shape[0]
        u = np.zeros((nc, 3))
        u[:, 0] = U0 * (1.0 + 0.01 * normal(seed, 2, nc))
        u[:, 1] = 0.01 * U0 * normal(seed, 3, nc)
        u[:, 2] = 0.01 * U0 * normal(seed, 4, nc)
        p = p0 * (1.0 + 0.01 * normal(seed, 1, nc))
        T = T0 * (1.0 + 0.01 * normal(seed, 0, nc))
        return T, p, u

    c = Case(f"boundary_layer_{nx}x{ny}x{nz}", mesh, params, 100, init)
    c.lines = mesh.lines_along(1)
    c.tmu = c.nut0 = None
    nc = nx * ny * nz
    if sa:
        c.nut0 = np.full(nc, nut_inf)
    elif viscous == 2:
        c.tmu = np.full(nc, float(sa_eddy_viscosity(nut_inf, rho0, mu0)))
    return c


def oblique_shock_cube(n: int = 256, seed: int = 0, sweeps: int = 8, precision: str = "mixed",
                       flux: str = "hlle", limiter: str = "barth") -> Case:
    T1, p1, M1 = 300.0, 1e5, 2.0
    a1 = math.sqrt(GAMMA * RTILDE * T1)
    U1 = M1 * a1
    inflow = bc("supersonicInflow", T=T1, pg=p1, u=(U1, 0.0, 0.0))
    outflow = bc("supersonicOutflow", T=T1, pg=p1, u=(U1, 0.0, 0.0))
    # x-min supersonic inflow, the rest supersonic outflow
    mesh = GeneratedMesh("hex", n=(n, n, n), L=(1.0, 1.0, 1.0),
                         bc_side=(0, 1, 1, 1, 1, 1), bcs=[inflow, outflow])
    params = default_params(flux=flux, limiter=limiter, solver="sgs", gauss_seidel_iter=sweeps,
                            cflmax=50.0, precision=precision)
    # shock plane through the centre, normal tilted 30 degrees from x in x-y
    th = math.radians(30.0)
    nrm = np.array([math.cos(th), math.sin(th), 0.0])
    Mn = M1 * nrm[0]
    g = GAMMA
    p2 = p1 * (1 + 2 * g / (g + 1) * (Mn * Mn - 1))
    r1 = p1 / (RTILDE * T1)
    r2 = r1 * (g + 1) * Mn * Mn / ((g - 1) * Mn * Mn + 2)
    T2 = p2 / (RTILDE * r2)
    u1 = np.array([U1, 0.0, 0.0])
    un1 = float(u1 @ nrm)
    un2 = un1 * r1 / r2
    u2 = u1 + (un2 - un1) * nrm

    def init(cc):
        nc = cc.shape[0]
        s = (cc - 0.5) @ nrm
        down = s > 0
        T = np.where(down, T2, T1)
        p = np.where(down, p2, p1)
        u = np.where(down[:, None], u2[None, :], u1[None, :])
        T = T * (1.0 + 0.005 * normal(seed, 0, nc))
        p = p * (1.0 + 0.005 * normal(seed, 1, nc))
        u = u * (1.0 + 0.005 * normal(seed, 2, nc))[:, None]
        return T, p, u

    return Case(f"oblique_shock_cube_{n}", mesh, params, 200, init)
