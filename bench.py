"""Benchmark of the steady implicit step (residual, Jacobians, LU, multi-colour
SGS, Newton update) on the 128^3 split-tet Taylor-Green grid.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fpsi|reference]

One step = one implicit pseudo-time step over every cell: FP64 residual
(MUSCL + Venkatakrishnan + Roe), FP32 Jacobian blocks and LU, 8 symmetric
multi-colour SGS sweeps in FP32 (defect correction), FP64 Newton update.
Metric: cell-iterations per second.  Under torchrun each rank runs an
independent replica of the grid on its own GPU (the path is not partitioned
across GPUs); timing is CUDA events on the library's stream, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-iters/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """SM clocks and clock-event reasons sampled over the timed region: NVML
    read every 20 ms from a thread (the same counters nvidia-smi prints),
    or an nvidia-smi sampler when NVML is unavailable.  Read-only."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        parts = [p for p in vis.split(",") if p.strip()]
        # the CUDA index maps to the NVML index through CUDA_VISIBLE_DEVICES
        self.index = int(parts[index]) if index < len(parts) and parts[index].strip().isdigit() else index
        self.samples, self.stop, self.thread, self.p, self.f = [], None, None, None, None

    def _nvml_loop(self, h, nv):
        bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while True:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), [n for n, b in zip(self.NAMES, bits) if r & b]))
            except Exception:  # noqa: BLE001
                pass
            if self.stop.wait(0.02):
                break

    def __enter__(self):
        try:
            import threading

            import pynvml as nv

            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, args=(h, nv), daemon=True)
            self.thread.start()
            return self
        except Exception:  # noqa: BLE001
            self.thread = None
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            t0 = time.time()  # wait for the first sample before the timed region
            while time.time() - t0 < 3 and not Path(self.f.name).read_text().strip():
                time.sleep(0.02)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(2)
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        if self.thread is not None:
            rows = self.samples
            src = "nvml"
        elif self.p is not None:
            self.f.flush()
            rows = []
            for r in Path(self.f.name).read_text().splitlines():
                r = r.split(",")
                try:
                    rows.append((float(r[1]), float(r[2]),
                                 [nm for nm, v in zip(self.NAMES, r[5:9]) if v.strip().lower() == "active"]))
                except (ValueError, IndexError):
                    continue
            src = "nvidia-smi"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm = [r[0] for r in rows]
        reasons = sorted({n for r in rows for n in r[2]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(r[1] for r in rows) if rows else None, "reasons": reasons,
                "samples": len(sm), "source": src}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def dist_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def sgs_launch_sequence(ncolours, sweeps):
    """colours launched by one step's sweeps: forward then backward, a
    colour that directly follows itself is not relaunched"""
    seq, last = [], -1
    for _ in range(sweeps):
        for k in list(range(ncolours)) + list(range(ncolours - 1, -1, -1)):
            if k != last:
                seq.append(k)
                last = k
    return seq


def sgs_colour_bytes(colour, nint, tb, tx, slot=25):
    """algorithmic bytes of one launch of each colour: per cell LU 25*tb +
    B 5*tb + x write 5*tx; per interior face side the off-diagonal slot
    (25 values, or 15 in the compact Roe form) + index 4 + neighbour x 5*tx"""
    per_cell = (30 * tb + 5 * tx) + nint * (slot * tb + 4 + 5 * tx)
    return np.bincount(colour, weights=per_cell.astype(np.float64))


def sgs_bytes_per_step(colour_bytes, sweeps):
    seq = sgs_launch_sequence(len(colour_bytes), sweeps)
    return float(sum(colour_bytes[k] for k in seq)), len(seq)


def kernel_bytes(name, nc, nfi, nbf, sweeps, tb, tx, sgs_step_bytes=None, compact=False):
    """algorithmic bytes of one step of each kernel (every array the kernel
    must touch counted once: FP64 8 B, FP32 4 B, index 4 B).  compact: the
    inviscid SGS system keeps its face Jacobians as 24-value face records
    (9 coefficients per direction + U + n) and 15-value sweep slots"""
    nf = nfi + nbf
    qf = 96  # reconstructed face states of both sides (+ spectral radii) per face
    if compact:
        jac_out = nf * 24 * tb
        # each face side needs its direction's 9 coefficients and U, n
        asm_faces = (2 * nfi + nbf) * 15 * tb + 2 * nfi * 15 * tb
    else:
        jac_out = (nfi * 2 + nbf) * 25 * tb
        asm_faces = (2 * nfi + nbf) * 25 * tb + 2 * nfi * 25 * tb
    return {
        "bc_state": nbf * (4 + 24 + 40 + 40),
        # q + Minv + vol per cell; per face cl,cr 8 + rL,rR 48 + n 24, the
        # two face-list entries 8 and the face-state write; boundary states
        "grad_limiter": nc * (40 + 48 + 8) + nf * (8 + 48 + 24 + 8 + qf) + nbf * 40,
        # face states, n and area in, the 48 B flux record out
        "face_flux": nf * (qf + 32 + 48),
        "cell_residual": nc * (40 + 8 + 40 + 8) + nf * 48,
        "face_jacobian": nf * (qf + 32) + jac_out,
        # the inviscid SGS systems' flux and compact Jacobian records in one pass
        "face_flux_jac": nf * (qf + 32 + 48) + jac_out,
        # q, src, dtau, vol; LU + B slots, pivots, Jacobi start; each face
        # block read once for the diagonal sum, interior ones written once
        # more into the off-diagonal slots
        "assemble_lu": nc * (40 + 40 + 8 + 8 + 30 * tb + 4 + 5 * tx) + asm_faces,
        "sgs_colour": sgs_step_bytes,
        "update": nc * (80 + 5 * tx),
    }.get(name)


def build_case(args):
    """the bench workload: the Taylor-Green split-tet grid (default), the
    turbulent boundary-layer block with line SGS and the viscous terms, or
    the oblique-shock hex cube"""
    from flowpsi_b200 import cases

    if args.workload == "bl":
        return cases.boundary_layer_block(args.bl_nx, args.bl_ny, args.bl_nz,
                                          precision=args.precision, viscous=args.viscous,
                                          solver="lsgs",
                                          sa=args.viscous == 2 and args.turb == "sa")
    if args.workload == "shock":
        return cases.oblique_shock_cube(args.n, seed=args.seed, sweeps=args.sweeps,
                                        precision=args.precision)
    return cases.taylor_green_tets(args.n, seed=args.seed, sweeps=args.sweeps,
                                   precision=args.precision)


def workload_name(args) -> str:
    if args.workload == "bl":
        turb = f"_{args.turb}" if args.viscous == 2 else ""
        return f"boundary_layer_{args.bl_nx}x{args.bl_ny}x{args.bl_nz}_visc{args.viscous}{turb}"
    if args.workload == "shock":
        return f"oblique_shock_cube_{args.n}"
    return f"taylor_green_tets_{args.n}"


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class OracleSample:
    """the oracle (the C++ restatement) on a smaller grid of the same
    workload with every requested host thread (residual, Jacobians and
    assembly in parallel), its SGS in the reference's sequential cell order
    (linearSolverSGS.loci:150-329, one thread) or multi-colour (parallel)"""

    def __init__(self, args, threads: int, n_sample: int, order: str = "sequential"):
        from flowpsi_b200 import cases
        from oracle import Oracle
        from oracle.oracle import set_threads

        self.threads = set_threads(threads)
        case = cases.taylor_green_tets(n_sample, seed=args.seed, sweeps=args.sweeps,
                                       precision=args.precision)
        self.case = case
        self.o = Oracle(case.mesh, case.params)
        T, p, u = case.initial_state(self.o.geometry()["cellcenter"])
        self.o.set_state(T, p, u)
        self.colour = greedy_colours(case.mesh) if order == "multicolour" else None
        self.order = order
        self.ncells = self.o.ncells

    def step(self) -> float:
        t0 = time.perf_counter()
        self.o.newton_step(colour=self.colour)
        return time.perf_counter() - t0


def cpu_oracle_rate(args, threads: int, n_sample: int, order: str, budget_s: float,
                    min_steps: int = 2):
    """cell-iterations per second of the oracle over steps until budget_s
    of CPU time (at least min_steps), after one warm-up step"""
    s = OracleSample(args, threads, n_sample, order)
    s.step()  # warm-up
    dt, steps = 0.0, 0
    while steps < min_steps or dt < budget_s:
        dt += s.step()
        steps += 1
    return s.ncells * steps / dt, s.ncells, dt, steps


def greedy_colours(mesh) -> np.ndarray:
    a = mesh.arrays()
    nc = a.ncells
    inner = a.cr >= 0
    cl, cr = a.cl[inner], a.cr[inner]
    nbr = [[] for _ in range(nc)]
    for x, y in zip(cl.tolist(), cr.tolist()):
        nbr[x].append(y)
        nbr[y].append(x)
    col = np.full(nc, -1, np.int32)
    for c in range(nc):
        used = {col[m] for m in nbr[c] if col[m] >= 0}
        k = 0
        while k in used:
            k += 1
        col[c] = k
    return col


def run_reference(args, ws, rank):
    """reference arm: the CPU restatement of the reference path (oracle port)
    with every host thread, one bounded sample per step"""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    smp = OracleSample(args, threads, args.cpu_n, "sequential")
    for _ in range(args.warmup):
        smp.step()
    times = [smp.step() for _ in range(args.steps)]
    total_dt = sum(times)
    rates = [smp.ncells / t for t in times]
    value = statistics.median(rates)
    sample = (f"taylor_green_tets {args.cpu_n}^3 x 6 = {6 * args.cpu_n ** 3} cells, "
              f"one implicit step per timed step, {args.sweeps} SGS sweeps in the reference's "
              f"sequential cell order; CPU {cpu_model()}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-iters/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_dt / max(args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": f"taylor_green_tets_{args.n}", "sample_cells": 6 * args.cpu_n ** 3,
                   "precision": args.precision, "sgs_sweeps": args.sweeps},
        "cpu_baseline": {"value": value, "unit": "cell-iters/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "cell-iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


RT_AIR, GAMMA = 8314.4621 / 28.96, 1.4


def _rho_energy(T, p, u):
    rho = p / (RT_AIR * T)
    return rho, rho * (RT_AIR * T / (GAMMA - 1.0) + 0.5 * (u * u).sum(1))


def _drop_arm(solver, case, drop, max_steps, chunk, model=None):
    """device ms and steps until the density residual (rtrms) falls below
    drop x its step-0 value.  Without a model: fpsi_run_timed in chunks
    (CUDA events on the library's stream).  With a model: one
    fpsi_newton_step_ex per step from the learned start with the rejection
    rule, timed by the host clock around the steps (its host decisions and
    copies are part of the cost)."""
    solver.set_state(*case.initial_state(solver.geometry()["cellcenter"]))
    r0, done, ms_tot, reached, rejected = None, 0, 0.0, None, 0
    if model is None:
        while done < max_steps and reached is None:
            hist, ms = solver.run_timed(chunk)
            if r0 is None:
                r0 = hist[0]["rtrms"]
            for k, h in enumerate(hist):
                if h["rtrms"] < drop * r0:
                    reached = done + k
                    ms_tot += ms * k / chunk
                    break
            else:
                ms_tot += ms
            done += chunk
    else:
        # one untimed learned step first: the context builds its cell graph
        # for the network and allocates the inference and rejection buffers
        # once per mesh, as the other arms' setup does; then the state is
        # reset, which also drops that step's update from the features
        solver.newton_step_ex(start="learned", model=model, reject=True)
        solver.set_state(*case.initial_state(solver.geometry()["cellcenter"]))
        t0 = time.perf_counter()
        for k in range(max_steps):
            r = solver.newton_step_ex(start="learned", model=model, reject=True)
            rejected += int(r["rejected"])
            if r0 is None:
                r0 = r["rtrms"]
            if r["after"]["rtrms"] < drop * r0:
                reached = k + 1
                break
        ms_tot = 1e3 * (time.perf_counter() - t0)
    return {"steps": reached, "ms": ms_tot if reached is not None else None, "r0": r0,
            "rejected": rejected if model is not None else None,
            "timer": "host clock, per-step decisions" if model is not None else
            "CUDA events on the library stream"}, solver.get_state()


def time_to_drop(n: int, drop: float = 1e-8, max_steps: int = 400, chunk: int = 10,
                 seed: int = 0, learned: bool = True):
    """Time to a 1e-8 drop of the density residual on the steady split-tet
    case (farfield_tets: the 128^3 x 6 jittered Kuhn grid of the
    Taylor-Green workload with farfield sides, M=0.5 freestream with 1%
    noise, Roe + MUSCL + Venkatakrishnan, 8 SGS sweeps, CFL 50): plain FP64,
    MIXED from the reference's Jacobi start, and MIXED from the learned start
    (a model trained first on 16^3 x 6 grids of the same case, seeds 1-4).
    Each arm reports steps, ms and the largest density and energy difference
    of its final state from the FP64 arm's and from the converged state (the
    FP64 run continued, untimed, to a 1e-12 drop)."""
    from flowpsi_b200 import FlowPsi, cases

    out = {"case": f"farfield_tets_{n}", "cells": 6 * n ** 3, "drop": drop}
    c64 = cases.farfield_tets(n, seed=seed, precision="fp64")
    s = FlowPsi(c64.mesh, c64.params)
    s.keep_blocks(False)
    out["fp64"], st64 = _drop_arm(s, c64, drop, max_steps, chunk)
    r0, extra = out["fp64"]["r0"], 0
    while extra < 400:
        hist = s.run(chunk)
        extra += chunk
        if hist[-1]["rtrms"] < 1e-12 * r0:
            break
    out["converged"] = {"extra_fp64_steps": extra, "drop": hist[-1]["rtrms"] / r0}
    rho_c, e_c = _rho_energy(*s.get_state())
    s.close()
    del s
    rho64, e64 = _rho_energy(*st64)

    def vs_converged(rho, e):
        return {"rho": float(np.abs(rho - rho_c).max() / np.abs(rho_c).max()),
                "rho_e0": float(np.abs(e - e_c).max() / np.abs(e_c).max())}

    out["fp64"]["max_rel_diff_vs_converged"] = vs_converged(rho64, e64)
    c32 = cases.farfield_tets(n, seed=seed, precision="mixed")
    s = FlowPsi(c32.mesh, c32.params)
    s.keep_blocks(learned)
    arms = [("mixed", None)]
    if learned:
        from flowpsi_b200.learned import train_on_case

        model, info = train_on_case(lambda sd: cases.farfield_tets(16, seed=sd, precision="fp64"),
                                    seeds=(1, 2, 3, 4), steps_per_seed=12, train_steps=1500,
                                    batch=16384)
        out["training"] = info
        arms.append(("mixed_learned", model))
    for name, model in arms:
        out[name], st = _drop_arm(s, c32, drop, max_steps, chunk, model)
        rho, e = _rho_energy(*st)
        out[name]["max_rel_diff_vs_fp64"] = {
            "rho": float(np.abs(rho - rho64).max() / np.abs(rho64).max()),
            "rho_e0": float(np.abs(e - e64).max() / np.abs(e64).max())}
        out[name]["max_rel_diff_vs_converged"] = vs_converged(rho, e)
    if learned:
        model.close()
    s.close()
    f = out["fp64"]["ms"]
    for name, _ in arms:
        m = out[name]["ms"]
        out[name]["speedup_vs_fp64"] = (f / m) if f and m else None
    return out


def bl_time_to_drop(drop: float = 1e-8, max_steps: int = 16000, chunk: int = 100) -> dict:
    """Config 3 to a 1e-8 drop: the 256x128x64 flat-plate boundary layer
    (first spacing 1e-6, growth 1.15, M 0.3, Re 1e6), Spalart-Allmaras,
    line SGS over the wall-normal lines, CFL 50; plain FP64 and MIXED, each
    timed with CUDA events in chunks of `chunk` steps"""
    from flowpsi_b200 import FlowPsi, cases

    out = {"case": "boundary_layer_256x128x64_sa", "cells": 256 * 128 * 64, "drop": drop}
    for prec in ("fp64", "mixed"):
        case = cases.boundary_layer_block(256, 128, 64, precision=prec, viscous=2, solver="lsgs",
                                          sa=True)
        s = FlowPsi(case.mesh, case.params)
        s.set_lines(case.lines)
        s.set_state(*case.initial_state(s.geometry()["cellcenter"]))
        s.set_nutilde(case.nut0)
        r0, done, ms, reached, hist_out = None, 0, 0.0, None, []
        while done < max_steps and reached is None:
            hist, dt = s.run_timed(chunk)
            r0 = r0 or hist[0]["rtrms"]
            for k, h in enumerate(hist):
                if h["rtrms"] < drop * r0:
                    reached = done + k
                    ms += dt * k / chunk
                    break
            else:
                ms += dt
            done += chunk
            if done % 1000 == 0:
                hist_out.append((done, hist[-1]["rtrms"] / r0))
        out[prec] = {"steps": reached, "ms": ms if reached is not None else None,
                     "drop_every_1000": hist_out, "timer": "CUDA events on the library stream"}
        s.close()
    f, m = out["fp64"]["ms"], out["mixed"]["ms"]
    out["mixed"]["speedup_vs_fp64"] = (f / m) if f and m else None
    return out


def run_fpsi(args, ws, rank, local):
    from flowpsi_b200 import FlowPsi
    from flowpsi_b200 import _native as N

    if not N.lib().fpsi_device_available():
        raise SystemExit("no CUDA device: the fpsi arm has no CPU fallback")
    t0 = time.perf_counter()
    case = build_case(args)
    solver = FlowPsi(case.mesh, case.params)
    if case.params.solver == 1:  # line SGS over the case's wall-normal lines
        solver.set_lines(case.lines)
    else:
        solver.keep_blocks(False)
    if getattr(case, "tmu", None) is not None:
        solver.set_eddy_viscosity(case.tmu)
    if getattr(case, "nut0", None) is not None:
        solver.set_nutilde(case.nut0)
    log(f"[rank {rank}] setup {time.perf_counter() - t0:.1f}s: {solver.ncells} cells, "
        f"{solver.nfaces} faces, {solver.ncolours} colours, "
        f"{solver.device_bytes / 1e9:.2f} GB device")
    geo = solver.geometry()
    T0, p0, u0 = case.initial_state(geo["cellcenter"])
    solver.set_state(T0, p0, u0)
    nc, nf = solver.ncells, solver.nfaces
    arr = case.mesh.arrays()
    inner = np.asarray(arr.cr) >= 0
    nfi = int(inner.sum())
    nbf = nf - nfi
    nint = (np.bincount(np.asarray(arr.cl)[inner], minlength=nc)
            + np.bincount(np.asarray(arr.cr)[inner], minlength=nc))
    hist_w = solver.run(args.warmup) if args.warmup > 0 else []
    dist_barrier(ws)
    with Clocks(local) as clk:
        hist, ms = solver.run_timed(args.steps)
    ms = dist_max(ms, ws)
    clocks = clk.summary()
    value = nc * args.steps * ws / (ms / 1e3)

    # per-kernel device times (separate run, events around every launch)
    kt = solver.kernel_times(args.profile_steps)
    tb = 4 if args.precision in ("ref", "mixed") else 8
    tx = 4 if args.precision == "mixed" else 8
    # inviscid systems relaxed by multi-colour SGS keep compact face Jacobians
    compact = case.params.viscous == 0 and case.params.solver == 0
    peaks, src = load_peaks()
    peak = float(peaks["hbm_gbs"])
    kernels = {}
    sgs_step = None
    if case.params.solver == 0:
        cb = sgs_colour_bytes(solver.colours(), nint, tb, tx, slot=15 if compact else 25)
        sgs_step, _ = sgs_bytes_per_step(cb, case.params.gauss_seidel_iter)
    for name, (kms, launches) in kt.items():
        b = kernel_bytes(name, nc, nfi, nbf, args.sweeps, tb, tx, sgs_step, compact)
        per_step_ms = kms / args.profile_steps
        kernels[name] = {"ms_per_step": per_step_ms, "launches_per_step": launches / args.profile_steps,
                         "gbs": None if b is None else b / (per_step_ms / 1e3) / 1e9}
    dom = max((k for k in kernels if kernels[k]["gbs"] is not None),
              key=lambda k: kernels[k]["ms_per_step"])
    dk = kernels[dom]
    b_launch = (kernel_bytes(dom, nc, nfi, nbf, args.sweeps, tb, tx, sgs_step, compact)
                / dk["launches_per_step"])
    avg_launch_s = dk["ms_per_step"] / dk["launches_per_step"] / 1e3
    achieved = b_launch / avg_launch_s / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        key = f"{dom}:{args.precision}:{args.n}" if args.workload == "tgv" else None
        traffic = json.loads(tf.read_text()).get(key) if key else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": dom,
                "peak_source": src, "bytes_per_launch": b_launch}

    # end to end through the public API: per step the state goes host ->
    # device from pinned memory, one implicit step runs, the new state and the
    # residual norms come back
    import torch

    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    Th, ph, uh = pin(T0), pin(p0), pin(u0)
    outs = (pin(np.empty(nc)), pin(np.empty(nc)), pin(np.empty(3 * nc)))
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    solver.set_state(Th, ph, uh)
    solver.newton_step()  # first touch of the pinned pages
    solver.get_state(out=outs)
    dist_barrier(ws)
    t1 = time.perf_counter()
    for _ in range(e2e_steps):
        solver.set_state(Th, ph, uh)
        solver.newton_step()
        solver.get_state(out=outs)
    e2e_s = dist_max(time.perf_counter() - t1, ws)
    e2e = {"value": nc * e2e_steps * ws / e2e_s, "unit": "cell-iters/s",
           "h2d_bytes_per_step": 5 * 8 * nc, "d2h_bytes_per_step": 5 * 8 * nc + 64,
           "steps": e2e_steps, "timer": "host wall clock, synchronous API"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        r, ncs, dt, k = cpu_oracle_rate(args, threads, args.cpu_n, "sequential", args.cpu_budget)
        r2, _, dt2, k2 = cpu_oracle_rate(args, threads, args.cpu_n, "multicolour", args.cpu_budget)
        cpu = {"value": r, "unit": "cell-iters/s", "cores": threads, "kind": "port",
               "cpu": cpu_model(),
               "sample": f"taylor_green_tets {args.cpu_n}^3 x 6 = {ncs} cells, {k} implicit "
                         f"steps ({dt:.1f} s); residual, Jacobians and assembly on {threads} "
                         f"threads, SGS in the reference's sequential cell order (one thread)",
               "multicolour": {"value": r2, "steps": k2, "seconds": dt2,
                               "sample": "the same grid with multi-colour SGS on every thread"}}

    converge = None
    if args.converge_n > 0 and rank == 0 and ws == 1:
        # second half of the metric: time to a 1e-8 residual drop on the
        # steady split-tet case, FP64 against FP32 relaxation (MIXED) from
        # the reference's start and from the learned start
        solver.close()
        converge = time_to_drop(args.converge_n, learned=not args.no_learned)

    launches = sum(v[1] for v in kt.values()) / args.profile_steps * args.steps
    line = {
        "metric": METRIC, "value": value, "unit": "cell-iters/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 residual + f32 blocks/sweeps" if args.precision == "mixed" else args.precision,
        "data": {"tgv": "synthetic (seeded Taylor-Green on a jittered split-tet grid)",
                 "bl": "synthetic (seeded noise on a flat-plate block; SA nu~ from 3 nu_inf)",
                 "shock": "synthetic (seeded oblique Mach-2 shock on a hex cube)"}[args.workload],
        "config": {"workload": workload_name(args), "cells": nc, "faces": nf,
                   "colours": solver.ncolours, "precision": args.precision,
                   "flux": {v: k for k, v in N.FLUX.items()}[case.params.flux],
                   "limiter": {v: k for k, v in N.LIMITER.items()}[case.params.limiter],
                   "solver": "lsgs" if case.params.solver == 1 else "sgs",
                   "sgs_sweeps": case.params.gauss_seidel_iter,
                   "parallelism": f"replicas{ws}",
                   "launch": ("CUDA graph of one step, captured at the second step of each run "
                              "and replayed" if case.params.step_graphs else "kernel launches"),
                   "l2": "inputs larger than L2 (%.1f GB resident)" % (solver.device_bytes / 1e9)},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(round(launches)),
        "clocks": clocks,
        "kernels": kernels,
        "time_to_1e-8": converge,
        "resid_first": hist[0]["rtrms"] if hist else None,
        "resid_last": hist[-1]["rtrms"] if hist else None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    solver.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fpsi", choices=["fpsi", "reference"])
    ap.add_argument("--n", type=int, default=128, help="hexes per direction (x6 tets)")
    ap.add_argument("--sweeps", type=int, default=8)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "ref", "mixed"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--profile-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-n", type=int, default=48)
    ap.add_argument("--cpu-budget", type=float, default=12.0,
                    help="seconds of CPU time per cpu_baseline variant")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="tgv", choices=["tgv", "bl", "shock"])
    ap.add_argument("--bl-nx", type=int, default=256)
    ap.add_argument("--bl-ny", type=int, default=128)
    ap.add_argument("--bl-nz", type=int, default=64)
    ap.add_argument("--viscous", type=int, default=2, help="bl: 0 inviscid, 1 laminar, 2 turbulent")
    ap.add_argument("--turb", default="sa", choices=["sa", "frozen"],
                    help="bl turbulent: SA nu~ transport or a frozen eddy viscosity")
    ap.add_argument("--converge-n", type=int, default=128,
                    help="split-tet farfield grid (n^3 x 6) of the time-to-1e-8 runs (0: skip)")
    ap.add_argument("--bl-drop", action="store_true",
                    help="only config 3 to a 1e-8 drop (boundary layer, SA, line SGS), FP64 and MIXED")
    ap.add_argument("--no-learned", action="store_true",
                    help="time-to-1e-8 without the learned-start arm")
    args = ap.parse_args()
    if args.bl_drop:
        print(json.dumps({"time_to_1e-8": bl_time_to_drop()}), flush=True)
        return
    if args.warmup < 3:
        log("warning: fewer than 3 warm-up steps")
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_fpsi(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
