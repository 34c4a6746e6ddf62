"""Learned starting iterate of the block relaxation (host side).

No counterpart in the reference; the hook is the relaxation's starting
iterate (linearSolverSGS.loci:57-69).  The network, its training and its
inference run in the library's CUDA kernels (flowpsi_b200/csrc/gnn.cu); this
module drives them: snapshot generation from the solver itself and
training.  Inside a Newton step the start is used through
FlowPsi.newton_step_ex(start="learned", model=...), which runs in the
library (fpsi_newton_step_ex): a step that does not lower the FP64 density
residual is undone and redone from the reference's Jacobi start D^-1 B.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .solver import FlowPsi

_fp = C.POINTER(C.c_float)


class LearnedStart:
    """The network's weights (independent of the mesh) and its training set;
    one model serves any FlowPsi context."""

    def __init__(self, seed: int = 0):
        h = C.c_void_p()
        N.check(N.lib().fpsi_gnn_create(C.byref(h), seed), "fpsi_gnn_create")
        self._h = h
        self.n_params = int(N.lib().fpsi_gnn_num_params(h))

    def close(self):
        if getattr(self, "_h", None):
            N.lib().fpsi_gnn_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def get_params(self) -> np.ndarray:
        w = np.empty(self.n_params, np.float32)
        N.check(N.lib().fpsi_gnn_get_params(self._h, w.ctypes.data_as(_fp)), "fpsi_gnn_get_params")
        return w

    def set_params(self, w) -> None:
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == self.n_params
        N.check(N.lib().fpsi_gnn_set_params(self._h, w.ctypes.data_as(_fp)), "fpsi_gnn_set_params")

    def add_snapshot(self, solver: FlowPsi, dq) -> None:
        """features of solver's assembled system and its converged update"""
        d = np.ascontiguousarray(dq, np.float64).reshape(-1)
        N.check(N.lib().fpsi_gnn_add_snapshot(self._h, solver._ctx, N.dptr(d)),
                "fpsi_gnn_add_snapshot")

    @property
    def n_snapshots(self) -> int:
        return int(N.lib().fpsi_gnn_num_snapshots(self._h))

    def snapshot(self, i: int):
        """(features [nc,40], target [nc,5], x_J [nc,5], scales rs|xs [10]) of
        snapshot i, caller cell order"""
        nc = int(N.lib().fpsi_gnn_snapshot_cells(self._h, i))
        if nc < 0:
            raise IndexError(i)
        f, t, xj = (np.empty((nc, 40), np.float32), np.empty((nc, 5), np.float32),
                    np.empty((nc, 5), np.float32))
        sc = np.empty(10, np.float32)
        N.check(N.lib().fpsi_gnn_get_snapshot(self._h, i, f.ctypes.data_as(_fp),
                                              t.ctypes.data_as(_fp), xj.ctypes.data_as(_fp),
                                              sc.ctypes.data_as(_fp)), "fpsi_gnn_get_snapshot")
        return f, t, xj, sc

    def loss_grad(self, i: int, batch: int | None = None, seed: int = 0):
        """mean squared error on snapshot i over about `batch` cells (all by
        default) and its gradient"""
        g = np.empty(self.n_params, np.float32)
        loss = C.c_double()
        nb = batch if batch is not None else (1 << 62)
        N.check(N.lib().fpsi_gnn_loss_grad(self._h, i, nb, seed, C.byref(loss),
                                           g.ctypes.data_as(_fp)), "fpsi_gnn_loss_grad")
        return loss.value, g

    def train(self, nsteps: int, batch: int = 65536, seed: int = 0, lr: float = 1e-3):
        out = np.empty(max(nsteps, 1))
        N.check(N.lib().fpsi_gnn_train(self._h, nsteps, batch, seed, lr, N.dptr(out)),
                "fpsi_gnn_train")
        return out[:nsteps]

    def predict(self, solver: FlowPsi, want: bool = False):
        """set solver's next starting iterate to the learned one"""
        x0 = np.empty(solver.ncells * 5) if want else None
        N.check(N.lib().fpsi_gnn_predict(self._h, solver._ctx, N.dptr(x0)), "fpsi_gnn_predict")
        return None if x0 is None else x0.reshape(-1, 5)


def converged_update(solver: FlowPsi, rtol: float = 1e-10, max_sweeps: int = 400) -> np.ndarray:
    """dq of solver's assembled system, swept from the current iterate until
    ||B - A dq|| <= rtol ||B||"""
    solver.sweeps_to_tolerance(rtol, max_sweeps)
    return solver.get_iterate()


def make_snapshots(model: LearnedStart, case, steps: int, rtol: float = 1e-10,
                   every: int = 1) -> list[float]:
    """run `steps` implicit steps of `case` (a FlowPsi case with the SGS
    solver and the diagonal blocks kept) and add (system, converged dq)
    pairs; returns the residual history"""
    s = FlowPsi(case.mesh, case.params)
    s.keep_blocks(True)
    T, p, u = case.initial_state(s.geometry()["cellcenter"])
    s.set_state(T, p, u)
    hist = []
    for k in range(steps):
        _, r = s.residual(want_src=False)
        hist.append(r["rtrms"])
        s.assemble()
        if k % every == 0:
            model.add_snapshot(s, converged_update(s, rtol))
            s.assemble()  # back to the reference's start for the solver's own step
        s.sweeps(case.params.gauss_seidel_iter)
        s.update()
    s.close()
    return hist


def train_on_case(make_case, seeds, steps_per_seed: int, train_steps: int,
                  batch: int = 65536, rtol: float = 1e-8, lr: float = 1e-3,
                  model_seed: int = 0) -> tuple[LearnedStart, dict]:
    """A model trained on (system, converged dq) snapshots of the first
    steps_per_seed implicit steps of make_case(seed) for every seed (FP64
    systems, dq swept to rtol), then train_steps Adam steps.  Returns the
    model and a summary (snapshots, final loss, seconds)."""
    import time

    m = LearnedStart(seed=model_seed)
    t0 = time.perf_counter()
    for sd in seeds:
        make_snapshots(m, make_case(sd), steps_per_seed, rtol=rtol)
    t1 = time.perf_counter()
    losses = m.train(train_steps, batch=batch, seed=model_seed, lr=lr)
    t2 = time.perf_counter()
    return m, {"snapshots": m.n_snapshots, "train_steps": train_steps, "batch": batch,
               "loss_first": float(losses[0]) if len(losses) else None,
               "loss_last": float(np.mean(losses[-50:])) if len(losses) else None,
               "snapshot_s": t1 - t0, "train_s": t2 - t1}


def sweeps_to_tolerance(solver: FlowPsi, start: str, rtol: float = 1e-3,
                        model: LearnedStart | None = None, max_sweeps: int = 200) -> int:
    """symmetric sweeps the assembled system needs from a given start
    ('zero', 'jacobi' -- the reference's D^-1 B -- or 'learned')"""
    if start == "zero":
        solver.set_iterate(np.zeros((solver.ncells, 5)))
    elif start == "jacobi":
        solver.assemble()  # the assembly leaves D^-1 B as the iterate
    elif start == "learned":
        model.predict(solver)
    else:
        raise ValueError(start)
    return solver.sweeps_to_tolerance(rtol, max_sweeps)


def _time_inference(argv=None) -> dict:
    """Wall time of the learned start's inference (features, the three
    tensor-core layers with the head, the start written into the solver's
    iterate) on an assembled Taylor-Green tet system of n^3 x 6 cells, and
    of training steps on one snapshot of it."""
    import argparse
    import json
    import time

    from . import cases

    ap = argparse.ArgumentParser(prog="python -m flowpsi_b200.learned")
    ap.add_argument("--n", type=int, default=64, help="hexes per direction (x6 tets)")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--train-steps", type=int, default=0)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "ref", "mixed"])
    a = ap.parse_args(argv)
    case = cases.taylor_green_tets(a.n, precision=a.precision)
    s = FlowPsi(case.mesh, case.params)
    s.keep_blocks(True)
    s.set_state(*case.initial_state(s.geometry()["cellcenter"]))
    s.residual(want_src=False)
    s.assemble()
    m = LearnedStart(seed=1)
    m.predict(s)  # first pass allocates the activations
    ts = []
    for _ in range(a.reps):
        t0 = time.perf_counter()
        m.predict(s)
        ts.append(time.perf_counter() - t0)
    out = {"cells": s.ncells, "predict_ms_min": 1e3 * min(ts), "predict_ms_median": 1e3 * float(np.median(ts)),
           "precision": a.precision}
    if a.train_steps > 0:
        s.sweeps(4)
        m.add_snapshot(s, s.get_iterate())
        m.train(1, batch=s.ncells)
        t0 = time.perf_counter()
        m.train(a.train_steps, batch=s.ncells)
        out["train_step_ms"] = 1e3 * (time.perf_counter() - t0) / a.train_steps
    m.close()
    s.close()
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    _time_inference()
