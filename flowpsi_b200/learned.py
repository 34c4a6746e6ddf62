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

    def save(self, path) -> None:
        """the parameters (BF16 values held as FP32, in the library's
        packing order) to an .npy file"""
        np.save(path, self.get_params())

    @classmethod
    def load(cls, path) -> "LearnedStart":
        """a model whose parameters are those saved by save(); the training
        set is not saved"""
        w = np.load(path)
        m = cls()
        if w.dtype != np.float32 or w.ndim != 1 or w.size != m.n_params:
            m.close()
            raise ValueError(f"{path}: expected {m.n_params} float32 parameters, got "
                             f"{w.size} {w.dtype}")
        m.set_params(w)
        return m

    def add_snapshot(self, solver: FlowPsi, dq) -> None:
        """features of solver's assembled system and its converged update"""
        d = np.ascontiguousarray(dq, np.float64).reshape(-1)
        N.check(N.lib().fpsi_gnn_add_snapshot(self._h, solver._ctx, N.dptr(d)),
                "fpsi_gnn_add_snapshot")

    def add_snapshot_region(self, solver: FlowPsi, dq, lo, hi, halo: int = 3) -> None:
        """a snapshot of the cells whose centroids lie in the box [lo, hi);
        the loss counts only cells more than `halo` hops inside it"""
        d = np.ascontiguousarray(dq, np.float64).reshape(-1)
        lo = np.ascontiguousarray(lo, np.float64)
        hi = np.ascontiguousarray(hi, np.float64)
        N.check(N.lib().fpsi_gnn_add_snapshot_region(self._h, solver._ctx, N.dptr(d), N.dptr(lo),
                                                     N.dptr(hi), halo),
                "fpsi_gnn_add_snapshot_region")

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


def _solve_to(solver: FlowPsi, rtol: float, max_sweeps: int, every: int = 10) -> int:
    """symmetric sweeps from the current iterate, checked every `every`
    sweeps, until ||B - A x|| <= rtol ||B||; returns the sweeps made"""
    done = 0
    while done < max_sweeps:
        nb, nr = solver.linear_residual()
        if nr <= rtol * nb:
            break
        k = min(every, max_sweeps - done)
        solver.sweeps(k)
        done += k
    return done


def tgv_state(cellcenter: np.ndarray, seed: int):
    """Taylor-Green state at M = 0.1 x amplitude, amplitude 0.5 + U(0,1)
    from the seed, with 1% seeded noise in every variable: the family of
    states the learned start is trained and evaluated on"""
    from . import cases

    amp = 0.5 + float(cases.uniform(seed, 17, 1)[0])
    T, p, u = cases.taylor_green_tets(2, amplitude=amp).initial_state(cellcenter)
    nc = cellcenter.shape[0]
    T = T * (1.0 + 0.01 * cases.normal(seed, 20, nc))
    p = p * (1.0 + 0.01 * cases.normal(seed, 21, nc))
    u = u + 0.01 * np.abs(u).max() * np.stack([cases.normal(seed, 22 + k, nc) for k in range(3)], 1)
    return T, p, u


def config4(n: int = 128, train_seeds=range(40), eval_seeds=range(40, 50), snaps_per_seed: int = 10,
            train_steps: int = 20000, batch: int = 65536, box_hex: int = 32, rtol: float = 1e-6,
            max_sweeps: int = 300, lin_tol: float = 1e-3, eval_steps: int = 6,
            precision: str = "ref", log=print) -> dict:
    """The learned start at the training scale of the specification: the
    n^3 x 6 jittered split-tet grid, Taylor-Green states from train_seeds
    (tgv_state), snaps_per_seed Newton systems each from the first steps,
    dq swept to rtol, kept as region snapshots of box_hex^3 hexes (random
    corners) so that 400 of them fit in memory; train_steps Adam steps
    (lr 1e-3) on batches of `batch` cells; then, on the states of
    eval_seeds, the sweeps to lin_tol and their wall time from the zero,
    Jacobi and learned starts on the same systems (the run takes the
    reference's steps).  Returns a summary."""
    import time

    from . import cases

    case = cases.taylor_green_tets(n, seed=0, precision=precision)
    s = FlowPsi(case.mesh, case.params)
    s.keep_blocks(True)
    cc = s.geometry()["cellcenter"]
    L = 2.0 * np.pi
    hb = box_hex * L / n
    m = LearnedStart(seed=0)
    t0 = time.perf_counter()
    for sd in train_seeds:
        s.set_state(*tgv_state(cc, sd))
        for k in range(snaps_per_seed):
            s.residual(want_src=False)
            s.assemble()
            _solve_to(s, rtol, max_sweeps)
            dq = s.get_iterate()
            lo = cases.uniform(sd, 100 + k, 3) * (L - hb)
            m.add_snapshot_region(s, dq, lo, lo + hb, 3)
            s.assemble()
            s.sweeps(case.params.gauss_seidel_iter)
            s.update()
        log(f"seed {sd}: {m.n_snapshots} snapshots, {time.perf_counter() - t0:.0f} s")
    t1 = time.perf_counter()
    losses = m.train(train_steps, batch=batch, seed=0, lr=1e-3)
    t2 = time.perf_counter()
    log(f"trained: loss {losses[:20].mean():.4g} -> {losses[-200:].mean():.4g} in {t2 - t1:.0f} s")
    res = {k: {"sweeps": 0, "ms": 0.0} for k in ("zero", "jacobi", "learned")}
    r0 = {"jacobi": [], "learned": []}
    for sd in eval_seeds:
        s.set_state(*tgv_state(cc, sd))
        for k in range(eval_steps):
            s.residual(want_src=False)
            s.assemble()
            for start in ("zero", "jacobi", "learned"):
                ta = time.perf_counter()
                if start == "zero":
                    s.set_iterate(np.zeros((s.ncells, 5)))
                elif start == "jacobi":
                    s.assemble()
                else:
                    m.predict(s)
                if start != "zero":
                    nb, nr = s.linear_residual()
                    r0[start].append(nr / nb)
                sw = _solve_to(s, lin_tol, max_sweeps, every=1)
                res[start]["ms"] += 1e3 * (time.perf_counter() - ta)
                res[start]["sweeps"] += sw
            s.assemble()
            s.sweeps(case.params.gauss_seidel_iter)
            s.update()
    out = {"cells": s.ncells, "snapshots": m.n_snapshots, "box_hex": box_hex,
           "snapshot_s": t1 - t0, "train_s": t2 - t1, "train_steps": train_steps, "batch": batch,
           "loss_first": float(losses[:20].mean()), "loss_last": float(losses[-200:].mean()),
           "eval": res, "initial_residual": {k: float(np.mean(v)) for k, v in r0.items()},
           "lin_tol": lin_tol, "eval_seeds": [int(x) for x in eval_seeds], "eval_steps": eval_steps}
    m.close()
    s.close()
    return out


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
    import sys

    if "--config4" in sys.argv:
        import json

        args = [a for a in sys.argv[1:] if a != "--config4"]
        kw = {}
        for a in args:  # key=value overrides, e.g. n=64 train_steps=2000
            k, v = a.split("=")
            kw[k] = range(*map(int, v.split(":"))) if ":" in v else (float(v) if "." in v or "e" in v else int(v))
        print(json.dumps(config4(**kw)), flush=True)
    else:
        _time_inference()
