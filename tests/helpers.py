"""Shared test utilities: seeded face states, flux scales, comparisons."""
from __future__ import annotations

import numpy as np

RT = 8314.4621 / 28.96
GAMMA = 1.4


def face_states(n: int, seed: int, jump: float = 0.3, speed: float = 200.0):
    """Seeded random face data: qL, qR packed [pg, T, u, v, w], unit normals,
    areas.  Pressures and temperatures are log-normal (always positive)."""
    rng = np.random.default_rng(seed)

    def st():
        q = np.empty((n, 5))
        q[:, 0] = 1e5 * np.exp(jump * rng.standard_normal(n))
        q[:, 1] = 300.0 * np.exp(0.7 * jump * rng.standard_normal(n))
        q[:, 2:] = speed * rng.standard_normal((n, 3))
        return q

    qL, qR = st(), st()
    an = rng.standard_normal((n, 3))
    an /= np.linalg.norm(an, axis=1)[:, None]
    area = rng.uniform(0.1, 2.0, n)
    return qL, qR, an, area


def flux_scale(qL, qR, an, area, pamb=0.0):
    """Per face and component, the magnitude of the terms a face flux is
    built from: area * sum over both states of |mass flux| * |conserved
    variable| + |pressure terms|, with |u.n| + a as the transport speed.
    Flux errors are measured relative to this scale, which does not vanish
    when the flux itself cancels."""
    out = np.zeros((qL.shape[0], 5))
    for q in (qL, qR):
        pg, T, u = q[:, 0], q[:, 1], q[:, 2:5]
        rho = (pg + pamb) / (RT * T)
        a = np.sqrt(GAMMA * RT * T)
        s = np.abs(np.einsum("ij,ij->i", u, an)) + a
        e0 = RT * T / (GAMMA - 1) + 0.5 * np.einsum("ij,ij->i", u, u)
        m = rho * s
        out[:, 0] += m
        out[:, 1:4] += (m * np.abs(u).max(axis=1))[:, None] + np.abs(pg)[:, None]
        out[:, 4] += m * e0 + np.abs(pg + pamb) * s
    return out * area[:, None]


def rel_to_scale(a, b, scale):
    return float(np.max(np.abs(a - b) / scale))


def src_scale(flux_abs_sum):
    return flux_abs_sum


def block_rel(a, b):
    """max |a-b| relative to the largest entry of each block"""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).reshape(b.shape[0], -1).max(axis=1)
    s = np.where(s > 0, s, 1.0)
    d = np.abs(a - b).reshape(a.shape[0], -1).max(axis=1)
    return float(np.max(d / s))
