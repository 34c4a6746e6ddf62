"""CPU checks of the learned start's CPU replica (oracle/gnn_oracle.py),
which the device forward, backward and inference are compared with in
tests/test_gpu_learned.py."""
import math

import numpy as np
import torch

from oracle import gnn_oracle as G


def test_gelu_is_the_tanh_form_within_its_published_bound():
    """The network's GELU is the tanh approximation of Hendrycks and Gimpel
    (2016), 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), evaluated as
    z sigmoid(2u).  Against the exact z Phi(z) = 0.5 z (1 + erf(z/sqrt 2))
    its largest deviation is 4.73e-4 (at |z| = 2.70).  The sigmoid form is
    the same function (0.5 (1 + tanh u) = sigmoid(2u)) without the
    cancellation of 1 + tanh(u) for negative z: where the tanh form keeps
    its digits the two agree to round-off."""
    z = torch.linspace(-12.0, 12.0, 240001, dtype=torch.float64)
    exact = 0.5 * z * (1.0 + torch.erf(z / math.sqrt(2.0)))
    got = G.gelu_tanh(z)
    assert float((got - exact).abs().max()) < 4.8e-4
    u = math.sqrt(2.0 / math.pi) * (z + 0.044715 * z ** 3)
    tanh_form = 0.5 * z * (1.0 + torch.tanh(u))
    kept = z.abs() < 2.0  # where 1 + tanh(u) keeps its digits in FP64
    assert float(((got - tanh_form).abs() / tanh_form.abs().clamp_min(1e-300))[kept].max()) < 1e-12


def test_neighbour_mean_is_sum_then_reciprocal():
    """the mean of the face neighbours' rows is formed as the device forms
    it: the FP32 sum of the rows times the FP32 reciprocal of the degree"""
    cl = np.array([0, 0, 1, 2, 0], np.int32)
    cr = np.array([1, 2, 2, 3, -1], np.int32)  # the last face is a boundary face
    A = G.neighbour_mean_matrix(4, cl, cr)
    h = torch.tensor(np.random.default_rng(1).standard_normal((4, 3)), dtype=torch.float32)
    got = A(h)
    for c, nbrs in enumerate([[1, 2], [0, 2], [0, 1, 3], [2]]):
        s = torch.zeros(3, dtype=torch.float32)
        for o in sorted(nbrs):
            s = s + h[o]
        want = s * (np.float32(1.0) / np.float32(len(nbrs)))
        assert torch.equal(got[c], want)
