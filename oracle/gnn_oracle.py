"""CPU oracle of the learned-start network (torch CPU autograd).

TEST INFRASTRUCTURE: restates the network of flowpsi_b200/csrc/gnn.cu in
torch on the CPU, with the same BF16-rounded weights, the same BF16
rounding of the layer inputs (features, neighbour means and hidden
activations; gradients pass straight through the rounding) and FP32
arithmetic, to check the device's loss and gradients.
"""
from __future__ import annotations

import numpy as np
import torch

NIN, W, NOUT, NLAYER = 40, 64, 5, 3


def unpack(w: np.ndarray):
    """flat FP32 masters -> list of tensors (rounded to BF16 as the device
    uses them)"""
    t = torch.from_numpy(np.ascontiguousarray(w, np.float32)).to(torch.bfloat16).to(torch.float32)
    t = t.clone().requires_grad_(True)
    parts, o = [], 0
    for l in range(NLAYER):
        fin = NIN if l == 0 else W
        parts.append((o, o + W * fin, (W, fin)))
        o += W * fin
        parts.append((o, o + W * fin, (W, fin)))
        o += W * fin
        parts.append((o, o + W, (W,)))
        o += W
    parts.append((o, o + NOUT * W, (NOUT, W)))
    o += NOUT * W
    parts.append((o, o + NOUT, (NOUT,)))
    o += NOUT
    assert o == t.numel()
    return t, [t[a:b].view(*shape) for a, b, shape in parts]


class NeighbourMean:
    """mean of the face neighbours' rows as the device forms it: the rows
    summed in FP32, then multiplied by the FP32 reciprocal of the degree
    (k_layer_tc / k_layer_ws: sum * (1.0f / deg)); for degrees that are not
    powers of two this differs in the last bits from summing rows / deg"""

    def __init__(self, nc: int, cl: np.ndarray, cr: np.ndarray):
        inner = cr >= 0
        a, b = cl[inner].astype(np.int64), cr[inner].astype(np.int64)
        rows = np.concatenate([a, b])
        cols = np.concatenate([b, a])
        deg = np.bincount(rows, minlength=nc).astype(np.float32)
        with np.errstate(divide="ignore"):
            inv = np.where(deg > 0, np.float32(1.0) / deg, np.float32(0.0)).astype(np.float32)
        self.S = torch.sparse_coo_tensor(np.vstack([rows, cols]), np.ones(len(rows), np.float32),
                                         (nc, nc)).coalesce()
        self.inv = torch.from_numpy(inv)

    def __call__(self, h: torch.Tensor) -> torch.Tensor:
        return torch.sparse.mm(self.S, h) * self.inv[:, None]


def neighbour_mean_matrix(nc: int, cl: np.ndarray, cr: np.ndarray) -> NeighbourMean:
    return NeighbourMean(nc, cl, cr)


def bf16(x: torch.Tensor) -> torch.Tensor:
    """round to BF16 in the forward pass, identity in the backward pass"""
    return x + (x.to(torch.bfloat16).to(torch.float32) - x).detach()


def gelu_tanh(z: torch.Tensor) -> torch.Tensor:
    """GELU in its tanh form (Hendrycks and Gimpel 2016),
    0.5 z (1 + tanh(u)) with u = sqrt(2/pi) (z + 0.044715 z^3), evaluated as
    the device does, z sigmoid(2u): the same function without the
    cancellation of 1 + tanh(u) for negative z"""
    u = 0.7978845608028654 * (z + 0.044715 * z * z * z)
    return z * torch.sigmoid(2.0 * u)


def loss_and_grad(w: np.ndarray, feat: np.ndarray, target: np.ndarray, A: torch.Tensor,
                  mask: np.ndarray | None = None):
    """mean squared error over all cells, or over the cells where mask is
    true, and its gradient"""
    flat, p = unpack(w)
    h = torch.from_numpy(np.ascontiguousarray(feat, np.float32))
    for l in range(NLAYER):
        ws, wn, b = p[3 * l], p[3 * l + 1], p[3 * l + 2]
        hb = bf16(h)  # the layer input as the network sees it (FP32 features rounded)
        agg = bf16(A(hb))  # mean of the neighbours' inputs, rounded
        h = bf16(gelu_tanh(hb @ ws.T + agg @ wn.T + b))
    y = h @ p[-2].T + p[-1]
    t = torch.from_numpy(np.ascontiguousarray(target, np.float32))
    if mask is None:
        loss = ((y - t) ** 2).mean()
    else:
        mk = torch.from_numpy(np.asarray(mask, bool))
        loss = ((y - t)[mk] ** 2).mean()
    loss.backward()
    return float(loss), flat.grad.numpy().copy(), y.detach().numpy()


def groups():
    """(name, start, end) of each parameter block in the flat layout"""
    out, o = [], 0
    for l in range(NLAYER):
        fin = NIN if l == 0 else W
        for nm, n in (("ws", W * fin), ("wn", W * fin), ("b", W)):
            out.append((f"{nm}{l}", o, o + n))
            o += n
    out.append(("wo", o, o + NOUT * W))
    o += NOUT * W
    out.append(("bo", o, o + NOUT))
    return out
