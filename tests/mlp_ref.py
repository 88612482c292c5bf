"""float64 numpy restatement of libbsz's cost-model MLP (test helper only).

Parameter layout (bsz_mlp_params): for each layer l, W_l as a row-major
[fan_in, fan_out] matrix, then b_l.  Hidden layers use ReLU, the output
layer is linear; the loss is mean((p - y)^2)."""

from __future__ import annotations

import numpy as np


def dims_of(in_dim: int, hidden: int, layers: int) -> list[int]:
    return [in_dim] + [hidden] * layers + [1]


def unpack(params: np.ndarray, dims: list[int]):
    ws, bs, off = [], [], 0
    for a, b in zip(dims[:-1], dims[1:]):
        ws.append(params[off:off + a * b].reshape(a, b).astype(np.float64))
        off += a * b
        bs.append(params[off:off + b].astype(np.float64))
        off += b
    assert off == params.size
    return ws, bs


def forward(params, dims, x):
    ws, bs = unpack(params, dims)
    acts = [np.asarray(x, np.float64)]
    for l, (w, b) in enumerate(zip(ws, bs)):
        z = acts[-1] @ w + b
        acts.append(np.maximum(z, 0) if l + 1 < len(ws) else z)
    return acts


def loss_and_grad(params, dims, x, y):
    ws, bs = unpack(params, dims)
    acts = forward(params, dims, x)
    p = acts[-1][:, 0]
    n = x.shape[0]
    loss = float(np.mean((p - y) ** 2))
    delta = (2.0 * (p - y) / n)[:, None]
    gw, gb = [None] * len(ws), [None] * len(ws)
    for l in range(len(ws) - 1, -1, -1):
        gw[l] = acts[l].T @ delta
        gb[l] = delta.sum(0)
        if l > 0:
            delta = (delta @ ws[l].T) * (acts[l] > 0)
    flat = np.concatenate([np.concatenate([w.ravel(), b]) for w, b in zip(gw, gb)])
    return loss, flat


def adam_step(params, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    c1 = 1 - b1 ** step
    c2 = 1 - b2 ** step
    return params - lr * ((m / c1) / (np.sqrt(v / c2) + eps) + wd * params), m, v
