"""CPU oracle of the variant selector's cost model (test infrastructure only).

float64 restatement of the perceptron the library trains and runs on the GPU
(kernel_mlp.cu, select_device.cuh): 16 features -> 64 ReLU -> 64 ReLU -> 3
outputs (predicted log-microseconds of LOP3, M4R, TC), and of its loss
L = sum(m * (f(x) - y)^2) / (2 sum(m)) with analytic gradients, in the
library's weight layout (W1[16][64], b1, W2[64][64], b2, W3[64][3], b3).
Also the selector's heuristic rule, for computing its choices offline.
"""
from __future__ import annotations

import numpy as np

F, H, O = 16, 64, 3
N_WEIGHTS = F * H + H + H * H + H + H * O + O


def unpack(w: np.ndarray):
    w = np.asarray(w, dtype=np.float64)
    i = 0
    out = []
    for shape in ((F, H), (H,), (H, H), (H,), (H, O), (O,)):
        k = int(np.prod(shape))
        out.append(w[i:i + k].reshape(shape))
        i += k
    return out


def pack(parts) -> np.ndarray:
    return np.concatenate([np.asarray(p, dtype=np.float64).ravel() for p in parts])


def forward(w: np.ndarray, x: np.ndarray) -> np.ndarray:
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1 = np.maximum(np.asarray(x, np.float64) @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    return h2 @ W3 + b3


def loss_grad(w: np.ndarray, x: np.ndarray, y: np.ndarray, m: np.ndarray):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x, y, m = (np.asarray(a, np.float64) for a in (x, y, m))
    a1 = x @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    out = h2 @ W3 + b3
    msum = m.sum()
    e = out - y
    loss = 0.5 * float((m * e * e).sum()) / msum
    dout = m * e / msum
    gW3, gb3 = h2.T @ dout, dout.sum(0)
    d2 = (dout @ W3.T) * (a2 > 0)
    gW2, gb2 = h1.T @ d2, d2.sum(0)
    d1 = (d2 @ W2.T) * (a1 > 0)
    gW1, gb1 = x.T @ d1, d1.sum(0)
    return loss, pack([gW1, gb1, gW2, gb2, gW3, gb3])


def heuristic_choice(cfg: dict, f: np.ndarray, T: int, tc_ok: bool) -> int:
    """The selector's threshold rule (variants 2 LOP3, 3 M4R, 4 TC)."""
    allowed = cfg["allowed"]
    if (tc_ok and allowed & (1 << 4) and T >= cfg["tc_min_tiles"] and f[2] >= cfg["tc_min_occ"]
            and f[6] >= cfg["tc_min_dense"]):
        return 4
    if allowed & (1 << 3) and f[6] >= cfg["m4r_min_dense"]:
        return 3
    if allowed & (1 << 2):
        return 2
    return 3 if allowed & (1 << 3) else 2
