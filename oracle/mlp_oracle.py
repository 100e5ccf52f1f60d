"""CPU oracle of the surrogate MLP (test infrastructure only).

Restates the network of netflux_b200/csrc/mlp.cu in numpy: 7 inputs (plus a
constant 1 carrying the first layer's bias) -> 4 x 128 SiLU -> 5 outputs, with
BF16 rounding (round to nearest even) applied where the kernels round: the
inputs, the weights, every stored activation (Z and H), and the gradients dZ
that the backward pass stores; sums are FP32. With ``bf16=False`` the same
network runs in float64 without rounding, which the finite-difference check
uses to pin the backward formulas.

The reference has no learned component; the parameter layout is the
library's (nf_mlp_param_count values, padded shapes).
"""
from typing import Dict, Tuple

import numpy as np

H, KIN, NOUT, NIN, NO = 128, 16, 16, 7, 5
OFF_W0 = 0
OFF_W1 = OFF_W0 + H * KIN
OFF_W2 = OFF_W1 + H * H
OFF_W3 = OFF_W2 + H * H
OFF_B1 = OFF_W3 + H * H
OFF_B2 = OFF_B1 + H
OFF_B3 = OFF_B2 + H
OFF_W4 = OFF_B3 + H
OFF_B4 = OFF_W4 + NOUT * H
N_PARAM = OFF_B4 + NOUT


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray) -> Dict[str, np.ndarray]:
    p = np.asarray(p)
    return {"W0": p[OFF_W0:OFF_W1].reshape(H, KIN), "W1": p[OFF_W1:OFF_W2].reshape(H, H),
            "W2": p[OFF_W2:OFF_W3].reshape(H, H), "W3": p[OFF_W3:OFF_B1].reshape(H, H),
            "b1": p[OFF_B1:OFF_B2], "b2": p[OFF_B2:OFF_B3], "b3": p[OFF_B3:OFF_W4],
            "W4": p[OFF_W4:OFF_B4].reshape(NOUT, H), "b4": p[OFF_B4:N_PARAM]}


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params: np.ndarray, feat: np.ndarray, bf16_round: bool = True) -> Tuple[np.ndarray, dict]:
    """Outputs [n][5] and the saved activations."""
    dt = np.float32 if bf16_round else np.float64
    rnd = bf16 if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    P = {k: np.asarray(v, dtype=dt) for k, v in unpack(params).items()}
    n = feat.shape[0]
    X0 = np.zeros((n, KIN), dt)
    X0[:, :NIN] = feat
    X0[:, NIN] = 1.0
    X0 = rnd(X0)
    Z0 = X0 @ rnd(P["W0"]).T
    Zs, Hs = [rnd(Z0)], [rnd(_silu(Z0))]
    for l in (1, 2, 3):
        Z = Hs[-1] @ rnd(P[f"W{l}"]).T + P[f"b{l}"]
        Zs.append(rnd(Z))
        Hs.append(rnd(_silu(Z)))
    Y = Hs[-1] @ rnd(P["W4"]).T + P["b4"]
    return Y[:, :NO], {"X0": X0, "Z": Zs, "H": Hs, "P": P}


def loss_and_grad(params: np.ndarray, feat: np.ndarray, target: np.ndarray,
                  bf16_round: bool = True) -> Tuple[float, np.ndarray]:
    """Mean squared error over n x 5 outputs and its gradient (padded layout)."""
    rnd = bf16 if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    Y, s = forward(params, feat, bf16_round)
    P, X0, Zs, Hs = s["P"], s["X0"], s["Z"], s["H"]
    n = feat.shape[0]
    e = Y - target
    loss = float(np.mean(np.asarray(e, np.float64) ** 2))
    dY = np.zeros((n, NOUT), Y.dtype)
    dY[:, :NO] = (2.0 / (n * NO)) * e
    dZ = rnd(dY)
    g = np.zeros(N_PARAM, np.float64)
    g[OFF_W4:OFF_B4] = (dZ.T @ Hs[3]).ravel()
    g[OFF_B4:N_PARAM] = dZ.sum(axis=0)
    dH = dZ @ rnd(P["W4"])
    for l in (3, 2, 1):
        dZ = rnd(dH * _dsilu(Zs[l]))
        g[{1: OFF_W1, 2: OFF_W2, 3: OFF_W3}[l]:{1: OFF_W2, 2: OFF_W3, 3: OFF_B1}[l]] = (dZ.T @ Hs[l - 1]).ravel()
        g[{1: OFF_B1, 2: OFF_B2, 3: OFF_B3}[l]:{1: OFF_B2, 2: OFF_B3, 3: OFF_W4}[l]] = dZ.sum(axis=0)
        dH = dZ @ rnd(P[f"W{l}"])
    dZ = rnd(dH * _dsilu(Zs[0]))
    g[OFF_W0:OFF_W1] = (dZ.T @ X0).ravel()
    return loss, g


def init_params(seed: int) -> np.ndarray:
    """Random parameters with the padded entries zero (uniform, 1/sqrt(fan_in))."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAM, np.float32)
    u = lambda shape, fan: rng.uniform(-1, 1, shape) / np.sqrt(fan)
    p[OFF_W0:OFF_W1] = np.pad(u((H, NIN + 1), NIN), ((0, 0), (0, KIN - NIN - 1))).ravel()
    for off in (OFF_W1, OFF_W2, OFF_W3):
        p[off:off + H * H] = u(H * H, H)
    p[OFF_B1:OFF_W4] = u(3 * H, H)
    p[OFF_W4:OFF_B4] = np.pad(u((NO, H), H), ((0, NOUT - NO), (0, 0))).ravel()
    p[OFF_B4:OFF_B4 + NO] = u(NO, H)
    return p
