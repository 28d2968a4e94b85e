"""CPU reference of the subgrid-closure MLP (TEST INFRASTRUCTURE: the reference the tests hold the
library's tensor-core MLP kernels against; only ``tests/`` may import it).

The closure has no counterpart in the reference (CRUNA has no learned component).  The network maps
12 features (9 velocity-gradient components, density, temperature, filter width; normalised by a
per-feature mean and scale) through 64 -> 64 hidden units with GELU (erf form) to 6 subgrid-stress
components (tau_11, tau_22, tau_33, tau_12, tau_13, tau_23 in normalised units).  Parameters are kept
in FP32, in this order (5382 values): W1[64][12], b1[64], W2[64][64], b2[64], W3[6][64], b3[6].

``forward_bf16`` / ``grad_bf16`` restate the library's arithmetic: features, weights and hidden
activations rounded to BF16 (round to nearest even) as tensor-core operands, products accumulated
in FP32 or better, biases and GELU in FP32.  ``forward_exact`` / ``grad_exact`` are the same network
in FP64 without rounding: the gradient the BF16 kernels approximate.
"""
from __future__ import annotations

import math
from typing import Dict, Tuple

import numpy as np

IN, HID, OUT = 12, 64, 6
SHAPES = (("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (OUT, HID)),
          ("b3", (OUT,)))
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p: np.ndarray) -> Dict[str, np.ndarray]:
    out, o = {}, 0
    for name, shp in SHAPES:
        k = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + k], dtype=np.float64).reshape(shp)
        o += k
    return out


def pack(d: Dict[str, np.ndarray]) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def normalise(X, in_mean, in_scale):
    return (np.asarray(X, np.float64) - np.asarray(in_mean, np.float64)) / np.asarray(in_scale, np.float64)


def forward_bf16(p, X, in_mean, in_scale, out_scale):
    """Physical outputs (n, 6) as the kernel computes them."""
    w = unpack(p)
    x = bf16(normalise(X, in_mean, in_scale).astype(np.float32))
    h1 = bf16(gelu(x @ bf16(w["W1"]).T + w["b1"].astype(np.float32)))
    h2 = bf16(gelu(h1 @ bf16(w["W2"]).T + w["b2"].astype(np.float32)))
    y = h2 @ bf16(w["W3"]).T + w["b3"].astype(np.float32)
    return y * np.asarray(out_scale, np.float64)


def forward_exact(p, X, in_mean, in_scale, out_scale):
    w = unpack(p)
    x = normalise(X, in_mean, in_scale)
    h1 = gelu(x @ w["W1"].T + w["b1"])
    h2 = gelu(h1 @ w["W2"].T + w["b2"])
    return (h2 @ w["W3"].T + w["b3"]) * np.asarray(out_scale, np.float64)


def loss_exact(p, X, Y, in_mean, in_scale, out_scale) -> float:
    """Mean squared error in normalised output units: mean((y_n - Y/out_scale)^2) over n x 6."""
    yn = forward_exact(p, X, in_mean, in_scale, out_scale) / np.asarray(out_scale, np.float64)
    t = np.asarray(Y, np.float64) / np.asarray(out_scale, np.float64)
    return float(np.mean((yn - t) ** 2))


def grad_exact(p, X, Y, in_mean, in_scale, out_scale) -> Tuple[float, np.ndarray]:
    """Loss and its exact gradient with respect to the packed parameters (FP64 backpropagation)."""
    w = unpack(p)
    n = X.shape[0]
    x = normalise(X, in_mean, in_scale)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = gelu(z1)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = gelu(z2)
    y = h2 @ w["W3"].T + w["b3"]
    t = np.asarray(Y, np.float64) / np.asarray(out_scale, np.float64)
    L = float(np.mean((y - t) ** 2))
    dy = 2.0 * (y - t) / (n * OUT)
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ w["W3"]) * gelu_grad(z2)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * gelu_grad(z1)
    g["W1"], g["b1"] = dz1.T @ x, dz1.sum(0)
    return L, pack(g)


def grad_bf16(p, X, Y, in_mean, in_scale, out_scale) -> Tuple[float, np.ndarray]:
    """The kernel's gradient: tensor-core operands (x, h1, h2, W, dy, dz2, dz1) rounded to BF16; the
    bias gradients are sums of the rounded dy, dz2, dz1 (the kernel forms them on the tensor core with
    a row of ones)."""
    w = unpack(p)
    n = X.shape[0]
    x = bf16(normalise(X, in_mean, in_scale).astype(np.float32))
    W1, W2, W3 = bf16(w["W1"]), bf16(w["W2"]), bf16(w["W3"])
    z1 = x @ W1.T + w["b1"]
    h1 = bf16(gelu(z1))
    z2 = h1 @ W2.T + w["b2"]
    h2 = bf16(gelu(z2))
    y = h2 @ W3.T + w["b3"]
    t = np.asarray(Y, np.float64) / np.asarray(out_scale, np.float64)
    L = float(np.mean((y - t) ** 2))
    dy = 2.0 * (y - t) / (n * OUT)
    dyb = bf16(dy)
    g = {"W3": dyb.T @ h2, "b3": dyb.sum(0)}
    dz2 = (dyb @ W3) * gelu_grad(z2)
    dz2b = bf16(dz2)
    g["W2"], g["b2"] = dz2b.T @ h1, dz2b.sum(0)
    dz1 = (dz2b @ W2) * gelu_grad(z1)
    dz1b = bf16(dz1)
    g["W1"], g["b1"] = dz1b.T @ x, dz1b.sum(0)
    return L, pack(g)


def init_params(seed: int) -> np.ndarray:
    """Uniform fan-in initialisation, +-1/sqrt(fan_in), from numpy PCG64(seed) (the library's
    cruna_mlp_create uses its own generator; tests set parameters explicitly)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    d = {}
    for name, shp in SHAPES:
        fan_in = shp[-1] if name.startswith("W") else (IN if name == "b1" else HID)
        d[name] = rng.uniform(-1.0, 1.0, size=shp) / math.sqrt(fan_in)
    return pack(d)
