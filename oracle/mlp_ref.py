"""CPU reference of the learned split proposer's MLP (forward and backward).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA training kernels
(marigold_b200/csrc/mgbvh_mlp.cu). float64 arithmetic on the BF16-rounded
weights the kernels use; the kernels accumulate in FP32, so gradients agree
to FP32 rounding.

Network: 24 -> 64 -> 64 -> 49, exact GELU, parameters in one flat vector
W1[64x24] b1[64] W2[64x64] b2[64] W3[49x64] b3[49] (8,945 values). Outputs
0..47 are position logits (axis * 16 + bucket), output 48 the refine logit.
Loss per sample: softmax cross-entropy over the 48 position logits (when the
label is valid) + binary cross-entropy of the refine logit against the gain
flag; the batch loss is the mean over samples.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

IN, H, OUT, NPOS = 24, 64, 49, 48
OFF = {"W1": 0, "b1": 1536, "W2": 1600, "b2": 5696, "W3": 5760, "b3": 8896}
NPARAM = 8945
NO_LABEL = 0xFFFFFFFF


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[0:1536].reshape(H, IN), p[1536:1600], p[1600:5696].reshape(H, H), p[5696:5760],
            p[5760:8896].reshape(OUT, H), p[8896:8945])


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(p_bf16, x):
    W1, b1, W2, b2, W3, b3 = unpack(p_bf16)
    x = np.asarray(x, np.float64)
    z1 = x @ W1.T + b1
    a1 = gelu(z1)
    z2 = a1 @ W2.T + b2
    a2 = gelu(z2)
    return a2 @ W3.T + b3, (x, z1, a1, z2, a2)


def loss_and_grad(p_bf16, x, label, gain):
    """Mean loss over the batch and its gradient w.r.t. the parameters."""
    W1, b1, W2, b2, W3, b3 = unpack(p_bf16)
    out, (x, z1, a1, z2, a2) = forward(p_bf16, x)
    B = x.shape[0]
    label = np.asarray(label, np.uint64)
    gain = np.asarray(gain, np.float64)
    d3 = np.zeros_like(out)
    valid = label < NPOS  # NO_LABEL and anything out of range: no position loss
    pos = out[:, :NPOS]
    m = pos.max(axis=1, keepdims=True)
    e = np.exp(pos - m)
    prob = e / e.sum(axis=1, keepdims=True)
    lab = np.where(valid, label, 0).astype(np.int64)
    ce = -np.log(prob[np.arange(B), lab])
    d3[:, :NPOS] = prob
    d3[np.arange(B), lab] -= 1.0
    d3[~valid, :NPOS] = 0.0
    l48 = out[:, NPOS]
    sig = 1.0 / (1.0 + np.exp(-l48))
    bce = np.logaddexp(0.0, l48) - gain * l48
    d3[:, NPOS] = sig - gain
    loss = (np.where(valid, ce, 0.0).sum() + bce.sum()) / B
    d3 /= B
    g = np.zeros(NPARAM)
    g[OFF["W3"]:OFF["W3"] + OUT * H] = (d3.T @ a2).ravel()
    g[OFF["b3"]:OFF["b3"] + OUT] = d3.sum(axis=0)
    d2 = (d3 @ W3) * gelu_grad(z2)
    g[OFF["W2"]:OFF["W2"] + H * H] = (d2.T @ a1).ravel()
    g[OFF["b2"]:OFF["b2"] + H] = d2.sum(axis=0)
    d1 = (d2 @ W2) * gelu_grad(z1)
    g[OFF["W1"]:OFF["W1"] + H * IN] = (d1.T @ x).ravel()
    g[OFF["b1"]:OFF["b1"] + H] = d1.sum(axis=0)
    return loss, g
