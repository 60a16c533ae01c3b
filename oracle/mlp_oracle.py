"""CPU oracle for the warm-start network (TEST INFRASTRUCTURE ONLY).

The forward and backward passes of the 3-layer ReLU MLP in numpy FP64, with
the device's rounding points made explicit: the GEMM operands (inputs,
weights, hidden activations, output gradients) are BF16, every product is
accumulated exactly enough in FP64 to stand for the device's FP32
accumulation. loss = (1/B) sum_b sum_j w_j (out_bj - t_bj)^2.
"""
import numpy as np


def bf16(a):
    """Round float32/float64 values to bfloat16 (round to nearest even), as float64."""
    x = np.asarray(a, dtype=np.float32).copy()
    u = x.view(np.uint32)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.view(np.float32).astype(np.float64)


def forward(X, W1, b1, W2, b2, W3, b3):
    """X BF16-valued; returns (Out, H1, H2) with H1, H2 rounded to BF16."""
    Z1 = bf16(X) @ bf16(W1).T + b1
    H1 = bf16(np.maximum(Z1, 0.0))
    Z2 = H1 @ bf16(W2).T + b2
    H2 = bf16(np.maximum(Z2, 0.0))
    Out = H2 @ bf16(W3).T + b3
    return Out, H1, H2


def gradients(X, T, w, W1, b1, W2, b2, W3, b3):
    B = X.shape[0]
    Out, H1, H2 = forward(X, W1, b1, W2, b2, W3, b3)
    E = Out - T
    loss = float((w * E * E).sum() / B)
    dOut = 2.0 * w * E / B
    dOut_h = bf16(dOut)
    gW3 = dOut_h.T @ H2
    gb3 = dOut.sum(axis=0)
    dH2 = dOut_h @ bf16(W3)
    dZ2 = dH2 * (H2 > 0)
    dZ2_h = bf16(dZ2)
    gW2 = dZ2_h.T @ H1
    gb2 = dZ2.sum(axis=0)
    dH1 = dZ2_h @ bf16(W2)
    dZ1 = dH1 * (H1 > 0)
    dZ1_h = bf16(dZ1)
    gW1 = dZ1_h.T @ bf16(X)
    gb1 = dZ1.sum(axis=0)
    return loss, dict(W1=gW1, b1=gb1, W2=gW2, b2=gb2, W3=gW3, b3=gb3)
