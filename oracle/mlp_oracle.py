"""TEST INFRASTRUCTURE, NOT PRODUCT CODE: the insertion-proposal network's
forward and backward pass restated in numpy (FP64) as the checker of the
CUDA training kernels (ermod_openacc_b200/csrc/mlp.cu).

The network has no reference counterpart (erdst inserts uniformly).  Weight
matrices are used rounded to BF16 (round to nearest even, as the device's
conversion), biases in FP32; the loss is the mean binary cross-entropy with
logits.  Pinned by a finite-difference check of its own gradient
(tests/test_mlp_oracle.py).
"""
from __future__ import annotations

import numpy as np

NIN, NH = 64, 128


def layout():
    o, n = {}, 0
    for name, size in (("W1", NH * NIN), ("b1", NH), ("W2", NH * NH), ("b2", NH), ("W3", NH * NH), ("b3", NH),
                       ("w4", NH), ("b4", 1)):
        o[name] = (n, size)
        n += size
    o["n"] = n
    return o


def bf16_round(x):
    """FP32 -> BF16 -> FP32 with round-to-nearest-even (NaN/Inf not handled)."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def tf32_round(x):
    """FP32 -> TF32 (10-bit mantissa) -> FP32, round to nearest with ties away from zero, as the
    device's cvt.rna.tf32.f32 stages the hidden layers' inputs for the tensor cores."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x1000) >> 13) << 13
    return r.astype(np.uint32).view(np.float32)


def unpack(p, round_weights=True):
    L = layout()
    get = lambda k: np.asarray(p[L[k][0]:L[k][0] + L[k][1]])
    # the device: BF16 weight matrices, FP32 biases; unrounded: the parameters as given (FP64 checks)
    rw = (lambda a: bf16_round(a).astype(np.float64)) if round_weights else (lambda a: a.astype(np.float64))
    rb = (lambda a: a.astype(np.float32).astype(np.float64)) if round_weights else (lambda a: a.astype(np.float64))
    W1 = rw(get("W1")).reshape(NH, NIN)
    W2 = rw(get("W2")).reshape(NH, NH)
    W3 = rw(get("W3")).reshape(NH, NH)
    w4 = rw(get("w4"))
    return W1, rb(get("b1")), W2, rb(get("b2")), W3, rb(get("b3")), w4, float(rb(get("b4"))[0])


def forward(p, x, round_weights=True, tf32_inputs=False):
    """Logits and the activations (x, h1, h2, h3).  tf32_inputs: each hidden layer's input is
    rounded to TF32 before its product, as the device's tensor-core forward stages it (the
    activations returned, which the backward pass uses, stay unrounded)."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p, round_weights)
    x = np.asarray(x, dtype=np.float64)
    t = (lambda a: tf32_round(a).astype(np.float64)) if tf32_inputs else (lambda a: a)
    h1 = np.maximum(t(x) @ W1.T + b1, 0.0)
    h1 = h1.astype(np.float32).astype(np.float64) if tf32_inputs else h1
    h2 = np.maximum(t(h1) @ W2.T + b2, 0.0)
    h2 = h2.astype(np.float32).astype(np.float64) if tf32_inputs else h2
    h3 = np.maximum(t(h2) @ W3.T + b3, 0.0)
    s = h3 @ w4 + b4
    return s, (x, h1, h2, h3)


def loss_and_grad(p, x, y, round_weights=True, tf32_inputs=False, acts=None):
    """Mean BCE-with-logits loss and its gradient w.r.t. the parameter vector
    (w.r.t. the weights as used, i.e. after BF16 rounding; the TF32 rounding of the
    forward's inputs, when asked, is passed straight through).  acts: given hidden
    activations (h1, h2, h3) to differentiate at instead of this module's own forward
    pass -- the device's, so that a TF32 rounding that falls the other way on one
    side of a rounding boundary does not count as a backward-pass error."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p, round_weights)
    if acts is None:
        s, (x, h1, h2, h3) = forward(p, x, round_weights, tf32_inputs)
    else:
        x = np.asarray(x, dtype=np.float64)
        h1, h2, h3 = (np.asarray(a, dtype=np.float64) for a in acts)
        s = h3 @ w4 + b4
    y = np.asarray(y, dtype=np.float64)
    n = len(s)
    loss = np.mean(np.logaddexp(0.0, s) - y * s)
    gs = (1.0 / (1.0 + np.exp(-s)) - y) / n
    L = layout()
    g = np.zeros(L["n"])
    put = lambda k, v: g.__setitem__(slice(L[k][0], L[k][0] + L[k][1]), np.ravel(v))
    put("w4", gs @ h3)
    put("b4", [gs.sum()])
    d3 = np.outer(gs, w4) * (h3 > 0)
    put("W3", d3.T @ h2)
    put("b3", d3.sum(axis=0))
    d2 = (d3 @ W3) * (h2 > 0)
    put("W2", d2.T @ h1)
    put("b2", d2.sum(axis=0))
    d1 = (d2 @ W2) * (h1 > 0)
    put("W1", d1.T @ x)
    put("b1", d1.sum(axis=0))
    return loss, g
