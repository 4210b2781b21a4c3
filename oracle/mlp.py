"""CPU restatement of the learned cache-admission network -- TEST
INFRASTRUCTURE ONLY (the checker for dycgraph_b200/csrc/policy.cu; the product
never imports it).

The network is POLICY_F -> 64 -> 64 -> 1 with ReLU, parameters laid out as
W1[F x H] b1[H] W2[H x H] b2[H] W3[H] b3 (FP32 master copy). The GPU kernels
round inputs and parameters to bfloat16 (round to nearest even) and
accumulate in FP32; the tensor-core inference also carries the first layer's
activations as two bfloat16 parts (hi + lo, ~2^-17 relative). This
restatement applies the same input and parameter rounding and computes in
float64 with exact activations, so the two agree to within that activation
split and FP32 accumulation error (the tests' tolerance: 1e-4 relative +
1e-5 absolute for inference). It has no counterpart in
the reference, whose admission is a decayed activity count
(include/framework/variants/driver.cuh:486-515).
"""
import numpy as np

F, H = 8, 64
OFF_W1 = 0
OFF_B1 = F * H
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
PARAMS = OFF_B3 + 1


def bf16_round(a):
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return (u & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(F, H), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def _prep(x, p, rounding):
    x = np.asarray(x, dtype=np.float32).reshape(-1, F)
    p = np.asarray(p, dtype=np.float32)
    if rounding:
        x = bf16_round(x)
        p = bf16_round(p)
    return x.astype(np.float64), p.astype(np.float64)


def forward(x, p, rounding=True):
    """Predictions for the rows of x."""
    x, p = _prep(x, p, rounding)
    W1, b1, W2, b2, W3, b3 = unpack(p)
    h1 = np.maximum(x @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    return h2 @ W3 + b3


def loss_grad(x, y, p, rounding=True):
    """(sum of squared errors, its gradient w.r.t. the parameters used)."""
    x, pp = _prep(x, p, rounding)
    return loss_grad64(x, y, pp)


def finite_difference(x, y, p, idx, eps=1e-6):
    """Central differences of the loss (no rounding) at parameter indices idx."""
    p = np.asarray(p, dtype=np.float64)
    out = []
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp = _loss64(x, y, q)
        q[i] -= 2 * eps
        lm = _loss64(x, y, q)
        out.append((lp - lm) / (2 * eps))
    return np.asarray(out)


def _loss64(x, y, p):
    x = np.asarray(x, dtype=np.float64).reshape(-1, F)
    W1, b1, W2, b2, W3, b3 = unpack(p)
    h2 = np.maximum(np.maximum(x @ W1 + b1, 0.0) @ W2 + b2, 0.0)
    d = h2 @ W3 + b3 - np.asarray(y, dtype=np.float64)
    return float(np.sum(d * d))


def loss_grad64(x, y, p):
    """Gradient in float64 without any rounding (for the finite-difference check)."""
    x = np.asarray(x, dtype=np.float64).reshape(-1, F)
    y = np.asarray(y, dtype=np.float64)
    p = np.asarray(p, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(p)
    a1 = x @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    d = h2 @ W3 + b3 - y
    dy = 2.0 * d
    g = np.zeros(PARAMS)
    g[OFF_W3:OFF_B3] = h2.T @ dy
    g[OFF_B3] = dy.sum()
    dh2 = np.outer(dy, W3) * (a2 > 0)
    g[OFF_W2:OFF_B2] = (h1.T @ dh2).ravel()
    g[OFF_B2:OFF_W3] = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (a1 > 0)
    g[OFF_W1:OFF_B1] = (x.T @ dh1).ravel()
    g[OFF_B1:OFF_W2] = dh1.sum(0)
    return float(np.sum(d * d)), g


def glorot_params(seed=0):
    """Random parameters for tests: Glorot-uniform weights, small biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    for off, fi, fo in ((OFF_W1, F, H), (OFF_W2, H, H), (OFF_W3, H, 1)):
        a = np.sqrt(6.0 / (fi + fo))
        p[off:off + fi * fo] = rng.uniform(-a, a, fi * fo)
    p[OFF_B1:OFF_W2] = rng.uniform(0, 0.1, H)
    p[OFF_B2:OFF_W3] = rng.uniform(0, 0.1, H)
    p[OFF_B3] = 0.05
    return p
