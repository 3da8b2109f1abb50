"""ORACLE / TEST INFRASTRUCTURE ONLY: the CPU reference of the scheduler MLP.

float64 forward and backward of the same network the GPU kernels implement
(hacs_b200/csrc/sched.cu): 5 inputs -> 3 hidden layers of 64 ReLU units -> 4
outputs, loss = mean over samples and outputs of (y - t)^2; parameters packed
W1[5][64] b1 W2[64][64] b2 W3[64][64] b3 W4[64][4] b4.  Also the BF16 forward
(round-to-nearest-even to bfloat16 of inputs, weights and each hidden layer's
activations, fp32-class accumulation).  The gradient is pinned by central finite
differences in tests/test_sched_cpu.py.
"""
import numpy as np

N_IN, N_H, N_OUT = 5, 64, 4
SHAPES = [(N_IN, N_H), (N_H,), (N_H, N_H), (N_H,), (N_H, N_H), (N_H,), (N_H, N_OUT), (N_OUT,)]
N_PARAMS = sum(int(np.prod(s)) for s in SHAPES)


def unpack(w):
    out, off = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(w[off:off + n], dtype=np.float64).reshape(s))
        off += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(p, dtype=np.float64).reshape(-1) for p in parts])


def forward(w, X):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(X @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    h3 = np.maximum(h2 @ W3 + b3, 0.0)
    return h3 @ W4 + b4, (X, h1, h2, h3)


def loss_grad(w, X, Y):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(w)
    Yp, (X, h1, h2, h3) = forward(w, X)
    n = X.shape[0]
    e = Yp - np.asarray(Y, dtype=np.float64)
    loss = float((e * e).sum() / (n * N_OUT))
    dy = 2.0 * e / (n * N_OUT)
    gW4, gb4 = h3.T @ dy, dy.sum(0)
    d3 = (dy @ W4.T) * (h3 > 0)
    gW3, gb3 = h2.T @ d3, d3.sum(0)
    d2 = (d3 @ W3.T) * (h2 > 0)
    gW2, gb2 = h1.T @ d2, d2.sum(0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    gW1, gb1 = X.T @ d1, d1.sum(0)
    return loss, pack([gW1, gb1, gW2, gb2, gW3, gb3, gW4, gb4])


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    x = np.asarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def forward_bf16(w, X):
    W1, b1, W2, b2, W3, b3, W4, b4 = [bf16(p.astype(np.float32)).astype(np.float64) for p in unpack(w)]
    x = bf16(np.asarray(X, dtype=np.float32)).astype(np.float64)
    h1 = bf16(np.maximum(x @ W1 + b1, 0.0).astype(np.float32)).astype(np.float64)
    h2 = bf16(np.maximum(h1 @ W2 + b2, 0.0).astype(np.float32)).astype(np.float64)
    h3 = bf16(np.maximum(h2 @ W3 + b3, 0.0).astype(np.float32)).astype(np.float64)
    return h3 @ W4 + b4
