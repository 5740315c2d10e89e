"""CPU reference of the learned-preconditioner network (test infrastructure
only: it checks the library's BF16 training kernels, csrc/mlp.cu).

Float64 arithmetic with BF16 rounding (round to nearest even) at exactly the
points where the GPU kernels round: the input, the weights, each hidden
activation after ReLU, the output gradient and each hidden-layer gradient
before it enters a GEMM.  Parameter layout as the library's: W1 (112 x 256),
b1, W2 (256 x 256), b2, W3 (256 x 144), b3, each W row-major (in x out).
"""
import numpy as np

N_IN, N_H, N_OUT = 112, 256, 144


def bf16(x):
    """Round float32 values to BF16 (nearest, ties to even); returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    shapes = [(N_IN, N_H), (N_H,), (N_H, N_H), (N_H,), (N_H, N_OUT), (N_OUT,)]
    out, o = [], 0
    for s in shapes:
        n = int(np.prod(s))
        out.append(p[o:o + n].reshape(s))
        o += n
    return out


def forward_backward(params, X, T):
    """(sum of squared errors, gradient of the mean squared error) in the
    library's parameter layout."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    W1b, W2b, W3b = bf16(W1), bf16(W2), bf16(W3)
    Xb = bf16(X)
    pre1 = Xb @ W1b + b1
    A1 = bf16(np.maximum(pre1, 0.0))
    pre2 = A1 @ W2b + b2
    A2 = bf16(np.maximum(pre2, 0.0))
    out = A2 @ W3b + b3
    e = out - T
    R = X.shape[0]
    g = 2.0 * e / (R * N_OUT)
    gb = bf16(g)
    dW3 = A2.T @ gb
    db3 = g.sum(0)
    dH2 = (gb @ W3b.T) * (pre2 > 0)
    dH2b = bf16(dH2)
    dW2 = A1.T @ dH2b
    db2 = dH2.sum(0)
    dH1 = (dH2b @ W2b.T) * (pre1 > 0)
    dH1b = bf16(dH1)
    dW1 = Xb.T @ dH1b
    db1 = dH1.sum(0)
    grads = np.concatenate([a.ravel() for a in (dW1, db1, dW2, db2, dW3, db3)])
    return float((e * e).sum()), grads
