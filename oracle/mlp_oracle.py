"""CPU restatement of the collision MLP's forward and backward passes.

TEST INFRASTRUCTURE ONLY: the checker of picopic_b200's tensor-core MLP
kernels (pcg_mlp.cu).  It computes the same network (13 -> 128 -> 128 -> 6,
ReLU, loss mean((y - t)^2)) in float64, optionally rounding every GEMM
operand to bfloat16 (round to nearest even) as the kernels do, so that the
kernels' gradients can be compared with an exact restatement.
"""
import numpy as np

from picopic_b200.mlp import unpack


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_backward(params: np.ndarray, x: np.ndarray, t: np.ndarray, round_bf16: bool = True):
    """Loss, gradient (flat, float64) and outputs of the network."""
    q = bf16 if round_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    p = unpack(np.asarray(params, dtype=np.float32))
    w1, w2, w3 = q(p["w1"]), q(p["w2"]), q(p["w3"])
    b1, b2, b3 = (np.asarray(p[k], dtype=np.float64) for k in ("b1", "b2", "b3"))
    X = q(x)
    z1 = X @ w1 + b1
    h1 = np.maximum(z1, 0.0)
    H1 = q(h1.astype(np.float32))
    z2 = H1 @ w2 + b2
    h2 = np.maximum(z2, 0.0)
    H2 = q(h2.astype(np.float32))
    y = H2 @ w3 + b3
    n = x.shape[0] * y.shape[1]
    e = y - t
    loss = float(np.sum(e * e) / n)
    dy = q((2.0 * e / n).astype(np.float32))
    dh2 = q(((dy @ w3.T) * (H2 > 0)).astype(np.float32))
    dh1 = q(((dh2 @ w2.T) * (H1 > 0)).astype(np.float32))
    grads = {"w3": H2.T @ dy, "b3": dy.sum(0), "w2": H1.T @ dh2, "b2": dh2.sum(0),
             "w1": X.T @ dh1, "b1": dh1.sum(0)}
    flat = np.concatenate([grads[k].ravel() for k in ("w1", "b1", "w2", "b2", "w3", "b3")])
    return loss, flat, y
