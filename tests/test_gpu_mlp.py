"""The tensor-core MLP kernels against the CPU restatement (oracle/mlp_oracle.py).

Forward outputs match the bfloat16-operand restatement to RTOL_FWD = 1e-2 of
the output scale (FP32 accumulation order and rare bf16 rounding flips of
hidden activations); the full-batch gradient matches it to RTOL_GRAD = 2e-2
in the relative 2-norm, and the exact float64 network (no bf16 rounding) to
RTOL_GRAD_EXACT = 5e-2.  Training reduces the loss of a smooth regression.
"""
import numpy as np
import pytest

from oracle.mlp_oracle import forward_backward

pytestmark = pytest.mark.gpu

RTOL_FWD = 1e-2
RTOL_GRAD = 2e-2
RTOL_GRAD_EXACT = 5e-2


def _data(rows, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(rows, 13)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2], np.tanh(x[:, 3] - x[:, 4]), x[:, 5] ** 2 / 4,
                  np.cos(x[:, 6]) * x[:, 7], 0.3 * x[:, 8:11].sum(1), np.abs(x[:, 11]) - x[:, 12]], 1)
    return x, t.astype(np.float32)


def test_forward_matches_oracle():
    from picopic_b200.mlp import Mlp
    m = Mlp(seed=3)
    x, t = _data(1000, 1)
    y = m.forward(x)
    _, _, yo = forward_backward(m.params, x, t)
    assert np.abs(y - yo).max() <= RTOL_FWD * np.abs(yo).max()


def test_gradient_matches_oracle():
    from picopic_b200.mlp import Mlp
    m = Mlp(seed=4)
    x, t = _data(777, 2)  # not a multiple of the 64-row block
    g, loss = m.gradient(x, t)
    lo, go, _ = forward_backward(m.params, x, t)
    le, ge, _ = forward_backward(m.params, x, t, round_bf16=False)
    assert abs(loss - lo) <= 1e-3 * lo
    assert np.linalg.norm(g - go) <= RTOL_GRAD * np.linalg.norm(go)
    assert np.linalg.norm(g - ge) <= RTOL_GRAD_EXACT * np.linalg.norm(ge)


def test_training_reduces_loss():
    from picopic_b200.mlp import Mlp
    m = Mlp(seed=5)
    x, t = _data(20000, 3)
    _, l0 = m.gradient(x, t)
    m.set_data(x, t)
    m.train(600, batch=1024, lr=2e-3)
    _, l1 = m.gradient(x, t)
    assert l1 < 0.3 * l0


@pytest.mark.parametrize("rows", [1000, 20000])
def test_forward_on_tcgen05_matches(rows):
    """The tcgen05 forward pass (pcg_mlp_forward_tc: UMMA from shared-memory
    descriptors, FP32 accumulators in tensor memory) against the mma.sync one
    on the same BF16 operands: within RTOL_TC = 5e-3 of the output scale
    (FP32 sum order, and the rare hidden activation whose BF16 rounding it
    flips), and against the restatement within RTOL_FWD; a partial last tile
    and several tiles per CTA."""
    from picopic_b200.mlp import Mlp
    m = Mlp(seed=5)
    x, t = _data(rows, 7)
    y = m.forward(x)
    y_tc, ms = m.forward_tc(x)
    assert ms > 0
    scale = np.abs(y).max()
    assert np.abs(y_tc - y).max() <= 5e-3 * scale
    assert np.median(np.abs(y_tc - y)) <= 1e-5 * scale
    _, _, yo = forward_backward(m.params, x, t)
    assert np.abs(y_tc - yo).max() <= RTOL_FWD * np.abs(yo).max()
