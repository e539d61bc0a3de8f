"""The CPU reference of the surrogate's algebra (oracle/surrogate_ref.py) pinned without a GPU: with the BF16 rounding
taken out, its backward pass equals central differences of its own loss, layer by layer; and its BF16 rounding is
round-to-nearest-even on the top 16 bits."""

import numpy as np
import pytest

from oracle import surrogate_ref as ref


def test_bf16_rounds_to_nearest_even():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 2**-8 + 2**-20, 1.0 + 3 * 2**-8, -2.5, 0.0], np.float32)
    got = ref.bf16(x)
    assert list(got) == [1.0, 1.0, 1.0 + 2**-7, 1.0 + 2**-6, -2.5, 0.0]


@pytest.mark.parametrize("delta", [0.0, 0.7])
def test_backward_equals_central_differences(monkeypatch, delta):
    monkeypatch.setattr(ref, "bf16", lambda a: np.asarray(a, dtype=np.float64))
    monkeypatch.setattr(ref, "FLOAT", np.float64)
    rng = np.random.default_rng(0)
    shapes = [(16, 8), (16, 16), (6, 16)]  # two hidden layers, 2 heads of 3 outputs
    heads, nt, M = 2, 3, 5
    p = rng.standard_normal(sum(r * c + r for r, c in shapes)) * 0.5
    feat = rng.standard_normal((M, 8))
    tgt = rng.standard_normal((M, nt))
    wts = rng.poisson(1.0, (M, heads)).astype(np.float64) + 0.5

    def loss_of(q):
        pred, _, _ = ref.forward(feat, [(w.astype(np.float64), b) for w, b in ref.unpack(q, shapes)])
        return ref.loss_grad(pred.astype(np.float64), tgt, wts, heads, nt, delta)[1]

    layers = ref.unpack(p, shapes)
    pred, a, z = ref.forward(feat, layers)
    dpred, _ = ref.loss_grad(pred.astype(np.float64), tgt, wts, heads, nt, delta)
    grads = ref.backward(dpred, layers, a, z)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    eps = 1e-6
    for k in rng.choice(p.size, 60, replace=False):
        d = np.zeros_like(p)
        d[k] = eps
        fd = (loss_of(p + d) - loss_of(p - d)) / (2 * eps)
        assert abs(fd - flat[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (k, fd, flat[k])
