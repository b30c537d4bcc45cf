"""The FP64 encoder oracle on the CPU: its analytic gradients against central
finite differences of its own loss, and its BF16 rounding helper."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import encoder_oracle as EO


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 3.140625, 1e-3])
    r = EO.bf16(x)
    assert r[0] == 1.0 and r[3] == -2.5 and r[4] == 0.0 and r[5] == 3.140625
    assert r[1] == 1.0  # a tie rounds to the even mantissa
    assert r[2] == 1.0 + 2 ** -7
    assert abs(r[6] - 1e-3) <= 1e-3 * 2 ** -8


@pytest.mark.parametrize("name", EO.NAMES)
def test_gradients_match_finite_differences(name):
    rng = np.random.default_rng(7)
    V, K = 40, 128
    t = EO.random_tensors(rng, V, K)
    doc_ptr, words = EO.random_batch(rng, V, 6, 9)
    docs = np.arange(6)
    target = EO.random_target(rng, 6, K)
    ora = EO.EncoderOracle(t)
    g = ora.run(doc_ptr, words, docs, target, rounding=False)["grads"][name]
    idx = [tuple(rng.integers(0, s) for s in t[name].shape) for _ in range(6)]
    if name == "E":  # rows of words that occur in the batch
        idx = [(int(words[i]), int(rng.integers(0, 256))) for i in rng.integers(0, len(words), 6)]
    h = 1e-5
    for ix in idx:
        plus = {k: v.copy() for k, v in t.items()}
        minus = {k: v.copy() for k, v in t.items()}
        plus[name][ix] += h
        minus[name][ix] -= h
        fd = (EO.EncoderOracle(plus).loss(doc_ptr, words, docs, target) -
              EO.EncoderOracle(minus).loss(doc_ptr, words, docs, target)) / (2 * h)
        assert abs(fd - g[ix]) <= 1e-6 + 1e-4 * abs(g[ix]), (name, ix, fd, g[ix])
