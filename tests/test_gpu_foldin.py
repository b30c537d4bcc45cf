"""Fold-in of held-out documents against a frozen model, and the encoder's
warm start, on the GPU against the FP64 oracle; and what the trained encoder
gains over random initial topics and over the untrained encoder (held-out
log-likelihood per sweep)."""
from __future__ import annotations

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200.configs import MINI, SMALL
from test_gpu_parity import assert_draws_match, assert_ll_close, snapshot_of

pytestmark = pytest.mark.gpu

K, ALPHA, BETA = 1024, 50.0 / 1024, 0.01


@pytest.fixture(scope="module")
def split():
    c = cb.Corpus.generate(MINI.gen)
    perm = np.random.default_rng(0).permutation(c.num_docs)
    cut = c.num_docs * 3 // 4
    return c.split_docs(np.sort(perm[:cut])), c.split_docs(np.sort(perm[cut:]))


def test_frozen_phi_sampling_matches_oracle(split):
    train, held = split
    with cb.LDA(train, K, ALPHA, BETA, seed=3) as m:
        m.iterate(4)
        phi, nk = m.phi()
    seed = 9
    with cb.LDA(held, K, ALPHA, BETA, seed=seed) as f:
        f.set_frozen_phi(phi, nk)
        for it in (1, 2):
            s = snapshot_of(f, held)
            z_ora, margin, ll = s.sample(seed, it, phi=phi, nk=nk)
            st = f.iterate(1)[0]
            assert st["status"] == 0
            assert_ll_close(st["loglik"], ll)
            assert_draws_match(f.topics(), z_ora, margin)
        _, own_nk = f.phi(dense=False)
        assert own_nk.sum() == held.num_tokens  # its own counts are still rebuilt


def test_set_frozen_phi_rejects_inconsistent_counts(split):
    _, held = split
    with cb.LDA(held, K, ALPHA, BETA, seed=1) as f:
        phi = np.zeros((held.num_words, K), dtype=np.int32)
        phi[0, 0] = 5
        nk = np.zeros(K, dtype=np.int32)
        with pytest.raises(cb.CuldaError):
            f.set_frozen_phi(phi, nk)
        nk[0] = 5
        f.set_frozen_phi(phi, nk)
        f.set_frozen_phi(None, None)
        assert f.iterate(1)[0]["status"] == 0


def test_warm_start_matches_oracle(split):
    train, held = split
    with cb.LDA(train, K, ALPHA, BETA, seed=3) as m:
        m.iterate(3)
        phi, nk = m.phi()
    seed = 12
    with cb.LDA(held, K, ALPHA, BETA, seed=seed) as f, cb.Encoder(held.num_words, K, 1024, seed=2) as enc:
        f.set_frozen_phi(phi, nk)
        f.set_proposal(enc, mix=0.05)
        cdf = f.proposal()
        s = snapshot_of(f, held)
        f.warm_start()
        z_ora, margin = s.warm_start(seed, cdf, phi=phi, nk=nk)
        assert_draws_match(f.topics(), z_ora, margin)
        assert f.iterate(1)[0]["status"] == 0


def test_encoder_warm_start_gains_on_held_out_docs():
    """Train on 3/4 of a corpus (plain CGS, states 21-40 accumulated), train the
    encoder on those states, then fold in the other quarter: the trained
    encoder's warm start beats random initial topics at every one of the first
    sweeps, and beats the same network untrained at the first sweep."""
    c = cb.Corpus.generate(SMALL.gen)
    perm = np.random.default_rng(1).permutation(c.num_docs)
    cut = c.num_docs * 3 // 4
    train, held = c.split_docs(np.sort(perm[:cut])), c.split_docs(np.sort(perm[cut:]))
    curves = {}
    with cb.LDA(train, K, ALPHA, BETA, seed=5) as m:
        m.iterate(20)
        for _ in range(20):
            m.iterate(1)
            m.accumulate_theta()
        phi, nk = m.phi()
        for mode in ("random", "untrained", "trained"):
            with cb.LDA(held, K, ALPHA, BETA, seed=7) as f, cb.Encoder(c.num_words, K, 512, seed=1) as enc:
                f.set_frozen_phi(phi, nk)
                if mode == "trained":
                    m.init_encoder(enc, seed=3)
                    m.train_encoder(enc, 20, seed=1)
                if mode != "random":
                    f.set_proposal(enc, mix=0.05)
                    f.warm_start()
                curves[mode] = [s["loglik"] for s in f.iterate(5)]
    assert curves["trained"][0] > curves["random"][0] + 0.1, curves
    assert all(e > r for e, r in zip(curves["trained"], curves["random"])), curves
    assert curves["trained"][0] > curves["untrained"][0], curves
