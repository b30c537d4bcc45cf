"""Metropolis-Hastings iterations and the learned proposal on the GPU.

MH draws on a frozen snapshot must equal the FP64 oracle (oracle_mh_fp64) for
every token whose decisions all lie at least 1e-6 (relative) from their
boundaries, with the doc proposal alone and mixed with the encoder's
proposal table; MH iterations keep the integer state exact; training on the
sampler's states lowers the encoder's cross-entropy, and the trained proposal
is accepted more often than the untrained one."""
from __future__ import annotations

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200.configs import MINI, SMALL, TINY
from test_gpu_parity import assert_counts_exact, snapshot_of

pytestmark = pytest.mark.gpu

BOUNDARY_TOL = 1e-6


def assert_mh_matches(z_gpu, z_ora, margin):
    far = margin >= BOUNDARY_TOL
    bad = (z_gpu != z_ora) & far
    assert not bad.any(), f"{int(bad.sum())} tokens differ beyond the tolerance, first {np.flatnonzero(bad)[:5]}"
    assert (z_gpu != z_ora).mean() < 1e-3


@pytest.mark.parametrize("gen,k", [(TINY.gen, 64), (MINI.gen, 1024)], ids=["tiny-k64", "mini-k1024"])
def test_mh_doc_proposal_matches_oracle(gen, k):
    c = cb.Corpus.generate(gen)
    seed = 17
    with cb.LDA(c, k, 50.0 / 1024, 0.01, seed=seed) as m:
        m.iterate(3)
        s = snapshot_of(m, c)
        z_gpu = m.mh_snapshot(11, steps=4)
        z_ora, margin = s.mh(seed, 11, 4)
        assert_mh_matches(z_gpu, z_ora, margin)
        assert np.array_equal(m.topics(), s.z)  # the state is untouched


def test_mh_encoder_proposal_matches_oracle():
    c = cb.Corpus.generate(MINI.gen)
    seed = 23
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=seed) as m, cb.Encoder(c.num_words, 1024, 1024, seed=3) as enc:
        m.iterate(2)
        m.set_proposal(enc, mix=0.05)
        cdf = m.proposal()
        assert np.all(np.diff(cdf, axis=1) >= 0)
        assert np.allclose(cdf[:, -1], 1.0, atol=1e-4)
        s = snapshot_of(m, c)
        z_gpu = m.mh_snapshot(7, steps=6)
        z_ora, margin = s.mh(seed, 7, 6, cdf=cdf)
        assert_mh_matches(z_gpu, z_ora, margin)


def test_iterate_mh_keeps_counts_exact():
    c = cb.Corpus.generate(MINI.gen)
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=5) as m:
        m.iterate(2)
        _, ll0 = m.sample_snapshot(1000)
        st = m.iterate_mh(6, steps=2)
        assert all(x["status"] == 0 for x in st)
        assert all(0.0 < x["accept_rate"] <= 1.0 for x in st)
        assert [x["iteration"] for x in st] == list(range(3, 9))
        assert_counts_exact(m, c)
        _, ll1 = m.sample_snapshot(1000)
        assert ll1 > ll0
        # plain iterations continue the numbering after MH ones
        assert m.iterate(1)[0]["iteration"] == 9
        assert_counts_exact(m, c)


def test_trained_proposal_is_accepted_more_often():
    """From the same state (plain iterations 1-20, states 11-20 accumulated)
    and with the same MH budget, the proposal of the encoder after training is
    accepted more often than before training, and its cross-entropy fell."""
    c = cb.Corpus.generate(SMALL.gen)
    accept = {}
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=41) as m, cb.Encoder(c.num_words, 1024, 512, seed=1) as enc:
        m.iterate(10)
        for _ in range(10):
            m.iterate(1)
            m.accumulate_theta()
        z_start = m.topics()
        for mode in ("untrained", "trained"):
            if mode == "trained":
                m.init_encoder(enc, seed=3)
                losses = [m.train_encoder(enc, 1, seed=e) for e in range(20)]
                assert losses[-1] < losses[0] - 0.2, losses
            m.set_topics(z_start)
            m.set_proposal(enc, mix=0.05)
            st = m.iterate_mh(2, steps=2)
            accept[mode] = float(np.mean([x["accept_rate"] for x in st]))
            assert_counts_exact(m, c)
    assert accept["trained"] > accept["untrained"], accept
