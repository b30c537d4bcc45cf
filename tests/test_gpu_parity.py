"""CUDA path against the oracle, through the C ABI.

Integer state (phi, n_k, theta CSR, initial topics) must be bit-exact.  Topic
draws on a frozen snapshot must equal the FP64 oracle's for every token whose
uniform lies at least 1e-6 (relative to S+Q) from a bucket boundary; the
per-token log-likelihood must agree to 1e-6 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200.configs import MINI, TINY
from culda_cgs_b200.corpus import GenConfig
from oracle import oracle as O

BOUNDARY_TOL = 1e-6   # relative distance of u*(S+Q) to a bucket boundary
LL_RTOL = 1e-6

pytestmark = pytest.mark.gpu


def snapshot_of(m: cb.LDA, c: cb.Corpus, z=None) -> O.Snapshot:
    z = m.topics() if z is None else z
    return O.Snapshot.build(c.word_ptr, c.doc_ids, c.doc_ptr, z, m.k, m.alpha, m.beta)


def assert_counts_exact(m: cb.LDA, c: cb.Corpus) -> O.Snapshot:
    s = snapshot_of(m, c)
    phi, nk = m.phi()
    a, ja, max_ia, cur = m.theta()
    assert np.array_equal(nk, s.nk)
    assert np.array_equal(phi, s.phi)
    assert np.array_equal(max_ia, s.max_ia)
    assert np.array_equal(cur, s.cur_ia)
    assert np.array_equal(a, s.theta_a)
    assert np.array_equal(ja, s.theta_ja)
    assert s.valid(phi=phi, nk=nk, theta_a=a, theta_ja=ja, cur_ia=cur) == (0, 0)
    return s


def assert_ll_close(got, want):
    """Per-token log-likelihoods agree to 1e-6 relative (absolute below |LL| = 1)."""
    assert abs(got - want) <= LL_RTOL * max(1.0, abs(want)), (got, want)


def assert_draws_match(z_gpu, z_ora, margin, check_rate=True):
    far = margin >= BOUNDARY_TOL
    bad = (z_gpu != z_ora) & far
    assert not bad.any(), (f"{int(bad.sum())} tokens differ beyond the boundary tolerance; "
                           f"first at {np.flatnonzero(bad)[:5]} margins {margin[bad][:5]}")
    if check_rate:  # near-boundary tokens are rare
        assert (z_gpu != z_ora).mean() < 1e-3


CASES = [  # name, corpus, K, lanes per token, item tokens (0 = auto), sampler register budget (0 = auto)
    ("tiny-k64-g8", TINY.gen, 64, 8, 0, 0),
    ("tiny-k64-g1-hot", TINY.gen, 64, 1, 64, 0),
    ("tiny-k32-g2", TINY.gen, 32, 2, 0, 0),
    ("mini-k1024-g4", MINI.gen, 1024, 4, 0, 0),
    ("mini-k1024-g8-hot", MINI.gen, 1024, 8, 300, 0),
    ("mini-k1024-g16", MINI.gen, 1024, 16, 0, 0),
    ("mini-k1024-g32", MINI.gen, 1024, 32, 0, 0),
    ("mini-k256-g1", MINI.gen, 256, 1, 0, 0),
    ("mini-k4096-g8", MINI.gen, 4096, 8, 0, 0),
    ("mini-k1024-g8-b10", MINI.gen, 1024, 8, 0, 10),
    ("mini-k1024-g4-b10-hot", MINI.gen, 1024, 4, 300, 10),
    ("mini-k1024-g16-b10", MINI.gen, 1024, 16, 0, 10),
    ("tiny-k64-g8-b10", TINY.gen, 64, 8, 0, 10),
    ("tiny-k64-flat", TINY.gen, 64, -1, 0, 0),
    ("tiny-k32-flat-hot", TINY.gen, 32, -1, 40, 0),
    ("mini-k1024-flat", MINI.gen, 1024, -1, 0, 0),
    ("mini-k1024-flat-hot", MINI.gen, 1024, -1, 300, 0),
    ("mini-k256-flat", MINI.gen, 256, -1, 0, 0),
    ("mini-k4096-flat", MINI.gen, 4096, -1, 0, 0),
    ("mini-k1024-flat-b8-hot", MINI.gen, 1024, -1, 300, 8),
]


@pytest.fixture(scope="module")
def corpora():
    return {id(g): cb.Corpus.generate(g) for g in (TINY.gen, MINI.gen)}


@pytest.mark.parametrize("name,gen,k,g,item_tokens,blocks", CASES, ids=[c[0] for c in CASES])
def test_counts_exact_and_snapshot_draws(corpora, name, gen, k, g, item_tokens, blocks):
    c = corpora[id(gen)]
    seed = 1234
    with cb.LDA(c, k, 50.0 / 1024, 0.01, seed=seed, group_lanes=g, item_tokens=item_tokens,
                sample_blocks=blocks) as m:
        assert m.info()["sample_blocks"] == (blocks or (9 if g == -1 else 8))
        z0 = m.topics()
        assert np.array_equal(z0, O.init_topics(c.num_tokens, k, seed))
        s0 = assert_counts_exact(m, c)
        # the first iteration samples snapshot 0 with Philox iteration 1
        z1_ora, margin, ll0 = s0.sample(seed, 1)
        st = m.iterate(1)[0]
        assert st["iteration"] == 1 and st["status"] == 0
        assert_ll_close(st["loglik"], ll0)
        z1 = m.topics()
        assert_draws_match(z1, z1_ora, margin)
        s1 = assert_counts_exact(m, c)
        assert st["theta_nnz"] == int((s1.theta_a != 0).sum())
        L = np.diff(c.doc_ptr)
        assert st["row_entries"] == int((L * (s1.cur_ia - s1.max_ia[:-1])).sum())
        # a few more iterations, then a frozen-snapshot draw
        m.iterate(3)
        s = assert_counts_exact(m, c)
        z_gpu, ll_gpu = m.sample_snapshot(77)
        z_ora, margin, ll_ora = s.sample(seed, 77)
        assert_draws_match(z_gpu, z_ora, margin)
        assert_ll_close(ll_gpu, ll_ora)
        # the snapshot draw left the state untouched
        assert np.array_equal(m.topics(), s.z)


def test_input_token_order_matches_the_oracle(corpora):
    """CULDA_FLAG_NO_REORDER keeps tokens in input order (no token index):
    the counts and draws still match the oracle."""
    c = corpora[id(MINI.gen)]
    seed = 4321
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=seed, flags=cb.CULDA_FLAG_NO_REORDER) as m:
        s0 = assert_counts_exact(m, c)
        z1_ora, margin, ll0 = s0.sample(seed, 1)
        st = m.iterate(1)[0]
        assert st["status"] == 0
        assert_ll_close(st["loglik"], ll0)
        assert_draws_match(m.topics(), z1_ora, margin)
        assert_counts_exact(m, c)


@pytest.mark.parametrize("g,blocks", [(1, 8), (4, 8), (8, 8), (32, 8), (8, 10), (-1, 8)])
def test_long_chain_keeps_device_state_consistent(g, blocks):
    """~10M draws per sampler variant: tokens whose target lands within a rounding
    of a bucket boundary must still get a topic (the sampler's error word stays 0)."""
    from culda_cgs_b200.configs import SMALL

    c = cb.Corpus.generate(SMALL.gen)
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=21 + g, group_lanes=g, sample_blocks=blocks) as m:
        stats = m.iterate(10)
        assert all(s["status"] == 0 for s in stats)
        assert stats[-1]["loglik"] > stats[0]["loglik"]
        assert_counts_exact(m, c)


def test_deterministic_replay(corpora):
    c = corpora[id(MINI.gen)]
    runs = []
    for _ in range(2):
        with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=99) as m:
            lls = [s["loglik"] for s in m.iterate(4)]
            runs.append((m.topics(), lls))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]


def test_loglik_joint_matches_oracle(corpora):
    c = corpora[id(MINI.gen)]
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=5) as m:
        m.iterate(2)
        s = snapshot_of(m, c)
        assert m.loglik_joint() == pytest.approx(s.loglik_joint(), rel=1e-10)


def test_loglik_improves(corpora):
    c = corpora[id(MINI.gen)]
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=5) as m:
        j0 = m.loglik_joint()
        lls = [s["loglik"] for s in m.iterate(15)]
        assert m.loglik_joint() > j0
        assert lls[-1] > lls[0]


# ---------------------------------------------------------------- edge cases
def _corpus(doc_of_token_by_word):
    """Corpus from a list (per word) of doc-id lists."""
    ids = np.concatenate([np.asarray(x, dtype=np.int32) for x in doc_of_token_by_word])
    wp = np.concatenate([[0], np.cumsum([len(x) for x in doc_of_token_by_word])])
    D = int(ids.max()) + 1
    dp = np.concatenate([[0], np.cumsum(np.bincount(ids, minlength=D))])
    return cb.Corpus.from_arrays(dp, wp, ids)


EDGE = {
    "single-token": [[0]],
    "one-doc": [[0] * 7, [0] * 3, [0]],
    "one-token-docs": [[0, 1, 2, 3], [4, 5], [6]],
    "empty-words": [[0, 1], [], [1, 2], [], []],
    "doc-longer-than-k": [[0] * 300, [0] * 200, [0, 1] * 20, [1]],
    "hot-word": [list(range(50)) * 40, [3, 7]],
}


@pytest.mark.parametrize("name", list(EDGE))
@pytest.mark.parametrize("g", [1, 8, -1])
def test_edge_corpora(name, g):
    c = _corpus(EDGE[name])
    k = 32
    with cb.LDA(c, k, 0.1, 0.01, seed=3, group_lanes=g, item_tokens=64) as m:
        s0 = assert_counts_exact(m, c)
        z1_ora, margin, ll0 = s0.sample(3, 1)
        st = m.iterate(1)[0]
        assert_ll_close(st["loglik"], ll0)
        assert_draws_match(m.topics(), z1_ora, margin, check_rate=False)
        assert_counts_exact(m, c)


def test_set_topics_all_same_topic():
    c = cb.Corpus.generate(TINY.gen)
    with cb.LDA(c, 64, 0.1, 0.01, seed=3) as m:
        m.set_topics(np.full(c.num_tokens, 5, dtype=np.uint16))
        s = assert_counts_exact(m, c)
        assert (s.nk[5] == c.num_tokens) and (s.cur_ia - s.max_ia[:-1] == 32).all()
        m.iterate(2)
        assert_counts_exact(m, c)


def test_set_topics_rejects_out_of_range():
    c = cb.Corpus.generate(TINY.gen)
    with cb.LDA(c, 64, 0.1, 0.01, seed=3) as m:
        z = m.topics()
        z[10] = 64
        with pytest.raises(cb.CuldaError):
            m.set_topics(z)


def test_longest_allowed_document():
    """A doc of 65535 tokens (the 16-bit count limit) split over two words."""
    n = 65535
    doc_ids = np.r_[np.zeros(n, dtype=np.int32), np.ones(3, dtype=np.int32)]
    c = cb.Corpus.from_arrays(np.array([0, n, n + 3]), np.array([0, n // 2, n + 3]), doc_ids)
    with cb.LDA(c, 64, 0.1, 0.01, seed=2) as m:
        m.iterate(1)
        assert_counts_exact(m, c)


@pytest.mark.parametrize("min_len", [1, 40, 300, -1])
@pytest.mark.parametrize("k", [64, 1024])
def test_theta_rebuild_bins_match_the_oracle(corpora, min_len, k):
    """Docs of at least min_len tokens rebuilt by a whole CTA each (1: every
    doc; -1: none): theta, n_k and the draws still match the oracle."""
    c = corpora[id(MINI.gen)]
    seed = 808
    with cb.LDA(c, k, 50.0 / k, 0.01, seed=seed, theta_min_len=min_len) as m:
        info = m.info()
        L = np.diff(c.doc_ptr)
        assert info["theta_min_len"] == max(min_len, 0)
        assert info["theta_long_docs"] == (int((L >= min_len).sum()) if min_len > 0 else 0)
        s0 = assert_counts_exact(m, c)
        z1_ora, margin, ll0 = s0.sample(seed, 1)
        st = m.iterate(1)[0]
        assert st["status"] == 0
        assert_ll_close(st["loglik"], ll0)
        assert_draws_match(m.topics(), z1_ora, margin)
        s1 = assert_counts_exact(m, c)
        assert st["theta_nnz"] == int((s1.theta_a != 0).sum())
        assert st["row_entries"] == int((L * (s1.cur_ia - s1.max_ia[:-1])).sum())
        m.iterate(2)
        assert_counts_exact(m, c)


def test_theta_rebuild_block_bin_on_the_longest_document():
    """The 65535-token document (the 16-bit count limit) rebuilt by a CTA."""
    n = 65535
    doc_ids = np.r_[np.zeros(n, dtype=np.int32), np.ones(3, dtype=np.int32)]
    c = cb.Corpus.from_arrays(np.array([0, n, n + 3]), np.array([0, n // 2, n + 3]), doc_ids)
    with cb.LDA(c, 64, 0.1, 0.01, seed=2, theta_min_len=1000) as m:
        assert m.info()["theta_long_docs"] == 1
        m.iterate(1)
        assert_counts_exact(m, c)
