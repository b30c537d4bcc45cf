"""The oracle itself: counts, CSR layout, sampling rule and likelihoods against
small pure-Python restatements of the reference's algorithm."""
from __future__ import annotations

import math

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200.configs import TINY
from oracle import oracle as O


@pytest.fixture(scope="module")
def tiny():
    c = cb.Corpus.generate(TINY.gen)
    z = O.init_topics(c.num_tokens, TINY.k, 11)
    return c, O.Snapshot.build(c.word_ptr, c.doc_ids, c.doc_ptr, z, TINY.k, TINY.alpha, TINY.beta)


def test_snapshot_is_valid(tiny):
    _, s = tiny
    assert s.valid() == (0, 0)
    assert s.nk.sum() == len(s.z) and (s.phi.sum(axis=1) == np.diff(s.word_ptr)).all()


def test_doc_rev_matches_reference_order(tiny):
    c, s = tiny
    assert np.array_equal(s.doc_tok, c.doc_tokens())
    for d in range(s.num_docs):  # ascending token ids inside a doc, all of the doc's tokens
        seg = s.doc_tok[s.doc_ptr[d]:s.doc_ptr[d + 1]]
        assert (np.diff(seg) > 0).all() and (s.doc_ids[seg] == d).all()


def test_theta_layout_and_rows(tiny):
    _, s = tiny
    L = np.diff(s.doc_ptr)
    cap = np.diff(s.max_ia)
    assert (cap == (np.minimum(L, s.k) + 31) // 32 * 32).all()
    for d in range(s.num_docs):
        b, e, cur = s.max_ia[d], s.max_ia[d + 1], s.cur_ia[d]
        a, ja = s.theta_a[b:e], s.theta_ja[b:e]
        nnz = int((a != 0).sum())
        assert (a[:nnz] > 0).all() and (a[nnz:] == 0).all() and (ja[nnz:] == 0).all()
        assert (np.diff(ja[:nnz]) > 0).all()
        assert cur == b + (nnz + 31) // 32 * 32
        hist = np.bincount(s.z[s.doc_tok[s.doc_ptr[d]:s.doc_ptr[d + 1]]], minlength=s.k)
        assert np.array_equal(hist[ja[:nnz]], a[:nnz])


def test_validators_catch_errors(tiny):
    _, s = tiny
    phi = s.phi.copy()
    phi[0, 0] += 1
    assert s.valid(phi=phi)[0] == 1
    nk = s.nk.copy()
    nk[3] += 1
    assert s.valid(nk=nk)[0] == 2
    a = s.theta_a.copy()
    a[0] += 1
    assert s.valid(theta_a=a)[1] == 3
    cur = s.cur_ia.copy()
    cur[0] += 32
    assert s.valid(cur_ia=cur)[1] == 5


def _py_sample(s: O.Snapshot, seed, iteration):
    """Slow restatement of lda_train_kernel.cu:65-259 in Python floats."""
    alpha, beta = s.alpha, s.beta
    z_out = np.empty_like(s.z)
    logs = 0.0
    for w in range(s.num_words):
        hist = np.bincount(s.z[s.word_ptr[w]:s.word_ptr[w + 1]], minlength=s.k)
        ph = [(hist[j] + beta) / (s.nk[j] + s.num_words * beta) for j in range(s.k)]
        q = sum(alpha * p for p in ph)
        for t in range(s.word_ptr[w], s.word_ptr[w + 1]):
            d = s.doc_ids[t]
            row = [(int(s.theta_a[i]), int(s.theta_ja[i])) for i in range(s.max_ia[d], s.cur_ia[d]) if s.theta_a[i]]
            S = sum(a * ph[j] for a, j in row)
            x = int(O.philox4x32_10((t & 0xFFFFFFFF, t >> 32, iteration, 0), (seed & 0xFFFFFFFF, seed >> 32))[0])
            T = O.uniform(x) * (S + q)
            if T < S:
                cum = 0.0
                for a, j in row:
                    cum += a * ph[j]
                    if cum > T:
                        z_out[t] = j
                        break
            else:
                cum = S
                for j in range(s.k):
                    cum += alpha * ph[j]
                    if cum > T:
                        z_out[t] = j
                        break
                else:
                    z_out[t] = s.k - 1
            L = s.doc_ptr[d + 1] - s.doc_ptr[d]
            logs += math.log((S + q) / (L + s.k * alpha))
    return z_out, logs / len(s.z)


def test_sampling_rule_matches_python_restatement(tiny):
    _, s = tiny
    z_new, margin, ll = s.sample(seed=5, iteration=3)
    z_py, ll_py = _py_sample(s, 5, 3)
    ok = margin > 1e-9
    assert ok.mean() > 0.99
    assert np.array_equal(z_new[ok], z_py[ok])
    assert ll == pytest.approx(ll_py, rel=1e-12)
    assert (margin >= 0).all() and (margin <= 0.5).all()


def test_sampling_is_a_function_of_seed_and_iteration(tiny):
    _, s = tiny
    a = s.sample(1, 1)[0]
    assert np.array_equal(a, s.sample(1, 1)[0])
    assert not np.array_equal(a, s.sample(1, 2)[0])
    assert not np.array_equal(a, s.sample(2, 1)[0])


def test_sampling_distribution_matches_conditional(tiny):
    """Averaged over many iterations the draws follow p(k) ~ (n_dk + alpha) phihat_wk."""
    _, s = tiny
    t = int(s.word_ptr[0])  # a token of the most frequent word
    d = int(s.doc_ids[t])
    hist = np.bincount(s.z[s.word_ptr[0]:s.word_ptr[1]], minlength=s.k)
    ph = (hist + s.beta) / (s.nk + s.num_words * s.beta)
    ndk = np.zeros(s.k)
    for i in range(s.max_ia[d], s.cur_ia[d]):
        if s.theta_a[i]:
            ndk[s.theta_ja[i]] = s.theta_a[i]
    p = (ndk + s.alpha) * ph
    p /= p.sum()
    draws = np.array([s.sample(9, it)[0][t] for it in range(1, 2001)])
    emp = np.bincount(draws, minlength=s.k) / len(draws)
    assert np.abs(emp - p).max() < 0.04


def test_joint_loglik_matches_python(tiny):
    _, s = tiny
    a, b, K, V, D = s.alpha, s.beta, s.k, s.num_words, s.num_docs
    ll = K * (math.lgamma(V * b) - V * math.lgamma(b)) + D * (math.lgamma(K * a) - K * math.lgamma(a))
    for w in range(V):
        ll += sum(math.lgamma(x + b) for x in s.phi[w])
    ll -= sum(math.lgamma(x + V * b) for x in s.nk)
    for d in range(D):
        hist = np.bincount(s.z[s.doc_tok[s.doc_ptr[d]:s.doc_ptr[d + 1]]], minlength=K)
        ll += sum(math.lgamma(x + a) for x in hist) - math.lgamma(s.doc_ptr[d + 1] - s.doc_ptr[d] + K * a)
    assert s.loglik_joint() == pytest.approx(ll, rel=1e-10)


def test_half_conversion():
    cases = {0.0: 0x0000, 1.0: 0x3C00, -2.0: 0xC000, 65504.0: 0x7BFF, 1e9: 0x7C00, 6.0e-8: 0x0001,
             5.960464477539063e-08: 0x0001, 2.9802322387695312e-08: 0x0000, 1.0009765625: 0x3C01,
             1.00048828125: 0x3C00, 1.00146484375: 0x3C02, 6.103515625e-05: 0x0400}
    for x, h in cases.items():
        assert O.float_to_half(x) == h, x
    xs = np.float32(np.random.default_rng(0).lognormal(-8, 4, 20000))
    assert np.array_equal(np.array([O.float_to_half(float(x)) for x in xs], dtype=np.uint16),
                          xs.astype(np.float16).view(np.uint16))


def test_token_selection_sampler_equals_the_full_oracle(tiny):
    """oracle_sample_tokens_fp64 (rows counted on the fly, all host threads)
    gives the draws, margins and log-likelihood of the whole-corpus oracle,
    for every token and for any ascending selection."""
    c, s = tiny
    r = O.RowSnapshot.build(c.word_ptr, c.doc_ids, c.doc_ptr, s.z, s.k, TINY.alpha, TINY.beta)
    assert np.array_equal(r.nk, s.nk) and np.array_equal(r.theta_a, s.theta_a) and np.array_equal(r.cur_ia, s.cur_ia)
    z_all, m_all, ll_all = s.sample(5, 3)
    z, m, ll_tok, (t_log, t_doc) = r.sample_tokens(5, 3)
    assert np.array_equal(z, z_all) and np.array_equal(m, m_all)
    assert (t_log - t_doc) / len(z) == pytest.approx(ll_all, rel=1e-12)
    assert ll_tok.sum() == pytest.approx(t_log - t_doc, rel=1e-12)
    sel = np.sort(np.random.default_rng(0).choice(len(s.z), 700, replace=False))
    z2, m2, ll2, _ = r.sample_tokens(5, 3, sel)
    assert np.array_equal(z2, z_all[sel]) and np.array_equal(m2, m_all[sel]) and np.allclose(ll2, ll_tok[sel])


def test_token_selection_sampler_splits_a_hot_word_into_runs():
    """A word of 70,000 tokens is cut into runs of 32,768 that share one
    counted row: the draws equal the whole-corpus oracle's."""
    rng = np.random.default_rng(3)
    D, K = 40, 64
    hot = np.sort(rng.integers(0, D, 70_000)).astype(np.int32)
    cold = [np.sort(rng.integers(0, D, n)).astype(np.int32) for n in (5, 300, 1)]
    doc_ids = np.concatenate([hot, *cold])
    word_ptr = np.concatenate([[0], np.cumsum([len(hot)] + [len(x) for x in cold])]).astype(np.int64)
    doc_ptr = np.concatenate([[0], np.cumsum(np.bincount(doc_ids, minlength=D))]).astype(np.int64)
    z = O.init_topics(len(doc_ids), K, 9)
    s = O.Snapshot.build(word_ptr, doc_ids, doc_ptr, z, K, 0.1, 0.01)
    r = O.RowSnapshot.build(word_ptr, doc_ids, doc_ptr, z, K, 0.1, 0.01)
    z_all, m_all, ll_all = s.sample(7, 2)
    zr, mr, _, (t_log, t_doc) = r.sample_tokens(7, 2)
    assert np.array_equal(zr, z_all) and np.array_equal(mr, m_all)
    assert (t_log - t_doc) / len(z) == pytest.approx(ll_all, rel=1e-12)
    sel = np.r_[np.arange(0, 70_000, 7), 70_000 + np.arange(306)]
    zs, ms, _, _ = r.sample_tokens(7, 2, sel)
    assert np.array_equal(zs, z_all[sel]) and np.array_equal(ms, m_all[sel])
