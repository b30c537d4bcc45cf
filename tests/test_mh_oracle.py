"""The Metropolis-Hastings restatement (oracle_mh_fp64) on the CPU: from any
start, enough steps on one frozen snapshot draw from the plain sampler's
conditional p(k) ~ (n_dk + alpha) phihat_wk, with the doc proposal alone and
mixed with an independent proposal table; and the corpus split used for
fold-in keeps every document's words."""
from __future__ import annotations

import numpy as np
import pytest
from scipy import stats

import culda_cgs_b200 as cb
from culda_cgs_b200.configs import TINY
from culda_cgs_b200.corpus import GenConfig
from oracle import oracle as O


def _snapshot(k=16, seed=4):
    c = cb.Corpus.generate(GenConfig(num_words=60, num_topics=4, num_docs=12, len_law=0, len_a=20.0, len_min=5,
                                     len_max=40, seed=seed))
    z = O.init_topics(c.num_tokens, k, seed)
    return c, O.Snapshot.build(c.word_ptr, c.doc_ids, c.doc_ptr, z, k, 0.5, 0.05)


def _conditional(s: O.Snapshot, t: int) -> np.ndarray:
    w = int(np.searchsorted(s.word_ptr, t, side="right") - 1)
    d = int(s.doc_ids[t])
    ndk = np.bincount(s.z[s.doc_tok[s.doc_ptr[d]:s.doc_ptr[d + 1]]], minlength=s.k).astype(np.float64)
    ph = (s.phi[w].astype(np.float64) + s.beta) / (s.nk + s.num_words * s.beta)
    p = (ndk + s.alpha) * ph
    return p / p.sum()


@pytest.mark.parametrize("with_table", [False, True])
def test_mh_draws_from_the_frozen_conditional(with_table):
    c, s = _snapshot()
    cdf = None
    if with_table:
        rng = np.random.default_rng(1)
        q = rng.dirichlet(np.full(s.k, 0.3), size=s.num_docs) * 0.9 + 0.1 / s.k
        cdf = np.cumsum(q, axis=1).astype(np.float32)
    # an independence sampler started far from the mode mixes geometrically:
    # 80 steps leave no start-state bias visible at this sample size
    runs = 3000
    picks = np.empty((runs, len(s.z)), dtype=np.int64)
    for r in range(runs):
        picks[r] = s.mh(seed=99, iteration=r + 1, steps=80, cdf=cdf)[0]
    for t in (0, len(s.z) // 2, len(s.z) - 1):
        p = _conditional(s, t)
        obs = np.bincount(picks[:, t], minlength=s.k)
        exp = p * runs
        keep = exp >= 5
        chi = ((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum() + \
            (obs[~keep].sum() - exp[~keep].sum()) ** 2 / max(exp[~keep].sum(), 1e-9)
        assert stats.chi2.sf(chi, int(keep.sum())) > 1e-3, (t, chi)


def test_split_docs_keeps_vocabulary_and_documents():
    c = cb.Corpus.generate(TINY.gen)
    a = c.split_docs(np.arange(0, c.num_docs, 2))
    b = c.split_docs(np.arange(1, c.num_docs, 2))
    assert a.num_words == b.num_words == c.num_words
    assert a.num_tokens + b.num_tokens == c.num_tokens

    def bags(x):
        w_of = np.repeat(np.arange(x.num_words), np.diff(x.word_ptr))
        dt = x.doc_tokens()
        return [sorted(w_of[dt[x.doc_ptr[d]:x.doc_ptr[d + 1]]]) for d in range(x.num_docs)]

    full = bags(c)
    assert bags(a) == full[0::2] and bags(b) == full[1::2]
