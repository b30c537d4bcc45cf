"""CUDA path against the oracle on the benchmark corpora themselves.

The toy-corpus parity tests (test_gpu_parity.py) cannot reach the shapes
where the sampler's special cases meet: words split over several CTAs (hot
rows, double-buffered topics), theta far larger than L2, 50,000-token
documents near the 16-bit count packing, and K = 4096 rows on the uneven
corpus.  Here, on the 1M-token small corpus, the 60M-token scale corpus and
the 118M-token uneven corpus (K = 1024 and 4096):

* integer state after an iteration is bit-exact against the oracle's recount:
  the initial topics (Philox), n_k, the theta CSR (thetaA / thetaJA / MaxIA /
  CurIA) and phi (densely on the small and scale corpora; on the uneven one
  the non-zero entries of each block of 50,000 words, counted on the device
  by culda_update_phi, against the host's sorted (word, topic) counts);
* one sampling pass on the frozen snapshot matches the FP64 oracle
  (oracle_sample_tokens_fp64) for every token whose target lies at least 1e-6
  (relative to S+Q) from a bucket boundary: on every token of the small and
  scale corpora and of the uneven corpus at K = 1024, and on the uneven corpus
  at K = 4096 on a selection holding every 61st token of each split word, all
  tokens of the longest documents and of 2,000 random words;
* where every token is drawn, the per-token log-likelihood agrees to 1e-6
  relative.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200.configs import SCALE, SMALL, UNEVEN
from oracle import oracle as O

BOUNDARY_TOL = 1e-6   # relative distance of u*(S+Q) to a bucket boundary
LL_RTOL = 1e-6
NEAR_BOUNDARY_MAX = 1e-3  # tokens allowed to differ (all of them near a boundary)

pytestmark = pytest.mark.gpu

# name, workload, K, sampler variant (lanes per token; -1 = the flat walk), draw every token
CASES = [
    ("small-k1024-flat", SMALL, 1024, -1, True),
    ("small-k1024-g8", SMALL, 1024, 8, True),
    ("scale-k1024-flat", SCALE, 1024, -1, True),
    ("uneven-k1024-flat", UNEVEN, 1024, -1, True),
    ("uneven-k4096-flat", UNEVEN, 4096, -1, False),
]

_CORPORA: dict[str, cb.Corpus] = {}


def corpus_of(wl) -> cb.Corpus:
    key = wl.name
    if key not in _CORPORA:
        _CORPORA.clear()  # one large corpus in host memory at a time
        _CORPORA[key] = cb.Corpus.generate(wl.gen)
    return _CORPORA[key]


def assert_theta_exact(m: cb.LDA, r: O.RowSnapshot):
    a, ja, max_ia, cur = m.theta()
    assert np.array_equal(max_ia, r.max_ia), "thetaMaxIA differs"
    assert np.array_equal(cur, r.cur_ia), "thetaCurIA differs"
    assert np.array_equal(a, r.theta_a), "thetaA differs"
    assert np.array_equal(ja, r.theta_ja), "thetaJA differs"


def assert_phi_blocks_exact(c: cb.Corpus, z: np.ndarray, k: int, block_words: int = 50_000):
    """phi recounted on the device from the context's topics, block by block of
    words, against the host's sorted (word, topic) counts of the same block."""
    import torch

    lib = cb.lib()
    wp = c.word_ptr
    d_wp = torch.from_numpy(wp).cuda()
    d_z = torch.from_numpy(z.view(np.int16)).cuda()
    d_nk = torch.zeros(k, dtype=torch.int32, device="cuda")
    d_phi = torch.empty(block_words * k, dtype=torch.int32, device="cuda")
    for w0 in range(0, c.num_words, block_words):
        nb = min(block_words, c.num_words - w0)
        st = lib.culda_update_phi(k, nb, C.c_void_p(d_wp.data_ptr() + 8 * w0), C.c_void_p(d_z.data_ptr()),
                                  C.c_void_p(d_phi.data_ptr()), C.c_void_p(d_nk.data_ptr()), None)
        assert st == 0, lib.culda_last_error(None)
        blk = d_phi[:nb * k]
        idx = torch.nonzero(blk).flatten()
        got_idx, got_cnt = idx.cpu().numpy(), blk[idx].cpu().numpy()
        t0, t1 = int(wp[w0]), int(wp[w0 + nb])
        words = np.repeat(np.arange(nb, dtype=np.int64), np.diff(wp[w0:w0 + nb + 1]))
        keys = words * k + z[t0:t1].astype(np.int64)
        want_idx, want_cnt = np.unique(keys, return_counts=True)
        assert np.array_equal(got_idx, want_idx), f"phi non-zeros differ in words {w0}..{w0 + nb}"
        assert np.array_equal(got_cnt, want_cnt), f"phi counts differ in words {w0}..{w0 + nb}"
    torch.cuda.synchronize()


def selection(c: cb.Corpus, item_tokens: int, rng) -> np.ndarray:
    """Every 61st token of each split (hot) word, every token of the 8 longest
    documents and of 2,000 random words, as ascending token indices."""
    wp = c.word_ptr
    lens = np.diff(wp)
    parts = []
    for w in np.flatnonzero(lens > item_tokens):
        parts.append(np.arange(wp[w], wp[w + 1], 61, dtype=np.int64))
    for w in rng.choice(c.num_words, 2000, replace=False):
        parts.append(np.arange(wp[w], wp[w + 1], dtype=np.int64))
    longest = np.argsort(np.diff(c.doc_ptr))[-8:]
    parts.append(np.flatnonzero(np.isin(c.doc_ids, longest)).astype(np.int64))
    return np.unique(np.concatenate(parts))


@pytest.mark.parametrize("name,wl,k,g,every_token", CASES, ids=[x[0] for x in CASES])
def test_benchmark_corpus_counts_and_draws(name, wl, k, g, every_token):
    c = corpus_of(wl)
    seed = 20 + k // 1024
    alpha, beta = 50.0 / k, 0.01
    with cb.LDA(c, k, alpha, beta, seed=seed, group_lanes=g) as m:
        info = m.info()
        if wl is not SMALL:
            assert info["num_hot"] > 0, "the benchmark corpora split their largest words"
        z0 = m.topics()
        assert np.array_equal(z0, O.init_topics(c.num_tokens, k, seed)), "initial topics differ"
        st = m.iterate(1)[0]
        assert st["status"] == 0, st
        z1 = m.topics()
        r = O.RowSnapshot.build(c.word_ptr, c.doc_ids, c.doc_ptr, z1, k, alpha, beta)
        _, nk = m.phi(dense=False)
        assert np.array_equal(nk, r.nk), "n_k differs"
        assert_theta_exact(m, r)
        assert st["theta_nnz"] == int((r.theta_a != 0).sum())
        if c.num_words * k <= 200_000_000:
            phi, _ = m.phi()
            ph_o, nk_o = O.phi_counts(c.num_words, k, c.word_ptr, z1)
            assert np.array_equal(phi, ph_o) and np.array_equal(nk_o, nk), "phi differs"
            del phi, ph_o
        else:
            assert_phi_blocks_exact(c, z1, k)

        # one pass on the frozen snapshot (Philox iteration 2) against the FP64 oracle
        z_gpu, ll_gpu = m.sample_snapshot(2)
        sel = None if every_token else selection(c, info["item_tokens"], np.random.default_rng(k))
        z_ora, margin, _, (t_log, t_doc) = r.sample_tokens(seed, 2, sel, per_token_ll=False)
        got = z_gpu if sel is None else z_gpu[sel]
        far = margin >= BOUNDARY_TOL
        bad = (got != z_ora) & far
        assert not bad.any(), (f"{int(bad.sum())} of {len(got)} tokens differ beyond the boundary tolerance; "
                               f"first at {np.flatnonzero(bad)[:5]}")
        assert (got != z_ora).mean() < NEAR_BOUNDARY_MAX
        if sel is None:
            ll_ora = (t_log - t_doc) / c.num_tokens
            assert abs(ll_gpu - ll_ora) <= LL_RTOL * abs(ll_ora), (ll_gpu, ll_ora)
        else:
            assert len(sel) > 100_000
        # the snapshot pass left the chain untouched; two more iterations keep
        # theta and n_k consistent with the topics
        assert np.array_equal(m.topics(), z1)
        assert all(s["status"] == 0 for s in m.iterate(2))
        z3 = m.topics()
        r3 = O.RowSnapshot.build(c.word_ptr, c.doc_ids, c.doc_ptr, z3, k, alpha, beta)
        assert_theta_exact(m, r3)
        assert np.array_equal(m.phi(dense=False)[1], r3.nk)
