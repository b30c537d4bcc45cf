"""Doc-chunk data parallelism on one GPU: two chunk contexts of one corpus,
their counts summed on the device, stand in for two ranks.

(Ranks on separate GPUs exchange the same buffers with an NCCL all-reduce,
exchange_counts; one GPU runs the two chunks one after the other, with the
sum done by the test, so no kernel waits on another.)

* The summed chunk counts (culda_count_phi) equal the oracle's counts of the
  whole corpus, before and after iterations.
* A chunk context sampling against the summed counts (culda_set_shared_phi)
  draws, on the frozen snapshot, what the FP64 oracle draws for the chunk's
  tokens with the whole corpus's phi and n_k and the chunk's theta, away from
  bucket boundaries.
* With one chunk, ChunkedLDA samples what a plain context samples.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200.chunked import ChunkedLDA, chunk_corpus, partition_docs
from culda_cgs_b200.configs import MINI
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _vp(t, offset=0):
    return C.c_void_p(t.data_ptr() + 4 * offset)


def _global_topics(c, bounds, chunk_topics):
    """The chunks' topics placed back at the whole corpus's token positions."""
    z = np.empty(c.num_tokens, dtype=np.uint16)
    for r, zc in enumerate(chunk_topics):
        keep = (c.doc_ids >= bounds[r]) & (c.doc_ids < bounds[r + 1])
        z[keep] = zc  # both word-major with ascending doc ids inside a word
    return z


def test_two_chunks_on_one_gpu_match_the_whole_corpus():
    import torch

    c = cb.Corpus.generate(MINI.gen)
    k, alpha, beta, seed = 1024, 50.0 / 1024, 0.01, 41
    V = c.num_words
    b = partition_docs(c.doc_ptr, 2)
    chunks = [chunk_corpus(c, int(b[r]), int(b[r + 1])) for r in range(2)]
    models = [cb.LDA(ch, k, alpha, beta, seed=seed + r) for r, ch in enumerate(chunks)]
    lib = cb.lib()
    try:
        local = [torch.zeros(V * k + k, dtype=torch.int32, device="cuda") for _ in range(2)]
        shared = torch.zeros(V * k + k, dtype=torch.int32, device="cuda")

        def exchange():
            for m, buf in zip(models, local):
                assert lib.culda_count_phi(m._ctx, _vp(buf), _vp(buf, V * k)) == 0, lib.culda_last_error(m._ctx)
            torch.add(local[0], local[1], out=shared)
            torch.cuda.synchronize()

        exchange()
        for m in models:
            assert lib.culda_set_shared_phi(m._ctx, _vp(shared), _vp(shared, V * k)) == 0
        for it in range(3):
            z = _global_topics(c, b, [m.topics() for m in models])
            phi_o, nk_o = O.phi_counts(V, k, c.word_ptr, z)
            got = shared.cpu().numpy()
            assert np.array_equal(got[:V * k].reshape(V, k), phi_o), f"summed phi differs before iteration {it + 1}"
            assert np.array_equal(got[V * k:], nk_o)
            # each chunk's draws against the summed counts, on the frozen snapshot
            for r, (m, ch) in enumerate(zip(models, chunks)):
                s = O.Snapshot.build(ch.word_ptr, ch.doc_ids, ch.doc_ptr, m.topics(), k, alpha, beta)
                z_ora, margin, ll_ora = s.sample(seed + r, 50 + it, phi=phi_o, nk=nk_o)
                z_gpu, ll_gpu = m.sample_snapshot(50 + it)
                far = margin >= 1e-6
                assert not ((z_gpu != z_ora) & far).any()
                assert abs(ll_gpu - ll_ora) <= 1e-6 * abs(ll_ora)
            for m in models:
                assert m.iterate(1)[0]["status"] == 0
            exchange()
    finally:
        for m in models:
            lib.culda_set_shared_phi(m._ctx, None, None)
            m.close()


def test_one_chunk_samples_what_a_plain_context_samples():
    c = cb.Corpus.generate(MINI.gen)
    k, alpha, beta, seed = 1024, 50.0 / 1024, 0.01, 9
    with cb.LDA(c, k, alpha, beta, seed=seed) as plain, ChunkedLDA(c, k, alpha, beta, seed=seed) as dp:
        assert dp.doc_range == (0, c.num_docs)
        assert np.array_equal(dp.topics(), plain.topics())
        s_plain = plain.iterate(2)
        s_dp = dp.iterate(2)
        for a, b in zip(s_plain, s_dp):
            assert abs(a["loglik"] - b["loglik_global"]) <= 1e-6 * abs(a["loglik"])
        # draws near a bucket boundary may differ; nothing else may
        assert (dp.topics() != plain.topics()).mean() < 1e-3
        phi, nk = dp.phi()
        z = dp.topics()
        phi_o, nk_o = O.phi_counts(c.num_words, k, c.word_ptr, z)
        assert np.array_equal(phi, phi_o) and np.array_equal(nk, nk_o)
