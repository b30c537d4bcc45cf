"""Doc-chunk data parallelism: one rank per GPU, each sampling one chunk of the
documents against word-topic counts summed over every chunk.

The reference's -g N -c N path (src_culda/train/MultiChunkMultiGPUequal.h:88-172)
drives N GPUs from one process: each samples its chunk against the same phi
replica, phi is collected on GPU 0, summed and copied back
(src_culda/model/model_phi.cpp:105-144), and phiHead is rebuilt everywhere.
Here each rank is its own process (torch.distributed, NCCL over NVLink):

* `partition_docs` is the doc -> chunk map of the reference's format tool
  (src_format/format.cpp:107-132): chunks of consecutive documents, each
  closed as soon as it holds at least ceil(N / chunks) tokens;
* `chunk_corpus` is one chunk over the whole vocabulary (doc ids renumbered
  from the chunk's first document);
* `exchange_counts` is the phi reduction: one in-place sum all-reduce of the
  chunk's V*K word-topic counts and K topic totals, held in one buffer;
* `ChunkedLDA` is one rank: its context samples its chunk against the summed
  counts (culda_set_shared_phi), then writes its chunk's new counts
  (culda_count_phi) into the buffer that the next exchange sums.

Every rank takes the same collective steps in the same order; the per-token
log-likelihood of an iteration is the sum of the chunks' terms over the total
token count.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._ffi import check, lib
from .corpus import BorrowedCorpus, Corpus
from .lda import LDA


def partition_docs(doc_ptr, num_chunks: int) -> np.ndarray:
    """Chunk boundaries [num_chunks + 1] in doc ids (format.cpp:107-132):
    chunk c takes documents from where chunk c-1 stopped until its token
    count reaches ceil(N / num_chunks) or the documents run out."""
    doc_ptr = np.asarray(doc_ptr, dtype=np.int64)
    if num_chunks < 1:
        raise ValueError("num_chunks must be at least 1")
    d_total = len(doc_ptr) - 1
    n = int(doc_ptr[-1] - doc_ptr[0])
    per_chunk = (n + num_chunks - 1) // num_chunks
    bounds = np.zeros(num_chunks + 1, dtype=np.int64)
    d = 0
    for c in range(num_chunks):
        bounds[c] = d
        if d < d_total:
            # the first doc at which the chunk's running size reaches per_chunk
            target = doc_ptr[d] + per_chunk
            e = int(np.searchsorted(doc_ptr, target, side="left"))
            d = min(max(e, d + 1), d_total)
    bounds[num_chunks] = d
    return bounds


def chunk_corpus(corpus: Corpus, d0: int, d1: int) -> BorrowedCorpus:
    """Documents [d0, d1) of `corpus` over its whole vocabulary, doc ids
    renumbered from 0; tokens stay word-major with ascending doc ids."""
    ids = corpus.doc_ids
    word_of = np.repeat(np.arange(corpus.num_words, dtype=np.int64), np.diff(corpus.word_ptr))
    keep = (ids >= d0) & (ids < d1)
    new_ids = (ids[keep] - d0).astype(np.int32)
    word_ptr = np.concatenate([[0], np.cumsum(np.bincount(word_of[keep], minlength=corpus.num_words))])
    doc_ptr = corpus.doc_ptr[d0:d1 + 1] - corpus.doc_ptr[d0]
    return BorrowedCorpus(doc_ptr.astype(np.int64), word_ptr.astype(np.int64), new_ids)


def exchange_counts(counts, group=None) -> None:
    """Sums the chunks' counts in place over the ranks of `group` (a flat
    int32 tensor: V*K word-topic counts then K topic totals).  One rank: no-op."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)


class ChunkedLDA:
    """One rank of a doc-chunk data-parallel chain (one process per GPU)."""

    def __init__(self, corpus: Corpus, k: int, alpha: float, beta: float, seed: int = 1, rank: int = 0,
                 world: int = 1, device: int = 0, group=None, **kw):
        import torch

        self.rank, self.world, self.group = rank, world, group
        bounds = partition_docs(corpus.doc_ptr, world)
        self.doc_range = (int(bounds[rank]), int(bounds[rank + 1]))
        self.chunk = chunk_corpus(corpus, *self.doc_range)
        self.num_tokens_total = corpus.num_tokens
        # each chunk draws from its own Philox key: a token index repeats across chunks
        self.lda = LDA(self.chunk, k, alpha, beta, seed=(seed + (rank << 40)) & (2**64 - 1), device=device, **kw)
        self.k, self.num_words = int(k), corpus.num_words
        self.device = torch.device("cuda", device)
        self.counts = torch.zeros(self.num_words * self.k + self.k, dtype=torch.int32, device=self.device)
        self._exchange()
        check(lib().culda_set_shared_phi(self.lda._ctx, self._ptr(0), self._ptr(self.num_words * self.k)),
              self.lda._ctx)

    def _ptr(self, offset: int) -> C.c_void_p:
        return C.c_void_p(self.counts.data_ptr() + 4 * offset)

    def _exchange(self) -> None:
        import torch

        check(lib().culda_count_phi(self.lda._ctx, self._ptr(0), self._ptr(self.num_words * self.k)), self.lda._ctx)
        exchange_counts(self.counts, self.group)
        torch.cuda.current_stream(self.device).synchronize()

    def iterate(self, n: int = 1) -> list[dict]:
        """n iterations: sample the chunk against the summed counts, rebuild
        its theta, then sum the new counts over the chunks.  Each returned
        dict is the chunk's statistics plus `loglik_global`, the per-token
        log-likelihood of the whole corpus."""
        import torch
        import torch.distributed as dist

        out = []
        for _ in range(n):
            st = self.lda.iterate(1)[0]
            self._exchange()
            ll = torch.tensor([st["loglik"] * self.chunk.num_tokens], dtype=torch.float64, device=self.device)
            if dist.is_available() and dist.is_initialized() and dist.get_world_size(self.group) > 1:
                dist.all_reduce(ll, op=dist.ReduceOp.SUM, group=self.group)
            st["loglik_global"] = float(ll.item()) / self.num_tokens_total
            out.append(st)
        return out

    def phi(self) -> tuple[np.ndarray, np.ndarray]:
        """The summed word-topic counts [V x K] and topic totals of the current topics."""
        c = self.counts.cpu().numpy()
        return c[:self.num_words * self.k].reshape(self.num_words, self.k), c[self.num_words * self.k:]

    def topics(self) -> np.ndarray:
        return self.lda.topics()

    def close(self) -> None:
        if self.lda is not None:
            check(lib().culda_set_shared_phi(self.lda._ctx, None, None), self.lda._ctx)
            self.lda.close()
            self.lda = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
