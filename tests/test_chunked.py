"""Doc-chunk data parallelism on the host (no GPU): the chunk map, the chunk
corpora, and the count exchange between two gloo ranks.

* partition_docs gives the `.chunk` file's doc ranges of the library's writer,
  which is byte-identical to the reference's format tool
  (src_format/format.cpp:107-132);
* the chunk corpora partition the tokens: together they hold every token of
  every word once, with the chunk's doc ids;
* two gloo ranks, each holding one chunk's counts of the same topic
  assignment, sum them with exchange_counts into exactly the counts of the
  whole corpus (the reduction of src_culda/model/model_phi.cpp:105-144).
"""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200.chunked import chunk_corpus, partition_docs
from culda_cgs_b200.configs import MINI, TINY

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.parametrize("wl", [TINY, MINI], ids=["tiny", "mini"])
@pytest.mark.parametrize("n", [1, 2, 3, 8])
def test_partition_matches_the_chunk_file(tmp_path, wl, n):
    c = cb.Corpus.generate(wl.gen)
    c.write(str(tmp_path / "x"), n)
    ends = [int(line.split()[1]) for line in (tmp_path / "x.chunk").read_text().splitlines() if line.strip()]
    b = partition_docs(c.doc_ptr, n)
    assert b[0] == 0 and list(b[1:]) == ends


def test_partition_edge_cases():
    # more chunks than documents: the last chunks are empty, as the reference leaves them
    assert list(partition_docs(np.array([0, 5, 9]), 4)) == [0, 1, 2, 2, 2]
    # empty documents stay with the chunk that reached its size before them
    dp = np.array([0, 3, 3, 3, 6, 6, 9])
    assert list(partition_docs(dp, 3)) == [0, 1, 4, 6]
    # one chunk: everything
    assert list(partition_docs(dp, 1)) == [0, 6]
    with pytest.raises(ValueError):
        partition_docs(dp, 0)


def test_chunk_corpora_partition_the_tokens():
    c = cb.Corpus.generate(MINI.gen)
    b = partition_docs(c.doc_ptr, 3)
    ids, wp = c.doc_ids, c.word_ptr
    word_of = np.repeat(np.arange(c.num_words), np.diff(wp))
    got = []
    for r in range(3):
        ch = chunk_corpus(c, int(b[r]), int(b[r + 1]))
        assert ch.num_words == c.num_words and ch.num_docs == b[r + 1] - b[r]
        assert np.array_equal(np.diff(ch.doc_ptr), np.diff(c.doc_ptr)[b[r]:b[r + 1]])
        cw = np.repeat(np.arange(ch.num_words), np.diff(ch.word_ptr))
        got.append(np.stack([cw, ch.doc_ids.astype(np.int64) + b[r]]))
        # word-major with ascending doc ids inside each word
        key = cw.astype(np.int64) * c.num_docs + ch.doc_ids
        assert (np.diff(key) >= 0).all()
    allp = np.concatenate(got, axis=1)
    order = np.lexsort((allp[1], allp[0]))
    assert np.array_equal(allp[:, order], np.stack([word_of, ids.astype(np.int64)]))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _chunk_counts(c, z_full, lo, hi, k):
    """Counts [V*K + K] of the tokens of docs [lo, hi) (test-side recount)."""
    word_of = np.repeat(np.arange(c.num_words, dtype=np.int64), np.diff(c.word_ptr))
    keep = (c.doc_ids >= lo) & (c.doc_ids < hi)
    phi = np.bincount(word_of[keep] * k + z_full[keep], minlength=c.num_words * k)
    nk = np.bincount(z_full[keep], minlength=k)
    return np.concatenate([phi, nk]).astype(np.int32)


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch
    import torch.distributed as dist

    import culda_cgs_b200 as cb
    from culda_cgs_b200.chunked import exchange_counts, partition_docs
    from culda_cgs_b200.configs import MINI
    from oracle import oracle as O

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        c = cb.Corpus.generate(MINI.gen)
        k = 256
        z = O.init_topics(c.num_tokens, k, 7).astype(np.int64)
        b = partition_docs(c.doc_ptr, world)
        counts = torch.from_numpy(_chunk_counts(c, z, int(b[rank]), int(b[rank + 1]), k))
        exchange_counts(counts)
        whole = _chunk_counts(c, z, 0, c.num_docs, k)
        out.put((rank, bool(np.array_equal(counts.numpy(), whole)), int(counts[-k:].sum())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sum_their_chunk_counts_to_the_whole_corpus():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in procs)
    n = cb.Corpus.generate(MINI.gen).num_tokens
    assert [r[0] for r in res] == [0, 1]
    assert all(ok and total == n for _, ok, total in res)
