"""Corpus files (src_format word-first format), the synthetic generator and the loader."""
from __future__ import annotations

import filecmp
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200 import CuldaError
from culda_cgs_b200._ffi import CULDA_ERR_FORMAT, CULDA_ERR_IO, CULDA_ERR_UNSUPPORTED
from culda_cgs_b200.configs import SMALL, TINY, MINI
from culda_cgs_b200.corpus import GenConfig

ROOT = Path(__file__).resolve().parent.parent
REF_FORMAT = ROOT / "oracle" / "_ref" / "format"
SUFFIXES = ["vocab", "doc.idx", "chunk", "word.idx", "word.data"]


def test_generator_shapes_and_invariants():
    c = cb.Corpus.generate(TINY.gen)
    dp, wp, ids = c.doc_ptr, c.word_ptr, c.doc_ids
    assert dp[0] == 0 and dp[-1] == c.num_tokens and wp[0] == 0 and wp[-1] == c.num_tokens
    assert (np.diff(dp) >= TINY.gen.len_min).all() and (np.diff(dp) <= TINY.gen.len_max).all()
    assert (np.diff(wp) > 0).all()  # ids by first appearance: every word occurs
    assert ids.min() >= 0 and ids.max() < c.num_docs
    for w in range(c.num_words):  # docs ascending inside a word
        seg = ids[wp[w]:wp[w + 1]]
        assert (np.diff(seg) >= 0).all()
    assert (np.bincount(ids, minlength=c.num_docs) == np.diff(dp)).all()


def test_generator_is_deterministic_and_thread_independent():
    a = cb.Corpus.generate(MINI.gen)
    b = cb.Corpus.generate(GenConfig(**{**MINI.gen.__dict__, "threads": 1}))
    assert np.array_equal(a.doc_ids, b.doc_ids) and np.array_equal(a.word_ptr, b.word_ptr)
    c = cb.Corpus.generate(GenConfig(**{**MINI.gen.__dict__, "seed": 2}))
    assert not np.array_equal(a.doc_ptr, c.doc_ptr)


def test_generator_length_laws():
    c = cb.Corpus.generate(SMALL.gen)
    L = c.doc_lengths
    assert abs(L.mean() - 100) < 1.0 and abs(L.std() - 10) < 0.5  # Poisson(100)
    assert 0.9e6 < c.num_tokens < 1.1e6
    # Zipf head: word 0 (first seen) is among the most frequent
    wl = np.diff(c.word_ptr)
    assert wl.max() > 50 * np.median(wl)


def test_write_load_roundtrip(tmp_path):
    c = cb.Corpus.generate(TINY.gen)
    c.write(str(tmp_path / "t"))
    d = cb.Corpus.load(str(tmp_path / "t"))
    assert (d.num_docs, d.num_words, d.num_tokens) == (c.num_docs, c.num_words, c.num_tokens)
    assert np.array_equal(d.doc_ids, c.doc_ids) and np.array_equal(d.doc_ptr, c.doc_ptr)
    doc = cb.Document().loadDocument(str(tmp_path / "t"), 1)
    assert doc.numTokens == c.num_tokens


@pytest.mark.skipif(not REF_FORMAT.exists(), reason="reference format tool not built")
@pytest.mark.parametrize("chunks", [1, 3])
def test_writer_matches_reference_format_tool(tmp_path, chunks):
    """Our direct writer equals src_format/format.cpp run on the text rendering."""
    c = cb.Corpus.generate(TINY.gen)
    c.write_text(str(tmp_path / "corpus.txt"))
    c.write(str(tmp_path / "mine"), chunks)
    subprocess.run([str(REF_FORMAT), "corpus.txt", "ref", str(chunks)], cwd=tmp_path, check=True,
                   capture_output=True)
    names = ["vocab", "doc.idx", "chunk"]
    if chunks == 1:
        names += ["word.idx", "word.data"]
    else:
        names += [f"word.{s}{i}" for s in ("idx", "data") for i in range(chunks)]
    for n in names:
        assert filecmp.cmp(tmp_path / f"mine.{n}", tmp_path / f"ref.{n}", shallow=False), n


def _write(c, path):
    c.write(str(path))
    return str(path)


def test_load_missing_files(tmp_path):
    c = cb.Corpus.generate(TINY.gen)
    p = _write(c, tmp_path / "t")
    for suf in SUFFIXES:
        q = tmp_path / f"m_{suf.replace('.', '_')}"
        _write(c, q)
        os.remove(f"{q}.{suf}")
        with pytest.raises(CuldaError) as e:
            cb.Corpus.load(str(q))
        assert e.value.status == CULDA_ERR_IO, suf
    assert cb.Corpus.load(p).num_tokens == c.num_tokens


def test_load_chunk_mismatch_and_multichunk(tmp_path):
    c = cb.Corpus.generate(TINY.gen)
    p = _write(c, tmp_path / "t")
    with pytest.raises(CuldaError) as e:
        cb.Corpus.load(p, 2)
    assert e.value.status == CULDA_ERR_UNSUPPORTED
    with open(p + ".chunk", "a") as f:
        f.write("1 5\n")
    with pytest.raises(CuldaError) as e:
        cb.Corpus.load(p, 1)
    assert e.value.status == CULDA_ERR_FORMAT


def test_load_corrupted_payload(tmp_path):
    c = cb.Corpus.generate(TINY.gen)
    p = _write(c, tmp_path / "t")
    data = np.fromfile(p + ".word.data", dtype=np.int32)
    bad = data.copy()
    bad[3] = c.num_docs + 7  # doc id out of range
    bad.tofile(p + ".word.data")
    with pytest.raises(CuldaError) as e:
        cb.Corpus.load(p)
    assert e.value.status == CULDA_ERR_FORMAT
    data[:-5].tofile(p + ".word.data")  # truncated
    with pytest.raises(CuldaError) as e:
        cb.Corpus.load(p)
    assert e.value.status == CULDA_ERR_FORMAT
    swapped = data.copy()
    i = int(np.argmax(data != data[0]))
    swapped[0], swapped[i] = swapped[i], swapped[0]  # doc lengths no longer match .doc.idx? (counts equal)
    swapped.tofile(p + ".word.data")
    assert cb.Corpus.load(p).num_tokens == c.num_tokens


def test_borrowed_corpus_arrays():
    c = cb.Corpus.generate(TINY.gen)
    b = cb.Corpus.from_arrays(c.doc_ptr, c.word_ptr, c.doc_ids)
    assert np.array_equal(b.doc_tokens(), c.doc_tokens())
