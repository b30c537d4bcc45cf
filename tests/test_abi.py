"""The C ABI surface: every declared entry point is exported, and the host-side
checks run without a GPU."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200 import _ffi
from culda_cgs_b200.configs import TINY

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "culda_b200.h"


def declared_functions() -> set[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"\b(culda_\w+)\s*\(", text))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", str(_ffi.library_path())], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert names <= exported, names - exported
    assert {n for n in exported if n.startswith("culda_")} == names  # nothing else leaks
    assert names == set(_ffi.SIGNATURES)


def test_version_and_status_strings():
    lib = cb.lib()
    assert b"sm_100a" in lib.culda_version()
    assert lib.culda_status_string(0) == b"ok"
    assert lib.culda_status_string(-8) == b"no CUDA device"


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the status without a device")
def test_trim_memory_without_a_device():
    assert cb.lib().culda_trim_memory(0) == _ffi.CULDA_ERR_NO_DEVICE


def _params(**kw):
    d = dict(k=64, alpha=0.1, beta=0.01, seed=1, device=0, group_lanes=0, item_tokens=0, flags=0, sample_blocks=0)
    d.update(kw)
    return _ffi.Params(**d)


@pytest.mark.parametrize("kw", [dict(k=48), dict(k=0), dict(k=8192), dict(alpha=0.0), dict(beta=-1.0),
                                dict(group_lanes=3), dict(group_lanes=-2), dict(sample_blocks=7), dict(group_lanes=1, sample_blocks=10),
                                dict(group_lanes=1, sample_blocks=9), dict(group_lanes=-1, sample_blocks=10),
                                dict(group_lanes=8, flags=_ffi.CULDA_FLAG_AUTOTUNE), dict(item_tokens=70000),
                                dict(item_tokens=-1)])
def test_create_rejects_bad_params(kw):
    c = cb.Corpus.generate(TINY.gen)
    ctx = C.c_void_p()
    p = _params(**kw)
    assert cb.lib().culda_create(c.c_ptr, C.byref(p), C.byref(ctx)) == _ffi.CULDA_ERR_INVALID_ARG
    assert not ctx.value


def test_create_rejects_inconsistent_corpus():
    c = cb.Corpus.generate(TINY.gen)
    dp = c.doc_ptr.copy()
    dp[-1] += 1
    b = cb.Corpus.from_arrays(dp, c.word_ptr, c.doc_ids)
    ctx = C.c_void_p()
    assert cb.lib().culda_create(b.c_ptr, C.byref(_params()), C.byref(ctx)) == _ffi.CULDA_ERR_FORMAT


def test_create_rejects_docs_over_16bit_counts():
    n = 70000
    b = cb.Corpus.from_arrays(np.array([0, n]), np.array([0, n]), np.zeros(n, dtype=np.int32))
    ctx = C.c_void_p()
    assert cb.lib().culda_create(b.c_ptr, C.byref(_params()), C.byref(ctx)) == _ffi.CULDA_ERR_UNSUPPORTED


def test_create_without_device_fails_cleanly(has_gpu):
    if has_gpu:
        pytest.skip("a device is present")
    c = cb.Corpus.generate(TINY.gen)
    ctx = C.c_void_p()
    assert cb.lib().culda_create(c.c_ptr, C.byref(_params()), C.byref(ctx)) == _ffi.CULDA_ERR_NO_DEVICE
    assert b"no CUDA device" in cb.lib().culda_last_error(None)


def build_items(word_ptr, item_tokens):
    wp = np.ascontiguousarray(word_ptr, dtype=np.int64)
    lib = cb.lib()
    nhot = C.c_int32()
    n = lib.culda_build_items(len(wp) - 1, wp.ctypes.data_as(C.POINTER(C.c_int64)), item_tokens, None, 0,
                              C.byref(nhot))
    items = (_ffi.Item * n)()
    assert lib.culda_build_items(len(wp) - 1, wp.ctypes.data_as(C.POINTER(C.c_int64)), item_tokens, items, n,
                                 C.byref(nhot)) == n
    return [(it.begin, it.count, it.word, it.hot, it.first) for it in items], nhot.value


def test_build_items_splits_hot_words_and_covers_every_token():
    lens = np.array([5000, 0, 3, 2500, 2501, 1, 0, 7])
    wp = np.concatenate([[0], np.cumsum(lens)])
    items, nhot = build_items(wp, 2500)
    assert nhot == 2
    counts = [it[1] for it in items]
    assert counts == sorted(counts, reverse=True) and max(counts) <= 2500
    covered = np.zeros(wp[-1], dtype=int)
    for b, n, w, hot, first in items:
        assert wp[w] <= b and b + n <= wp[w + 1]
        covered[b:b + n] += 1
        assert (hot >= 0) == (lens[w] > 2500)
    assert (covered == 1).all()
    assert sum(it[4] for it in items) == int((lens > 0).sum())  # one first item per non-empty word


def _items_reference(lens, item_tokens):
    """Words in order, words longer than item_tokens cut into ns slices of
    ceil(len / ns) tokens (the last shorter), then a stable sort by size,
    largest first."""
    out, hot, off = [], 0, 0
    for w, n in enumerate(lens):
        if n > item_tokens:
            ns = -(-n // item_tokens)
            sz = -(-n // ns)
            for i in range(ns):
                b, e = off + i * sz, min(off + (i + 1) * sz, off + n)
                if e > b:
                    out.append((b, e - b, w, hot, 1 if i == 0 else 0))
            hot += 1
        elif n > 0:
            out.append((off, n, w, -1, 1))
        off += n
    return sorted(out, key=lambda x: -x[1]), hot


@pytest.mark.parametrize("item_tokens", [7, 300, 4096])
def test_build_items_matches_a_stable_sort_of_the_slices(item_tokens):
    rng = np.random.default_rng(item_tokens)
    lens = rng.zipf(1.3, size=3000).clip(0, 20000) * rng.integers(0, 2, size=3000)
    wp = np.concatenate([[0], np.cumsum(lens)])
    items, nhot = build_items(wp, item_tokens)
    ref, ref_hot = _items_reference([int(x) for x in lens], item_tokens)
    assert nhot == ref_hot
    assert items == ref


def test_build_segments_runs_of_one_doc_inside_items():
    lens = np.array([70, 5, 1, 40])
    wp = np.concatenate([[0], np.cumsum(lens)])
    # word 0: doc 3 x 70 (one long run), word 1: docs 1,1,2,2,2, word 2: doc 0, word 3: docs 4 x 40
    doc_ids = np.array([3] * 70 + [1, 1, 2, 2, 2] + [0] + [4] * 40, dtype=np.int32)
    items = build_items_struct(wp, 50)
    lib = cb.lib()
    n = lib.culda_build_segments(len(doc_ids), doc_ids.ctypes.data_as(C.POINTER(C.c_int32)), items, len(items), 32,
                                 None, 0)
    seg = np.zeros(n, dtype=np.int32)
    assert lib.culda_build_segments(len(doc_ids), doc_ids.ctypes.data_as(C.POINTER(C.c_int32)), items, len(items),
                                    32, seg.ctypes.data_as(C.POINTER(C.c_int32)), n) == n
    covered = np.zeros(len(doc_ids), dtype=int)
    for it in items:
        starts = list(seg[it.seg_begin:it.seg_begin + it.seg_count]) + [it.begin + it.count]
        assert starts[0] == it.begin
        for a, b in zip(starts[:-1], starts[1:]):
            assert 0 < b - a <= 32 and (doc_ids[a:b] == doc_ids[a]).all()
            covered[a:b] += 1
    assert (covered == 1).all()
    # word 0 (70 tokens of one doc) is split into two items of 35, each cut into 32 + 3;
    # word 1 -> 2 (docs 1 and 2); word 2 -> 1; word 3 (40 of one doc) -> 32 + 8
    assert n == 4 + 2 + 1 + 2


def build_items_struct(word_ptr, item_tokens):
    wp = np.ascontiguousarray(word_ptr, dtype=np.int64)
    lib = cb.lib()
    nhot = C.c_int32()
    n = lib.culda_build_items(len(wp) - 1, wp.ctypes.data_as(C.POINTER(C.c_int64)), item_tokens, None, 0,
                              C.byref(nhot))
    items = (_ffi.Item * n)()
    lib.culda_build_items(len(wp) - 1, wp.ctypes.data_as(C.POINTER(C.c_int64)), item_tokens, items, n, C.byref(nhot))
    return items
