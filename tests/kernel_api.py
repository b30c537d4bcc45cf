"""Helpers for driving the kernel-level C entry points with device buffers.

Device memory comes from torch (plumbing only); every computation goes
through the library's C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

import culda_cgs_b200 as cb
from culda_cgs_b200 import _ffi


def dev(a: np.ndarray):
    import torch

    a = np.ascontiguousarray(a)
    if a.dtype == np.uint16:
        a = a.view(np.int16)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    if a.dtype == np.uint8:
        return torch.from_numpy(a.copy()).cuda()
    return torch.from_numpy(a.copy()).cuda()


def host(t, dtype) -> np.ndarray:
    return t.cpu().numpy().view(dtype)


def ptr(t) -> int:
    return t.data_ptr()


@dataclass
class Problem:
    """One corpus and topic assignment laid out for the kernel-level API."""
    corpus: cb.Corpus
    k: int
    alpha: float
    beta: float
    z: np.ndarray
    items: object          # ctypes array of _ffi.Item (with segments)
    num_items: int
    num_hot: int
    hot: object            # ctypes array of the hot items
    num_hot_items: int
    seg_start: np.ndarray
    cap: int
    d: dict                # device tensors


def prepare(corpus: cb.Corpus, k: int, alpha: float, beta: float, z: np.ndarray, item_tokens: int = 256) -> Problem:
    import torch

    lib = cb.lib()
    wp, dp, ids = corpus.word_ptr, corpus.doc_ptr, corpus.doc_ids
    nhot = C.c_int32()
    wpc = np.ascontiguousarray(wp, dtype=np.int64)
    n = lib.culda_build_items(corpus.num_words, wpc.ctypes.data_as(C.POINTER(C.c_int64)), item_tokens, None, 0,
                              C.byref(nhot))
    items = (_ffi.Item * n)()
    assert lib.culda_build_items(corpus.num_words, wpc.ctypes.data_as(C.POINTER(C.c_int64)), item_tokens, items, n,
                                 C.byref(nhot)) == n
    idc = np.ascontiguousarray(ids, dtype=np.int32)
    nseg = lib.culda_build_segments(len(ids), idc.ctypes.data_as(C.POINTER(C.c_int32)), items, n, 32, None, 0)
    seg = np.zeros(nseg, dtype=np.int32)
    assert lib.culda_build_segments(len(ids), idc.ctypes.data_as(C.POINTER(C.c_int32)), items, n, 32,
                                    seg.ctypes.data_as(C.POINTER(C.c_int32)), nseg) == nseg
    hot_list = [items[i] for i in range(n) if items[i].hot >= 0]
    hot = (_ffi.Item * max(1, len(hot_list)))(*hot_list)
    # theta layout: capacity roundup32(min(L_d, K)) per doc, rows start empty
    L = np.diff(dp)
    capd = (np.minimum(L, k) + 31) // 32 * 32
    starts = np.concatenate([[0], np.cumsum(capd)])[:-1].astype(np.int32)
    rows = np.stack([starts, starts], axis=1).astype(np.int32).ravel()
    cap = int(capd.sum())
    d = {
        "word_ptr": dev(wp.astype(np.int64)), "doc_ptr": dev(dp.astype(np.int64)), "doc_ids": dev(idc),
        "doc_tok": dev(corpus.doc_tokens()), "z": dev(z.astype(np.uint16)),
        "z_out": torch.zeros(len(ids), dtype=torch.int16, device="cuda"),
        "rows": dev(rows), "theta": torch.zeros(cap, dtype=torch.int32, device="cuda"),
        "nk": torch.zeros(k, dtype=torch.int32, device="cuda"),
        "stats": torch.zeros(3, dtype=torch.int64, device="cuda"),
        "items": dev(np.frombuffer(bytes(items), dtype=np.uint8)),
        "hot": dev(np.frombuffer(bytes(hot), dtype=np.uint8)),
        "seg": dev(seg), "ll": torch.zeros(1, dtype=torch.float64, device="cuda"),
        "err": torch.zeros(1, dtype=torch.int32, device="cuda"),
        "ws_theta": torch.zeros(lib.culda_update_theta_workspace(k, corpus.num_docs) // 4 + 64, dtype=torch.int32,
                                device="cuda"),
    }
    return Problem(corpus, k, float(np.float32(alpha)), float(np.float32(beta)), z, items, n, nhot.value, hot,
                   len(hot_list), seg, cap, d)


def update_theta(p: Problem) -> int:
    lib = cb.lib()
    d = p.d
    return lib.culda_update_theta(p.k, p.corpus.num_docs, ptr(d["doc_ptr"]), ptr(d["doc_tok"]), ptr(d["z"]), None,
                                  ptr(d["rows"]), ptr(d["theta"]), ptr(d["nk"]), ptr(d["stats"]), ptr(d["ws_theta"]),
                                  d["ws_theta"].numel() * 4, None)


def sample_args(p: Problem, seed: int, iteration: int, group_lanes: int = 8) -> _ffi.SampleArgs:
    d = p.d
    c = p.corpus
    return _ffi.SampleArgs(
        k=p.k, alpha=p.alpha, beta=p.beta, num_docs=c.num_docs, num_words=c.num_words, num_tokens=c.num_tokens,
        word_ptr=ptr(d["word_ptr"]), doc_ids=ptr(d["doc_ids"]), topics_in=ptr(d["z"]), topics_out=ptr(d["z_out"]),
        theta=ptr(d["theta"]), theta_rows=ptr(d["rows"]), nk=ptr(d["nk"]), items=ptr(d["items"]),
        seg_start=ptr(d["seg"]), num_segs=len(p.seg_start), num_items=p.num_items, num_hot=p.num_hot,
        hot_items=ptr(d["hot"]) if p.num_hot_items else None, num_hot_items=p.num_hot_items, theta_capacity=p.cap,
        seed=seed, iteration=iteration, group_lanes=group_lanes, loglik_sum=ptr(d["ll"]), error=ptr(d["err"]))


def doc_term(p: Problem) -> float:
    L = np.diff(p.corpus.doc_ptr).astype(np.float64)
    return float((L * np.log(L + p.k * p.alpha)).sum())
