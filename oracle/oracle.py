"""TEST INFRASTRUCTURE ONLY: numpy front end of oracle/liboracle.so.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product never does.  See oracle/cgs_oracle.cpp for what each
function restates (with reference file:line).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _HERE / "liboracle.so"
        if not path.exists():
            from . import build_oracle

            build_oracle.build_oracle_lib()
        _lib = C.CDLL(str(path))
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def philox4x32_10(ctr, key) -> np.ndarray:
    c = _c(ctr, np.uint32)
    k = _c(key, np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().oracle_philox4x32_10(_p(c), _p(k), _p(out))
    return out


def uniform(x: int) -> float:
    f = lib().oracle_uniform
    f.restype = C.c_double
    return f(C.c_uint32(x))


def init_topics(n: int, k: int, seed: int) -> np.ndarray:
    z = np.empty(n, dtype=np.uint16)
    lib().oracle_init_topics(C.c_int64(n), C.c_int32(k), C.c_uint64(seed), _p(z))
    return z


def doc_rev(num_docs: int, doc_ids, doc_ptr) -> np.ndarray:
    doc_ids = _c(doc_ids, np.int32)
    doc_ptr = _c(doc_ptr, np.int64)
    out = np.empty(len(doc_ids), dtype=np.int32)
    lib().oracle_doc_rev(C.c_int32(num_docs), C.c_int64(len(doc_ids)), _p(doc_ids), _p(doc_ptr), _p(out))
    return out


def theta_layout(num_docs: int, k: int, doc_ptr) -> np.ndarray:
    doc_ptr = _c(doc_ptr, np.int64)
    max_ia = np.empty(num_docs + 1, dtype=np.int32)
    f = lib().oracle_theta_layout
    f.restype = C.c_int64
    f(C.c_int32(num_docs), C.c_int32(k), _p(doc_ptr), _p(max_ia))
    return max_ia


def phi_counts(num_words: int, k: int, word_ptr, z) -> tuple[np.ndarray, np.ndarray]:
    word_ptr = _c(word_ptr, np.int64)
    z = _c(z, np.uint16)
    phi = np.empty((num_words, k), dtype=np.int32)
    nk = np.empty(k, dtype=np.int32)
    lib().oracle_phi_counts(C.c_int32(num_words), C.c_int32(k), _p(word_ptr), _p(z), _p(phi), _p(nk))
    return phi, nk


def phi_head_f16(num_words: int, k: int, beta: float, phi, nk) -> np.ndarray:
    phi = _c(phi, np.int32)
    nk = _c(nk, np.int32)
    out = np.empty((num_words, k), dtype=np.uint16)
    lib().oracle_phi_head_f16(C.c_int32(num_words), C.c_int32(k), C.c_float(beta), _p(phi), _p(nk), _p(out))
    return out


def float_to_half(x: float) -> int:
    f = lib().oracle_float_to_half
    f.restype = C.c_uint16
    return int(f(C.c_float(x)))


def theta_csr(num_docs: int, k: int, doc_ptr, doc_tok, z, max_ia):
    doc_ptr, doc_tok, z, max_ia = _c(doc_ptr, np.int64), _c(doc_tok, np.int32), _c(z, np.uint16), _c(max_ia, np.int32)
    cap = int(max_ia[-1])
    a = np.empty(cap, dtype=np.int16)
    ja = np.empty(cap, dtype=np.int16)
    cur = np.empty(num_docs, dtype=np.int32)
    lib().oracle_theta_csr(C.c_int32(num_docs), C.c_int32(k), _p(doc_ptr), _p(doc_tok), _p(z), _p(max_ia), _p(a),
                           _p(ja), _p(cur))
    return a, ja, cur


def valid_phi(num_words, k, word_ptr, z, phi, nk) -> int:
    return lib().oracle_valid_phi(C.c_int32(num_words), C.c_int32(k), _p(_c(word_ptr, np.int64)), _p(_c(z, np.uint16)),
                                  _p(_c(phi, np.int32)), _p(_c(nk, np.int32)))


def valid_theta(num_docs, k, doc_ptr, doc_tok, z, a, ja, max_ia, cur_ia) -> int:
    return lib().oracle_valid_theta(C.c_int32(num_docs), C.c_int32(k), _p(_c(doc_ptr, np.int64)),
                                    _p(_c(doc_tok, np.int32)), _p(_c(z, np.uint16)), _p(_c(a, np.int16)),
                                    _p(_c(ja, np.int16)), _p(_c(max_ia, np.int32)), _p(_c(cur_ia, np.int32)))


class CpuCgs:
    """The OpenMP host sampler (oracle/cgs_cpu.cpp): the CPU baseline."""

    def __init__(self, doc_ptr, word_ptr, doc_ids, k, alpha, beta, seed, threads=0):
        self._keep = (_c(doc_ptr, np.int64), _c(word_ptr, np.int64), _c(doc_ids, np.int32))
        self.num_tokens = len(self._keep[2])
        f = lib().cpu_cgs_create
        f.restype = C.c_void_p
        self._h = C.c_void_p(f(C.c_int32(len(self._keep[0]) - 1), C.c_int32(len(self._keep[1]) - 1),
                               C.c_int64(self.num_tokens), _p(self._keep[0]), _p(self._keep[1]),
                               _p(self._keep[2]), C.c_int32(k), C.c_float(alpha), C.c_float(beta),
                               C.c_uint64(seed), C.c_int32(threads)))
        self.threads = lib().cpu_cgs_threads(self._h)

    def iterate(self, n=1):
        sec = np.zeros(n)
        ll = np.zeros(n)
        lib().cpu_cgs_iterate(self._h, C.c_int(n), _p(sec), _p(ll))
        return sec, ll

    def topics(self) -> np.ndarray:
        z = np.empty(self.num_tokens, dtype=np.uint16)
        lib().cpu_cgs_topics(self._h, _p(z))
        return z

    def close(self):
        if self._h:
            lib().cpu_cgs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Snapshot:
    """Counts of one topic assignment, built by the oracle from scratch."""
    num_docs: int
    num_words: int
    k: int
    alpha: float
    beta: float
    word_ptr: np.ndarray
    doc_ids: np.ndarray
    doc_ptr: np.ndarray
    doc_tok: np.ndarray
    z: np.ndarray
    phi: np.ndarray
    nk: np.ndarray
    theta_a: np.ndarray
    theta_ja: np.ndarray
    max_ia: np.ndarray
    cur_ia: np.ndarray

    @classmethod
    def build(cls, word_ptr, doc_ids, doc_ptr, z, k, alpha, beta) -> "Snapshot":
        word_ptr, doc_ids, doc_ptr = _c(word_ptr, np.int64), _c(doc_ids, np.int32), _c(doc_ptr, np.int64)
        z = _c(z, np.uint16)
        d = len(doc_ptr) - 1
        v = len(word_ptr) - 1
        doc_tok = doc_rev(d, doc_ids, doc_ptr)
        phi, nk = phi_counts(v, k, word_ptr, z)
        max_ia = theta_layout(d, k, doc_ptr)
        a, ja, cur = theta_csr(d, k, doc_ptr, doc_tok, z, max_ia)
        return cls(d, v, k, float(np.float32(alpha)), float(np.float32(beta)), word_ptr, doc_ids, doc_ptr, doc_tok, z,
                   phi, nk, a, ja, max_ia, cur)

    def sample(self, seed: int, iteration: int, phi=None, nk=None):
        """(z_new, margin, loglik): one FP64 draw per token on this snapshot;
        with phi / nk given, against those fixed word-topic counts (fold-in)."""
        n = len(self.z)
        z_out = np.empty(n, dtype=np.uint16)
        margin = np.empty(n, dtype=np.float64)
        terms = np.zeros(2, dtype=np.float64)
        fixed = _c(phi, np.int32) if phi is not None else None
        nk_used = _c(nk, np.int32) if phi is not None else self.nk
        lib().oracle_sample_fixed_fp64(C.c_int32(self.num_docs), C.c_int32(self.num_words), C.c_int32(self.k),
                                       C.c_float(self.alpha), C.c_float(self.beta), _p(self.word_ptr),
                                       _p(self.doc_ids), _p(self.doc_ptr), _p(self.z), _p(nk_used), _p(self.theta_a),
                                       _p(self.theta_ja), _p(self.max_ia), _p(self.cur_ia), C.c_uint64(seed),
                                       C.c_uint32(iteration), _p(fixed) if fixed is not None else None, _p(z_out),
                                       _p(margin), _p(terms))
        return z_out, margin, (terms[0] - terms[1]) / n

    def mh(self, seed: int, iteration: int, steps: int, cdf=None):
        """(z_new, margin): one Metropolis-Hastings pass from this snapshot
        (oracle_mh_fp64); cdf is the [D x K] float32 proposal prefix table or None."""
        n = len(self.z)
        z_out = np.empty(n, dtype=np.uint16)
        margin = np.empty(n, dtype=np.float64)
        c = None if cdf is None else _c(cdf, np.float32)
        lib().oracle_mh_fp64(C.c_int32(self.num_docs), C.c_int32(self.num_words), C.c_int32(self.k),
                             C.c_float(self.alpha), C.c_float(self.beta), _p(self.word_ptr), _p(self.doc_ids),
                             _p(self.doc_ptr), _p(self.doc_tok), _p(self.z), _p(self.nk),
                             _p(c) if c is not None else None, C.c_uint64(seed), C.c_uint32(iteration),
                             C.c_int32(steps), _p(z_out), _p(margin))
        return z_out, margin

    def warm_start(self, seed: int, cdf, phi=None, nk=None):
        """(z, margin): topics drawn from q_d(k) * phihat_wk (oracle_warm_start)."""
        n = len(self.z)
        z_out = np.empty(n, dtype=np.uint16)
        margin = np.empty(n, dtype=np.float64)
        phi = _c(self.phi if phi is None else phi, np.int32)
        nk = _c(self.nk if nk is None else nk, np.int32)
        c = _c(cdf, np.float32)
        lib().oracle_warm_start(C.c_int32(self.num_docs), C.c_int32(self.num_words), C.c_int32(self.k),
                                C.c_float(self.beta), _p(self.word_ptr), _p(self.doc_ids), _p(phi), _p(nk), _p(c),
                                C.c_uint64(seed), _p(z_out), _p(margin))
        return z_out, margin

    def loglik_joint(self) -> float:
        f = lib().oracle_loglik_joint
        f.restype = C.c_double
        return f(C.c_int32(self.num_docs), C.c_int32(self.num_words), C.c_int32(self.k), C.c_float(self.alpha),
                 C.c_float(self.beta), _p(self.word_ptr), _p(self.doc_ptr), _p(self.doc_tok), _p(self.z))

    def valid(self, z=None, phi=None, nk=None, theta_a=None, theta_ja=None, cur_ia=None) -> tuple[int, int]:
        z = self.z if z is None else z
        vp = valid_phi(self.num_words, self.k, self.word_ptr, z, self.phi if phi is None else phi,
                       self.nk if nk is None else nk)
        vt = valid_theta(self.num_docs, self.k, self.doc_ptr, self.doc_tok, z,
                         self.theta_a if theta_a is None else theta_a, self.theta_ja if theta_ja is None else theta_ja,
                         self.max_ia, self.cur_ia if cur_ia is None else cur_ia)
        return vp, vt


@dataclass
class RowSnapshot:
    """n_k and the theta CSR of one topic assignment, without the V x K phi
    table (which does not fit at a million words and K = 4096): the rows the
    samplers read.  Built by the oracle from scratch."""
    num_docs: int
    num_words: int
    k: int
    alpha: float
    beta: float
    word_ptr: np.ndarray
    doc_ids: np.ndarray
    doc_ptr: np.ndarray
    z: np.ndarray
    nk: np.ndarray
    theta_a: np.ndarray
    theta_ja: np.ndarray
    max_ia: np.ndarray
    cur_ia: np.ndarray

    @classmethod
    def build(cls, word_ptr, doc_ids, doc_ptr, z, k, alpha, beta) -> "RowSnapshot":
        word_ptr, doc_ids, doc_ptr = _c(word_ptr, np.int64), _c(doc_ids, np.int32), _c(doc_ptr, np.int64)
        z = _c(z, np.uint16)
        d = len(doc_ptr) - 1
        doc_tok = doc_rev(d, doc_ids, doc_ptr)
        max_ia = theta_layout(d, k, doc_ptr)
        a, ja, cur = theta_csr(d, k, doc_ptr, doc_tok, z, max_ia)
        del doc_tok
        nk = np.bincount(z, minlength=k).astype(np.int32)
        return cls(d, len(word_ptr) - 1, k, float(np.float32(alpha)), float(np.float32(beta)), word_ptr, doc_ids,
                   doc_ptr, z, nk, a, ja, max_ia, cur)

    def sample_tokens(self, seed: int, iteration: int, sel=None, per_token_ll: bool = True):
        """(z_new, margin, ll_tok, (sum log(S+Q), sum doc term)) for the tokens
        `sel` (ascending word-major indices; None = all), one FP64 draw each
        (oracle_sample_tokens_fp64); ll_tok is None unless per_token_ll."""
        sel_arr = None if sel is None else _c(sel, np.int64)
        n = len(self.z) if sel_arr is None else len(sel_arr)
        if sel_arr is not None and n > 1:
            assert (np.diff(sel_arr) > 0).all(), "selection must be ascending"
        z_out = np.empty(n, dtype=np.uint16)
        margin = np.empty(n, dtype=np.float64)
        ll_tok = np.empty(n, dtype=np.float64) if per_token_ll else None
        terms = np.zeros(2, dtype=np.float64)
        lib().oracle_sample_tokens_fp64(
            C.c_int32(self.num_docs), C.c_int32(self.num_words), C.c_int32(self.k), C.c_float(self.alpha),
            C.c_float(self.beta), _p(self.word_ptr), _p(self.doc_ids), _p(self.doc_ptr), _p(self.z), _p(self.nk),
            _p(self.theta_a), _p(self.theta_ja), _p(self.max_ia), _p(self.cur_ia), C.c_uint64(seed),
            C.c_uint32(iteration), C.c_int64(n), _p(sel_arr) if sel_arr is not None else None, _p(z_out), _p(margin),
            _p(ll_tok) if ll_tok is not None else None, _p(terms))
        return z_out, margin, ll_tok, (float(terms[0]), float(terms[1]))


def reference_slots(word_ptr) -> tuple[np.ndarray, np.ndarray]:
    """(slot_word, slot_range [slots x 2]): the reference's slots of a corpus
    (oracle_reference_slots, doc_chunk.cpp:148-205)."""
    wp = _c(word_ptr, np.int64)
    v = len(wp) - 1
    cap = v + 2 * 57 + 16  # slices of the long words add at most N / (N // 56) + 1 slots
    sw = np.empty(cap, dtype=np.int32)
    sr = np.empty(2 * cap, dtype=np.int64)
    f = lib().oracle_reference_slots
    f.restype = C.c_int32
    ns = f(C.c_int32(v), _p(wp), _p(sw), _p(sr))
    return sw[:ns].copy(), sr[:2 * ns].reshape(ns, 2).copy()


def loglik_reference(snapshot: "Snapshot", num_tokens: int, slot_word, slot_range, phi_head_f16_table) -> float:
    """The log-likelihood the reference prints (oracle_loglik_reference)."""
    s = snapshot
    f = lib().oracle_loglik_reference
    f.restype = C.c_double
    sw = _c(slot_word, np.int32)
    sr = _c(slot_range, np.int64)
    ph = _c(phi_head_f16_table, np.uint16)
    return f(C.c_int32(s.num_words), C.c_int32(s.k), C.c_float(s.alpha), C.c_int64(num_tokens), C.c_int32(len(sw)),
             _p(sw), _p(sr), _p(s.doc_ids), _p(s.doc_ptr), _p(ph), _p(s.theta_a), _p(s.theta_ja), _p(s.max_ia),
             _p(s.cur_ia))
