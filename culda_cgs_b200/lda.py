"""The sampler context (culda_ctx) and the reference's training driver.

`LDA` owns one corpus on one GPU and runs iterations; `LDATrain` reproduces
the reference's one-GPU driver loop and its per-iteration line
(src_culda/train/SingleChunkSingleGPU.h:70-127):

    Iteration %3d: %6.2f sec, %3.2f sec, logLikelyhood = %.8f, %5.3f M
"""
from __future__ import annotations

import ctypes as C
import sys
from dataclasses import dataclass

import numpy as np

from . import _ffi
from ._ffi import check, lib
from .corpus import Corpus


@dataclass
class Argument:
    """The reference's CLI arguments (src_culda/model/culda_argument.h:50-82)."""
    numGPUs: int = 1  # noqa: N815
    k: int = 1024
    iteration: int = 100
    numChunks: int = 1  # noqa: N815
    alpha: float = 50.0 / 1024.0
    beta: float = 0.01
    inputFilePrefix: str = ""  # noqa: N815
    outputFilePrefix: str = ""  # noqa: N815


def _u16p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint16))


def _i32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class LDA:
    """One corpus resident on one GPU (culda_create ... culda_destroy)."""

    def __init__(self, corpus: Corpus, k: int, alpha: float, beta: float, seed: int = 1, device: int = 0,
                 group_lanes: int = 0, item_tokens: int = 0, flags: int = 0, sample_blocks: int = 0,
                 theta_min_len: int = 0):
        self.corpus = corpus
        self.k = int(k)
        self.alpha = float(np.float32(alpha))
        self.beta = float(np.float32(beta))
        self.num_tokens = corpus.num_tokens
        self.num_docs = corpus.num_docs
        self.num_words = corpus.num_words
        self.seed = int(seed)
        p = _ffi.Params(self.k, alpha, beta, seed, device, group_lanes, item_tokens, flags, sample_blocks,
                        theta_min_len)
        self._ctx = C.c_void_p()
        check(lib().culda_create(corpus.c_ptr, C.byref(p), C.byref(self._ctx)))

    def _check(self, status: int) -> None:
        check(status, self._ctx)

    @staticmethod
    def _stats(st, n) -> list[dict]:
        return [{name: getattr(s, name) for name, _ in _ffi.IterStats._fields_} for s in st[:n]]

    def iterate(self, n: int = 1) -> list[dict]:
        st = (_ffi.IterStats * max(n, 1))()
        self._check(lib().culda_iterate(self._ctx, int(n), st))
        return self._stats(st, n)

    # ---------------------------------------------------- learned proposal
    def accumulate_theta(self) -> None:
        """Adds the current doc-topic counts to the encoder's training targets."""
        self._check(lib().culda_accumulate_theta(self._ctx))

    def init_encoder(self, encoder, seed: int = 1) -> None:
        """Word embeddings from the current topics' word profiles (a random projection)."""
        self._check(lib().culda_encoder_init_from_phi(self._ctx, encoder.handle, int(seed)))

    def train_encoder(self, encoder, epochs: int, seed: int = 1) -> float:
        loss = C.c_double()
        self._check(lib().culda_train_encoder(self._ctx, encoder.handle, int(epochs), int(seed), C.byref(loss)))
        return loss.value

    def set_proposal(self, encoder, mix: float = 0.05) -> None:
        """The encoder's per-doc distributions (mixed with mix / K) become the
        independent MH proposal; None drops it."""
        self._check(lib().culda_set_proposal(self._ctx, encoder.handle if encoder is not None else None,
                                             float(mix)))

    def proposal(self) -> np.ndarray:
        cdf = np.empty((self.num_docs, self.k), dtype=np.float32)
        self._check(lib().culda_get_proposal(self._ctx, cdf.ctypes.data_as(C.c_void_p)))
        return cdf

    def iterate_mh(self, n: int = 1, steps: int = 2) -> list[dict]:
        st = (_ffi.IterStats * max(n, 1))()
        self._check(lib().culda_iterate_mh(self._ctx, int(n), int(steps), st))
        return self._stats(st, n)

    def mh_snapshot(self, iteration: int, steps: int = 2) -> np.ndarray:
        z = np.empty(self.num_tokens, dtype=np.uint16)
        self._check(lib().culda_mh_snapshot(self._ctx, int(iteration), int(steps), z.ctypes.data_as(C.c_void_p)))
        return z

    # -------------------------------------------------------------- fold-in
    def set_frozen_phi(self, phi, nk) -> None:
        """Sample this corpus against fixed word-topic counts (None: own counts)."""
        if phi is None:
            self._check(lib().culda_set_frozen_phi(self._ctx, None, None))
            return
        phi = np.ascontiguousarray(phi, dtype=np.int32)
        nk = np.ascontiguousarray(nk, dtype=np.int32)
        assert phi.shape == (self.num_words, self.k) and nk.shape == (self.k,)
        self._check(lib().culda_set_frozen_phi(self._ctx, phi.ctypes.data_as(C.c_void_p),
                                               nk.ctypes.data_as(C.c_void_p)))

    def warm_start(self) -> None:
        """Topics drawn from the proposal (set_proposal) times phihat."""
        self._check(lib().culda_warm_start(self._ctx))

    def topics(self) -> np.ndarray:
        z = np.empty(self.num_tokens, dtype=np.uint16)
        self._check(lib().culda_get_topics(self._ctx, _u16p(z)))
        return z

    def set_topics(self, z: np.ndarray) -> None:
        z = np.ascontiguousarray(z, dtype=np.uint16)
        assert z.shape == (self.num_tokens,)
        self._check(lib().culda_set_topics(self._ctx, _u16p(z)))

    # ------------------------------------------------- checkpoint / resume
    @property
    def next_iteration(self) -> int:
        return int(lib().culda_next_iteration(self._ctx))

    def set_iteration(self, iteration: int) -> None:
        self._check(lib().culda_set_iteration(self._ctx, int(iteration)))

    def save(self, path) -> None:
        """The chain's state (topics in input order, next iteration, settings)
        as an .npz file."""
        np.savez_compressed(path, topics=self.topics(), next_iteration=self.next_iteration, k=self.k,
                            alpha=self.alpha, beta=self.beta, seed=self.seed, num_tokens=self.num_tokens)

    def restore(self, path) -> None:
        """Resume a chain saved by save() on the same corpus and settings."""
        f = np.load(path)
        if int(f["num_tokens"]) != self.num_tokens or int(f["k"]) != self.k or int(f["seed"]) != self.seed or \
                float(f["alpha"]) != self.alpha or float(f["beta"]) != self.beta:
            raise ValueError("checkpoint does not match this corpus and these settings")
        self.set_topics(f["topics"])
        self.set_iteration(int(f["next_iteration"]))

    def phi(self, dense: bool = True) -> tuple[np.ndarray | None, np.ndarray]:
        nk = np.empty(self.k, dtype=np.int32)
        phi = np.empty((self.num_words, self.k), dtype=np.int32) if dense else None
        self._check(lib().culda_get_phi(self._ctx, _i32p(phi) if dense else None, _i32p(nk)))
        return phi, nk

    def theta(self) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        cap = lib().culda_theta_capacity(self._ctx)
        a = np.empty(cap, dtype=np.int16)
        ja = np.empty(cap, dtype=np.int16)
        max_ia = np.empty(self.num_docs + 1, dtype=np.int32)
        cur_ia = np.empty(self.num_docs, dtype=np.int32)
        self._check(lib().culda_get_theta(self._ctx, a.ctypes.data_as(C.POINTER(C.c_int16)),
                                          ja.ctypes.data_as(C.POINTER(C.c_int16)), _i32p(max_ia), _i32p(cur_ia)))
        return a, ja, max_ia, cur_ia

    def sample_snapshot(self, iteration: int) -> tuple[np.ndarray, float]:
        z = np.empty(self.num_tokens, dtype=np.uint16)
        ll = C.c_double()
        self._check(lib().culda_sample_snapshot(self._ctx, int(iteration), _u16p(z), C.byref(ll)))
        return z, ll.value

    def info(self) -> dict:
        i = _ffi.Info()
        self._check(lib().culda_get_info(self._ctx, C.byref(i)))
        return {name: getattr(i, name) for name, _ in _ffi.Info._fields_}

    def loglik_joint(self) -> float:
        ll = C.c_double()
        self._check(lib().culda_loglik_joint(self._ctx, C.byref(ll)))
        return ll.value

    def close(self) -> None:
        if self._ctx:
            lib().culda_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def LDATrain(doc: Corpus, arg: Argument, seed: int = 1, out=sys.stdout) -> LDA:  # noqa: N802
    """The reference's one-GPU training loop with its per-iteration line."""
    k = (arg.k + 31) // 32 * 32  # src_culda/main.cpp:132-135
    model = LDA(doc, k, arg.alpha, arg.beta, seed=seed)
    elapsed = 0.0
    for _ in range(arg.iteration):
        s = model.iterate(1)[0]
        elapsed += s["seconds"]
        out.write("Iteration %3d: %6.2f sec, %3.2f sec, logLikelyhood = %.8f, %5.3f M\n"
                  % (s["iteration"], elapsed, s["seconds"], s["loglik"], doc.num_tokens / s["seconds"] / 1e6))
    return model
