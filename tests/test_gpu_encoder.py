"""The document encoder on the GPU (tensor-core forward and backward, Adam)
against the FP64 oracle of oracle/encoder_oracle.py, which rounds to BF16
where the CUDA path stores BF16.  Tolerances: loss 1e-3 relative, q 2e-3
absolute, each gradient tensor 2e-2 in relative Frobenius norm (FP32
accumulation order and operands on the other side of a BF16 rounding
boundary are the only differences)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200 import _ffi
from oracle import encoder_oracle as EO

pytestmark = pytest.mark.gpu

TENSORS = {"E": _ffi.CULDA_ENC_E, "W1": _ffi.CULDA_ENC_W1, "b1": _ffi.CULDA_ENC_B1, "W2": _ffi.CULDA_ENC_W2,
           "b2": _ffi.CULDA_ENC_B2, "W3": _ffi.CULDA_ENC_W3, "b3": _ffi.CULDA_ENC_B3}


class Encoder:
    def __init__(self, V, K, max_batch, seed=1, lr=0.0):
        self.V, self.K = V, K
        p = _ffi.EncoderParams(num_words=V, k=K, max_batch=max_batch, device=0, seed=seed, lr=lr)
        self.h = C.c_void_p()
        assert cb.lib().culda_encoder_create(C.byref(p), C.byref(self.h)) == 0, cb.lib().culda_last_error(None)

    def close(self):
        cb.lib().culda_encoder_destroy(self.h)

    def get(self, name, grad=False):
        which = TENSORS[name] + (_ffi.CULDA_ENC_GRAD if grad else 0)
        n = cb.lib().culda_encoder_tensor_size(self.h, which)
        out = np.empty(n, dtype=np.float32)
        assert cb.lib().culda_encoder_get_tensor(self.h, which, out.ctypes.data_as(C.c_void_p)) == 0
        return out

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32).ravel()
        assert cb.lib().culda_encoder_set_tensor(self.h, TENSORS[name], a.ctypes.data_as(C.c_void_p)) == 0


def _dev(a, dtype):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


SHAPES = {"E": lambda V, K: (V, 256), "W1": lambda V, K: (512, 256), "b1": lambda V, K: (512,),
          "W2": lambda V, K: (512, 512), "b2": lambda V, K: (512,), "W3": lambda V, K: (K, 512),
          "b3": lambda V, K: (K,)}


@pytest.mark.parametrize("batch,K", [(128, 128), (200, 256)])
def test_backward_matches_fp64_oracle(batch, K):
    rng = np.random.default_rng(batch + K)
    V, D = 300, 260
    t = EO.random_tensors(rng, V, K)
    t = {k: v.astype(np.float32).astype(np.float64) for k, v in t.items()}
    doc_ptr, words = EO.random_batch(rng, V, D, 40)
    docs = rng.permutation(D)[:batch].astype(np.int32)
    target = EO.random_target(rng, batch, K)
    enc = Encoder(V, K, batch)
    try:
        for k, v in t.items():
            enc.set(k, v)
        d_ptr, d_words, d_docs = _dev(doc_ptr, np.int64), _dev(words, np.int32), _dev(docs, np.int32)
        d_target = _dev(target, np.float32)
        loss = C.c_double()
        rc = cb.lib().culda_encoder_backward(enc.h, batch, _p(d_docs), _p(d_ptr), _p(d_words), _p(d_target),
                                             C.byref(loss), None)
        assert rc == 0, cb.lib().culda_last_error(None)
        ora = EO.EncoderOracle(t).run(doc_ptr, words, docs, target.astype(np.float32).astype(np.float64))
        assert abs(loss.value - ora["loss"]) <= 1e-3 * abs(ora["loss"])
        for name in EO.NAMES:
            got = enc.get(name, grad=True).reshape(SHAPES[name](V, K)).astype(np.float64)
            want = ora["grads"][name]
            rel = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30)
            assert rel < 2e-2, (name, rel)
        # forward alone gives the same q
        import torch

        probs = torch.zeros(batch, K, dtype=torch.float32, device="cuda")
        assert cb.lib().culda_encoder_forward(enc.h, batch, _p(d_docs), _p(d_ptr), _p(d_words), _p(probs),
                                              None) == 0
        q = probs.cpu().numpy().astype(np.float64)
        assert np.abs(q.sum(1) - 1).max() < 1e-4
        assert np.abs(q - ora["q"]).max() < 2e-3
    finally:
        enc.close()


def test_training_fits_a_learnable_target():
    """Targets that are a function of the document's words: Adam steps on the
    GPU bring the cross-entropy far below its starting value."""
    rng = np.random.default_rng(3)
    V, K, D = 512, 128, 1024
    doc_ptr, words = EO.random_batch(rng, V, D, 30)
    # topic of a doc: the majority of word // 4 (mod K) over its tokens
    target = np.full((D, K), 0.02 / K)
    for d in range(D):
        w = words[doc_ptr[d]:doc_ptr[d + 1]] // 4 % K
        target[d, np.bincount(w, minlength=K).argmax()] += 0.98
    enc = Encoder(V, K, 256, seed=5, lr=3e-3)
    try:
        d_ptr, d_words, d_target = _dev(doc_ptr, np.int64), _dev(words, np.int32), _dev(target, np.float32)
        losses = []
        for step in range(240):
            b0 = (step * 256) % D
            docs = _dev(np.arange(b0, b0 + 256), np.int32)
            import torch

            tgt = d_target[b0:b0 + 256].contiguous()
            loss = C.c_double()
            assert cb.lib().culda_encoder_train_step(enc.h, 256, _p(docs), _p(d_ptr), _p(d_words), _p(tgt),
                                                     C.byref(loss), None) == 0
            losses.append(loss.value)
            del torch
        assert np.mean(losses[-8:]) < 0.5 * np.mean(losses[:4])
    finally:
        enc.close()


def test_rejects_bad_arguments():
    enc = Encoder(100, 128, 128)
    try:
        import torch

        z = torch.zeros(1024, dtype=torch.int64, device="cuda")
        probs = torch.zeros(256 * 128, dtype=torch.float32, device="cuda")
        assert cb.lib().culda_encoder_forward(enc.h, 129 + 128, None, _p(z), _p(z), _p(probs), None) \
            == _ffi.CULDA_ERR_INVALID_ARG
    finally:
        enc.close()
    bad = _ffi.EncoderParams(num_words=10, k=100, max_batch=128, device=0, seed=1)
    h = C.c_void_p()
    assert cb.lib().culda_encoder_create(C.byref(bad), C.byref(h)) == _ffi.CULDA_ERR_INVALID_ARG
