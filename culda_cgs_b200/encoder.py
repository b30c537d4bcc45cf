"""The document encoder of the learned Metropolis-Hastings proposal (a ctypes
host over culda_encoder_* in libculda_b200.so)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi
from ._ffi import check, lib

TENSORS = {"E": _ffi.CULDA_ENC_E, "W1": _ffi.CULDA_ENC_W1, "b1": _ffi.CULDA_ENC_B1, "W2": _ffi.CULDA_ENC_W2,
           "b2": _ffi.CULDA_ENC_B2, "W3": _ffi.CULDA_ENC_W3, "b3": _ffi.CULDA_ENC_B3}


class Encoder:
    """Embedding bag over V words -> 2 x 512 GELU -> softmax over K topics.
    max_batch is also the batch size of LDA.train_encoder."""

    def __init__(self, num_words: int, k: int, max_batch: int = 512, seed: int = 1, device: int = 0,
                 lr: float = 3e-3):
        self.num_words, self.k = int(num_words), int(k)
        p = _ffi.EncoderParams(num_words=self.num_words, k=self.k, max_batch=int(max_batch), device=int(device),
                               seed=int(seed), lr=float(lr))
        self.handle = C.c_void_p()
        check(lib().culda_encoder_create(C.byref(p), C.byref(self.handle)))

    def shape(self, name: str) -> tuple:
        n = lib().culda_encoder_tensor_size(self.handle, TENSORS[name])
        return {"E": (self.num_words, 256), "W1": (512, 256), "W2": (512, 512), "W3": (self.k, 512)}.get(name, (n,))

    def get(self, name: str, grad: bool = False) -> np.ndarray:
        which = TENSORS[name] + (_ffi.CULDA_ENC_GRAD if grad else 0)
        out = np.empty(self.shape(name), dtype=np.float32)
        check(lib().culda_encoder_get_tensor(self.handle, which, out.ctypes.data_as(C.c_void_p)))
        return out

    def set(self, name: str, value) -> None:
        a = np.ascontiguousarray(value, dtype=np.float32)
        check(lib().culda_encoder_set_tensor(self.handle, TENSORS[name], a.ctypes.data_as(C.c_void_p)))

    def close(self) -> None:
        if self.handle:
            lib().culda_encoder_destroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
