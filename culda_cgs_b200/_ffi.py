"""ctypes binding of include/culda_b200.h (libculda_b200.so).

The shared library is loaded from the package directory; there is no Python
or CPU fallback: if the library is missing the import of any entry point
raises, so a run without the native code fails loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libculda_b200.so"

i32, i64, u16, u32, u64, f32, f64 = C.c_int32, C.c_int64, C.c_uint16, C.c_uint32, C.c_uint64, C.c_float, C.c_double
P = C.POINTER

CULDA_OK = 0
CULDA_ERR_INVALID_ARG = -1
CULDA_ERR_IO = -2
CULDA_ERR_FORMAT = -3
CULDA_ERR_CUDA = -4
CULDA_ERR_OOM = -5
CULDA_ERR_UNSUPPORTED = -6
CULDA_ERR_DEVICE_STATE = -7
CULDA_ERR_NO_DEVICE = -8

CULDA_LEN_POISSON, CULDA_LEN_LOGNORMAL, CULDA_LEN_PARETO = 0, 1, 2
CULDA_NOALLOC_SCRATCH_BYTES = 8 << 20  # include/culda_b200.h
CULDA_FLAG_NO_GRAPH, CULDA_FLAG_VERBOSE, CULDA_FLAG_NO_REORDER, CULDA_FLAG_AUTOTUNE = 1, 2, 4, 8
CULDA_SAMPLER_FLAT = -1


class Corpus(C.Structure):
    _fields_ = [("num_docs", i32), ("num_words", i32), ("num_tokens", i64), ("doc_ptr", P(i64)),
                ("word_ptr", P(i64)), ("doc_ids", P(i32)), ("word_label", P(i32)), ("owned", i32)]


class Vocab(C.Structure):
    _fields_ = [("num_words", i32), ("offsets", P(i64)), ("bytes", C.c_void_p)]


class GenParams(C.Structure):
    _fields_ = [("num_words", i32), ("num_topics", i32), ("num_docs", i32), ("len_law", i32), ("zipf_s", f64),
                ("word_conc", f64), ("doc_conc", f64), ("len_a", f64), ("len_b", f64), ("len_min", i32),
                ("len_max", i32), ("seed", u64), ("threads", i32)]


class Params(C.Structure):
    _fields_ = [("k", i32), ("alpha", f32), ("beta", f32), ("seed", u64), ("device", i32), ("group_lanes", i32),
                ("item_tokens", i32), ("flags", i32), ("sample_blocks", i32), ("theta_min_len", i32)]


class IterStats(C.Structure):
    _fields_ = [("iteration", i32), ("status", i32), ("seconds", f64), ("loglik", f64), ("tokens_per_sec", f64),
                ("row_entries", i64), ("theta_nnz", i64), ("token_nnz", i64), ("sample_seconds", f64),
                ("rebuild_seconds", f64), ("accept_rate", f64)]


class Info(C.Structure):
    _fields_ = [("num_items", i32), ("num_hot", i32), ("num_hot_items", i32), ("item_tokens", i32),
                ("group_lanes", i32), ("sample_grid", i32), ("sample_blocks", i32), ("theta_grid", i32),
                ("kernels_per_iteration", i32),
                ("theta_capacity", i64), ("device_bytes", i64), ("doc_term", f64), ("tuned", i32),
                ("tune_ms", f32), ("theta_min_len", i32), ("theta_long_docs", i32), ("theta_tune_ms", f32)]


class Item(C.Structure):
    _fields_ = [("begin", i64), ("count", i32), ("word", i32), ("hot", i32), ("first", i32), ("seg_begin", i32),
                ("seg_count", i32)]


class SampleArgs(C.Structure):
    _fields_ = [("k", i32), ("alpha", f32), ("beta", f32), ("num_docs", i32), ("num_words", i32),
                ("num_tokens", i64), ("word_ptr", C.c_void_p), ("doc_ids", C.c_void_p), ("topics_in", C.c_void_p),
                ("topics_out", C.c_void_p), ("theta", C.c_void_p), ("theta_rows", C.c_void_p), ("nk", C.c_void_p),
                ("items", C.c_void_p), ("seg_start", C.c_void_p), ("num_segs", i32), ("num_items", i32),
                ("num_hot", i32),
                ("hot_items", C.c_void_p),
                ("num_hot_items", i32), ("theta_capacity", i64), ("seed", u64), ("iteration", u32),
                ("group_lanes", i32), ("loglik_sum", C.c_void_p), ("error", C.c_void_p)]


# every symbol the header declares, with its signature
CULDA_GEMM_F32, CULDA_GEMM_BIAS_GELU, CULDA_GEMM_GELU_BWD = 0, 1, 2


class GemmArgs(C.Structure):
    _fields_ = [("m", i32), ("n", i32), ("k", i32), ("a", C.c_void_p), ("lda", i32), ("b", C.c_void_p),
                ("ldb", i32), ("epilogue", i32), ("alpha", f32), ("out_f32", C.c_void_p), ("out_bf16", C.c_void_p),
                ("out_bf16_t", C.c_void_p), ("ldo", i32), ("ld_t", i32), ("bias", C.c_void_p), ("pre", C.c_void_p),
                ("colsum", C.c_void_p), ("error", C.c_void_p), ("k_splits", i32)]


CULDA_ENC_EMBED, CULDA_ENC_HIDDEN = 256, 512
CULDA_ENC_E, CULDA_ENC_W1, CULDA_ENC_B1, CULDA_ENC_W2, CULDA_ENC_B2, CULDA_ENC_W3, CULDA_ENC_B3 = range(7)
CULDA_ENC_GRAD = 16


class EncoderParams(C.Structure):
    _fields_ = [("num_words", i32), ("k", i32), ("max_batch", i32), ("device", i32), ("seed", u64), ("lr", f32),
                ("beta1", f32), ("beta2", f32), ("eps", f32)]


SIGNATURES = {
    "culda_status_string": (C.c_char_p, [C.c_int]),
    "culda_version": (C.c_char_p, []),
    "culda_corpus_generate": (C.c_int, [P(GenParams), P(P(Corpus))]),
    "culda_corpus_load": (C.c_int, [C.c_char_p, C.c_int, P(P(Corpus))]),
    "culda_corpus_write": (C.c_int, [P(Corpus), C.c_char_p, C.c_int]),
    "culda_corpus_write_text": (C.c_int, [P(Corpus), C.c_char_p]),
    "culda_corpus_free": (None, [P(Corpus)]),
    "culda_corpus_doc_tokens": (C.c_int, [P(Corpus), P(i32)]),
    "culda_vocab_free": (None, [P(Vocab)]),
    "culda_corpus_from_text": (C.c_int, [C.c_char_p, i32, P(P(Corpus)), P(P(Vocab))]),
    "culda_format_write": (C.c_int, [P(Corpus), P(Vocab), C.c_char_p, C.c_int]),
    "culda_format_text": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, i32]),
    "culda_create": (C.c_int, [P(Corpus), P(Params), P(C.c_void_p)]),
    "culda_iterate": (C.c_int, [C.c_void_p, C.c_int, P(IterStats)]),
    "culda_set_topics": (C.c_int, [C.c_void_p, P(u16)]),
    "culda_get_topics": (C.c_int, [C.c_void_p, P(u16)]),
    "culda_get_phi": (C.c_int, [C.c_void_p, P(i32), P(i32)]),
    "culda_get_theta": (C.c_int, [C.c_void_p, P(C.c_int16), P(C.c_int16), P(i32), P(i32)]),
    "culda_theta_capacity": (i64, [C.c_void_p]),
    "culda_num_tokens": (i64, [C.c_void_p]),
    "culda_sample_snapshot": (C.c_int, [C.c_void_p, u32, P(u16), P(f64)]),
    "culda_loglik_joint": (C.c_int, [C.c_void_p, P(f64)]),
    "culda_get_info": (C.c_int, [C.c_void_p, P(Info)]),
    "culda_last_error": (C.c_char_p, [C.c_void_p]),
    "culda_destroy": (None, [C.c_void_p]),
    "culda_trim_memory": (C.c_int, [i32]),
    "culda_build_items": (i64, [i32, P(i64), i32, P(Item), i64, P(i32)]),
    "culda_build_segments": (i64, [i64, P(i32), P(Item), i32, i32, P(i32), i64]),
    "culda_update_phi": (C.c_int, [i32, i32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "culda_compute_phi_head": (C.c_int, [i32, f32, i32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "culda_update_theta_workspace": (C.c_size_t, [i32, i32]),
    "culda_update_theta": (C.c_int, [i32, i32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "culda_sample_workspace": (C.c_size_t, [i32, i32, i32]),
    "culda_sample": (C.c_int, [P(SampleArgs), C.c_void_p, C.c_size_t, C.c_void_p]),
    "culda_sample_noalloc": (C.c_int, [P(SampleArgs), C.c_void_p]),
    "culda_loglik": (C.c_int, [C.c_void_p, f64, i64, P(f64), C.c_void_p]),
    "culda_gemm_bf16": (C.c_int, [P(GemmArgs), C.c_void_p]),
    "culda_encoder_create": (C.c_int, [P(EncoderParams), P(C.c_void_p)]),
    "culda_encoder_destroy": (C.c_int, [C.c_void_p]),
    "culda_encoder_tensor_size": (i64, [C.c_void_p, i32]),
    "culda_encoder_get_tensor": (C.c_int, [C.c_void_p, i32, C.c_void_p]),
    "culda_encoder_set_tensor": (C.c_int, [C.c_void_p, i32, C.c_void_p]),
    "culda_encoder_forward": (C.c_int, [C.c_void_p, i32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "culda_encoder_backward": (C.c_int, [C.c_void_p, i32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, P(f64),
                                         C.c_void_p]),
    "culda_encoder_train_step": (C.c_int, [C.c_void_p, i32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           P(f64), C.c_void_p]),
    "culda_accumulate_theta": (C.c_int, [C.c_void_p]),
    "culda_train_encoder": (C.c_int, [C.c_void_p, C.c_void_p, i32, u64, P(f64)]),
    "culda_encoder_init_from_phi": (C.c_int, [C.c_void_p, C.c_void_p, u64]),
    "culda_set_proposal": (C.c_int, [C.c_void_p, C.c_void_p, f32]),
    "culda_get_proposal": (C.c_int, [C.c_void_p, C.c_void_p]),
    "culda_iterate_mh": (C.c_int, [C.c_void_p, i32, i32, P(IterStats)]),
    "culda_mh_snapshot": (C.c_int, [C.c_void_p, u32, i32, C.c_void_p]),
    "culda_set_frozen_phi": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "culda_next_iteration": (u32, [C.c_void_p]),
    "culda_set_iteration": (C.c_int, [C.c_void_p, u32]),
    "culda_warm_start": (C.c_int, [C.c_void_p]),
    "culda_count_phi": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "culda_set_shared_phi": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise RuntimeError(f"{_LIB_PATH} is missing: run `python -m culda_cgs_b200.build` "
                               "(the sampler has no fallback path)")
        h = C.CDLL(str(_LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def library_path() -> Path:
    return _LIB_PATH


class CuldaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} [{lib().culda_status_string(status).decode()}]")
        self.status = status


def check(status: int, ctx=None) -> None:
    if status != CULDA_OK:
        msg = lib().culda_last_error(ctx)
        raise CuldaError(status, msg.decode() if msg else "")
