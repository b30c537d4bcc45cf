"""B200-native collapsed-Gibbs LDA sampler, a drop-in for CuLDA_CGS's one-GPU path.

The compute path is hand-written sm_100a CUDA behind the C ABI in
include/culda_b200.h (libculda_b200.so); this package is a thin ctypes host
over it that mirrors the reference's host interface (Document, Argument,
LDATrain).
"""
from ._ffi import CULDA_FLAG_AUTOTUNE, CULDA_FLAG_NO_GRAPH, CULDA_FLAG_NO_REORDER, CULDA_FLAG_VERBOSE, CuldaError, lib, library_path
from .corpus import BorrowedCorpus, Corpus, Document, GenConfig, format_text
from .encoder import Encoder
from .lda import LDA, Argument, LDATrain

__all__ = ["CuldaError", "lib", "library_path", "Corpus", "BorrowedCorpus", "Document", "GenConfig", "format_text",
           "LDA", "Argument", "LDATrain", "Encoder"]
