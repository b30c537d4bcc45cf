"""Corpus in CuLDA_CGS's word-first format, backed by the C ABI.

Mirrors the reference's `Document` (src_culda/model/doc.h:20-50):
`Document.loadDocument(prefix, numChunks)` reads the src_format files and
exposes numDocs / numWords / numTokens; the arrays are the reference's
docIndices (doc_ptr), wordIndices (word_ptr) and wordTokens (doc_ids).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _ffi
from ._ffi import check, lib


@dataclass(frozen=True)
class GenConfig:
    """Parameters of the seeded synthetic LDA corpus (culda_gen_params)."""
    num_words: int
    num_topics: int
    num_docs: int
    len_law: int = _ffi.CULDA_LEN_POISSON
    len_a: float = 100.0
    len_b: float = 0.0
    len_min: int = 10
    len_max: int = 1000
    zipf_s: float = 1.05
    word_conc: float = 0.1
    doc_conc: float = 0.1
    seed: int = 1
    threads: int = 0

    def to_c(self) -> _ffi.GenParams:
        return _ffi.GenParams(self.num_words, self.num_topics, self.num_docs, self.len_law, self.zipf_s,
                              self.word_conc, self.doc_conc, self.len_a, self.len_b, self.len_min, self.len_max,
                              self.seed, self.threads)


class Corpus:
    """A corpus owned by the library (culda_corpus)."""

    def __init__(self, ptr: C.POINTER(_ffi.Corpus)):
        self._ptr = ptr
        self._vocab = None  # culda_vocab of a corpus read from text
        c = ptr.contents
        self.num_docs = int(c.num_docs)
        self.num_words = int(c.num_words)
        self.num_tokens = int(c.num_tokens)

    # --- construction
    @classmethod
    def generate(cls, cfg: GenConfig) -> "Corpus":
        out = C.POINTER(_ffi.Corpus)()
        p = cfg.to_c()
        check(lib().culda_corpus_generate(C.byref(p), C.byref(out)))
        return cls(out)

    @classmethod
    def load(cls, prefix: str, num_chunks: int = 1) -> "Corpus":
        out = C.POINTER(_ffi.Corpus)()
        check(lib().culda_corpus_load(str(prefix).encode(), int(num_chunks), C.byref(out)))
        return cls(out)

    @classmethod
    def from_text(cls, path: str, threads: int = 0) -> "Corpus":
        """Parse a text corpus, one document per line: a title field, then the
        document's tokens (src_format/format.cpp:64-90).  Word ids follow first
        appearance; the token strings are in `vocab`."""
        out = C.POINTER(_ffi.Corpus)()
        voc = C.POINTER(_ffi.Vocab)()
        check(lib().culda_corpus_from_text(str(path).encode(), int(threads), C.byref(out), C.byref(voc)))
        c = cls(out)
        c._vocab = voc
        return c

    @property
    def vocab(self) -> list[str] | None:
        """Token strings by word id (None unless the corpus was read from text);
        bytes that are not UTF-8 are kept as surrogate escapes."""
        if not self._vocab:
            return None
        v = self._vocab.contents
        off = np.ctypeslib.as_array(v.offsets, shape=(v.num_words + 1,))
        raw = C.string_at(v.bytes, int(off[-1])) if off[-1] else b""
        return [raw[off[i]:off[i + 1]].decode("utf-8", "surrogateescape") for i in range(v.num_words)]

    @classmethod
    def from_arrays(cls, doc_ptr, word_ptr, doc_ids) -> "BorrowedCorpus":
        return BorrowedCorpus(doc_ptr, word_ptr, doc_ids)

    # --- I/O
    def write(self, prefix: str, num_chunks: int = 1) -> None:
        """The src_format files; `.vocab` holds the token strings of a corpus
        read from text, else "w<label>" names."""
        if self._vocab:
            check(lib().culda_format_write(self._ptr, self._vocab, str(prefix).encode(), int(num_chunks)))
        else:
            check(lib().culda_corpus_write(self._ptr, str(prefix).encode(), int(num_chunks)))

    def write_text(self, path: str) -> None:
        check(lib().culda_corpus_write_text(self._ptr, str(path).encode()))

    # --- arrays (copies)
    @property
    def doc_ptr(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._ptr.contents.doc_ptr, shape=(self.num_docs + 1,)).copy()

    @property
    def word_ptr(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._ptr.contents.word_ptr, shape=(self.num_words + 1,)).copy()

    @property
    def doc_ids(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._ptr.contents.doc_ids, shape=(self.num_tokens,)).copy()

    def split_docs(self, docs) -> "BorrowedCorpus":
        """The corpus restricted to the given docs (renumbered 0.. in the given
        order) over the same vocabulary: word ids and V are kept, so a model
        trained on the other docs applies to it (fold-in of held-out docs)."""
        docs = np.asarray(docs, dtype=np.int64)
        remap = np.full(self.num_docs, -1, dtype=np.int64)
        remap[docs] = np.arange(len(docs))
        ids = self.doc_ids
        word_of = np.repeat(np.arange(self.num_words), np.diff(self.word_ptr))
        keep = remap[ids] >= 0
        new_ids = remap[ids[keep]]
        new_words = word_of[keep]
        order = np.lexsort((new_ids, new_words))  # word-major, ascending doc id within a word
        new_ids = new_ids[order].astype(np.int32)
        counts = np.bincount(new_words, minlength=self.num_words)
        word_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        lens = np.diff(self.doc_ptr)[docs]
        doc_ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        return BorrowedCorpus(doc_ptr, word_ptr, new_ids)

    def doc_tokens(self) -> np.ndarray:
        """docRevIdx: word-major token ids grouped by doc (doc_chunk.cpp:225-255)."""
        out = np.empty(self.num_tokens, dtype=np.int32)
        check(lib().culda_corpus_doc_tokens(self._ptr, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    @property
    def doc_lengths(self) -> np.ndarray:
        return np.diff(self.doc_ptr)

    @property
    def c_ptr(self):
        return self._ptr

    # reference spellings
    @property
    def numDocs(self) -> int:  # noqa: N802
        return self.num_docs

    @property
    def numWords(self) -> int:  # noqa: N802
        return self.num_words

    @property
    def numTokens(self) -> int:  # noqa: N802
        return self.num_tokens

    def close(self) -> None:
        if self._ptr:
            lib().culda_corpus_free(self._ptr)
            self._ptr = None
        if getattr(self, "_vocab", None):
            lib().culda_vocab_free(self._vocab)
            self._vocab = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def format_text(in_path: str, out_prefix: str, num_chunks: int = 1, threads: int = 0) -> None:
    """The reference's `format input output_prefix numChunks` tool
    (src_format/format.cpp:19-165): text corpus in, the five word-first files
    out, byte-identical, parsed on `threads` host threads (0 = all)."""
    check(lib().culda_format_text(str(in_path).encode(), str(out_prefix).encode(), int(num_chunks), int(threads)))


class BorrowedCorpus(Corpus):
    """A corpus descriptor over caller-owned numpy arrays (not freed by the library)."""

    def __init__(self, doc_ptr, word_ptr, doc_ids):
        self._doc_ptr = np.ascontiguousarray(doc_ptr, dtype=np.int64)
        self._word_ptr = np.ascontiguousarray(word_ptr, dtype=np.int64)
        self._doc_ids = np.ascontiguousarray(doc_ids, dtype=np.int32)
        self._c = _ffi.Corpus(len(self._doc_ptr) - 1, len(self._word_ptr) - 1, len(self._doc_ids),
                              self._doc_ptr.ctypes.data_as(C.POINTER(C.c_int64)),
                              self._word_ptr.ctypes.data_as(C.POINTER(C.c_int64)),
                              self._doc_ids.ctypes.data_as(C.POINTER(C.c_int32)), None, 0)
        super().__init__(C.pointer(self._c))

    def close(self) -> None:
        self._ptr = None


class Document(Corpus):
    """Reference spelling: Document().loadDocument(prefix, numChunks)."""

    def __init__(self, ptr=None):
        if ptr is not None:
            super().__init__(ptr)
        else:
            self._ptr = None
            self.num_docs = self.num_words = self.num_tokens = 0

    def loadDocument(self, prefix: str, numChunks: int = 1) -> "Document":  # noqa: N802,N803
        c = Corpus.load(prefix, numChunks)
        self._ptr, c._ptr = c._ptr, None
        Corpus.__init__(self, self._ptr)
        return self
