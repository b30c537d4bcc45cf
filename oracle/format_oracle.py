"""TEST INFRASTRUCTURE ONLY: pure-Python restatement of the reference's
preprocessing tool, the checker of culda_format_text / the `format` command.

Only tests/ import this module.  It follows src_format/format.cpp and
src_format/data_chunk.h step by step, for the small inputs the tests use:

- lines come from `getline` (split at b"\\n"); a line whose first
  `istringstream >> string` field is missing is skipped (format.cpp:64-70);
  fields are separated by the C locale's whitespace, the same set as
  `bytes.split()` (space, \\t \\n \\v \\f \\r);
- a token gets the next id the first time it is seen (vocab.cpp:24-31,
  format.cpp:75-76) and its doc id is appended once per occurrence
  (format.cpp:77-84);
- `.doc.idx` holds "docId tokensSoFar" per document (format.cpp:86);
- `.vocab` holds "token id" per word in id order (format.cpp:96-99);
- documents go to chunks in order until a chunk reaches
  ceil(numTokens / numChunks) tokens (format.cpp:104-132), `.chunk` holds
  "chunkId docIdEnd" per chunk;
- per chunk, `.word.idx` holds "wordId cumulativeEntries" for every word and
  `.word.data` the int32 doc ids, word-major (data_chunk.h:49-67), with the
  chunk id appended to both names when numChunks > 1 (data_chunk.h:35-43).
"""
from __future__ import annotations

import struct


def format_files(text: bytes, num_chunks: int = 1) -> dict[str, bytes]:
    """File suffix (".vocab", ".word.data0", ...) -> the bytes the tool writes."""
    num_chunks = max(1, int(num_chunks))  # format.cpp:27-28
    ids: dict[bytes, int] = {}
    words: list[bytes] = []
    word_docs: list[list[int]] = []
    doc_len: list[int] = []
    doc_idx = []
    n_tokens = 0
    for line in text.split(b"\n"):
        fields = line.split()
        if not fields:
            continue
        d = len(doc_len)
        for tok in fields[1:]:
            w = ids.get(tok)
            if w is None:
                w = ids[tok] = len(words)
                words.append(tok)
                word_docs.append([])
            word_docs[w].append(d)
            n_tokens += 1
        doc_idx.append(b"%d %d\n" % (d, n_tokens))
        doc_len.append(len(fields) - 1)

    out = {".vocab": b"".join(b"%s %d\n" % (t, i) for i, t in enumerate(words)), ".doc.idx": b"".join(doc_idx)}
    per_chunk = (n_tokens + num_chunks - 1) // num_chunks
    chunk_of = []
    chunk_lines = []
    d = 0
    for ch in range(num_chunks):
        size = 0
        while d < len(doc_len):
            size += doc_len[d]
            chunk_of.append(ch)
            d += 1
            if size >= per_chunk:
                break
        chunk_lines.append(b"%d %d\n" % (ch, d))
    out[".chunk"] = b"".join(chunk_lines)
    for ch in range(num_chunks):
        suffix = str(ch) if num_chunks > 1 else ""
        idx, data, off = [], [], 0
        for w in range(len(words)):
            mine = [doc for doc in word_docs[w] if chunk_of[doc] == ch]
            off += len(mine)
            idx.append(b"%d %d\n" % (w, off))
            data.append(struct.pack("<%di" % len(mine), *mine))
        out[".word.idx" + suffix] = b"".join(idx)
        out[".word.data" + suffix] = b"".join(data)
    return out
