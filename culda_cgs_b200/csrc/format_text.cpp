// format_text.cpp — a text corpus turned into CuLDA_CGS's word-first corpus on
// all host cores: the job of the reference's preprocessing tool
// (src_format/format.cpp:56-165), with the same output bytes.
//
// Input: one document per line (lines end at '\n').  A line's first
// whitespace-separated field is the document's title and is dropped; the other
// fields are its tokens; a line with no field at all is not a document
// (src_format/format.cpp:64-70).  Whitespace is the C locale's isspace set
// (space, \t \n \v \f \r), the set `istringstream >> string` splits on.  Word
// ids follow the order in which tokens first appear in the file
// (src_culda/model/vocab.cpp:24-31); each word's doc list holds one entry per
// occurrence, docs ascending (src_format/format.cpp:77-84).
//
// Parallel plan: the file is cut at line starts into one byte range per
// thread.  Each thread parses its range with a private open-addressing token
// table that numbers words by first appearance inside the range, and counts
// its tokens per local word.  The tables are then merged in range order: a
// word that is new to the merged table when range t is merged first appears in
// range t, at its local position, so the merged numbering is the file's
// first-appearance order.  A stable counting sort by word (per-range cursors
// laid out in range order) writes the word-major doc ids with docs ascending.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/culda_b200.h"
#include "internal.h"

namespace culda {
namespace {

inline bool is_space(unsigned char ch) { return ch == ' ' || (ch >= '\t' && ch <= '\r'); }

// 64-bit hash of a byte string: 8-byte words folded by multiply-xorshift, then
// the MurmurHash3 64-bit finaliser.
inline uint64_t token_hash(const char *p, uint32_t n) {
    uint64_t h = 0x9E3779B97F4A7C15ull ^ (uint64_t(n) * 0xC2B2AE3D27D4EB4Full);
    while (n >= 8) {
        uint64_t w;
        memcpy(&w, p, 8);
        h = (h ^ w) * 0xFF51AFD7ED558CCDull;
        h ^= h >> 32;
        p += 8;
        n -= 8;
    }
    if (n) {
        uint64_t w = 0;
        memcpy(&w, p, n);
        h = (h ^ w) * 0xFF51AFD7ED558CCDull;
        h ^= h >> 32;
    }
    h ^= h >> 33;
    h *= 0xC4CEB9FE1A85EC53ull;
    h ^= h >> 33;
    return h;
}

// Open-addressing (linear probing) map from a token's bytes to its id.  Keys
// point into the input buffer, which outlives the table.
class TokenTable {
  public:
    explicit TokenTable(size_t cap = 1 << 12) { reset(cap); }

    // Id of the token, or -1 with the free slot to insert at in *where.
    int32_t find(const char *p, uint32_t len, uint64_t h, size_t *where) const {
        size_t i = h & mask_;
        for (;;) {
            const Slot &s = slots_[i];
            if (!s.p) {
                *where = i;
                return -1;
            }
            if (s.hash == h && s.len == len && memcmp(s.p, p, len) == 0) return s.id;
            i = (i + 1) & mask_;
        }
    }

    void insert_at(size_t where, const char *p, uint32_t len, uint64_t h, int32_t id) {
        slots_[where] = Slot{h, p, len, id};
        if (++used_ * 2 > slots_.size()) grow();
    }

  private:
    struct Slot {
        uint64_t hash;
        const char *p;  // nullptr marks a free slot (tokens are never empty)
        uint32_t len;
        int32_t id;
    };
    std::vector<Slot> slots_;
    size_t mask_ = 0, used_ = 0;

    void reset(size_t cap) {
        slots_.assign(cap, Slot{0, nullptr, 0, -1});
        mask_ = cap - 1;
        used_ = 0;
    }
    void grow() {
        std::vector<Slot> old;
        old.swap(slots_);
        reset(old.size() * 2);
        for (const Slot &s : old) {
            if (!s.p) continue;
            size_t i = s.hash & mask_;
            while (slots_[i].p) i = (i + 1) & mask_;
            slots_[i] = s;
            ++used_;
        }
    }
};

// What one thread learns from its byte range.
struct RangeParse {
    std::vector<int32_t> tok;       // local word id of every token, in text order
    std::vector<int64_t> doc_len;   // tokens of every document, in text order
    std::vector<const char *> wp;   // local words in first-appearance order: bytes,
    std::vector<uint32_t> wl;       //   length
    std::vector<uint64_t> wh;       //   and hash
    std::vector<int64_t> cnt;       // tokens per local word
    bool too_long = false;          // a token of 4 GiB or more
};

void parse_range(const char *b, const char *e, RangeParse &out) {
    TokenTable tab;
    const char *p = b;
    while (p < e) {
        const char *eol = (const char *)memchr(p, '\n', (size_t)(e - p));
        if (!eol) eol = e;
        while (p < eol && is_space((unsigned char)*p)) ++p;
        if (p == eol) {  // no title: not a document (format.cpp:69)
            p = eol < e ? eol + 1 : e;
            continue;
        }
        while (p < eol && !is_space((unsigned char)*p)) ++p;  // the title
        int64_t n = 0;
        for (;;) {
            while (p < eol && is_space((unsigned char)*p)) ++p;
            if (p == eol) break;
            const char *s = p;
            while (p < eol && !is_space((unsigned char)*p)) ++p;
            if ((uint64_t)(p - s) > UINT32_MAX) {
                out.too_long = true;
                return;
            }
            uint32_t len = (uint32_t)(p - s);
            uint64_t h = token_hash(s, len);
            size_t where;
            int32_t id = tab.find(s, len, h, &where);
            if (id < 0) {
                id = (int32_t)out.wp.size();
                tab.insert_at(where, s, len, h, id);
                out.wp.push_back(s);
                out.wl.push_back(len);
                out.wh.push_back(h);
                out.cnt.push_back(0);
            }
            out.tok.push_back(id);
            ++out.cnt[(size_t)id];
            ++n;
        }
        out.doc_len.push_back(n);
        p = eol < e ? eol + 1 : e;
    }
}

// Range starts: equal byte shares moved forward to the next line start.
std::vector<size_t> line_aligned_bounds(const std::vector<char> &buf, int parts) {
    size_t size = buf.size();
    std::vector<size_t> b((size_t)parts + 1, size);
    b[0] = 0;
    for (int i = 1; i < parts; ++i) {
        size_t pos = std::max(b[(size_t)i - 1], size / (size_t)parts * (size_t)i);
        if (pos > 0 && pos < size && buf[pos - 1] != '\n') {
            const char *nl = (const char *)memchr(buf.data() + pos, '\n', size - pos);
            pos = nl ? (size_t)(nl - buf.data()) + 1 : size;
        }
        b[(size_t)i] = std::min(pos, size);
    }
    return b;
}

template <class T>
T *copy_out(const std::vector<T> &v) {
    T *p = (T *)malloc(std::max<size_t>(1, v.size()) * sizeof(T));
    if (p && !v.empty()) memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

}  // namespace
}  // namespace culda

using namespace culda;

extern "C" void culda_vocab_free(culda_vocab *v) {
    if (!v) return;
    free(v->offsets);
    free(v->bytes);
    free(v);
}

extern "C" int culda_corpus_from_text(const char *path, int32_t threads, culda_corpus **corpus_out,
                                      culda_vocab **vocab_out) {
    if (!path || !corpus_out) {
        set_global_error("culda_corpus_from_text: null argument");
        return CULDA_ERR_INVALID_ARG;
    }
    *corpus_out = nullptr;
    if (vocab_out) *vocab_out = nullptr;
    std::vector<char> buf;
    if (!read_file_bytes(path, buf)) {
        set_global_error("%s open failed", path);  // format.cpp:33-36
        return CULDA_ERR_IO;
    }
    int nt = threads > 0 ? threads : omp_get_max_threads();
    // at least 1 MiB of text per range
    nt = (int)std::max<size_t>(1, std::min<size_t>((size_t)nt, buf.size() >> 20));
    std::vector<size_t> bounds = line_aligned_bounds(buf, nt);
    std::vector<RangeParse> parts((size_t)nt);
#pragma omp parallel for num_threads(nt) schedule(static, 1)
    for (int t = 0; t < nt; ++t)
        parse_range(buf.data() + bounds[(size_t)t], buf.data() + bounds[(size_t)t + 1], parts[(size_t)t]);

    int64_t num_docs = 0, num_tokens = 0;
    for (const RangeParse &r : parts) {
        if (r.too_long) {
            set_global_error("%s: a token of 4 GiB or more", path);
            return CULDA_ERR_INVALID_ARG;
        }
        num_docs += (int64_t)r.doc_len.size();
        num_tokens += (int64_t)r.tok.size();
    }
    if (num_docs > INT32_MAX) {
        set_global_error("%s: %lld documents, more than int32 doc ids hold", path, (long long)num_docs);
        return CULDA_ERR_INVALID_ARG;
    }

    // Merge in range order: global first-appearance ids and word totals.
    TokenTable global;
    std::vector<const char *> gp;
    std::vector<uint32_t> gl;
    std::vector<int64_t> gcnt;
    std::vector<std::vector<int32_t>> remap((size_t)nt);
    for (int t = 0; t < nt; ++t) {
        const RangeParse &r = parts[(size_t)t];
        std::vector<int32_t> &m = remap[(size_t)t];
        m.resize(r.wp.size());
        for (size_t j = 0; j < r.wp.size(); ++j) {
            size_t where;
            int32_t id = global.find(r.wp[j], r.wl[j], r.wh[j], &where);
            if (id < 0) {
                if (gp.size() >= (size_t)INT32_MAX) {
                    set_global_error("%s: more distinct tokens than int32 word ids hold", path);
                    return CULDA_ERR_INVALID_ARG;
                }
                id = (int32_t)gp.size();
                global.insert_at(where, r.wp[j], r.wl[j], r.wh[j], id);
                gp.push_back(r.wp[j]);
                gl.push_back(r.wl[j]);
                gcnt.push_back(0);
            }
            m[j] = id;
            gcnt[(size_t)id] += r.cnt[j];
        }
    }
    const int32_t V = (int32_t)gp.size();

    std::vector<int64_t> word_ptr((size_t)V + 1, 0);
    for (int32_t w = 0; w < V; ++w) word_ptr[(size_t)w + 1] = word_ptr[(size_t)w] + gcnt[(size_t)w];
    std::vector<int64_t> doc_ptr((size_t)num_docs + 1, 0);
    std::vector<int32_t> doc_base((size_t)nt + 1, 0);
    {
        int64_t d = 0;
        for (int t = 0; t < nt; ++t) {
            doc_base[(size_t)t] = (int32_t)d;
            for (int64_t len : parts[(size_t)t].doc_len) {
                doc_ptr[(size_t)d + 1] = doc_ptr[(size_t)d] + len;
                ++d;
            }
        }
        doc_base[(size_t)nt] = (int32_t)d;
    }
    // Per-range start of each local word inside its global word's doc list:
    // earlier ranges (earlier docs) first, which keeps every list ascending.
    std::vector<std::vector<int64_t>> cursor((size_t)nt);
    {
        std::vector<int64_t> run(word_ptr.begin(), word_ptr.end() - 1);
        for (int t = 0; t < nt; ++t) {
            const RangeParse &r = parts[(size_t)t];
            std::vector<int64_t> &c = cursor[(size_t)t];
            c.resize(r.wp.size());
            for (size_t j = 0; j < r.wp.size(); ++j) {
                int32_t w = remap[(size_t)t][j];
                c[j] = run[(size_t)w];
                run[(size_t)w] += r.cnt[j];
            }
        }
    }
    int32_t *doc_ids = (int32_t *)malloc((size_t)std::max<int64_t>(1, num_tokens) * sizeof(int32_t));
    if (!doc_ids) {
        set_global_error("culda_corpus_from_text: out of host memory");
        return CULDA_ERR_OOM;
    }
#pragma omp parallel for num_threads(nt) schedule(static, 1)
    for (int t = 0; t < nt; ++t) {
        const RangeParse &r = parts[(size_t)t];
        std::vector<int64_t> &c = cursor[(size_t)t];
        size_t k = 0;
        int32_t d = doc_base[(size_t)t];
        for (int64_t len : r.doc_len) {
            for (int64_t i = 0; i < len; ++i, ++k) doc_ids[c[(size_t)r.tok[k]]++] = d;
            ++d;
        }
    }

    culda_corpus *c = (culda_corpus *)calloc(1, sizeof(culda_corpus));
    culda_vocab *v = vocab_out ? (culda_vocab *)calloc(1, sizeof(culda_vocab)) : nullptr;
    if (c) {
        c->owned = 1;
        c->num_docs = (int32_t)num_docs;
        c->num_words = V;
        c->num_tokens = num_tokens;
        c->doc_ptr = copy_out(doc_ptr);
        c->word_ptr = copy_out(word_ptr);
        c->doc_ids = doc_ids;
        doc_ids = nullptr;
    }
    bool ok = c && c->doc_ptr && c->word_ptr && (!vocab_out || v);
    if (ok && v) {
        std::vector<int64_t> off((size_t)V + 1, 0);
        for (int32_t w = 0; w < V; ++w) off[(size_t)w + 1] = off[(size_t)w] + gl[(size_t)w];
        v->num_words = V;
        v->offsets = copy_out(off);
        v->bytes = (char *)malloc((size_t)std::max<int64_t>(1, off[(size_t)V]));
        ok = v->offsets && v->bytes;
        if (ok)
            for (int32_t w = 0; w < V; ++w) memcpy(v->bytes + off[(size_t)w], gp[(size_t)w], gl[(size_t)w]);
    }
    free(doc_ids);
    if (!ok) {
        culda_corpus_free(c);
        culda_vocab_free(v);
        set_global_error("culda_corpus_from_text: out of host memory");
        return CULDA_ERR_OOM;
    }
    *corpus_out = c;
    if (vocab_out) *vocab_out = v;
    return CULDA_OK;
}

extern "C" int culda_format_text(const char *in_path, const char *out_prefix, int num_chunks, int32_t threads) {
    if (!in_path || !out_prefix) {
        set_global_error("culda_format_text: null argument");
        return CULDA_ERR_INVALID_ARG;
    }
    culda_corpus *c = nullptr;
    culda_vocab *v = nullptr;
    int rc = culda_corpus_from_text(in_path, threads, &c, &v);
    if (rc != CULDA_OK) return rc;
    rc = culda_format_write(c, v, out_prefix, num_chunks);
    culda_corpus_free(c);
    culda_vocab_free(v);
    return rc;
}
