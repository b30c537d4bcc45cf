// corpus.cpp — host side of the corpus: CuLDA_CGS's word-first files and a
// seeded synthetic LDA generator.
//
// File formats follow the reference's preprocessing tool and loader:
//   <prefix>.vocab       "token id" per word, id by first appearance   (src_format/format.cpp:75-76,97-99)
//   <prefix>.doc.idx     "docId cumulativeTokenEnd" per doc           (src_format/format.cpp:88)
//   <prefix>.chunk       "chunkId docEnd" per chunk                    (src_format/format.cpp:107-132)
//   <prefix>.word.idx    "wordId cumulativeTokenEnd" per word          (src_format/data_chunk.h:53-56)
//   <prefix>.word.data   int32 doc ids, word-major, docs ascending     (src_format/data_chunk.h:58-60)
// with a chunk-id suffix on the last two when there is more than one chunk
// (src_format/data_chunk.h:35-43, src_culda/model/doc.cpp:131-144).
#include <omp.h>

#include <algorithm>
#include <cerrno>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/culda_b200.h"
#include "internal.h"
#include "philox.h"

namespace culda {

// ------------------------------------------------------------------ errors
static thread_local std::string g_error;

void set_global_error(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
}

const char *global_error() { return g_error.c_str(); }

// ------------------------------------------------------------ file reading
bool read_file_bytes(const std::string &path, std::vector<char> &buf) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    if (fseek(f, 0, SEEK_END) != 0) {
        fclose(f);
        return false;
    }
    long sz = ftell(f);
    if (sz < 0) {
        fclose(f);
        return false;
    }
    rewind(f);
    buf.resize((size_t)sz + 1);
    size_t got = sz ? fread(buf.data(), 1, (size_t)sz, f) : 0;
    fclose(f);
    if (got != (size_t)sz) return false;
    buf[(size_t)sz] = '\0';
    buf.resize((size_t)sz);
    return true;
}

// Parse whitespace-separated integer pairs "a b" the way `stream >> a >> b`
// does: stop at the first token that is not an integer.
static void parse_pairs(const std::vector<char> &buf, std::vector<int64_t> &second) {
    const char *p = buf.data(), *end = buf.data() + buf.size();
    auto skip = [&]() {
        while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t' || *p == '\v' || *p == '\f')) ++p;
    };
    auto num = [&](int64_t &v) -> bool {
        skip();
        if (p >= end) return false;
        const char *q = p;
        bool neg = false;
        if (*q == '-' || *q == '+') neg = (*q++ == '-');
        if (q >= end || *q < '0' || *q > '9') return false;
        int64_t x = 0;
        while (q < end && *q >= '0' && *q <= '9') x = x * 10 + (*q++ - '0');
        v = neg ? -x : x;
        p = q;
        return true;
    };
    int64_t a, b;
    while (num(a) && num(b)) second.push_back(b);
}

static culda_corpus *new_corpus() {
    culda_corpus *c = (culda_corpus *)calloc(1, sizeof(culda_corpus));
    if (c) c->owned = 1;
    return c;
}

}  // namespace culda

using namespace culda;

extern "C" void culda_corpus_free(culda_corpus *c) {
    if (!c || !c->owned) return;
    free(c->doc_ptr);
    free(c->word_ptr);
    free(c->doc_ids);
    free(c->word_label);
    free(c);
}

// Checks shared by every corpus entry point: monotone prefixes that end at N,
// doc ids in range and doc lengths consistent with the token payload.
int culda::validate_corpus(const culda_corpus *c) {
    if (!c || c->num_docs <= 0 || c->num_words <= 0 || c->num_tokens <= 0 || !c->doc_ptr || !c->word_ptr ||
        !c->doc_ids) {
        set_global_error("corpus: empty or missing arrays");
        return CULDA_ERR_INVALID_ARG;
    }
    if (c->num_tokens >= (int64_t)INT32_MAX) {
        set_global_error("corpus: %lld tokens exceed the int32 token index", (long long)c->num_tokens);
        return CULDA_ERR_UNSUPPORTED;
    }
    if (c->doc_ptr[0] != 0 || c->word_ptr[0] != 0 || c->doc_ptr[c->num_docs] != c->num_tokens ||
        c->word_ptr[c->num_words] != c->num_tokens) {
        set_global_error("corpus: doc/word index totals (%lld, %lld) do not match %lld tokens",
                         (long long)c->doc_ptr[c->num_docs], (long long)c->word_ptr[c->num_words],
                         (long long)c->num_tokens);
        return CULDA_ERR_FORMAT;
    }
    for (int32_t d = 0; d < c->num_docs; ++d)
        if (c->doc_ptr[d + 1] < c->doc_ptr[d]) {
            set_global_error("corpus: doc index decreases at doc %d", d);
            return CULDA_ERR_FORMAT;
        }
    for (int32_t w = 0; w < c->num_words; ++w)
        if (c->word_ptr[w + 1] < c->word_ptr[w]) {
            set_global_error("corpus: word index decreases at word %d", w);
            return CULDA_ERR_FORMAT;
        }
    std::vector<int64_t> cnt((size_t)c->num_docs, 0);
    for (int64_t t = 0; t < c->num_tokens; ++t) {
        int32_t d = c->doc_ids[t];
        if (d < 0 || d >= c->num_docs) {
            set_global_error("corpus: token %lld has doc id %d outside [0, %d)", (long long)t, d, c->num_docs);
            return CULDA_ERR_FORMAT;
        }
        cnt[d]++;
    }
    for (int32_t d = 0; d < c->num_docs; ++d)
        if (cnt[d] != c->doc_ptr[d + 1] - c->doc_ptr[d]) {
            set_global_error("corpus: doc %d has %lld tokens in .word.data but length %lld in .doc.idx", d,
                             (long long)cnt[d], (long long)(c->doc_ptr[d + 1] - c->doc_ptr[d]));
            return CULDA_ERR_FORMAT;
        }
    return CULDA_OK;
}

extern "C" int culda_corpus_load(const char *prefix, int num_chunks, culda_corpus **out) {
    if (!prefix || !out) {
        set_global_error("culda_corpus_load: null argument");
        return CULDA_ERR_INVALID_ARG;
    }
    *out = nullptr;
    if (num_chunks != 1) {
        set_global_error("culda_corpus_load: %d chunks requested; only the one-GPU path (-c 1) is supported",
                         num_chunks);
        return CULDA_ERR_UNSUPPORTED;
    }
    std::string pre(prefix);
    std::vector<char> buf;
    // The reference opens the vocabulary first and stops when it is missing
    // (src_culda/main.cpp:172-173, src_culda/model/vocab.cpp:53-58); the
    // sampler itself never reads it.
    {
        FILE *f = fopen((pre + ".vocab").c_str(), "rb");
        if (!f) {
            set_global_error("Vocabulary file %s.vocab open failed", prefix);
            return CULDA_ERR_IO;
        }
        fclose(f);
    }
    std::vector<int64_t> doc_end, chunk_end, word_end;
    if (!read_file_bytes(pre + ".doc.idx", buf)) {
        set_global_error("File %s.doc.idx open failed", prefix);
        return CULDA_ERR_IO;
    }
    parse_pairs(buf, doc_end);
    if (!read_file_bytes(pre + ".chunk", buf)) {
        set_global_error("File %s.chunk open failed", prefix);
        return CULDA_ERR_IO;
    }
    parse_pairs(buf, chunk_end);
    if ((int)chunk_end.size() != num_chunks) {
        set_global_error("Error: numChunks(%d) does not match the chunk file", num_chunks);
        return CULDA_ERR_FORMAT;
    }
    if (!read_file_bytes(pre + ".word.idx", buf)) {
        set_global_error("File %s.word.idx open failed", prefix);
        return CULDA_ERR_IO;
    }
    parse_pairs(buf, word_end);
    std::vector<char> data;
    if (!read_file_bytes(pre + ".word.data", data)) {
        set_global_error("File %s.word.data open failed", prefix);
        return CULDA_ERR_IO;
    }
    if (doc_end.empty() || word_end.empty()) {
        set_global_error("corpus %s: empty doc or word index", prefix);
        return CULDA_ERR_FORMAT;
    }
    if (doc_end.size() >= (size_t)INT32_MAX || word_end.size() >= (size_t)INT32_MAX) {
        set_global_error("corpus %s: too many docs or words", prefix);
        return CULDA_ERR_UNSUPPORTED;
    }
    culda_corpus *c = new_corpus();
    if (!c) return CULDA_ERR_OOM;
    c->num_docs = (int32_t)doc_end.size();
    c->num_words = (int32_t)word_end.size();
    c->num_tokens = (int64_t)(data.size() / sizeof(int32_t));  // doc_chunk.cpp:143-144
    c->doc_ptr = (int64_t *)malloc(sizeof(int64_t) * (doc_end.size() + 1));
    c->word_ptr = (int64_t *)malloc(sizeof(int64_t) * (word_end.size() + 1));
    c->doc_ids = (int32_t *)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(c->num_tokens, 1));
    if (!c->doc_ptr || !c->word_ptr || !c->doc_ids) {
        culda_corpus_free(c);
        return CULDA_ERR_OOM;
    }
    c->doc_ptr[0] = 0;
    for (size_t i = 0; i < doc_end.size(); ++i) c->doc_ptr[i + 1] = doc_end[i];
    c->word_ptr[0] = 0;
    for (size_t i = 0; i < word_end.size(); ++i) c->word_ptr[i + 1] = word_end[i];
    if (c->num_tokens) memcpy(c->doc_ids, data.data(), sizeof(int32_t) * (size_t)c->num_tokens);
    if (chunk_end[0] != c->num_docs) {
        set_global_error("corpus %s: the one chunk ends at doc %lld but there are %d docs", prefix,
                         (long long)chunk_end[0], c->num_docs);
        culda_corpus_free(c);
        return CULDA_ERR_FORMAT;
    }
    int rc = validate_corpus(c);
    if (rc != CULDA_OK) {
        culda_corpus_free(c);
        return rc;
    }
    *out = c;
    return CULDA_OK;
}

// ---------------------------------------------------------------- writing
namespace {

// Buffered output file with a decimal integer formatter (the text files hold
// millions of "id value" lines).
class OutFile {
  public:
    explicit OutFile(const std::string &path) : f_(fopen(path.c_str(), "wb")) { buf_.reserve(kBuf); }
    ~OutFile() {
        if (f_) fclose(f_);
    }
    bool ok() const { return f_ != nullptr; }
    void put(const char *p, size_t n) {
        if (buf_.size() + n > kBuf) flush();
        if (n > kBuf) {
            if (fwrite(p, 1, n, f_) != n) bad_ = true;
            return;
        }
        buf_.insert(buf_.end(), p, p + n);
    }
    void put(char ch) { put(&ch, 1); }
    void put_int(int64_t v) {
        char tmp[24];
        char *e = tmp + sizeof(tmp), *p = e;
        uint64_t u = v < 0 ? 0 - (uint64_t)v : (uint64_t)v;
        do {
            *--p = char('0' + u % 10);
            u /= 10;
        } while (u);
        if (v < 0) *--p = '-';
        put(p, (size_t)(e - p));
    }
    // "a b\n", the `out << a << " " << b << endl` lines of the reference's files
    void pair_line(int64_t a, int64_t b) {
        put_int(a);
        put(' ');
        put_int(b);
        put('\n');
    }
    bool close() {
        if (!f_) return false;
        flush();
        bool good = !bad_ && ferror(f_) == 0;
        if (fclose(f_) != 0) good = false;
        f_ = nullptr;
        return good;
    }

  private:
    static constexpr size_t kBuf = 1 << 22;
    FILE *f_;
    std::vector<char> buf_;
    bool bad_ = false;
    void flush() {
        if (!buf_.empty() && fwrite(buf_.data(), 1, buf_.size(), f_) != buf_.size()) bad_ = true;
        buf_.clear();
    }
};

// The checks the writer needs: consistent prefixes and doc ids in range.
// Unlike validate_corpus it accepts empty corpora and any token count, as the
// reference's tool does.
int check_for_writing(const culda_corpus *c, const culda_vocab *v) {
    if (c->num_docs < 0 || c->num_words < 0 || c->num_tokens < 0 || !c->doc_ptr || !c->word_ptr ||
        (c->num_tokens > 0 && !c->doc_ids)) {
        set_global_error("corpus: negative sizes or missing arrays");
        return CULDA_ERR_INVALID_ARG;
    }
    if (v && (v->num_words != c->num_words || !v->offsets || (v->offsets[v->num_words] > 0 && !v->bytes))) {
        set_global_error("vocabulary: %d words for a corpus of %d", v->num_words, c->num_words);
        return CULDA_ERR_INVALID_ARG;
    }
    if (c->doc_ptr[0] != 0 || c->word_ptr[0] != 0 || c->doc_ptr[c->num_docs] != c->num_tokens ||
        c->word_ptr[c->num_words] != c->num_tokens) {
        set_global_error("corpus: doc/word index totals do not match %lld tokens", (long long)c->num_tokens);
        return CULDA_ERR_FORMAT;
    }
    for (int32_t w = 0; w < c->num_words; ++w)
        if (c->word_ptr[w + 1] < c->word_ptr[w]) {
            set_global_error("corpus: word index decreases at word %d", w);
            return CULDA_ERR_FORMAT;
        }
    for (int64_t t = 0; t < c->num_tokens; ++t)
        if (c->doc_ids[t] < 0 || c->doc_ids[t] >= c->num_docs) {
            set_global_error("corpus: token %lld has doc id %d outside [0, %d)", (long long)t, c->doc_ids[t],
                             c->num_docs);
            return CULDA_ERR_FORMAT;
        }
    return CULDA_OK;
}

}  // namespace

extern "C" int culda_format_write(const culda_corpus *c, const culda_vocab *vocab, const char *prefix,
                                  int num_chunks) {
    if (!c || !prefix) {
        set_global_error("culda_format_write: null argument");
        return CULDA_ERR_INVALID_ARG;
    }
    int rc = check_for_writing(c, vocab);
    if (rc != CULDA_OK) return rc;
    if (num_chunks <= 1) num_chunks = 1;  // src_format/format.cpp:27-28
    std::string pre(prefix);
    {
        OutFile f(pre + ".vocab");  // src_format/format.cpp:96-99
        if (!f.ok()) {
            set_global_error("%s.vocab open failed", prefix);
            return CULDA_ERR_IO;
        }
        for (int32_t w = 0; w < c->num_words; ++w) {
            if (vocab) {
                f.put(vocab->bytes + vocab->offsets[w], (size_t)(vocab->offsets[w + 1] - vocab->offsets[w]));
            } else {
                f.put('w');
                f.put_int(c->word_label ? c->word_label[w] : w);
            }
            f.put(' ');
            f.put_int(w);
            f.put('\n');
        }
        if (!f.close()) return CULDA_ERR_IO;
    }
    {
        OutFile f(pre + ".doc.idx");  // src_format/format.cpp:86
        if (!f.ok()) {
            set_global_error("%s.doc.idx open failed", prefix);
            return CULDA_ERR_IO;
        }
        for (int32_t d = 0; d < c->num_docs; ++d) f.pair_line(d, c->doc_ptr[d + 1]);
        if (!f.close()) return CULDA_ERR_IO;
    }
    // Doc -> chunk map by equal token counts (src_format/format.cpp:107-132).
    int64_t per_chunk = (c->num_tokens + num_chunks - 1) / num_chunks;
    std::vector<int32_t> chunk_start(num_chunks + 1, 0);
    {
        OutFile f(pre + ".chunk");
        if (!f.ok()) {
            set_global_error("%s.chunk open failed", prefix);
            return CULDA_ERR_IO;
        }
        int32_t d = 0;
        for (int ch = 0; ch < num_chunks; ++ch) {
            chunk_start[ch] = d;
            int64_t sz = 0;
            while (d < c->num_docs) {
                sz += c->doc_ptr[d + 1] - c->doc_ptr[d];
                ++d;
                if (sz >= per_chunk) break;
            }
            f.pair_line(ch, d);
        }
        chunk_start[num_chunks] = d;
        if (!f.close()) return CULDA_ERR_IO;
    }
    // Per chunk, every word's entries for the chunk's docs: a word's doc list
    // is ascending and a chunk is a doc range, so they are one contiguous run
    // (src_format/data_chunk.h:49-67 writes the same bytes from per-chunk lists).
    for (int ch = 0; ch < num_chunks; ++ch) {
        std::string idx_name = pre + ".word.idx", data_name = pre + ".word.data";
        if (num_chunks > 1) {
            idx_name += std::to_string(ch);
            data_name += std::to_string(ch);
        }
        OutFile fi(idx_name), fd(data_name);
        if (!fi.ok() || !fd.ok()) {
            set_global_error("%s open failed", (fi.ok() ? data_name : idx_name).c_str());
            return CULDA_ERR_IO;
        }
        const int32_t d0 = chunk_start[ch], d1 = chunk_start[ch + 1];
        int64_t off = 0;
        for (int32_t w = 0; w < c->num_words; ++w) {
            const int32_t *b = c->doc_ids + c->word_ptr[w], *e = c->doc_ids + c->word_ptr[w + 1];
            if (num_chunks > 1) {
                b = std::lower_bound(b, e, d0);
                e = std::lower_bound(b, e, d1);
            }
            off += e - b;
            if (e > b) fd.put((const char *)b, (size_t)(e - b) * sizeof(int32_t));
            fi.pair_line(w, off);
        }
        if (!fi.close() || !fd.close()) return CULDA_ERR_IO;
    }
    return CULDA_OK;
}

extern "C" int culda_corpus_write(const culda_corpus *c, const char *prefix, int num_chunks) {
    if (!c || !prefix) {
        set_global_error("culda_corpus_write: null argument");
        return CULDA_ERR_INVALID_ARG;
    }
    int rc = validate_corpus(c);
    if (rc != CULDA_OK) return rc;
    return culda_format_write(c, nullptr, prefix, num_chunks);
}

extern "C" int culda_corpus_write_text(const culda_corpus *c, const char *path) {
    if (!c || !path) return CULDA_ERR_INVALID_ARG;
    int rc = validate_corpus(c);
    if (rc != CULDA_OK) return rc;
    // Rebuild doc-major token lists.  Inside a doc the tokens come out in
    // ascending word id, which keeps the first-appearance id assignment of
    // src_format/format.cpp:75-76 identical to the corpus's own ids.
    std::vector<int64_t> cur(c->doc_ptr, c->doc_ptr + c->num_docs);
    std::vector<int32_t> words((size_t)c->num_tokens);
    for (int32_t w = 0; w < c->num_words; ++w)
        for (int64_t t = c->word_ptr[w]; t < c->word_ptr[w + 1]; ++t) words[cur[c->doc_ids[t]]++] = w;
    OutFile f(path);
    if (!f.ok()) {
        set_global_error("%s open failed", path);
        return CULDA_ERR_IO;
    }
    for (int32_t d = 0; d < c->num_docs; ++d) {
        f.put('d');
        f.put_int(d);
        for (int64_t i = c->doc_ptr[d]; i < c->doc_ptr[d + 1]; ++i) {
            f.put(" w", 2);
            f.put_int(c->word_label ? c->word_label[words[i]] : words[i]);
        }
        f.put('\n');
    }
    return f.close() ? CULDA_OK : CULDA_ERR_IO;
}

extern "C" int culda_corpus_doc_tokens(const culda_corpus *c, int32_t *doc_tok) {
    if (!c || !doc_tok) return CULDA_ERR_INVALID_ARG;
    std::vector<int64_t> cur(c->doc_ptr, c->doc_ptr + c->num_docs);
    for (int64_t t = 0; t < c->num_tokens; ++t) doc_tok[cur[c->doc_ids[t]]++] = (int32_t)t;
    return CULDA_OK;
}

// -------------------------------------------------------------- generator
namespace {

enum : uint32_t { kGenLen = 16, kGenTheta = 17, kGenTopic = 18, kGenPhi = 19, kGenWord = 20 };

// Sequential stream of Philox words for one (purpose, id) pair.
struct Stream {
    uint32_t k0, k1, id_lo, id_hi, purpose, ctr = 0;
    u32x4 buf;
    int pos = 4;
    Stream(uint64_t seed, uint32_t purpose_, uint64_t id)
        : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), id_lo((uint32_t)id), id_hi((uint32_t)(id >> 32)),
          purpose(purpose_) {}
    uint32_t next() {
        if (pos == 4) {
            u32x4 c = {id_lo, id_hi, ctr++, purpose};
            buf = philox4x32_10(c, k0, k1);
            pos = 0;
        }
        uint32_t v = pos == 0 ? buf.x : pos == 1 ? buf.y : pos == 2 ? buf.z : buf.w;
        ++pos;
        return v;
    }
    // 53-bit uniform in (0,1).
    double uniform() {
        uint64_t a = next() >> 5, b = next() >> 6;
        return ((double)(a * 67108864ull + b) + 0.5) * 0x1p-53;
    }
    // Box-Muller normal.
    double normal() {
        double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// log of a Gamma(a, 1) draw: Marsaglia and Tsang, "A Simple Method for
// Generating Gamma Variables" (ACM TOMS 26(3), 2000); shapes below one use
// their boost Gamma(a) = Gamma(a+1) * U^(1/a), kept in log space so tiny
// shapes do not underflow.
double log_gamma_draw(double a, Stream &s) {
    if (a < 1.0) return log_gamma_draw(a + 1.0, s) + std::log(s.uniform()) / a;
    const double d = a - 1.0 / 3.0, c = 1.0 / std::sqrt(9.0 * d);
    for (;;) {
        double x, v;
        do {
            x = s.normal();
            v = 1.0 + c * x;
        } while (v <= 0.0);
        v = v * v * v;
        double u = s.uniform();
        if (u < 1.0 - 0.0331 * x * x * x * x) return std::log(d * v);
        if (std::log(u) < 0.5 * x * x + d * (1.0 - v + std::log(v))) return std::log(d * v);
    }
}

// Dirichlet draw with concentrations conc[i] (or the scalar conc0 when conc
// is null) written as normalised probabilities.
void dirichlet_draw(int n, const double *conc, double conc0, Stream &s, double *out) {
    double mx = -INFINITY;
    for (int i = 0; i < n; ++i) {
        out[i] = log_gamma_draw(conc ? conc[i] : conc0, s);
        mx = std::max(mx, out[i]);
    }
    double sum = 0;
    for (int i = 0; i < n; ++i) {
        out[i] = std::exp(out[i] - mx);
        sum += out[i];
    }
    for (int i = 0; i < n; ++i) out[i] /= sum;
}

int64_t draw_length(const culda_gen_params *p, Stream &s) {
    double x = 0;
    if (p->len_law == CULDA_LEN_POISSON) {
        // inversion by sequential search (lambda <= 600 is checked by the caller)
        double u = s.uniform(), pk = std::exp(-p->len_a), F = pk;
        int64_t k = 0;
        while (u > F && k < 1000000) {
            ++k;
            pk *= p->len_a / (double)k;
            F += pk;
        }
        x = (double)k;
    } else if (p->len_law == CULDA_LEN_LOGNORMAL) {
        x = std::exp(p->len_a + p->len_b * s.normal());
    } else {
        x = p->len_b * std::pow(s.uniform(), -1.0 / p->len_a);
    }
    if (!(x < 4e18)) x = 4e18;
    int64_t l = (int64_t)std::llround(x);
    if (l < p->len_min) l = p->len_min;
    if (l > p->len_max) l = p->len_max;
    return l;
}

// Walker alias table built with Vose's method ("A Linear Algorithm for
// Generating Random Numbers with a Given Distribution", IEEE TSE 1991).
struct Alias {
    std::vector<double> thr;
    std::vector<int32_t> alias;
    std::vector<int32_t> small, large;
    void build(const double *p, int n) {
        thr.assign(n, 0.0);
        alias.assign(n, 0);
        small.clear();
        large.clear();
        for (int i = 0; i < n; ++i) {
            thr[i] = p[i] * n;
            (thr[i] < 1.0 ? small : large).push_back(i);
        }
        while (!small.empty() && !large.empty()) {
            int32_t s = small.back(), l = large.back();
            small.pop_back();
            large.pop_back();
            alias[s] = l;
            thr[l] = (thr[l] + thr[s]) - 1.0;
            (thr[l] < 1.0 ? small : large).push_back(l);
        }
        for (int32_t i : large) thr[i] = 1.0;
        for (int32_t i : small) thr[i] = 1.0;
    }
    int32_t draw(Stream &s, int n) const {
        int32_t i = (int32_t)bounded_from_bits(s.next(), (uint32_t)n);
        return s.uniform() < thr[i] ? i : alias[i];
    }
};

}  // namespace

extern "C" int culda_corpus_generate(const culda_gen_params *p, culda_corpus **out) {
    if (!p || !out) return CULDA_ERR_INVALID_ARG;
    *out = nullptr;
    if (p->num_words <= 0 || p->num_topics <= 0 || p->num_topics > 65535 || p->num_docs <= 0 || p->len_min < 1 ||
        p->len_max < p->len_min || p->word_conc <= 0 || p->doc_conc <= 0 || p->zipf_s < 0 ||
        p->len_law < 0 || p->len_law > 2 || (p->len_law == CULDA_LEN_POISSON && (p->len_a <= 0 || p->len_a > 600)) ||
        (p->len_law == CULDA_LEN_PARETO && (p->len_a <= 0 || p->len_b <= 0))) {
        set_global_error("culda_corpus_generate: invalid parameters");
        return CULDA_ERR_INVALID_ARG;
    }
    const int V = p->num_words, KG = p->num_topics, D = p->num_docs;
    int threads = p->threads > 0 ? p->threads : omp_get_max_threads();
    const uint64_t seed = p->seed;

    // 1. doc lengths
    std::vector<int64_t> doc_ptr((size_t)D + 1, 0);
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int d = 0; d < D; ++d) {
        Stream s(seed, kGenLen, (uint64_t)d);
        doc_ptr[(size_t)d + 1] = draw_length(p, s);
    }
    for (int d = 0; d < D; ++d) doc_ptr[(size_t)d + 1] += doc_ptr[d];
    const int64_t N = doc_ptr[D];
    if (N >= (int64_t)INT32_MAX) {
        set_global_error("culda_corpus_generate: %lld tokens exceed the int32 token index", (long long)N);
        return CULDA_ERR_UNSUPPORTED;
    }

    // 2. topic of every token: theta_d ~ Dir(doc_conc), z ~ theta_d
    std::vector<uint16_t> tok_topic((size_t)N);
#pragma omp parallel num_threads(threads)
    {
        std::vector<double> th((size_t)KG), cdf((size_t)KG);
#pragma omp for schedule(dynamic, 256)
        for (int d = 0; d < D; ++d) {
            Stream s(seed, kGenTheta, (uint64_t)d);
            dirichlet_draw(KG, nullptr, p->doc_conc, s, th.data());
            double acc = 0;
            for (int k = 0; k < KG; ++k) cdf[k] = (acc += th[k]);
            Stream st(seed, kGenTopic, (uint64_t)d);
            for (int64_t i = doc_ptr[d]; i < doc_ptr[(size_t)d + 1]; ++i) {
                double u = st.uniform() * acc;
                int k = (int)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
                tok_topic[(size_t)i] = (uint16_t)std::min(k, KG - 1);
            }
        }
    }

    // 3. group tokens by generating topic
    std::vector<int64_t> topic_ptr((size_t)KG + 1, 0);
    for (int64_t i = 0; i < N; ++i) topic_ptr[(size_t)tok_topic[(size_t)i] + 1]++;
    for (int k = 0; k < KG; ++k) topic_ptr[(size_t)k + 1] += topic_ptr[k];
    std::vector<int32_t> topic_tok((size_t)N);
    {
        std::vector<int64_t> cur(topic_ptr.begin(), topic_ptr.end() - 1);
        for (int64_t i = 0; i < N; ++i) topic_tok[(size_t)cur[tok_topic[(size_t)i]]++] = (int32_t)i;
    }
    std::vector<uint16_t>().swap(tok_topic);

    // 4. word of every token: phi_k ~ Dir(word_conc * V * p), p_r ~ r^-s, one
    //    alias table per topic, built and dropped inside the topic's task
    std::vector<double> zipf((size_t)V);
    {
        double sum = 0;
        for (int r = 0; r < V; ++r) sum += (zipf[r] = std::pow((double)(r + 1), -p->zipf_s));
        for (int r = 0; r < V; ++r) zipf[r] = p->word_conc * (double)V * zipf[r] / sum;
    }
    std::vector<int32_t> tok_word((size_t)N);
#pragma omp parallel num_threads(threads)
    {
        std::vector<double> ph((size_t)V);
        Alias al;
#pragma omp for schedule(dynamic, 1)
        for (int k = 0; k < KG; ++k) {
            if (topic_ptr[(size_t)k + 1] == topic_ptr[k]) continue;
            Stream s(seed, kGenPhi, (uint64_t)k);
            dirichlet_draw(V, zipf.data(), 0.0, s, ph.data());
            al.build(ph.data(), V);
            for (int64_t j = topic_ptr[k]; j < topic_ptr[(size_t)k + 1]; ++j) {
                int32_t i = topic_tok[(size_t)j];
                Stream sw(seed, kGenWord, (uint64_t)i);
                tok_word[(size_t)i] = al.draw(sw, V);
            }
        }
    }
    std::vector<int32_t>().swap(topic_tok);

    // 5. word ids by first appearance (src_format/format.cpp:75-76)
    std::vector<int32_t> new_id((size_t)V, -1), label;
    label.reserve((size_t)V);
    for (int64_t i = 0; i < N; ++i) {
        int32_t &nid = new_id[(size_t)tok_word[(size_t)i]];
        if (nid < 0) {
            nid = (int32_t)label.size();
            label.push_back(tok_word[(size_t)i]);
        }
        tok_word[(size_t)i] = nid;
    }
    const int32_t VE = (int32_t)label.size();

    // 6. word-major layout, docs ascending within a word (src_format/format.cpp:144-157)
    culda_corpus *c = new_corpus();
    if (!c) return CULDA_ERR_OOM;
    c->num_docs = D;
    c->num_words = VE;
    c->num_tokens = N;
    c->doc_ptr = (int64_t *)malloc(sizeof(int64_t) * ((size_t)D + 1));
    c->word_ptr = (int64_t *)calloc((size_t)VE + 1, sizeof(int64_t));
    c->doc_ids = (int32_t *)malloc(sizeof(int32_t) * (size_t)N);
    c->word_label = (int32_t *)malloc(sizeof(int32_t) * (size_t)VE);
    if (!c->doc_ptr || !c->word_ptr || !c->doc_ids || !c->word_label) {
        culda_corpus_free(c);
        return CULDA_ERR_OOM;
    }
    memcpy(c->doc_ptr, doc_ptr.data(), sizeof(int64_t) * ((size_t)D + 1));
    memcpy(c->word_label, label.data(), sizeof(int32_t) * (size_t)VE);
    for (int64_t i = 0; i < N; ++i) c->word_ptr[(size_t)tok_word[(size_t)i] + 1]++;
    for (int32_t w = 0; w < VE; ++w) c->word_ptr[(size_t)w + 1] += c->word_ptr[w];
    {
        std::vector<int64_t> cur(c->word_ptr, c->word_ptr + VE);
        for (int32_t d = 0; d < D; ++d)
            for (int64_t i = doc_ptr[d]; i < doc_ptr[(size_t)d + 1]; ++i)
                c->doc_ids[cur[(size_t)tok_word[(size_t)i]]++] = d;
    }
    *out = c;
    return CULDA_OK;
}
