/*
 * cgs_oracle.cpp — TEST INFRASTRUCTURE ONLY.
 *
 * Host FP64 restatement of CuLDA_CGS's one-GPU iteration, used as the checker
 * for the CUDA path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load this library; the product never links or calls it.
 *
 * What it restates (reference paths relative to the CuLDA_CGS tree):
 *   - doc-reverse index          src_culda/model/doc_chunk.cpp:225-255
 *   - theta row capacities       src_culda/model/model_theta.cpp:50-56,
 *                                src_culda/model/model_theta_chunk.cpp:74-85
 *   - phi / n_k counts           src_culda/kernel/lda_phi_kernel.cu:94-116
 *   - phiHead (FP16 table)       src_culda/kernel/lda_phi_kernel.cu:24-30
 *   - theta CSR compaction       src_culda/kernel/lda_theta_kernel.cu:33-85
 *   - sampling rule and buckets  src_culda/kernel/lda_train_kernel.cu:65-259
 *   - per-token log term         src_culda/kernel/lda_train_kernel.cu:258
 *   - validPhi / validTheta      src_culda/model/model_phi.cpp:194-280,
 *                                src_culda/model/model_theta_chunk.cpp:142-273
 * and two parts with no reference counterpart: the Philox4x32-10 counter RNG
 * (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3",
 * SC'11) and the Griffiths-Steyvers joint log-likelihood.
 *
 * Parity pins: Philox against the published known-answer vectors; counts,
 * theta layout and phiHead against outputs of the reference's own kernels
 * (tests/golden/, made by tests/golden/make_golden.py); the sampling rule and
 * the per-token log term are restated from the kernel source (the reference
 * draws from cuRAND XORWOW seeded by clock(), so its topic draws cannot be
 * replayed).
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" {

/* ---------------------------------------------------------------- Philox */
/* Philox4x32-10 from the SC'11 paper: 10 rounds of the 4x32 S-box with
 * multipliers 0xD2511F53 / 0xCD9E8D57 and a Weyl key schedule
 * 0x9E3779B9 / 0xBB67AE85. */
void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

static inline uint32_t philox_word0(uint64_t seed, uint64_t t, uint32_t iter, uint32_t purpose) {
    uint32_t ctr[4] = {(uint32_t)t, (uint32_t)(t >> 32), iter, purpose};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    oracle_philox4x32_10(ctr, key, out);
    return out[0];
}

/* Uniform in (0,1): (2*(x>>9)+1) * 2^-24, exact in float and double. */
double oracle_uniform(uint32_t x) { return (double)((((x >> 9) << 1) | 1u)) * 0x1p-24; }

/* Initial topics: z_t = floor(x0 * K / 2^32) with x0 = Philox(seed, {t, 0, 1}).
 * (The reference draws rand() % K after srand(time(NULL)), doc_chunk.cpp:259-264.) */
void oracle_init_topics(int64_t n, int32_t k, uint64_t seed, uint16_t *z) {
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < n; ++t) {
        uint32_t x = philox_word0(seed, (uint64_t)t, 0u, 1u);
        z[t] = (uint16_t)(((uint64_t)x * (uint64_t)k) >> 32);
    }
}

/* ------------------------------------------------------------- structure */
/* docRevIdx: the word-major token ids of each doc in ascending order
 * (doc_chunk.cpp:225-255). */
void oracle_doc_rev(int32_t num_docs, int64_t n, const int32_t *doc_ids, const int64_t *doc_ptr, int32_t *doc_tok) {
    std::vector<int64_t> cur(doc_ptr, doc_ptr + num_docs);
    for (int64_t t = 0; t < n; ++t) doc_tok[cur[doc_ids[t]]++] = (int32_t)t;
}

/* thetaMaxIA: row capacity roundup32(min(L_d, K)), rows back to back
 * (model_theta.cpp:50-56, model_theta_chunk.cpp:74-85). Returns the total. */
int64_t oracle_theta_layout(int32_t num_docs, int32_t k, const int64_t *doc_ptr, int32_t *max_ia) {
    int64_t off = 0;
    for (int32_t d = 0; d < num_docs; ++d) {
        int64_t len = doc_ptr[d + 1] - doc_ptr[d];
        if (len >= k) len = k;
        len = (len + 31) / 32 * 32;
        max_ia[d] = (int32_t)off;
        off += len;
    }
    max_ia[num_docs] = (int32_t)off;
    return off;
}

/* phi[w*K+k] and n_k (lda_phi_kernel.cu:94-116). */
void oracle_phi_counts(int32_t num_words, int32_t k, const int64_t *word_ptr, const uint16_t *z, int32_t *phi,
                       int32_t *nk) {
    std::memset(nk, 0, sizeof(int32_t) * (size_t)k);
#pragma omp parallel for schedule(dynamic, 64)
    for (int32_t w = 0; w < num_words; ++w) {
        int32_t *row = phi + (size_t)w * k;
        std::memset(row, 0, sizeof(int32_t) * (size_t)k);
        for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) row[z[t]]++;
    }
    for (int64_t t = word_ptr[0]; t < word_ptr[num_words]; ++t) nk[z[t]]++;
}

/* IEEE binary16 round-to-nearest-even of a float, from the format definition. */
uint16_t oracle_float_to_half(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t exp = (x >> 23) & 0xFFu;
    uint32_t man = x & 0x7FFFFFu;
    if (exp == 0xFFu) return (uint16_t)(sign | 0x7C00u | (man ? 0x200u : 0u));
    int32_t e = (int32_t)exp - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7C00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        uint32_t m = man | 0x800000u;
        uint32_t shift = (uint32_t)(14 - e);
        uint32_t half_m = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1u);
        uint32_t halfway = 1u << (shift - 1);
        if (rem > halfway || (rem == halfway && (half_m & 1u))) half_m++;
        return (uint16_t)(sign | half_m);
    }
    uint32_t h = sign | ((uint32_t)e << 10) | (man >> 13);
    uint32_t rem = man & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;
    return (uint16_t)h;
}

float oracle_half_to_float(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1Fu;
    uint32_t man = h & 0x3FFu;
    uint32_t x;
    if (exp == 0) {
        if (man == 0) {
            x = sign;
        } else {
            int e = -1;
            do {
                man <<= 1;
                ++e;
            } while (!(man & 0x400u));
            x = sign | ((uint32_t)(127 - 15 - e) << 23) | ((man & 0x3FFu) << 13);
        }
    } else if (exp == 31) {
        x = sign | 0x7F800000u | (man << 13);
    } else {
        x = sign | ((exp - 15 + 127) << 23) | (man << 13);
    }
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}

/* The reference's FP16 phiHead (lda_phi_kernel.cu:26-29): the quotient is
 * formed in float, (phi + beta) / (n_k + beta * V), then rounded to half. */
void oracle_phi_head_f16(int32_t num_words, int32_t k, float beta, const int32_t *phi, const int32_t *nk,
                         uint16_t *out) {
    for (int32_t w = 0; w < num_words; ++w)
        for (int32_t j = 0; j < k; ++j) {
            volatile float num = (float)phi[(size_t)w * k + j] + beta;
            volatile float den = (float)nk[j] + beta * (float)num_words;
            volatile float q = num / den;
            out[(size_t)w * k + j] = oracle_float_to_half(q);
        }
}

/* Theta CSR (lda_theta_kernel.cu:33-85): for each doc, the histogram of its
 * tokens' topics, non-zeros in ascending topic order from thetaMaxIA[d],
 * thetaCurIA[d] = start + roundup32(nnz); entries past nnz up to the row
 * capacity are zero (the memsets at model_theta_chunk.cpp:114-115). */
void oracle_theta_csr(int32_t num_docs, int32_t k, const int64_t *doc_ptr, const int32_t *doc_tok,
                      const uint16_t *z, const int32_t *max_ia, int16_t *theta_a, int16_t *theta_ja,
                      int32_t *cur_ia) {
#pragma omp parallel
    {
    std::vector<int32_t> dense((size_t)k);
#pragma omp for schedule(dynamic, 256)
    for (int32_t d = 0; d < num_docs; ++d) {
        std::fill(dense.begin(), dense.end(), 0);
        for (int64_t i = doc_ptr[d]; i < doc_ptr[d + 1]; ++i) dense[z[doc_tok[i]]]++;
        int32_t start = max_ia[d], cap_end = max_ia[d + 1], nnz = 0;
        for (int32_t j = start; j < cap_end; ++j) {
            theta_a[j] = 0;
            theta_ja[j] = 0;
        }
        for (int32_t j = 0; j < k; ++j)
            if (dense[j] > 0) {
                theta_a[start + nnz] = (int16_t)dense[j];
                theta_ja[start + nnz] = (int16_t)j;
                ++nnz;
            }
        cur_ia[d] = start + (nnz + 31) / 32 * 32;
    }
    }
}

/* Host recount checks of validPhi (model_phi.cpp:194-280) and validTheta
 * (model_theta_chunk.cpp:142-273), generalised from the hard-coded K = 1024.
 * Return 0 when consistent, else a positive code naming the first failed check. */
int oracle_valid_phi(int32_t num_words, int32_t k, const int64_t *word_ptr, const uint16_t *z, const int32_t *phi,
                     const int32_t *nk) {
    std::vector<int32_t> row((size_t)k), tot((size_t)k, 0);
    for (int32_t w = 0; w < num_words; ++w) {
        std::fill(row.begin(), row.end(), 0);
        for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) {
            if (z[t] >= k) return 3;
            row[z[t]]++;
            tot[z[t]]++;
        }
        for (int32_t j = 0; j < k; ++j)
            if (row[j] != phi[(size_t)w * k + j]) return 1;
    }
    for (int32_t j = 0; j < k; ++j)
        if (tot[j] != nk[j]) return 2;
    return 0;
}

int oracle_valid_theta(int32_t num_docs, int32_t k, const int64_t *doc_ptr, const int32_t *doc_tok, const uint16_t *z,
                       const int16_t *theta_a, const int16_t *theta_ja, const int32_t *max_ia, const int32_t *cur_ia) {
    std::vector<int32_t> dense((size_t)k), mask((size_t)k);
    for (int32_t d = 0; d < num_docs; ++d) {
        int32_t s = max_ia[d], e = max_ia[d + 1];
        if (s % 32 != 0 || e % 32 != 0) return 1; /* rows 32-aligned */
        int found = 0;
        for (int32_t j = s; j < e; ++j)
            if (theta_ja[j] == 0 && theta_a[j] != 0) {
                if (found) return 2; /* topic 0 at most once */
                found = 1;
            }
        std::fill(dense.begin(), dense.end(), 0);
        std::fill(mask.begin(), mask.end(), 0);
        for (int64_t i = doc_ptr[d]; i < doc_ptr[d + 1]; ++i) dense[z[doc_tok[i]]]++;
        for (int32_t j = s; j < e; ++j) {
            if (theta_a[j] == 0) continue;
            mask[theta_ja[j]] = 1;
            /* thetaA is int16 in the reference: compare in that width */
            if ((int16_t)dense[theta_ja[j]] != theta_a[j]) return 3; /* non-zero entry disagrees with the recount */
        }
        for (int32_t j = 0; j < k; ++j)
            if (!mask[j] && dense[j] != 0) return 4; /* topic missing from the row */
        /* the used region ends at start + roundup32(nnz) */
        int32_t nnz = 0;
        for (int32_t j = 0; j < k; ++j) nnz += dense[j] > 0;
        if (cur_ia[d] != s + (nnz + 31) / 32 * 32) return 5;
    }
    return 0;
}

/* ---------------------------------------------------------------- sampling */
/*
 * One sampling pass on a frozen snapshot in FP64 (lda_train_kernel.cu:65-259
 * restated).  For token t of word w in doc d:
 *   phihat_k = (n_wk + beta) / (n_k + V*beta)        (lda_phi_kernel.cu:26, in FP64)
 *   S = sum over the doc's row, ascending topic, of A_i * phihat_{JA_i}
 *   Q = alpha * sum_{k=0}^{K-1} phihat_k
 *   u = uniform(Philox(seed, {t_lo, t_hi, iteration, 0}).x0)
 *   T = u * (S + Q); T < S picks the first row entry whose running sum
 *   exceeds T, otherwise the first topic whose running alpha*phihat sum
 *   exceeds T - S.  (The reference tests u < S/(S+Q) and rescales, the same
 *   partition of (0,1).)
 * margin[t] = distance from T to the nearest bucket boundary / (S + Q); a
 * token whose margin is below the FP32 rounding budget may legitimately come
 * out differently on the GPU.  loglik_terms receives sum_t log(S+Q) and
 * sum_t log(L_d + K*alpha) (the reference's per-token log term,
 * lda_train_kernel.cu:258, summed in FP64 with Neumaier compensation).
 */
static inline void neumaier_add(double &sum, double &comp, double x) {
    double t = sum + x;
    if (std::fabs(sum) >= std::fabs(x))
        comp += (sum - t) + x;
    else
        comp += (x - t) + sum;
    sum = t;
}

/* phi_fixed [V x K] (with nk its totals) replaces the counts of z: fold-in
 * against a frozen model (no reference counterpart). */
void oracle_sample_fixed_fp64(int32_t num_docs, int32_t num_words, int32_t k, float alpha_f, float beta_f,
                              const int64_t *word_ptr, const int32_t *doc_ids, const int64_t *doc_ptr,
                              const uint16_t *z, const int32_t *nk, const int16_t *theta_a, const int16_t *theta_ja,
                              const int32_t *max_ia, const int32_t *cur_ia, uint64_t seed, uint32_t iteration,
                              const int32_t *phi_fixed, uint16_t *z_out, double *margin, double *loglik_terms);

void oracle_sample_fp64(int32_t num_docs, int32_t num_words, int32_t k, float alpha_f, float beta_f,
                        const int64_t *word_ptr, const int32_t *doc_ids, const int64_t *doc_ptr, const uint16_t *z,
                        const int32_t *nk, const int16_t *theta_a, const int16_t *theta_ja, const int32_t *max_ia,
                        const int32_t *cur_ia, uint64_t seed, uint32_t iteration, uint16_t *z_out, double *margin,
                        double *loglik_terms) {
    oracle_sample_fixed_fp64(num_docs, num_words, k, alpha_f, beta_f, word_ptr, doc_ids, doc_ptr, z, nk, theta_a,
                             theta_ja, max_ia, cur_ia, seed, iteration, nullptr, z_out, margin, loglik_terms);
}

void oracle_sample_fixed_fp64(int32_t num_docs, int32_t num_words, int32_t k, float alpha_f, float beta_f,
                              const int64_t *word_ptr, const int32_t *doc_ids, const int64_t *doc_ptr,
                              const uint16_t *z, const int32_t *nk, const int16_t *theta_a, const int16_t *theta_ja,
                              const int32_t *max_ia, const int32_t *cur_ia, uint64_t seed, uint32_t iteration,
                              const int32_t *phi_fixed, uint16_t *z_out, double *margin, double *loglik_terms) {
    const double alpha = alpha_f, beta = beta_f;
    const double vbeta = (double)num_words * beta;
    std::vector<double> inv((size_t)k), ph((size_t)k);
    std::vector<int32_t> hist((size_t)k);
    for (int32_t j = 0; j < k; ++j) inv[j] = 1.0 / ((double)nk[j] + vbeta);
    double s_log = 0, c_log = 0, s_doc = 0, c_doc = 0;
    for (int32_t w = 0; w < num_words; ++w) {
        std::fill(hist.begin(), hist.end(), 0);
        if (phi_fixed)
            std::copy(phi_fixed + (size_t)w * k, phi_fixed + (size_t)(w + 1) * k, hist.begin());
        else
            for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) hist[z[t]]++;
        double q = 0;
        for (int32_t j = 0; j < k; ++j) {
            ph[j] = ((double)hist[j] + beta) / ((double)nk[j] + vbeta);
            q += alpha * ph[j];
        }
        for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) {
            int32_t d = doc_ids[t];
            int32_t rs = max_ia[d], re = cur_ia[d];
            double s = 0;
            for (int32_t i = rs; i < re; ++i)
                if (theta_a[i] != 0) s += (double)(uint16_t)theta_a[i] * ph[(uint16_t)theta_ja[i]];
            double total = s + q;
            double u = oracle_uniform(philox_word0(seed, (uint64_t)t, iteration, 0u));
            double target = u * total;
            int32_t pick = -1;
            double lo = 0, hi = total;
            if (target < s) {
                double cum = 0;
                int32_t last = -1;
                for (int32_t i = rs; i < re; ++i) {
                    if (theta_a[i] == 0) continue;
                    double nxt = cum + (double)(uint16_t)theta_a[i] * ph[(uint16_t)theta_ja[i]];
                    last = i;
                    if (nxt > target) {
                        pick = (uint16_t)theta_ja[i];
                        lo = cum;
                        hi = nxt;
                        break;
                    }
                    cum = nxt;
                }
                if (pick < 0) { /* cannot happen in exact arithmetic */
                    pick = (uint16_t)theta_ja[last];
                    lo = cum;
                    hi = s;
                }
            } else {
                double cum = s;
                for (int32_t j = 0; j < k; ++j) {
                    double nxt = cum + alpha * ph[j];
                    if (nxt > target) {
                        pick = j;
                        lo = cum;
                        hi = nxt;
                        break;
                    }
                    cum = nxt;
                }
                if (pick < 0) {
                    pick = k - 1;
                    lo = cum;
                    hi = total;
                }
            }
            z_out[t] = (uint16_t)pick;
            if (margin) margin[t] = std::min(target - lo, hi - target) / total;
            int64_t len = doc_ptr[d + 1] - doc_ptr[d];
            neumaier_add(s_log, c_log, std::log(total));
            neumaier_add(s_doc, c_doc, std::log((double)len + (double)k * alpha));
        }
    }
    if (loglik_terms) {
        loglik_terms[0] = s_log + c_log;
        loglik_terms[1] = s_doc + c_doc;
    }
}

/*
 * The same FP64 rule as oracle_sample_fixed_fp64 (lda_train_kernel.cu:65-259,
 * per-token log term :258) for a selection of tokens:
 * sel holds ascending word-major token indices (NULL = every token), z_out,
 * margin and ll_tok (each may be NULL) are indexed like sel, and ll_tok[i] is
 * the token's log term log(S+Q) - log(L_d + K*alpha).  Each word's phi row is
 * counted from z on the fly (no V x K table), so corpora of any vocabulary
 * fit; the work runs on all host threads in runs of at most 32768 selected
 * tokens of one word (the rows of words cut into several runs are counted
 * once, first).  ll_terms receives sum log(S+Q) and sum log(L_d + K*alpha)
 * over the selection, each run's Neumaier sum added in run order.
 */
void oracle_sample_tokens_fp64(int32_t num_docs, int32_t num_words, int32_t k, float alpha_f, float beta_f,
                               const int64_t *word_ptr, const int32_t *doc_ids, const int64_t *doc_ptr,
                               const uint16_t *z, const int32_t *nk, const int16_t *theta_a,
                               const int16_t *theta_ja, const int32_t *max_ia, const int32_t *cur_ia, uint64_t seed,
                               uint32_t iteration, int64_t n_sel, const int64_t *sel, uint16_t *z_out,
                               double *margin, double *ll_tok, double *ll_terms) {
    (void)num_docs;
    const double alpha = alpha_f, beta = beta_f;
    const double vbeta = (double)num_words * beta;
    const int64_t total_tokens = word_ptr[num_words] - word_ptr[0];
    if (!sel) n_sel = total_tokens;
    auto token_at = [&](int64_t i) -> int64_t { return sel ? sel[i] : word_ptr[0] + i; };
    auto word_of = [&](int64_t t) -> int32_t {
        return (int32_t)(std::upper_bound(word_ptr, word_ptr + num_words + 1, t) - word_ptr - 1);
    };
    // runs: [begin, end) of the selection, all of one word, at most kRun long
    const int64_t kRun = 32768;
    struct Run { int64_t begin, end; int32_t word, shared_row; };
    std::vector<Run> runs;
    std::vector<int32_t> shared_words;
    for (int64_t i = 0; i < n_sel;) {
        const int32_t w = word_of(token_at(i));
        int64_t j = i;
        if (sel) {
            while (j < n_sel && sel[j] < word_ptr[w + 1]) ++j;
        } else {
            j = word_ptr[w + 1] - word_ptr[0];
        }
        const bool split = (j - i) > kRun;
        if (split) shared_words.push_back(w);
        for (int64_t b = i; b < j; b += kRun)
            runs.push_back({b, std::min(j, b + kRun), w, split ? (int32_t)shared_words.size() - 1 : -1});
        i = j;
    }
    std::vector<double> den((size_t)k);
    for (int32_t j = 0; j < k; ++j) den[j] = (double)nk[j] + vbeta;
    // phi rows of the words cut into several runs
    std::vector<double> shared((size_t)shared_words.size() * k);
#pragma omp parallel
    {
        std::vector<int32_t> hist((size_t)k);
#pragma omp for schedule(dynamic, 1)
        for (int64_t r = 0; r < (int64_t)shared_words.size(); ++r) {
            const int32_t w = shared_words[r];
            std::fill(hist.begin(), hist.end(), 0);
            for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) hist[z[t]]++;
            for (int32_t j = 0; j < k; ++j) shared[(size_t)r * k + j] = ((double)hist[j] + beta) / den[j];
        }
    }
    std::vector<double> run_log(runs.size() * 2), run_doc(runs.size() * 2);
#pragma omp parallel
    {
        std::vector<int32_t> hist((size_t)k);
        std::vector<double> own((size_t)k);
#pragma omp for schedule(dynamic, 1)
        for (int64_t r = 0; r < (int64_t)runs.size(); ++r) {
            const Run &run = runs[r];
            const int32_t w = run.word;
            const double *ph;
            if (run.shared_row >= 0) {
                ph = &shared[(size_t)run.shared_row * k];
            } else {
                std::fill(hist.begin(), hist.end(), 0);
                for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) hist[z[t]]++;
                for (int32_t j = 0; j < k; ++j) own[j] = ((double)hist[j] + beta) / den[j];
                ph = own.data();
            }
            double q = 0;
            for (int32_t j = 0; j < k; ++j) q += alpha * ph[j];
            double s_log = 0, c_log = 0, s_doc = 0, c_doc = 0;
            for (int64_t i = run.begin; i < run.end; ++i) {
                const int64_t t = token_at(i);
                const int32_t d = doc_ids[t];
                const int32_t rs = max_ia[d], re = cur_ia[d];
                double s = 0;
                for (int32_t e = rs; e < re; ++e)
                    if (theta_a[e] != 0) s += (double)(uint16_t)theta_a[e] * ph[(uint16_t)theta_ja[e]];
                const double tot = s + q;
                const double target = oracle_uniform(philox_word0(seed, (uint64_t)t, iteration, 0u)) * tot;
                int32_t pick = -1;
                double lo = 0, hi = tot;
                if (target < s) {
                    double cum = 0;
                    int32_t last = -1;
                    for (int32_t e = rs; e < re; ++e) {
                        if (theta_a[e] == 0) continue;
                        const double nxt = cum + (double)(uint16_t)theta_a[e] * ph[(uint16_t)theta_ja[e]];
                        last = e;
                        if (nxt > target) {
                            pick = (uint16_t)theta_ja[e];
                            lo = cum;
                            hi = nxt;
                            break;
                        }
                        cum = nxt;
                    }
                    if (pick < 0) {
                        pick = (uint16_t)theta_ja[last];
                        lo = cum;
                        hi = s;
                    }
                } else {
                    double cum = s;
                    for (int32_t j = 0; j < k; ++j) {
                        const double nxt = cum + alpha * ph[j];
                        if (nxt > target) {
                            pick = j;
                            lo = cum;
                            hi = nxt;
                            break;
                        }
                        cum = nxt;
                    }
                    if (pick < 0) {
                        pick = k - 1;
                        lo = cum;
                        hi = tot;
                    }
                }
                const double dl = std::log((double)(doc_ptr[d + 1] - doc_ptr[d]) + (double)k * alpha);
                if (z_out) z_out[i] = (uint16_t)pick;
                if (margin) margin[i] = std::min(target - lo, hi - target) / tot;
                if (ll_tok) ll_tok[i] = std::log(tot) - dl;
                neumaier_add(s_log, c_log, std::log(tot));
                neumaier_add(s_doc, c_doc, dl);
            }
            run_log[2 * r] = s_log;
            run_log[2 * r + 1] = c_log;
            run_doc[2 * r] = s_doc;
            run_doc[2 * r + 1] = c_doc;
        }
    }
    if (ll_terms) {
        double s1 = 0, c1 = 0, s2 = 0, c2 = 0;
        for (size_t r = 0; r < runs.size(); ++r) {
            neumaier_add(s1, c1, run_log[2 * r]);
            neumaier_add(s1, c1, run_log[2 * r + 1]);
            neumaier_add(s2, c2, run_doc[2 * r]);
            neumaier_add(s2, c2, run_doc[2 * r + 1]);
        }
        ll_terms[0] = s1 + c1;
        ll_terms[1] = s2 + c2;
    }
}

/* ------------------------------------ Metropolis-Hastings (no reference counterpart) */
/*
 * One MH pass from the snapshot z (input order), restating
 * culda_cgs_b200/csrc/learned.cu in FP64 on the same Philox words
 * (counter {t, iteration, 16 + step}): per token `steps` steps, even steps (all
 * steps when cdf is NULL) the doc proposal (n_dk + alpha) with acceptance
 * phihat_wk' / phihat_ws, odd steps the independent proposal given by the
 * prefix table cdf [D x K] with acceptance p(k') q(s) / (p(s) q(k')),
 * p(k) = (n_dk + alpha) phihat_wk.  margin[t]: the smallest relative distance
 * of any decision on the token's path (bucket choice, table search,
 * acceptance) to its boundary.
 */
static inline void philox_words(uint64_t seed, uint64_t t, uint32_t iter, uint32_t purpose, uint32_t out[4]) {
    uint32_t ctr[4] = {(uint32_t)t, (uint32_t)(t >> 32), iter, purpose};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    oracle_philox4x32_10(ctr, key, out);
}

static inline uint32_t bounded(uint32_t x, uint32_t n) { return (uint32_t)(((uint64_t)x * (uint64_t)n) >> 32); }

void oracle_mh_fp64(int32_t num_docs, int32_t num_words, int32_t k, float alpha_f, float beta_f,
                    const int64_t *word_ptr, const int32_t *doc_ids, const int64_t *doc_ptr, const int32_t *doc_tok,
                    const uint16_t *z, const int32_t *nk, const float *cdf, uint64_t seed, uint32_t iteration,
                    int32_t steps, uint16_t *z_out, double *margin) {
    const double alpha = alpha_f, beta = beta_f, vbeta = (double)num_words * beta, ka = (double)k * alpha;
    std::vector<int32_t> ndk((size_t)num_docs * k, 0);
    for (int32_t d = 0; d < num_docs; ++d)
        for (int64_t i = doc_ptr[d]; i < doc_ptr[d + 1]; ++i) ndk[(size_t)d * k + z[doc_tok[i]]]++;
    std::vector<double> ph((size_t)k);
    std::vector<int32_t> hist((size_t)k);
    for (int32_t w = 0; w < num_words; ++w) {
        std::fill(hist.begin(), hist.end(), 0);
        for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) hist[z[t]]++;
        for (int32_t j = 0; j < k; ++j) ph[j] = ((double)hist[j] + beta) / ((double)nk[j] + vbeta);
        for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) {
            const int32_t d = doc_ids[t];
            const int64_t d0 = doc_ptr[d];
            const double L = (double)(doc_ptr[d + 1] - d0);
            int32_t s = z[t];
            double m = INFINITY;
            for (int32_t step = 0; step < steps; ++step) {
                uint32_t x[4];
                philox_words(seed, (uint64_t)t, iteration, 16u + (uint32_t)step, x);
                int32_t kp;
                double ratio;
                if (!(cdf && (step & 1))) {
                    const double a = oracle_uniform(x[0]) * (L + ka);
                    m = std::min(m, std::fabs(a - L) / (L + ka));
                    if (a < L)
                        kp = z[doc_tok[d0 + bounded(x[1], (uint32_t)L)]];
                    else
                        kp = (int32_t)bounded(x[1], (uint32_t)k);
                    ratio = ph[kp] / ph[s];
                } else {
                    const float *row = cdf + (size_t)d * k;
                    const double total = row[k - 1];
                    const double T = oracle_uniform(x[1]) * total;
                    kp = k - 1;
                    for (int32_t j = 0; j < k; ++j)
                        if ((double)row[j] > T) {
                            kp = j;
                            break;
                        }
                    const double lo = kp > 0 ? (double)row[kp - 1] : 0.0;
                    m = std::min(m, std::min((double)row[kp] - T, T - lo) / total);
                    const double qk = (double)row[kp] - lo;
                    const double qs = (double)row[s] - (s > 0 ? (double)row[s - 1] : 0.0);
                    const double pk = ((double)ndk[(size_t)d * k + kp] + alpha) * ph[kp];
                    const double ps = ((double)ndk[(size_t)d * k + s] + alpha) * ph[s];
                    ratio = (pk * qs) / (ps * qk);
                }
                if (kp != s) {
                    const double u = oracle_uniform(x[2]);
                    if (ratio > 0) m = std::min(m, std::fabs(u - ratio) / ratio);
                    if (u < ratio) s = kp;
                }
            }
            z_out[t] = (uint16_t)s;
            if (margin) margin[t] = m;
        }
    }
}

/* Warm start (no reference counterpart; culda_cgs_b200/csrc/learned.cu): token
 * t of word w in doc d draws its topic from q_d(k) * phihat_wk, q_d(k) the
 * differences of the prefix table cdf [D x K], phihat from phi [V x K] and nk,
 * by inverse CDF in ascending topic with u = Philox(seed, {t, 0, 6}). */
void oracle_warm_start(int32_t num_docs, int32_t num_words, int32_t k, float beta_f, const int64_t *word_ptr,
                       const int32_t *doc_ids, const int32_t *phi, const int32_t *nk, const float *cdf, uint64_t seed,
                       uint16_t *z_out, double *margin) {
    (void)num_docs;
    const double beta = beta_f, vbeta = (double)num_words * beta;
    std::vector<double> ph((size_t)k), p((size_t)k);
    for (int32_t w = 0; w < num_words; ++w) {
        for (int32_t j = 0; j < k; ++j) ph[j] = ((double)phi[(size_t)w * k + j] + beta) / ((double)nk[j] + vbeta);
        for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) {
            const float *row = cdf + (size_t)doc_ids[t] * k;
            double total = 0;
            for (int32_t j = 0; j < k; ++j) {
                p[j] = ((double)row[j] - (j > 0 ? (double)row[j - 1] : 0.0)) * ph[j];
                total += p[j];
            }
            const double T = oracle_uniform(philox_word0(seed, (uint64_t)t, 0u, 6u)) * total;
            double cum = 0, lo = 0, hi = total;
            int32_t pick = k - 1;
            for (int32_t j = 0; j < k; ++j) {
                if (cum + p[j] > T) {
                    pick = j;
                    lo = cum;
                    hi = cum + p[j];
                    break;
                }
                cum += p[j];
            }
            z_out[t] = (uint16_t)pick;
            if (margin) margin[t] = std::min(T - lo, hi - T) / total;
        }
    }
}

/* ------------------------------------------- reference-compatible loglik */
/*
 * The value the reference prints (lda_train_kernel.cu:56-262 then
 * LDATrainPerplexity :273-356), with its own arithmetic:
 *   - phiHeadCache = FP16 phiHead widened to float (lda_train_kernel.cu:71),
 *     FP16 rounding of the float quotient (lda_phi_kernel.cu:26-29);
 *   - Q: per group of 32 topics a shfl_down tree of alpha*phi (16,8,4,2,1),
 *     then a lock-step Kogge-Stone scan of the 32 group sums (:68-99);
 *   - S: per 32-entry chunk of the doc's row a shfl_down tree of A*phi,
 *     accumulated chunk by chunk in float (:116-137);
 *   - term = logf((S+Q) / (float)(L_d + K*alpha)) summed in float by each warp
 *     over tokens start+w, start+w+32, ... of its slot (:104-106,256-262);
 *   - each warp sum truncated to int, only the first numWords*32 warp slots
 *     summed (:282-298, :338), divided by N (:355).
 * slot_word / slot_range are the slots of DocChunk::loadChunk (doc_chunk.cpp:148-205).
 */
static inline float warp_tree32(const float *v) {
    float a[32];
    for (int l = 0; l < 32; ++l) a[l] = v[l];
    for (int o = 16; o >= 1; o >>= 1)
        for (int l = 0; l < o; ++l) a[l] = a[l] + a[l + o];
    return a[0];
}

double oracle_loglik_reference(int32_t num_words, int32_t k, float alpha, int64_t num_tokens, int32_t num_slots,
                               const int32_t *slot_word, const int64_t *slot_range, const int32_t *doc_ids,
                               const int64_t *doc_ptr, const uint16_t *phi_head, const int16_t *theta_a,
                               const int16_t *theta_ja, const int32_t *max_ia, const int32_t *cur_ia) {
    int64_t total = 0;
    // slots are independent and the warp sums are integers after truncation,
    // so the slots may run on all host threads in any order
#pragma omp parallel reduction(+ : total)
    {
    std::vector<float> cache((size_t)k), qtree(32);
#pragma omp for schedule(dynamic, 16)
    for (int32_t s = 0; s < num_slots; ++s) {
        const int32_t w = slot_word[s];
        for (int32_t j = 0; j < k; ++j) cache[j] = oracle_half_to_float(phi_head[(size_t)w * k + j]);
        float grp[32];
        for (int g = 0; g < 32; ++g) {
            for (int l = 0; l < 32; ++l) grp[l] = 32 * g + l < k ? alpha * cache[32 * g + l] : 0.f;
            qtree[g] = warp_tree32(grp);
        }
        for (int o = 1; o < 32; o <<= 1) {
            float nv[32];
            for (int l = 0; l < 32; ++l) nv[l] = l >= o ? qtree[l - o] + qtree[l] : qtree[l];
            for (int l = 0; l < 32; ++l) qtree[l] = nv[l];
        }
        const float Q = qtree[31];
        for (int warp = 0; warp < 32; ++warp) {
            float sum = 0.0f;
            for (int64_t t = slot_range[2 * s] + warp; t < slot_range[2 * s + 1]; t += 32) {
                const int32_t d = doc_ids[t];
                float S = 0.f;
                for (int32_t base = max_ia[d]; base < cur_ia[d]; base += 32) {
                    float p[32];
                    for (int l = 0; l < 32; ++l) p[l] = (float)(int)theta_a[base + l] * cache[(uint16_t)theta_ja[base + l]];
                    S += warp_tree32(p);
                }
                const float den = (float)(doc_ptr[d + 1] - doc_ptr[d]) + (float)k * alpha;
                sum += logf((S + Q) / den);
            }
            if (s < num_words) total += (int64_t)(int)(double)sum;
        }
    }
    }
    return (double)total / (double)num_tokens;
}

/* The reference's slots (doc_chunk.cpp:148-205): words by length, longest
 * first; a word longer than 1.05 * (N / 56) tokens is cut into
 * ceil(len / ave) slices of ceil(len / slices) tokens.  The reference sorts
 * with std::sort on the length alone, which leaves the order of words of equal
 * length unspecified; here they keep ascending word id.  Writes num_slots
 * (at most num_words + N / ave + 1) slot words and [start, end) ranges, and
 * returns num_slots. */
int32_t oracle_reference_slots(int32_t num_words, const int64_t *word_ptr, int32_t *slot_word, int64_t *slot_range) {
    const int64_t n = word_ptr[num_words] - word_ptr[0];
    const int ave = (int)(n / 56);
    std::vector<int32_t> order((size_t)num_words);
    for (int32_t w = 0; w < num_words; ++w) order[(size_t)w] = w;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return word_ptr[a + 1] - word_ptr[a] > word_ptr[b + 1] - word_ptr[b];
    });
    int32_t ns = 0;
    for (int32_t w : order) {
        const int len = (int)(word_ptr[w + 1] - word_ptr[w]);
        if (ave > 0 && len > 1.05 * ave) {
            const int slices = (len + ave - 1) / ave;
            const int size = (len + slices - 1) / slices;
            for (int i = 0; i < slices; ++i) {
                const int64_t b = word_ptr[w] + (int64_t)size * i;
                int64_t e = b + size;
                if (e >= word_ptr[w + 1]) e = word_ptr[w + 1];
                slot_word[ns] = w;
                slot_range[2 * ns] = b;
                slot_range[2 * ns + 1] = e;
                ++ns;
            }
        } else {
            slot_word[ns] = w;
            slot_range[2 * ns] = word_ptr[w];
            slot_range[2 * ns + 1] = word_ptr[w + 1];
            ++ns;
        }
    }
    return ns;
}

/* ------------------------------------------------------ joint likelihood */
/*
 * log p(w, z) = K lgamma(V b) - sum_k lgamma(n_k + V b) + sum_{w,k: n>0} [lgamma(n_wk + b) - lgamma(b)]
 *             + D lgamma(K a) - sum_d lgamma(L_d + K a) + sum_{d,k: n>0} [lgamma(n_dk + a) - lgamma(a)]
 * (collapsed LDA joint, Griffiths & Steyvers, PNAS 2004), FP64, Neumaier sums.
 */
double oracle_loglik_joint(int32_t num_docs, int32_t num_words, int32_t k, float alpha_f, float beta_f,
                           const int64_t *word_ptr, const int64_t *doc_ptr, const int32_t *doc_tok, const uint16_t *z) {
    const double a = alpha_f, b = beta_f, vb = (double)num_words * b, ka = (double)k * a;
    const double lg_b = std::lgamma(b), lg_a = std::lgamma(a);
    double s = 0, c = 0;
    std::vector<int32_t> hist((size_t)k), nk((size_t)k, 0);
    for (int32_t w = 0; w < num_words; ++w) {
        std::fill(hist.begin(), hist.end(), 0);
        for (int64_t t = word_ptr[w]; t < word_ptr[w + 1]; ++t) hist[z[t]]++;
        for (int32_t j = 0; j < k; ++j)
            if (hist[j] > 0) {
                neumaier_add(s, c, std::lgamma((double)hist[j] + b) - lg_b);
                nk[j] += hist[j];
            }
    }
    neumaier_add(s, c, (double)k * std::lgamma(vb));
    for (int32_t j = 0; j < k; ++j) neumaier_add(s, c, -std::lgamma((double)nk[j] + vb));
    neumaier_add(s, c, (double)num_docs * std::lgamma(ka));
    for (int32_t d = 0; d < num_docs; ++d) {
        std::fill(hist.begin(), hist.end(), 0);
        for (int64_t i = doc_ptr[d]; i < doc_ptr[d + 1]; ++i) hist[z[doc_tok[i]]]++;
        neumaier_add(s, c, -std::lgamma((double)(doc_ptr[d + 1] - doc_ptr[d]) + ka));
        for (int32_t j = 0; j < k; ++j)
            if (hist[j] > 0) neumaier_add(s, c, std::lgamma((double)hist[j] + a) - lg_a);
    }
    return s + c;
}

} /* extern "C" */
