/*
 * cgs_cpu.cpp — TEST / BASELINE INFRASTRUCTURE ONLY.
 *
 * Host OpenMP collapsed-Gibbs sampler with the reference's sampling rule: a
 * frozen count snapshot per iteration, no self-exclusion, the sparse doc
 * bucket S = sum theta_dk phihat_wk over the doc's row (ascending topic) and
 * the dense word bucket Q = alpha sum_k phihat_wk, FP32 probabilities
 * (src_culda/kernel/lda_train_kernel.cu:65-259), followed by the count
 * rebuilds (lda_phi_kernel.cu:94-116, lda_theta_kernel.cu:33-85).  Uniforms
 * come from the same Philox4x32-10 stream as the GPU sampler, keyed on
 * (seed, token, iteration).  bench.py times it on the GPU host's cores as the
 * CPU baseline; it is never part of the product.
 */
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]);

namespace {

struct CpuCgs {
    int32_t D, V, K;
    int64_t N;
    float alpha, beta;
    uint64_t seed;
    int threads;
    uint32_t iteration = 1;
    std::vector<int64_t> word_ptr, doc_ptr;
    std::vector<int32_t> doc_ids, doc_tok, row_start, row_end;
    std::vector<uint16_t> z[2];
    int cur = 0;
    std::vector<uint32_t> theta;  // (count << 16) | topic
    std::vector<int32_t> nk;
};

inline uint32_t philox_x0(uint64_t seed, uint64_t t, uint32_t it, uint32_t purpose) {
    uint32_t c[4] = {(uint32_t)t, (uint32_t)(t >> 32), it, purpose}, k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)},
             o[4];
    oracle_philox4x32_10(c, k, o);
    return o[0];
}

inline void neumaier(float &s, float &c, float x) {
    const float t = s + x;
    if (std::fabs(s) >= std::fabs(x))
        c += (s - t) + x;
    else
        c += (x - t) + s;
    s = t;
}

void rebuild(CpuCgs &m) {
    const int K = m.K;
    std::vector<int64_t> nk_acc((size_t)K, 0);
#pragma omp parallel num_threads(m.threads)
    {
        std::vector<uint32_t> cnt((size_t)K, 0);
        std::vector<uint64_t> mask((size_t)(K + 63) / 64, 0);
        std::vector<int64_t> acc((size_t)K, 0);
        const uint16_t *z = m.z[m.cur].data();
#pragma omp for schedule(dynamic, 256)
        for (int32_t d = 0; d < m.D; ++d) {
            for (int64_t i = m.doc_ptr[d]; i < m.doc_ptr[d + 1]; ++i) {
                const uint16_t k = z[m.doc_tok[i]];
                if (cnt[k]++ == 0) mask[k >> 6] |= 1ull << (k & 63);
            }
            int32_t pos = m.row_start[d];
            for (size_t w = 0; w < mask.size(); ++w) {
                uint64_t b = mask[w];
                while (b) {
                    const int bit = __builtin_ctzll(b);
                    b &= b - 1;
                    const int k = (int)(w * 64 + bit);
                    m.theta[pos++] = (cnt[k] << 16) | (uint32_t)k;
                    acc[k] += cnt[k];
                    cnt[k] = 0;
                }
                mask[w] = 0;
            }
            const int32_t nnz = pos - m.row_start[d];
            const int32_t end = m.row_start[d] + (nnz + 31) / 32 * 32;
            for (int32_t j = pos; j < std::max(end, m.row_end[d]); ++j) m.theta[j] = 0;
            m.row_end[d] = end;
        }
#pragma omp critical
        for (int k = 0; k < K; ++k) nk_acc[k] += acc[k];
    }
    for (int k = 0; k < K; ++k) m.nk[k] = (int32_t)nk_acc[k];
}

double sample(CpuCgs &m) {
    const int K = m.K;
    std::vector<float> inv((size_t)K);
    const float vbeta = m.beta * (float)m.V;
    for (int k = 0; k < K; ++k) inv[k] = 1.0f / ((float)m.nk[k] + vbeta);
    const uint16_t *zin = m.z[m.cur].data();
    uint16_t *zout = m.z[1 - m.cur].data();
    double ll = 0.0;
#pragma omp parallel num_threads(m.threads) reduction(+ : ll)
    {
        std::vector<int32_t> hist((size_t)K);
        std::vector<float> ph((size_t)K), qc((size_t)K);
#pragma omp for schedule(dynamic, 16)
        for (int32_t w = 0; w < m.V; ++w) {
            const int64_t b = m.word_ptr[w], e = m.word_ptr[w + 1];
            if (b == e) continue;
            std::fill(hist.begin(), hist.end(), 0);
            for (int64_t t = b; t < e; ++t) hist[zin[t]]++;
            float qs = 0.f, qcmp = 0.f;
            for (int k = 0; k < K; ++k) {
                ph[k] = ((float)hist[k] + m.beta) * inv[k];
                neumaier(qs, qcmp, m.alpha * ph[k]);
                qc[k] = qs + qcmp;
            }
            const float Q = qc[K - 1];
            for (int64_t t = b; t < e; ++t) {
                const int32_t d = m.doc_ids[t];
                const uint32_t *row = m.theta.data() + m.row_start[d];
                const int32_t len = m.row_end[d] - m.row_start[d];
                float s = 0.f, c = 0.f;
                for (int32_t i = 0; i < len; ++i) {
                    const uint32_t en = row[i];
                    if (!(en >> 16)) break;  // rows are zero padded after the last non-zero
                    neumaier(s, c, (float)(en >> 16) * ph[en & 0xFFFFu]);
                }
                const float S = s + c, total = S + Q;
                const uint32_t x = philox_x0(m.seed, (uint64_t)t, m.iteration, 0u);
                const float u = (float)(((x >> 9) << 1) | 1u) * 5.9604644775390625e-08f;
                const float T = u * total;
                int topic = K - 1;
                if (T < S) {
                    float s2 = 0.f, c2 = 0.f;
                    for (int32_t i = 0; i < len; ++i) {
                        const uint32_t en = row[i];
                        if (!(en >> 16)) break;
                        neumaier(s2, c2, (float)(en >> 16) * ph[en & 0xFFFFu]);
                        topic = (int)(en & 0xFFFFu);
                        if (s2 + c2 > T) break;
                    }
                } else {
                    const float tq = T - S;
                    topic = (int)(std::upper_bound(qc.begin(), qc.end(), tq) - qc.begin());
                    if (topic >= K) topic = K - 1;
                }
                zout[t] = (uint16_t)topic;
                ll += (double)std::log(total);
            }
        }
    }
    return ll;
}

}  // namespace

extern "C" {

void *cpu_cgs_create(int32_t D, int32_t V, int64_t N, const int64_t *doc_ptr, const int64_t *word_ptr,
                     const int32_t *doc_ids, int32_t K, float alpha, float beta, uint64_t seed, int32_t threads) {
    CpuCgs *m = new CpuCgs();
    m->D = D;
    m->V = V;
    m->N = N;
    m->K = K;
    m->alpha = alpha;
    m->beta = beta;
    m->seed = seed;
    m->threads = threads > 0 ? threads : omp_get_max_threads();
    m->word_ptr.assign(word_ptr, word_ptr + V + 1);
    m->doc_ptr.assign(doc_ptr, doc_ptr + D + 1);
    m->doc_ids.assign(doc_ids, doc_ids + N);
    m->doc_tok.resize((size_t)N);
    {
        std::vector<int64_t> cur(doc_ptr, doc_ptr + D);
        for (int64_t t = 0; t < N; ++t) m->doc_tok[(size_t)cur[doc_ids[t]]++] = (int32_t)t;
    }
    m->row_start.resize((size_t)D);
    m->row_end.resize((size_t)D);
    int64_t off = 0;
    for (int32_t d = 0; d < D; ++d) {
        int64_t len = std::min<int64_t>(doc_ptr[d + 1] - doc_ptr[d], K);
        m->row_start[d] = m->row_end[d] = (int32_t)off;
        off += (len + 31) / 32 * 32;
    }
    m->theta.assign((size_t)off, 0u);
    m->nk.assign((size_t)K, 0);
    m->z[0].resize((size_t)N);
    m->z[1].resize((size_t)N);
#pragma omp parallel for num_threads(m->threads) schedule(static)
    for (int64_t t = 0; t < N; ++t)
        m->z[0][(size_t)t] = (uint16_t)(((uint64_t)philox_x0(seed, (uint64_t)t, 0u, 1u) * (uint64_t)K) >> 32);
    rebuild(*m);
    return m;
}

/* Runs n iterations; seconds[i] and loglik[i] (per-token, reference formula)
 * receive each iteration's wall time and snapshot log-likelihood. */
int cpu_cgs_iterate(void *h, int n, double *seconds, double *loglik) {
    CpuCgs &m = *(CpuCgs *)h;
    double doc_term = 0;
    for (int32_t d = 0; d < m.D; ++d) {
        const double L = (double)(m.doc_ptr[d + 1] - m.doc_ptr[d]);
        doc_term += L * std::log(L + (double)m.K * (double)m.alpha);
    }
    for (int i = 0; i < n; ++i) {
        const auto t0 = std::chrono::steady_clock::now();
        const double ll = sample(m);
        m.cur = 1 - m.cur;
        rebuild(m);
        ++m.iteration;
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) seconds[i] = std::chrono::duration<double>(t1 - t0).count();
        if (loglik) loglik[i] = (ll - doc_term) / (double)m.N;
    }
    return 0;
}

void cpu_cgs_topics(void *h, uint16_t *out) {
    CpuCgs &m = *(CpuCgs *)h;
    std::memcpy(out, m.z[m.cur].data(), sizeof(uint16_t) * (size_t)m.N);
}

int cpu_cgs_threads(void *h) { return ((CpuCgs *)h)->threads; }

void cpu_cgs_destroy(void *h) { delete (CpuCgs *)h; }

} /* extern "C" */
