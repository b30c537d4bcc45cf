// culda_main.cpp — the `culda` command: the reference's CLI and per-iteration
// output (src_culda/main.cpp:40-194, src_culda/train/SingleChunkSingleGPU.h:70-127)
// over the C ABI of libculda_b200.so.
//
//   culda -g 1 -c 1 -k <topics> -t <iterations> -a <alpha> -b <beta> -i <prefix> [-o <prefix>] [-s n]
//
// Extra options (off by default, so parsers of the reference's output keep
// working): -seed <n> (Philox key, default 1), -G <lanes> (a group sampler
// with that many lanes per token instead of the default warp-flattened walk),
// -j (print the FP64 joint log-likelihood on a separate line after
// each iteration), -z <file> (write the final topics as int16), -top <n>
// (words per topic in the -o report, default 20, 0 = all).  -o <prefix>,
// accepted and unused by the reference, writes the topic-word and doc-topic
// reports of the reference's commented-out saveWord / saveDoc.
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "culda_b200.h"

namespace {

struct Argument {  // src_culda/model/culda_argument.h:50-82
    int numGPUs = 1, k = 0, iteration = 0, numWorkers = 1, numChunks = 1;
    float alpha = 0.f, beta = 0.f;
    std::string inputFilePrefix, outputFilePrefix, topicsOut;
    unsigned long long seed = 1;
    int groupLanes = 0, topWords = 20;
    bool jointLL = false;
};

bool numerical(const char *s) {  // ISNumerical, main.cpp:26-36
    int c = 0;
    for (; *s; ++s) {
        if (!isdigit((unsigned char)*s)) return false;
        ++c;
    }
    return c > 0;
}

Argument parse(int argc, char **argv) {  // ParseArgument, main.cpp:40-161
    if (argc == 1) throw std::invalid_argument("No argument found");
    Argument a;
    bool have_k = false, have_t = false, have_a = false, have_b = false, have_i = false;
    for (int i = 1; i < argc; ++i) {
        std::string o = argv[i];
        auto need = [&](const char *what) -> const char * {
            if (i + 1 >= argc) throw std::invalid_argument(std::string("need to specify a value after ") + what);
            return argv[++i];
        };
        auto integer = [&](const char *what) -> int {
            const char *v = need(what);
            if (!numerical(v)) throw std::invalid_argument(std::string(what) + " should be followed by a positive integer");
            return atoi(v);
        };
        if (o == "-g") a.numGPUs = integer("-g");
        else if (o == "-k") { a.k = integer("-k"); have_k = true; }
        else if (o == "-t") { a.iteration = integer("-t"); have_t = true; }
        else if (o == "-s") a.numWorkers = integer("-s");
        else if (o == "-a") { a.alpha = (float)atof(need("-a")); have_a = true; }
        else if (o == "-b") { a.beta = (float)atof(need("-b")); have_b = true; }
        else if (o == "-c") a.numChunks = atoi(need("-c"));
        else if (o == "-i") { a.inputFilePrefix = need("-i"); have_i = true; }
        else if (o == "-o") a.outputFilePrefix = need("-o");
        else if (o == "-seed") a.seed = strtoull(need("-seed"), nullptr, 10);
        else if (o == "-G") a.groupLanes = integer("-G");
        else if (o == "-j") a.jointLL = true;
        else if (o == "-z") a.topicsOut = need("-z");
        else if (o == "-top") a.topWords = atoi(need("-top"));
        else break;  // the reference stops at the first unknown token
    }
    // The reference leaves these uninitialised when absent; here they are required.
    if (!have_k || !have_t || !have_a || !have_b || !have_i)
        throw std::invalid_argument("-k, -t, -a, -b and -i are required");
    if (a.k % 32 != 0) {
        printf("Warning: number of topics(k) has been rounded to multiples of 32.\n");
        a.k = (a.k + 31) / 32 * 32;
    }
    if (a.numWorkers <= 0) {
        printf("Warning: wrong number of workers.\n");
        a.numWorkers = 1;
    }
    if (a.numGPUs <= 0) a.numGPUs = 1;
    if (a.numGPUs > 1) {
        printf("Warning: number of GPUs(%d) is larger than the one-GPU path supports, rounded to 1\n", a.numGPUs);
        a.numGPUs = 1;
    }
    return a;
}

void print_argument(const Argument &a) {  // culda_argument.h:69-81
    printf("numGPUs     :%d\n", a.numGPUs);
    printf("k           :%d\n", a.k);
    printf("iteration   :%d\n", a.iteration);
    printf("numWorkers  :%d\n", a.numWorkers);
    printf("numChunks   :%d\n", a.numChunks);
    printf("alpha       :%.2f\n", a.alpha);
    printf("beta        :%.2f\n", a.beta);
    printf("prefix      :%s\n", a.inputFilePrefix.c_str());
    printf("outfile     :%s\n", a.outputFilePrefix.c_str());
    printf("\n");
}

// Token strings from "<prefix>.vocab" ("token id" per line, src_format/format.cpp:96-99);
// the word id as text for any word the file does not name.
std::vector<std::string> load_vocab(const std::string &prefix, int V) {
    std::vector<std::string> names((size_t)V);
    for (int w = 0; w < V; ++w) names[(size_t)w] = std::to_string(w);
    FILE *f = fopen((prefix + ".vocab").c_str(), "rb");
    if (!f) return names;
    std::string line;
    int ch;
    auto flush_line = [&]() {
        const size_t sp = line.find_last_of(' ');
        if (sp != std::string::npos && sp > 0 && sp + 1 < line.size()) {
            const long id = strtol(line.c_str() + sp + 1, nullptr, 10);
            if (id >= 0 && id < V) names[(size_t)id] = line.substr(0, sp);
        }
        line.clear();
    };
    while ((ch = fgetc(f)) != EOF) {
        if (ch == '\n')
            flush_line();
        else
            line.push_back((char)ch);
    }
    if (!line.empty()) flush_line();
    fclose(f);
    return names;
}

// -o <prefix>: the two model reports of the reference's commented-out
// ModelPhi::saveWord (model_phi.cpp:283-329) and ModelTheta::saveDoc
// (model_theta.cpp:207-242), in their layouts:
//   <prefix>.topwords   "topic, total, top words", then per topic with tokens
//                       "%4d total (token,count) ..." by count (ties: lower id
//                       first), the first -top n words (0: all)
//   <prefix>.doctopics  "Doc, total, top topics", then per doc
//                       "%4d| total (topic,count), ..." over all its topics
int write_reports(culda_ctx *ctx, const culda_corpus *corpus, const Argument &arg) {
    const int K = arg.k, V = corpus->num_words, D = corpus->num_docs;
    const int64_t N = corpus->num_tokens;
    std::vector<int32_t> phi((size_t)V * K), nk((size_t)K);
    std::vector<uint16_t> z((size_t)N);
    int rc = culda_get_phi(ctx, phi.data(), nk.data());
    if (rc == CULDA_OK) rc = culda_get_topics(ctx, z.data());
    if (rc != CULDA_OK) {
        fprintf(stderr, "Error: %s\n", culda_last_error(ctx));
        return rc;
    }
    const std::vector<std::string> names = load_vocab(arg.inputFilePrefix, V);
    std::string path = arg.outputFilePrefix + ".topwords";
    FILE *f = fopen(path.c_str(), "w");
    if (!f) {
        fprintf(stderr, "Error: writing %s failed\n", path.c_str());
        return CULDA_ERR_IO;
    }
    fprintf(f, "topic, total, top words\n");
    std::vector<int32_t> idx;
    for (int k = 0; k < K; ++k) {
        idx.clear();
        int64_t total = 0;
        for (int w = 0; w < V; ++w)
            if (phi[(size_t)w * K + k] > 0) {
                idx.push_back(w);
                total += phi[(size_t)w * K + k];
            }
        if (total <= 0) continue;
        const size_t top = arg.topWords > 0 ? std::min(idx.size(), (size_t)arg.topWords) : idx.size();
        std::partial_sort(idx.begin(), idx.begin() + (long)top, idx.end(), [&](int32_t a, int32_t b) {
            const int32_t ca = phi[(size_t)a * K + k], cb = phi[(size_t)b * K + k];
            return ca != cb ? ca > cb : a < b;
        });
        fprintf(f, "%4d %lld ", k, (long long)total);
        for (size_t i = 0; i < top; ++i)
            fprintf(f, "(%s,%d) ", names[(size_t)idx[i]].c_str(), phi[(size_t)idx[i] * K + k]);
        fprintf(f, "\n");
    }
    if (fclose(f) != 0) return CULDA_ERR_IO;

    std::vector<int32_t> doc_tok((size_t)N);
    rc = culda_corpus_doc_tokens(corpus, doc_tok.data());
    if (rc != CULDA_OK) return rc;
    path = arg.outputFilePrefix + ".doctopics";
    f = fopen(path.c_str(), "w");
    if (!f) {
        fprintf(stderr, "Error: writing %s failed\n", path.c_str());
        return CULDA_ERR_IO;
    }
    fprintf(f, "Doc, total, top topics\n");
    std::vector<uint16_t> topics;
    std::vector<std::pair<int, int>> freq;  // (topic, count)
    for (int d = 0; d < D; ++d) {
        topics.clear();
        for (int64_t i = corpus->doc_ptr[d]; i < corpus->doc_ptr[d + 1]; ++i) topics.push_back(z[(size_t)doc_tok[(size_t)i]]);
        std::sort(topics.begin(), topics.end());
        freq.clear();
        for (size_t i = 0; i < topics.size();) {
            size_t j = i;
            while (j < topics.size() && topics[j] == topics[i]) ++j;
            freq.emplace_back(topics[i], (int)(j - i));
            i = j;
        }
        std::stable_sort(freq.begin(), freq.end(), [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
            return a.second > b.second;
        });
        fprintf(f, "%4d| %lld ", d, (long long)topics.size());
        for (const auto &fr : freq) fprintf(f, "(%d,%d), ", fr.first, fr.second);
        fprintf(f, "\n");
    }
    return fclose(f) == 0 ? CULDA_OK : CULDA_ERR_IO;
}

}  // namespace

int main(int argc, char **argv) {
    printf("Parsing arguments ...\n");
    Argument arg;
    try {
        arg = parse(argc, argv);
    } catch (std::invalid_argument &e) {
        printf("Error: %s\n", e.what());
        return 1;
    }
    print_argument(arg);
    printf("Loading document ...\n");
    culda_corpus *corpus = nullptr;
    int rc = culda_corpus_load(arg.inputFilePrefix.c_str(), arg.numChunks, &corpus);
    if (rc != CULDA_OK) {
        fprintf(stderr, "Error: %s\n", culda_last_error(nullptr));
        return 2;
    }
    printf("numDocs  :  %d\n", corpus->num_docs);
    printf("numWords :  %d\n", corpus->num_words);
    printf("numTokens:  %lld\n\n", (long long)corpus->num_tokens);
    culda_params p{};
    p.k = arg.k;
    p.alpha = arg.alpha;
    p.beta = arg.beta;
    p.seed = arg.seed;
    p.device = 0;
    p.group_lanes = arg.groupLanes;
    culda_ctx *ctx = nullptr;
    rc = culda_create(corpus, &p, &ctx);
    if (rc != CULDA_OK) {
        fprintf(stderr, "Error: %s\n", culda_last_error(nullptr));
        culda_corpus_free(corpus);
        return 3;
    }
    double elapsed = 0;
    for (int ite = 0; ite < arg.iteration; ++ite) {
        culda_iter_stats st{};
        const auto b = std::chrono::steady_clock::now();
        rc = culda_iterate(ctx, 1, &st);
        const auto e = std::chrono::steady_clock::now();
        if (rc != CULDA_OK) {
            fprintf(stderr, "Error: %s\n", culda_last_error(ctx));
            break;
        }
        const double stamp = std::chrono::duration<double>(e - b).count();
        elapsed += stamp;
        printf("Iteration %3d: %6.2f sec, %3.2f sec, logLikelyhood = %.8f, %5.3f M\n", ite + 1, elapsed, stamp,
               st.loglik, (double)corpus->num_tokens / stamp / 1000000);
        if (arg.jointLL) {
            double ll = 0;
            if (culda_loglik_joint(ctx, &ll) == CULDA_OK)
                printf("joint loglik/token = %.10f\n", ll / (double)corpus->num_tokens);
        }
        fflush(stdout);
    }
    if (rc == CULDA_OK && !arg.topicsOut.empty()) {
        std::vector<uint16_t> z((size_t)corpus->num_tokens);
        rc = culda_get_topics(ctx, z.data());
        FILE *f = rc == CULDA_OK ? fopen(arg.topicsOut.c_str(), "wb") : nullptr;
        if (!f || fwrite(z.data(), 2, z.size(), f) != z.size()) {
            fprintf(stderr, "Error: writing %s failed\n", arg.topicsOut.c_str());
            rc = CULDA_ERR_IO;
        }
        if (f) fclose(f);
    }
    if (rc == CULDA_OK && !arg.outputFilePrefix.empty()) rc = write_reports(ctx, corpus, arg);
    printf("\n");
    culda_destroy(ctx);
    culda_corpus_free(corpus);
    return rc == CULDA_OK ? 0 : 4;
}
