// culda_main.cpp — the `culda` command: the reference's CLI and per-iteration
// output (src_culda/main.cpp:40-194, src_culda/train/SingleChunkSingleGPU.h:70-127)
// over the C ABI of libculda_b200.so.
//
//   culda -g 1 -c 1 -k <topics> -t <iterations> -a <alpha> -b <beta> -i <prefix> [-o <prefix>] [-s n]
//
// Extra options (off by default, so parsers of the reference's output keep
// working): -seed <n> (Philox key, default 1), -G <lanes> (sampler lanes per
// token), -j (print the FP64 joint log-likelihood on a separate line after
// each iteration), -z <file> (write the final topics as int16).  -o <prefix>,
// accepted and unused by the reference, writes <prefix>.topwords: each
// topic's token count and its 20 most frequent words.
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
    int groupLanes = 0;
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
    // -o: the model summary the reference's commented-out saveWord
    // (model_phi.cpp:283-329) would have written: per topic its token count
    // and its 20 most frequent words (word id:count)
    if (rc == CULDA_OK && !arg.outputFilePrefix.empty()) {
        const int K = arg.k, V = corpus->num_words;
        std::vector<int32_t> phi((size_t)V * K), nk((size_t)K);
        rc = culda_get_phi(ctx, phi.data(), nk.data());
        const std::string path = arg.outputFilePrefix + ".topwords";
        FILE *f = rc == CULDA_OK ? fopen(path.c_str(), "w") : nullptr;
        if (!f) {
            fprintf(stderr, "Error: writing %s failed\n", path.c_str());
            rc = CULDA_ERR_IO;
        } else {
            std::vector<int32_t> idx((size_t)V);
            for (int k = 0; k < K; ++k) {
                for (int w = 0; w < V; ++w) idx[(size_t)w] = w;
                const int top = std::min(20, V);
                std::partial_sort(idx.begin(), idx.begin() + top, idx.end(), [&](int32_t a, int32_t b) {
                    const int32_t ca = phi[(size_t)a * K + k], cb = phi[(size_t)b * K + k];
                    return ca != cb ? ca > cb : a < b;
                });
                fprintf(f, "topic %d tokens %d:", k, nk[(size_t)k]);
                for (int i = 0; i < top && phi[(size_t)idx[(size_t)i] * K + k] > 0; ++i)
                    fprintf(f, " %d:%d", idx[(size_t)i], phi[(size_t)idx[(size_t)i] * K + k]);
                fprintf(f, "\n");
            }
            fclose(f);
        }
    }
    printf("\n");
    culda_destroy(ctx);
    culda_corpus_free(corpus);
    return rc == CULDA_OK ? 0 : 4;
}
