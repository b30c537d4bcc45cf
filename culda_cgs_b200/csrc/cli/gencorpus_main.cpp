// gencorpus_main.cpp — the `gencorpus` command: writes a seeded synthetic LDA
// corpus (culda_corpus_generate) as the five src_format files the reference's
// `culda -i <prefix>` reads (src_format/format.cpp:92-165, data_chunk.h:49-67).
//
//   gencorpus -words V -topics KG -docs D -law poisson|lognormal|pareto
//             -a A [-b B] -min LMIN -max LMAX [-zipf S] [-wconc C] [-dconc C]
//             [-seed S] [-threads T] -o <prefix>
//
// Prints one JSON line {"num_docs":…, "num_words":…, "num_tokens":…} on
// success.  Host-only: it touches no GPU.  Exit status 1 for a bad command
// line, 2 when generation or writing fails.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "culda_b200.h"

static int usage() {
    fprintf(stderr,
            "Usage: gencorpus -words V -topics KG -docs D -law poisson|lognormal|pareto -a A [-b B] -min LMIN "
            "-max LMAX [-zipf S] [-wconc C] [-dconc C] [-seed S] [-threads T] -o prefix\n");
    return 1;
}

int main(int argc, char **argv) {
    culda_gen_params p{};
    p.zipf_s = 1.05;
    p.word_conc = 0.1;
    p.doc_conc = 0.1;
    p.seed = 1;
    p.len_law = -1;
    std::string out;
    for (int i = 1; i < argc; ++i) {
        const char *f = argv[i];
        if (i + 1 >= argc) return usage();
        const char *v = argv[++i];
        if (!strcmp(f, "-words")) p.num_words = atoi(v);
        else if (!strcmp(f, "-topics")) p.num_topics = atoi(v);
        else if (!strcmp(f, "-docs")) p.num_docs = atoi(v);
        else if (!strcmp(f, "-a")) p.len_a = atof(v);
        else if (!strcmp(f, "-b")) p.len_b = atof(v);
        else if (!strcmp(f, "-min")) p.len_min = atoi(v);
        else if (!strcmp(f, "-max")) p.len_max = atoi(v);
        else if (!strcmp(f, "-zipf")) p.zipf_s = atof(v);
        else if (!strcmp(f, "-wconc")) p.word_conc = atof(v);
        else if (!strcmp(f, "-dconc")) p.doc_conc = atof(v);
        else if (!strcmp(f, "-seed")) p.seed = strtoull(v, nullptr, 10);
        else if (!strcmp(f, "-threads")) p.threads = atoi(v);
        else if (!strcmp(f, "-o")) out = v;
        else if (!strcmp(f, "-law")) {
            if (!strcmp(v, "poisson")) p.len_law = CULDA_LEN_POISSON;
            else if (!strcmp(v, "lognormal")) p.len_law = CULDA_LEN_LOGNORMAL;
            else if (!strcmp(v, "pareto")) p.len_law = CULDA_LEN_PARETO;
            else return usage();
        } else {
            return usage();
        }
    }
    if (out.empty() || p.len_law < 0) return usage();
    culda_corpus *c = nullptr;
    if (culda_corpus_generate(&p, &c) != CULDA_OK) {
        fprintf(stderr, "%s\n", culda_last_error(nullptr));
        return 2;
    }
    const int rc = culda_corpus_write(c, out.c_str(), 1);
    if (rc != CULDA_OK) {
        fprintf(stderr, "%s\n", culda_last_error(nullptr));
    } else {
        printf("{\"num_docs\": %d, \"num_words\": %d, \"num_tokens\": %lld}\n", c->num_docs, c->num_words,
               (long long)c->num_tokens);
    }
    culda_corpus_free(c);
    return rc == CULDA_OK ? 0 : 2;
}
