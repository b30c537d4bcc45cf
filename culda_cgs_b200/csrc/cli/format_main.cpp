// format_main.cpp — the `format` command: the reference's preprocessing tool
// (src_format/format.cpp:19-165) over the C ABI of libculda_b200.so, parsing on
// all host cores (OMP_NUM_THREADS caps them).
//
//   format <input text> <output prefix> [numChunks, default 1]
//
// Writes <prefix>.vocab, .doc.idx, .chunk, .word.idx, .word.data (chunk-id
// suffixes on the last two when numChunks > 1) with the bytes the reference's
// tool writes, and prints its progress lines.  Exit status: 0 on success, 1
// for a wrong argument count (the usage line), 2 when a file cannot be opened
// or written (the reference prints the same messages and exits 0).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "culda_b200.h"

int main(int argc, char **argv) {
    if (argc != 3 && argc != 4) {
        printf("Usage:./format input output_prefix numChunks[default=1]\n");
        return 1;
    }
    int num_chunks = argc == 4 ? atoi(argv[3]) : 1;
    if (num_chunks <= 1) num_chunks = 1;

    printf("reading input file ...\n");
    fflush(stdout);
    culda_corpus *c = nullptr;
    culda_vocab *v = nullptr;
    if (culda_corpus_from_text(argv[1], 0, &c, &v) != CULDA_OK) {
        printf("%s\n", culda_last_error(nullptr));
        return 2;
    }
    // The reference's doc -> chunk map (format.cpp:104-132), for the report.
    const long long per_chunk = (c->num_tokens + num_chunks - 1) / num_chunks;
    std::vector<int> start(num_chunks + 1, 0);
    std::vector<long long> size(num_chunks, 0);
    int d = 0;
    for (int ch = 0; ch < num_chunks; ++ch) {
        start[ch] = d;
        while (d < c->num_docs) {
            size[ch] += c->doc_ptr[d + 1] - c->doc_ptr[d];
            ++d;
            if (size[ch] >= per_chunk) break;
        }
    }
    start[num_chunks] = d;
    printf("write vocabulary ...\n");
    printf("mapping chunks ...\n");
    printf("numChunks:%d\n", num_chunks);
    printf("numTokens:%lld\n", (long long)c->num_tokens);
    printf("perChunk :%lld\n", per_chunk);
    const std::string pre(argv[2]);
    for (int ch = 0; ch < num_chunks; ++ch) {
        std::string suffix = num_chunks > 1 ? std::to_string(ch) : std::string();
        printf("----\n");
        printf("chunkId:%d\n", ch);
        printf("numWords:%d\n", c->num_words);
        printf("doc range:%d - %d\n", start[ch], start[ch + 1]);
        printf("chunkSize:%lld\n", size[ch]);
        printf("%s.word.idx%s\n", pre.c_str(), suffix.c_str());
        printf("%s.word.data%s\n", pre.c_str(), suffix.c_str());
    }
    printf("chunk partitioning ...\n");
    printf("write chunks ...\n");
    for (int ch = 0; ch < num_chunks; ++ch) printf("writing chunk %d ...\n", ch);
    fflush(stdout);
    int rc = culda_format_write(c, v, argv[2], num_chunks);
    if (rc != CULDA_OK) printf("%s\n", culda_last_error(nullptr));
    culda_corpus_free(c);
    culda_vocab_free(v);
    return rc == CULDA_OK ? 0 : 2;
}
