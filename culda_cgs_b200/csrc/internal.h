// internal.h — declarations shared by the library's translation units.
#pragma once
#include <stdarg.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/culda_b200.h"

namespace culda {

// Thread-local message of the last failed call that has no context.
void set_global_error(const char *fmt, ...);
const char *global_error();

// Whole file into `buf`; false when it cannot be opened or read.
bool read_file_bytes(const std::string &path, std::vector<char> &buf);

// Host checks of a corpus descriptor (prefix arrays, doc ids, doc lengths).
int validate_corpus(const culda_corpus *c);

// cudaMalloc on the current device; when it runs out of memory, the
// context-block pool's unused reserve on that device is handed back and the
// allocation is tried once more (returns the CUDA status).
int device_malloc(void **p, size_t bytes);

// Device error word bits.
enum : int32_t {
    kErrTopicRange = 1,   // a topic >= K was found in the topic array
    kErrDocRange = 2,     // a doc id outside [0, D) reached the sampler
    kErrRowRange = 4,     // a theta row outside the theta array or misaligned
    kErrLongDoc = 8,      // a document longer than 65535 tokens
    kErrTimeout = 16,     // a bounded wait on an mbarrier gave up (the tile was not stored)
    kErrWordRange = 32    // a word id outside [0, V) reached the encoder
};

// Sampler block size and the dynamic shared memory it needs for K topics.
constexpr int kSampleThreads = 128;
constexpr int kThetaWarps = 8;

}  // namespace culda
