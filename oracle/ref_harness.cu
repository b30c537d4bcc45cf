// ref_harness.cu — TEST INFRASTRUCTURE.  Drives the reference's own host
// classes and kernels (compiled from its sources with oracle/ref_compat.h) on
// one GPU to record golden vectors: the initial count build of
// SingleChunkSingleGPU (src_culda/train/SingleChunkSingleGPU.h:15-41) on a
// given topic assignment, then optionally one sampling pass and its
// log-likelihood (SingleChunkSingleGPU.h:55-58,75-105).
//
// usage: ref_harness <prefix> <k> <alpha> <beta> <topics.bin int16[N]> <out_prefix> <sample 0|1>
// writes <out_prefix>.<name>.bin for phi, nk, phihead, theta_a, theta_ja,
// max_ia, cur_ia, doc_rev_idx, slot_word, slot_range, and (sample) z_new, loglik.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "kernel/lda_train_kernel.h"
#include "model/doc.h"
#include "model/model_phi.h"
#include "model/model_theta.h"
#include "model/vocab.h"

static void dump(const std::string &path, const void *p, size_t bytes) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f || fwrite(p, 1, bytes, f) != bytes) {
        fprintf(stderr, "write %s failed\n", path.c_str());
        exit(2);
    }
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc != 8) {
        fprintf(stderr, "usage: %s prefix k alpha beta topics.bin out_prefix sample\n", argv[0]);
        return 1;
    }
    const std::string prefix = argv[1], out = argv[6];
    const int k = atoi(argv[2]);
    const float alpha = (float)atof(argv[3]), beta = (float)atof(argv[4]);
    const int sample = atoi(argv[7]);

    Document doc;
    doc.loadDocument(prefix, 1);
    DocChunk *ch = doc.docChunkVec[0];
    {
        FILE *f = fopen(argv[5], "rb");
        if (!f || fread(ch->wordTopics, sizeof(short), ch->chunkNumTokens, f) != (size_t)ch->chunkNumTokens) {
            fprintf(stderr, "read %s failed\n", argv[5]);
            return 2;
        }
        fclose(f);
    }
    ch->allocGPU(0);
    ch->toGPU();
    ModelPhi modelPhi(k, 1, doc.numDocs, doc.numWords, 1);
    modelPhi.InitData(doc);
    modelPhi.UpdatePhiGPU(doc, 0);
    modelPhi.UpdatePhiHead(beta);
    ModelTheta modelTheta(k, doc.numDocs, doc.numWords, 1);
    modelTheta.InitData(doc);
    modelTheta.UpdateThetaGPU(doc);
    cudaDeviceSynchronize();
    modelPhi.MasterGPUToCPU();
    modelTheta.toCPU();
    cudaDeviceSynchronize();

    const size_t vk = (size_t)doc.numWords * k;
    ModelThetaChunk *th = modelTheta.thetaChunkVec[0];
    dump(out + ".phi.bin", modelPhi.hostPhiTopicWordShort[0], vk * sizeof(int));
    dump(out + ".nk.bin", modelPhi.hostPhiTopic[0], (size_t)k * sizeof(int));
    std::vector<unsigned short> head(vk);
    cudaMemcpy(head.data(), modelPhi.phiChunkVec[0]->devicePhiHead, vk * sizeof(unsigned short),
               cudaMemcpyDeviceToHost);
    dump(out + ".phihead.bin", head.data(), vk * sizeof(unsigned short));
    dump(out + ".theta_a.bin", th->hostThetaA, (size_t)th->chunkNNZ * sizeof(short));
    dump(out + ".theta_ja.bin", th->hostThetaJA, (size_t)th->chunkNNZ * sizeof(short));
    dump(out + ".max_ia.bin", th->hostThetaMaxIA, (size_t)(doc.numDocs + 1) * sizeof(int));
    dump(out + ".cur_ia.bin", th->hostThetaCurIA, (size_t)doc.numDocs * sizeof(int));
    dump(out + ".doc_rev_idx.bin", ch->docRevIdx, (size_t)ch->chunkNumTokens * sizeof(int));
    dump(out + ".slot_word.bin", ch->slotIdToWordId, (size_t)ch->numSlots * sizeof(int));
    dump(out + ".slot_range.bin", ch->slotIndices, (size_t)ch->numSlots * 2 * sizeof(long long));

    if (sample) {
        const int randStateSize = 256 * 20;
        curandState *rs = nullptr;
        cudaMalloc(&rs, sizeof(curandState) * randStateSize);
        initRandState<<<randStateSize / 256, 256>>>(rs);
        cudaDeviceSynchronize();
        LDAKernelTrain<<<ch->numSlots, TrainBlockSize>>>(
            k, alpha, beta, doc.numDocs, doc.numWords, ch->chunkNumTokens, ch->deviceWordIndices,
            ch->deviceSlotIdToWordId, ch->deviceSlotIndices, ch->deviceWordTokens, ch->deviceWordTopics,
            th->deviceThetaA, th->deviceThetaMaxIA, th->deviceThetaCurIA, th->deviceThetaJA, th->docIdStart,
            modelPhi.phiChunkVec[0]->devicePhiTopicWordShort, modelPhi.phiChunkVec[0]->devicePhiTopic,
            modelPhi.phiChunkVec[0]->devicePhiHead, rs, randStateSize, 0, ch->deviceWordPerplexity,
            ch->deviceDocRevIndices);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            fprintf(stderr, "LDAKernelTrain: %s\n", cudaGetErrorString(e));
            return 3;
        }
        double ll = LDATrainPerplexity(doc);
        ch->toCPU();
        dump(out + ".z_new.bin", ch->wordTopics, (size_t)ch->chunkNumTokens * sizeof(short));
        dump(out + ".loglik.bin", &ll, sizeof(double));
        printf("loglik %.10f\n", ll);
        cudaFree(rs);
    }
    printf("harness ok: D=%d V=%d N=%lld slots=%d nnzcap=%d\n", doc.numDocs, doc.numWords,
           (long long)ch->chunkNumTokens, ch->numSlots, th->chunkNNZ);
    return 0;
}
