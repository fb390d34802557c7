// Internal declarations of the batched EMCS path (batch.cu, capi.cu).
#pragma once
#include "engine.h"

namespace mqv {

// One replica of a batch as the batched kernels see it.
struct BatchRep {
    ModelDev md;
    StencilDev st;
    WolffDev w;
    Key key;
    uint32_t replica;
    uint32_t sweep0, cluster0;  // the member handle's counters when the run started
    int8_t* s;                  // state (reference site order)
    uint32_t* visited;          // Wolff scratch of the member handle
    int32_t* queue;
    const unsigned long long* cuts;  // the member's Metropolis cut table
    int D;                           // its maximum degree
};

// Device counters of a run: EMCS done, first EMCS of the current chunk
// (measurement slot = e - ebase).
struct BatchCtr {
    uint32_t e;
    uint32_t ebase;
};

constexpr int kBatchMetroThreads = 256;

// Device pointers and shapes the launchers need.
struct BatchLaunch {
    const BatchRep* reps;
    const int64_t* half_prefix;  // nrep + 1 prefix sums of n / 2
    const int32_t* block_rep;    // first replica of each metropolis block
    int64_t total_half;
    int metro_blocks;
    int meas_parts;              // measurement CTAs per replica
    int nrep;
    BatchCtr* ctr;
    long long* acc;              // slot-major accumulators
    int32_t* csize;              // cluster sizes: (slot * ncluster + c) * nrep + r
};

cudaError_t batch_launch_emcs(const BatchLaunch& b, cudaStream_t st, int ncluster, int nmetro, uint64_t* launches);
cudaError_t batch_launch_chunk_start(const BatchLaunch& b, cudaStream_t st, uint32_t e);
cudaError_t batch_launch_finalize(const BatchLaunch& b, cudaStream_t st, int nslots, double* out);

}  // namespace mqv
