// Batched elementary Monte Carlo steps over many independent int8
// simulations (replicas, temperatures, lattice sizes) on one GPU.
//
// MARQOV runs such a farm as one simulation per CPU thread
// (src/libmarqov/marqovscheduler.h:64-494); on the GPU the same farm is a
// handful of kernels per EMCS that each cover every replica:
//   batch_wolff_int8    one CTA per replica grows and flips its cluster,
//   batch_metro_int8    one launch per colour over the sites of that colour of
//                       all replicas (flattened, block -> first replica table),
//   batch_measure_int8  CTAs (part, replica) accumulate each replica's
//                       observables,
//   batch_tick          advances the EMCS counter.
// Every per-step number (sweep and cluster serials, measurement slot) is
// derived on the device from that counter, so the kernels of one EMCS form a
// fixed sequence: it is captured once into a CUDA graph and replayed.
// The per-replica arithmetic is that of the per-handle kernels, keyed by each
// replica's (seed, replica id, sweep, site), so a batched run equals running
// every member handle on its own, bit for bit.
#include <cuda_runtime.h>

#include "batch.h"
#include "int8_site.cuh"
#include "wolff_int8.cuh"

namespace mqv {

__global__ void batch_metro_int8(const BatchRep* __restrict__ reps, const int64_t* __restrict__ half_prefix,
                                 const int32_t* __restrict__ block_rep, int64_t total, int colour,
                                 const BatchCtr* __restrict__ ctr, int nmetro, int j)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int r = block_rep[blockIdx.x];
    while (g >= half_prefix[r + 1]) ++r;
    const BatchRep& R = reps[r];
    const uint32_t sweep = R.sweep0 + ctr->e * (uint32_t)nmetro + (uint32_t)j;
    int8_site(R.md, R.st, R.s, parity_site(R.st, g - half_prefix[r], colour), R.key, sweep, R.replica, R.cuts, R.D);
}

__global__ void __launch_bounds__(1024) batch_wolff_int8(const BatchRep* __restrict__ reps,
                                                         const BatchCtr* __restrict__ ctr, int ncluster, int c,
                                                         int32_t* __restrict__ csize, int nrep)
{
    const BatchRep& R = reps[blockIdx.x];
    const uint32_t e = ctr->e, slot = e - ctr->ebase;
    const uint32_t serial = R.cluster0 + e * (uint32_t)ncluster + (uint32_t)c;
    wolff_int8_cluster(R.w, R.st, R.s, R.visited, R.queue, csize + ((size_t)slot * ncluster + c) * nrep + blockIdx.x,
                       R.key, serial, tag(kWolffSeed, R.replica), tag(kWolffBond, R.replica));
}

__global__ void batch_measure_int8(const BatchRep* __restrict__ reps, const BatchCtr* __restrict__ ctr,
                                   long long* __restrict__ acc, int nrep)
{
    const BatchRep& R = reps[blockIdx.y];
    const uint32_t slot = ctr->e - ctr->ebase;
    measure_int8_part(R.md, R.st, R.s, acc + ((size_t)slot * nrep + blockIdx.y) * kAccStride, blockIdx.x, gridDim.x);
}

__global__ void batch_tick(BatchCtr* ctr) { ctr->e += 1u; }

__global__ void batch_chunk_start(BatchCtr* ctr, uint32_t e)
{
    ctr->e = e;
    ctr->ebase = e;
}

// acc/out: slot-major, entry k = slot * nrep + replica
__global__ void batch_finalize_int8(const BatchRep* __restrict__ reps, const long long* __restrict__ acc, int nslots,
                                    int nrep, double* __restrict__ out)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)nslots * nrep) return;
    const BatchRep& R = reps[k % nrep];
    finalize_int8_one(R.md, R.st.n, acc + (size_t)k * kAccStride, out + 4 * (size_t)k);
}

// ---- launchers (stream-ordered; all capturable) ------------------------------------

cudaError_t batch_launch_emcs(const BatchLaunch& b, cudaStream_t st, int ncluster, int nmetro, uint64_t* launches)
{
    for (int c = 0; c < ncluster; ++c) {
        batch_wolff_int8<<<b.nrep, 1024, 0, st>>>(b.reps, b.ctr, ncluster, c, b.csize, b.nrep);
        ++*launches;
    }
    for (int j = 0; j < nmetro; ++j)
        for (int colour = 0; colour < 2; ++colour) {
            batch_metro_int8<<<b.metro_blocks, kBatchMetroThreads, 0, st>>>(b.reps, b.half_prefix, b.block_rep,
                                                                             b.total_half, colour, b.ctr, nmetro, j);
            ++*launches;
        }
    batch_measure_int8<<<dim3(b.meas_parts, b.nrep), 256, 0, st>>>(b.reps, b.ctr, b.acc, b.nrep);
    batch_tick<<<1, 1, 0, st>>>(b.ctr);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t batch_launch_chunk_start(const BatchLaunch& b, cudaStream_t st, uint32_t e)
{
    batch_chunk_start<<<1, 1, 0, st>>>(b.ctr, e);
    return cudaGetLastError();
}

cudaError_t batch_launch_finalize(const BatchLaunch& b, cudaStream_t st, int nslots, double* out)
{
    const int64_t n = (int64_t)nslots * b.nrep;
    batch_finalize_int8<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(b.reps, b.acc, nslots, b.nrep, out);
    return cudaGetLastError();
}

}  // namespace mqv
