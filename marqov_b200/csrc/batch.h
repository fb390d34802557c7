// Internal declarations of the batched EMCS path (batch.cu, capi.cu).
#pragma once
#include "engine.h"

namespace mqv {

// One member of a batch as the batched kernels see it.
struct BatchRep {
    ModelDev md;
    StencilDev st;              // hypercubic members
    CSRDev csr;                 // CSR members
    int lat_kind;               // MQV_LATTICE_*
    const int32_t* order;       // CSR: sites grouped by colour
    WolffDev w;                 // int8 activation rule
    Key key;
    uint32_t replica;
    uint32_t sweep0, cluster0;  // the member handle's counters when the run started
    void* s;                    // state: int8_t or float, reference site order
    uint32_t* visited;          // Wolff scratch of the member handle
    int32_t* queue;
    const unsigned long long* cuts;  // int8: the member's Metropolis cut table
    int D;                           // int8: its maximum degree
    int resident;                    // runs in one CTA's shared memory (batch_resident), not in the graphs
    int tile;                        // labelling order (ccl_site): 0 site order, 2 16x16 tiles, 3 8x8x4 tiles
};

// Labelling order of a lattice: 2D stencils with len % 16 == 0 in 16 x 16
// tiles, 3D stencils with len % 8 == 0 in 8 x 8 x 4 tiles (256 sites, one
// CTA block of the labelling kernels each), others in site order.
inline int ccl_tile_kind(int lat_kind, int dim, int len)
{
    if (lat_kind != MQV_LATTICE_HYPERCUBIC) return 0;
    if (dim == 2 && len % 16 == 0) return 2;
    if (dim == 3 && len % 8 == 0) return 3;
    return 0;
}

// Sites of a member's lattice.
__host__ __device__ __forceinline__ int64_t rep_sites(const BatchRep& R)
{
    return R.lat_kind == MQV_LATTICE_HYPERCUBIC ? R.st.n : R.csr.n;
}

// Device counters of a run: EMCS done, first EMCS of the current chunk
// (measurement slot = e - ebase).
struct BatchCtr {
    uint32_t e;
    uint32_t ebase;
};

constexpr int kBatchMetroThreads = 256;

// Device tables and shapes the launchers need.  Colour c's work is the
// concatenation over members of their colour-c sites, each member's count
// ccount[r * ncol + c] padded to whole warp blocks of kAccSites sites:
// prefix + c * (nrep + 1) holds the padded prefix sums, block_rep +
// block_off[c] the first member of each CTA's first warp block,
// cbegin[r * ncol + c] member r's offset into its colour order.
struct BatchLaunch {
    const BatchRep* reps;
    int nrep;
    int f32;                     // float members (else int8)
    int ncol;                    // colours of the member with the most
    const int64_t* prefix;       // [ncol][nrep + 1]
    const int32_t* block_rep;    // [sum of blocks]
    const int32_t* cbegin;       // [nrep][ncol]
    const int32_t* ccount;       // [nrep][ncol] sites of each colour
    const int* block_off;        // host: [ncol] offsets into block_rep
    const int* blocks;           // host: [ncol] blocks of each colour
    const int64_t* total;        // host: [ncol] padded work items of each colour
    // measurement: member r's sites are split over meas_prefix[r + 1] -
    // meas_prefix[r] CTAs (about 4096 sites each); meas_rep[c] is CTA c's member
    const int32_t* meas_prefix;  // [nrep + 1]
    const int32_t* meas_rep;     // [meas_blocks]
    int meas_blocks;
    // site-level work (every site of every member) for the labelling Wolff
    const int64_t* site_prefix;  // [nrep + 1]
    const int32_t* site_block_rep;
    int64_t total_sites;
    int site_blocks;
    void* ccl_seeds;             // [nrep] seeds of the labelling Wolff
    int wolff_ccl;               // clusters by labelling (1) or by one CTA's breadth-first growth (0)
    BatchCtr* ctr;
    long long* acc;              // slot-major accumulators (int64, or FP64 in the same words)
    int32_t* csize;              // cluster sizes: (slot * ncluster + c) * nrep + r
};

cudaError_t batch_launch_emcs(const BatchLaunch& b, cudaStream_t st, int ncluster, int nmetro);
// EMCS e0 .. e0 + count - 1 of the resident members order[0 .. nres) (the
// largest with max_n sites), measurement slots from slot0 (smem_emcs.cu)
cudaError_t batch_launch_resident(const BatchLaunch& b, cudaStream_t st, const int32_t* order, int nres, size_t smem,
                                  uint32_t e0, int slot0, int count, int ncluster, int nmetro, int device);
// the same for members held by clusters of `ctas` CTAs (cluster_emcs.cu)
cudaError_t batch_launch_cluster(const BatchLaunch& b, cudaStream_t st, const int32_t* order, int nmem, int ctas,
                                 uint32_t e0, int slot0, int count, int ncluster, int nmetro);
int cluster_ctas(int64_t n);
bool cluster_launchable(int ctas);
cudaError_t batch_launch_chunk_start(const BatchLaunch& b, cudaStream_t st, uint32_t e);
cudaError_t batch_launch_finalize(const BatchLaunch& b, cudaStream_t st, int nslots, double* out);
// raw sums of the chunk's slots -> samples[r][e0 + slot][4] (n_total EMCS per member)
cudaError_t batch_launch_samples(const BatchLaunch& b, cudaStream_t st, int nslots, int e0, int n_total,
                                 double* samples);
// replica exchange of the step's disjoint pairs ([npairs][2] member ids) from
// the energies of the EMCS just done; perm/flags as batch_temper describes
cudaError_t batch_launch_temper(const BatchLaunch& b, cudaStream_t st, const int32_t* pairs, int npairs, uint32_t step,
                                uint64_t seed, double en_min, double en_max, int32_t* perm, int32_t* flags);
// kernel launches of one EMCS
inline uint64_t batch_launches_per_emcs(const BatchLaunch& b, int ncluster, int nmetro)
{
    int live = 0;
    for (int c = 0; c < b.ncol; ++c) live += b.total[c] > 0;
    const uint64_t ccl = b.site_blocks > 0 ? 5ull : 0ull;  // seed, local, hook, halve, flip
    return (uint64_t)ncluster * (b.wolff_ccl ? ccl : 1ull) + (uint64_t)nmetro * (uint64_t)live +
           (b.meas_blocks > 0 ? 2ull : 1ull);
}

}  // namespace mqv
