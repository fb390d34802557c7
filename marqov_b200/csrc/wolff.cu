// Wolff single-cluster updates for sm_100a: level-synchronous frontier BFS.
//
// Reference semantics (src/libmarqov/wolff.h:72-126 with
// src/libmarqov/embedder.h:66-93, Wolff<Ising<int>> src/hamiltonian/Ising.h:126-168,
// Wolff<Potts<Q>> src/hamiltonian/Potts.h:220-320): a bond between a cluster
// site and a candidate neighbour is activated by one uniform draw.  Here that
// draw is keyed by the undirected bond (lower id, cluster serial, upper id), so
// the grown cluster is the seed's connected component of activated bonds and
// does not depend on the visiting order -- a breadth-first frontier grows the
// same cluster as the reference's depth-first stack on the same draws.
//
// One CTA grows one cluster: the frontier lives in a global append-only queue
// (the queue is also the member list), membership in a bit per site set with
// atomicOr, and appends are compacted per warp with a ballot.  Spins are
// flipped after the growth, from the member list, so couplings always see the
// pre-flip state; the visited bits of the members are cleared afterwards so
// the bitmap is zero again for the next cluster.
#include <cuda_runtime.h>

#include <mutex>

#include "wolff_ccl.cuh"
#include "wolff_int8.cuh"

namespace mqv {

template <class Lat>
__global__ void __launch_bounds__(1024) wolff_int8(WolffDev w, Lat lat, int8_t* __restrict__ s,
                                                   uint32_t* __restrict__ visited, int32_t* __restrict__ queue,
                                                   int32_t* __restrict__ out_size, Key key, uint32_t serial,
                                                   uint32_t tg_seed, uint32_t tg_bond, int max_degree)
{
    __shared__ int32_t fbuf[2 * kWolffCap8];
    wolff_int8_cluster(w, lat, s, visited, queue, out_size, key, serial, tg_seed, tg_bond, max_degree, fbuf);
}

unsigned long long accept_cut(int pref, double dE, double beta);

// Wolff activation thresholds on u53 = word >> 11:
//  Ising<int>: add iff real() < prob, prob = -expm1(2 beta J): u53 < ceil(prob 2^53)
//  embedded Ising / Potts: add iff !update_accepted<2>(cpl): u53 >= cut(cpl)
WolffDev wolff_int8_params(const ModelDev& md)
{
    WolffDev w{};
    const double beta = md.beta;
    if (md.kind == MQV_MODEL_ISING) {
        w.mode = 0;
        const double prob = -expm1(2.0 * beta * md.J);
        if (!(prob > 0)) w.thr = 0;
        else {
            // smallest u53 with u53 * 2^-53 >= prob
            const double x = prob * 9007199254740992.0;
            unsigned long long c = (unsigned long long)x;
            if ((double)c < x) ++c;
            w.thr = c > (1ull << 53) ? (1ull << 53) : c;
        }
    } else if (md.kind == MQV_MODEL_POTTS) {
        w.mode = 2;
        w.q = md.q;
        // coupling k * (-0.5) for a neighbour in the seed's old state
        w.thr = accept_cut(2, md.k * -0.5, beta);
    } else {
        // embedded Ising: cpl = J * (s_cur flipped) * s_nbr = -J for an aligned neighbour
        w.mode = 1;
        w.thr = accept_cut(2, -md.J, beta);
    }
    return w;
}

cudaError_t launch_wolff_int8(Sim* s, int slot)
{
    const WolffDev w = wolff_int8_params(s->md);
    int8_t* st = (int8_t*)s->state[s->cur];
    const Key key = make_key(s->seed);
    const uint32_t serial = (uint32_t)s->cluster;
    int32_t* out = s->d_csize + slot;
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC)
        wolff_int8<<<1, 1024, 0, s->stream>>>(w, s->sten, st, s->d_visited, s->d_queue, out, key, serial,
                                              tag(kWolffSeed, s->replica), tag(kWolffBond, s->replica), s->max_degree);
    else
        wolff_int8<<<1, 1024, 0, s->stream>>>(w, s->csr, st, s->d_visited, s->d_queue, out, key, serial,
                                              tag(kWolffSeed, s->replica), tag(kWolffBond, s->replica), s->max_degree);
    s->launches++;
    s->cluster++;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// One cluster of one lattice by connected-component labelling (the batched
// path's kernels, wolff_ccl.cuh, over a one-member table): a fixed number of
// whole-lattice passes whatever the cluster's depth, where a breadth-first
// growth pays a CTA barrier per level -- thousands of levels for a critical
// cluster on a large lattice.  The labels are the handle's queue (n int32).

__global__ void single_rep_set(BatchRep* __restrict__ d, BatchRep r, BatchCtr* __restrict__ ctr, uint32_t serial)
{
    *d = r;
    ctr->e = serial;  // serial = cluster0 (0) + e * 1 + 0; slot = e - ebase = 0
    ctr->ebase = serial;
}

static BatchRep single_rep(const Sim* s)
{
    BatchRep r{};
    r.md = s->md;
    r.st = s->sten;
    r.csr = s->csr;
    r.lat_kind = s->lat_kind;
    r.order = s->d_order;
    if (!s->is_f32) r.w = wolff_int8_params(s->md);
    r.key = make_key(s->seed);
    r.replica = s->replica;
    r.sweep0 = (uint32_t)s->sweep;
    r.cluster0 = 0;
    r.s = s->state[s->cur];
    r.visited = s->d_visited;
    r.queue = s->d_queue;
    r.cuts = s->d_cuts;
    r.D = s->max_degree;
    r.tile = ccl_tile_kind(s->lat_kind, s->dim, s->len);
    return r;
}

template <bool F32>
static void launch_label_t(Sim* s, int32_t* csize)
{
    const int64_t n = s->n;
    const unsigned gb = (unsigned)((n + kBatchMetroThreads - 1) / kBatchMetroThreads);
    CclSeed* sd = (CclSeed*)s->d_seed1;
    single_rep_set<<<1, 1, 0, s->stream>>>(s->d_rep1, single_rep(s), s->d_ctr1, (uint32_t)s->cluster);
    ccl_seed<F32><<<1, 32, 0, s->stream>>>(s->d_rep1, s->d_ctr1, 1, 0, sd, csize, 1);
    ccl_local<F32><<<gb, kBatchMetroThreads, 0, s->stream>>>(s->d_rep1, s->d_sprefix1, s->d_sbrep1, n, sd, s->d_ctr1,
                                                             1, 0);
    ccl_hook<F32><<<gb, kBatchMetroThreads, 0, s->stream>>>(s->d_rep1, s->d_sprefix1, s->d_sbrep1, n, sd, s->d_ctr1,
                                                            1, 0);
    ccl_halve<<<gb, kBatchMetroThreads, 0, s->stream>>>(s->d_rep1, s->d_sprefix1, s->d_sbrep1, n);
    ccl_flip<F32><<<gb, kBatchMetroThreads, 0, s->stream>>>(s->d_rep1, s->d_sprefix1, s->d_sbrep1, n, sd, s->d_ctr1, 1,
                                                            0, csize, 1);
    s->launches += 6;
}

// The one-member tables of the labelling path, allocated on first use.
cudaError_t ensure_label_tables(Sim* s)
{
    if (s->d_sbrep1) return cudaSuccess;  // allocated last: all tables present
    const int64_t n = s->n;
    const int64_t gb = (n + kBatchMetroThreads - 1) / kBatchMetroThreads;
    const int64_t pre[2] = {0, n};
    cudaError_t e = cudaSuccess;
    if (!s->d_rep1) e = cudaMalloc(&s->d_rep1, sizeof(BatchRep));
    if (e == cudaSuccess && !s->d_ctr1) e = cudaMalloc(&s->d_ctr1, sizeof(BatchCtr));
    if (e == cudaSuccess && !s->d_seed1) e = cudaMalloc(&s->d_seed1, sizeof(CclSeed));
    if (e == cudaSuccess && !s->d_sprefix1) e = cudaMalloc(&s->d_sprefix1, sizeof(pre));
    // on the handle's stream, before the kernels that read them
    if (e == cudaSuccess) e = upload_sync(s->stream, s->d_sprefix1, pre, sizeof(pre));
    int32_t* brep = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&brep, sizeof(int32_t) * (size_t)gb);
    if (e == cudaSuccess) e = cudaMemsetAsync(brep, 0, sizeof(int32_t) * (size_t)gb, s->stream);
    if (e == cudaSuccess) s->d_sbrep1 = brep;
    else if (brep) cudaFree(brep);
    return e;
}

// n_emcs EMCS of a mid-size int8 lattice on a thread-block cluster
// (cluster_emcs.cu) through the one-member table; acc NULL: no measurement.
cudaError_t launch_emcs_cluster(Sim* s, int n_emcs, int ncluster, int nmetro, long long* acc, int32_t* csize)
{
    cudaError_t e = ensure_label_tables(s);
    if (e != cudaSuccess) return e;
    BatchRep r = single_rep(s);
    r.cluster0 = (uint32_t)s->cluster;
    single_rep_set<<<1, 1, 0, s->stream>>>(s->d_rep1, r, s->d_ctr1, 0u);
    BatchLaunch b{};
    b.reps = s->d_rep1;
    b.nrep = 1;
    b.acc = acc;
    b.csize = csize;
    e = batch_launch_cluster(b, s->stream, s->d_sbrep1, 1, cluster_ctas(s->n), 0u, 0, n_emcs, ncluster, nmetro);
    s->launches += 2;
    s->sweep += (uint64_t)n_emcs * (uint64_t)nmetro;
    s->cluster += (uint64_t)n_emcs * (uint64_t)ncluster;
    return e;
}

cudaError_t launch_wolff_label(Sim* s, int slot)
{
    const cudaError_t e = ensure_label_tables(s);
    if (e != cudaSuccess) return e;
    if (s->is_f32) launch_label_t<true>(s, s->d_csize + slot);
    else launch_label_t<false>(s, s->d_csize + slot);
    s->cluster++;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Wolff clusters for int8 models with scratch that is never allocated.
//
// mqv_wolff takes its queue, visited bitmap and cluster-size slots from
// device memory that the handle allocates on its first cluster.  A host that
// cannot have device memory allocated at that point -- one that budgets the
// whole of HBM up front for many resident lattices, or that must not let a
// cudaMalloc/cudaFree stall its other streams in the middle of a run -- uses
// mqv_wolff_noalloc instead, which draws the same clusters with the scratch
// below: one file-scope device array, sized for lattices of up to
// kNoAllocMaxSites sites, that exists from module load.
//
// What must start at zero: the visited bitmap.  The module load zero-fills
// the array, and every cluster clears the bits of its members before its
// kernel returns, so the bitmap is zero again between clusters.  The queue
// and size slots are written before they are read.
//
// The array is shared by every handle on a device: calls whose kernels may
// overlap (two streams, two host threads, two handles without ordering
// between them) race on it and must be serialised by the caller.
constexpr int64_t kNoAllocMaxSites = 1 << 20;  // 1,048,576 sites: 4 MiB queue + 128 KiB bitmap
constexpr int kNoAllocMaxClusters = 4096;      // size slots per chunk of clusters
constexpr size_t kNoAllocWords = (size_t)kNoAllocMaxSites + (size_t)kNoAllocMaxSites / 32 + kNoAllocMaxClusters;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

namespace {
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
uint32_t* g_noalloc_addr[kNoAllocMaxDevices] = {};
}  // namespace

int64_t wolff_noalloc_max_sites() { return kNoAllocMaxSites; }
int wolff_noalloc_max_clusters() { return kNoAllocMaxClusters; }

// Device address of the scratch on `device`, looked up once per device with
// that device current (the caller makes it current).  The first lookup may
// load the module, so the first call on a device has to come before any
// stream capture begins.
cudaError_t wolff_noalloc_scratch(int device, uint32_t** out)
{
    if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[device] = static_cast<uint32_t*>(p);
    }
    *out = g_noalloc_addr[device];
    return cudaSuccess;
}

// One cluster of the int8 Wolff update on the static scratch; the activation
// rule and the draws are those of launch_wolff_int8, so the cluster is the
// same.  The size lands in size slot `slot` of the scratch.
cudaError_t launch_wolff_int8_noalloc(Sim* s, uint32_t* scratch, int slot)
{
    const WolffDev w = wolff_int8_params(s->md);
    int32_t* queue = reinterpret_cast<int32_t*>(scratch);
    uint32_t* visited = scratch + kNoAllocMaxSites;
    int32_t* sizes = reinterpret_cast<int32_t*>(visited + kNoAllocMaxSites / 32);
    int8_t* st = (int8_t*)s->state[s->cur];
    const Key key = make_key(s->seed);
    const uint32_t serial = (uint32_t)s->cluster;
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC)
        wolff_int8<<<1, 1024, 0, s->stream>>>(w, s->sten, st, visited, queue, sizes + slot, key, serial,
                                              tag(kWolffSeed, s->replica), tag(kWolffBond, s->replica), s->max_degree);
    else
        wolff_int8<<<1, 1024, 0, s->stream>>>(w, s->csr, st, visited, queue, sizes + slot, key, serial,
                                              tag(kWolffSeed, s->replica), tag(kWolffBond, s->replica), s->max_degree);
    s->launches++;
    s->cluster++;
    return cudaGetLastError();
}

// Size slots of the scratch (for the copy of a chunk's sizes to the host).
const int32_t* wolff_noalloc_sizes(const uint32_t* scratch)
{
    return reinterpret_cast<const int32_t*>(scratch + kNoAllocMaxSites + kNoAllocMaxSites / 32);
}

}  // namespace mqv
