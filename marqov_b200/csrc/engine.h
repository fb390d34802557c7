// Internal declarations of the marqov_b200 engine (not part of the ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/marqov_b200.h"
#include "common.cuh"

namespace mqv {

// Observable accumulators of one measurement slot (int64, exact for integer
// models; float models keep FP64 sums in the double view of the same slot).
constexpr int kAccStride = 72;
enum AccIdx { kAccEne = 0, kAccMag = 1, kAccSq = 2, kAccQ4 = 3, kAccMagY = 4, kAccMagZ = 5, kAccPotts = 8 };

// Model parameters as the kernels see them.
struct ModelDev {
    int kind;
    int q;
    int proposal;
    int symd;
    double J, h, h2, k, delta, cap;
    double beta;
    // termselector of the lattice (src/libmarqov/metropolishelpers.h:402-430):
    // 0 = every onsite term acts on every site; 1 = SimpleBipartite
    // (src/lattice/simple_bipartite.h:22-41), onsite term p acts on the
    // sites whose coordinate sum has parity p -- the checkerboard colour.
    int termsel;
};

// Weights of onsite terms 0 and 1 at a site of sublattice (colour) `sub`.
MQV_HD double onsite_w0(const ModelDev& m, int sub) { return (m.termsel && sub) ? 0.0 : 1.0; }
MQV_HD double onsite_w1(const ModelDev& m, int sub) { return (m.termsel && !sub) ? 0.0 : 1.0; }

// Layout of the fused 2D Ising path: row y holds its even-x sites, then its
// odd-x sites (split rows); within each half, the 32 sites of a word (32
// consecutive sites of that parity, 32 bytes) are stored transposed, site s
// of the word at byte 4 (s & 7) + (s >> 3), so that bit 1 of byte k of the
// word's 32-bit lane i belongs to site 8k + i.
MQV_HD int64_t split_addr(int64_t y, int x, int len)
{
    const int m = x >> 1;
    return y * len + (x & 1) * (len >> 1) + (m & ~31) + 4 * (m & 7) + ((m >> 3) & 3);
}

// Periodic hypercubic stencil: neighbour order +x,-x,+y,-y,... of
// FixedDimRegularHypercubic::nbrs (src/lattice/regular_hypercubic.h:31-66).
struct StencilDev {
    int dim;
    int len;
    int64_t n;  // < 2^31: site indices fit 32 bits
    int64_t pows[4];
    int split;      // 2D state stored in split rows (see split_addr)
    int lg;         // log2(len) when len is a power of two, else -1
    uint64_t mlen;  // ceil(2^64 / len) otherwise: u / len = mulhi64(u, mlen), exact for 32-bit u
    // bond weights (bnds, e.g. RegularRandomBond): plane d holds the bond of
    // every site to its +d neighbour, fb[d n + i]; the bond to the -d
    // neighbour is that neighbour's +d bond.  NULL: every bond is 1.
    const int8_t* fb;
    MQV_HD uint32_t divlen(uint32_t u) const
    {
#ifdef __CUDA_ARCH__
        return (uint32_t)__umul64hi((unsigned long long)u, (unsigned long long)mlen);
#else
        return (uint32_t)(((unsigned __int128)u * mlen) >> 64);
#endif
    }
    // coordinate j of site i (shifts for power-of-two sides, multiply-high
    // division otherwise)
    MQV_HD int coord(int64_t i, int j) const
    {
        uint32_t u = (uint32_t)i;
        if (lg >= 0) return (int)((u >> (lg * j)) & (uint32_t)(len - 1));
        for (int k = 0; k < j; ++k) u = divlen(u);
        return (int)(u - divlen(u) * (uint32_t)len);
    }
    // device address of site i
    MQV_HD int64_t addr(int64_t i) const
    {
        if (!split) return i;
        return split_addr(coord(i, 1), coord(i, 0), len);  // split layouts are 2D
    }
    MQV_HD int degree(int64_t) const { return 2 * dim; }
    // pows[j] by selects: no dynamic index, so that a copy of the stencil in
    // a kernel stays in registers instead of local memory
    MQV_HD int64_t pow_of(int j) const { return j == 0 ? pows[0] : j == 1 ? pows[1] : j == 2 ? pows[2] : pows[3]; }
    MQV_HD int64_t nbr(int64_t i, int slot) const
    {
        const int j = slot >> 1;
        const int64_t p = pow_of(j);
        const int x = coord(i, j);
        if ((slot & 1) == 0) return x == len - 1 ? i - (int64_t)(len - 1) * p : i + p;
        return x == 0 ? i + (int64_t)(len - 1) * p : i - p;
    }
    MQV_HD int bond(int64_t i, int slot) const
    {
        if (!fb) return 1;
        const int64_t j = (slot & 1) ? nbr(i, slot) : i;
        return fb[(int64_t)(slot >> 1) * n + j];
    }
};

// The same stencil with its dimension, whether its side is a power of two
// and whether its state is stored in split rows fixed at compile time, for
// the per-site kernels: neighbour loops unroll (degree 2 D), each coordinate
// is computed once per site and shared by its two neighbours, the last
// coordinate needs no remainder, and index arithmetic stays in 32 bits
// (n < 2^31).  The neighbour order and the sites are those of StencilDev.
template <int D, bool P2, bool SPLIT = false>
struct StencilDim : StencilDev {
    MQV_HD explicit StencilDim(const StencilDev& s) : StencilDev(s) {}
    MQV_HD int degree(int64_t) const { return 2 * D; }
    MQV_HD int coord(int64_t i, int j) const
    {
        uint32_t u = (uint32_t)i;
        if (P2) return j == D - 1 ? (int)(u >> (lg * j)) : (int)((u >> (lg * j)) & (uint32_t)(len - 1));
        if (j >= 1) u = divlen(u);
        if (j >= 2) u = divlen(u);
        if (j == D - 1) return (int)u;  // u < len already
        return (int)(u - divlen(u) * (uint32_t)len);
    }
    MQV_HD int64_t addr(int64_t i) const
    {
        if (!SPLIT) return i;
        return split_addr(coord(i, 1), coord(i, 0), len);
    }
    MQV_HD int64_t nbr(int64_t i, int slot) const
    {
        const int j = slot >> 1;
        const uint32_t p = (uint32_t)pow_of(j), u = (uint32_t)i, w = (uint32_t)(len - 1) * p;
        const int x = coord(i, j);
        if ((slot & 1) == 0) return (int64_t)(x == len - 1 ? u - w : u + p);
        return (int64_t)(x == 0 ? u + w : u - p);
    }
    MQV_HD int bond(int64_t i, int slot) const
    {
        if (!fb) return 1;
        const int64_t j = (slot & 1) ? nbr(i, slot) : i;
        return fb[(int64_t)(slot >> 1) * n + j];
    }
};

// Call f(lat) with the stencil's dimension (2 or 3), power-of-two side and
// split-row storage fixed where possible (StencilDev otherwise).
template <class F>
__device__ __forceinline__ void with_dim(const StencilDev& st, F&& f)
{
    const bool p2 = st.lg >= 0;
    if (st.dim == 2) {
        if (st.split) {
            if (p2) f(StencilDim<2, true, true>(st));
            else f(StencilDim<2, false, true>(st));
        } else {
            if (p2) f(StencilDim<2, true>(st));
            else f(StencilDim<2, false>(st));
        }
    } else if (st.dim == 3 && !st.split) {
        if (p2) f(StencilDim<3, true>(st));
        else f(StencilDim<3, false>(st));
    } else {
        f(st);
    }
}

struct CSRDev {
    int64_t n;
    const int32_t* rp;
    const int32_t* ci;
    const int8_t* bonds;
    MQV_HD int64_t addr(int64_t i) const { return i; }
    MQV_HD int degree(int64_t i) const { return rp[i + 1] - rp[i]; }
    MQV_HD int64_t nbr(int64_t i, int slot) const { return ci[rp[i] + slot]; }
    MQV_HD int bond(int64_t i, int slot) const { return bonds ? bonds[rp[i] + slot] : 1; }
};

// Wolff activation rule of the int8 models.
struct WolffDev {
    int mode;               // 0 Ising exact, 1 embedded (threshold rule), 2 Potts
    unsigned long long thr; // Ising exact: u53 < thr adds; embedded/Potts: u53 >= thr adds
    int q;
};
// Shared memory of a breadth-first cluster kernel for the frontier of the
// current and of the next level (site ids; float models also the site's
// projection on the embedding direction), so that a level reads its sites
// from shared memory; a level larger than the buffer is read from the
// global queue.  int8: 2 x 4608 ids; float: 2 x 1536 (id, projection).
constexpr int kWolffSmem = 36864;
constexpr int kWolffCap8 = kWolffSmem / 8;
constexpr int kWolffCapF = kWolffSmem / 24;

// Threads given to one frontier site in a breadth-first cluster level: one
// per neighbour on stencils; on CSR graphs up to 8, a site of higher degree
// looping over its neighbours t0, t0 + lanes, ...
MQV_HD int wolff_lanes(const StencilDev& st, int) { return 2 * st.dim; }
MQV_HD int wolff_lanes(const CSRDev&, int max_degree) { return max_degree < 1 ? 1 : max_degree > 8 ? 8 : max_degree; }

// u53 cuts of an int8 model's Metropolis moves for lattices of maximum degree
// D, indexed as int8_site computes its dE index (host side).
std::vector<unsigned long long> int8_cut_table(const ModelDev& md, int D);
// Activation rule of an int8 model (host side, wolff.cu).
WolffDev wolff_int8_params(const ModelDev& md);

// The resident path (smem_emcs.cu): int8 lattices of at most this many
// sites run whole chunks of EMCS in the shared memory of one CTA.
constexpr int64_t kResidentMaxSites = 65536;
// batches launch their resident members in two classes, up to this many
// sites (several CTAs per SM) and above
constexpr int64_t kResSmall = 16384;
struct Sim;
bool resident_fits(const Sim* s);
// dynamic shared memory of the resident kernels for one lattice (smem_emcs.cu)
size_t resident_smem_for(const StencilDev& st);
// lattices of up to 8 x 32768 sites on a thread-block cluster (cluster_emcs.cu)
int cluster_ctas(int64_t n);
bool cluster_launchable(int ctas);

struct Sim;
// Smallest u53 rejected by update_accepted<pref>(dE, beta, .) (2^53: all accepted).
unsigned long long accept_cut(int pref, double dE, double beta);
cudaError_t launch_selftest_philox(uint64_t seed, uint32_t c1, uint32_t c2, uint32_t c3, int n,
                                   uint32_t* d_eng, uint32_t* d_cur, cudaStream_t st);

struct Sim {
    mqv_model_desc model{};
    ModelDev md{};
    int lat_kind = 0;
    int termsel = 0;  // lattice termselector (ModelDev::termsel)
    int dim = 0, len = 0;
    int64_t n = 0;
    int symd = 1;
    bool is_f32 = false;
    size_t state_bytes = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // state: two buffers; stencil sweeps ping-pong between them
    void* state[2] = {nullptr, nullptr};
    int cur = 0;
    bool initialised = false;
    // lattice
    StencilDev sten{};
    CSRDev csr{};
    int32_t* d_rp = nullptr;
    int32_t* d_ci = nullptr;
    int8_t* d_bonds = nullptr;
    int max_degree = 0;
    uint64_t lat_hash = 0;            // CSR: FNV-1a of row_ptr, col_idx and bonds
    std::vector<int32_t> colour_ptr;  // host
    int32_t* d_order = nullptr;       // sites grouped by colour
    // random numbers
    uint64_t seed = 0;
    uint32_t replica = 0;
    uint64_t sweep = 0;
    uint64_t cluster = 0;
    // fused 2D Ising path (ising2d.cu): state in split rows
    bool fused_ising2d = false;
    int num_sms = 148;
    int* d_status = nullptr;   // device error word of bounded waits
    int* d_counter = nullptr;  // tile counter of the fused sweep
    double thr_J = 0, thr_beta = -1;  // (J, beta) the cached 2D thresholds belong to
    unsigned long long thr_cut[5] = {};
    int sweep_cfg = -1;  // autotuned fused-sweep configuration (-1: not chosen yet)
    uint32_t flags = 0;  // MQV_FLAG_* of the run parameters
    // a device wait gave up: compute is refused until the state is set again
    bool failed = false;
    int cluster_ok = -1;  // the device co-schedules this lattice's thread-block cluster (-1: not asked yet)
    // one-shot injected timeout of the next fused band sweep (tests)
    int inject_row = -1;
    unsigned long long inject_wait_ns = 0;
    // int8 models: u53 cut of every possible dE (int8_cut_table), on the device
    unsigned long long* d_cuts = nullptr;
    int n_cuts = 0;
    double cuts_for[7] = {0, 0, 0, -1, 0, 0, 0};  // (J, h, k, beta, kind, h2, termsel) of the table
    // measurement
    int nslots = 0;
    long long* d_acc = nullptr;  // nslots * kAccStride
    double* d_obs = nullptr;     // nslots * 4
    // Wolff scratch
    uint32_t* d_visited = nullptr;  // n bits
    int32_t* d_queue = nullptr;     // n entries
    int32_t* d_csize = nullptr;     // cluster sizes, nslots_c entries
    int nslots_c = 0;
    // clusters of this lattice: MQV_WOLFF_AUTO (by size), _BFS or _LABEL, and
    // the one-member tables of the labelling kernels (wolff.cu)
    int wolff_algo = 0;
    struct BatchRep* d_rep1 = nullptr;
    struct BatchCtr* d_ctr1 = nullptr;
    void* d_seed1 = nullptr;
    int64_t* d_sprefix1 = nullptr;
    int32_t* d_sbrep1 = nullptr;
    uint64_t launches = 0;
};

void set_error(const std::string& msg);

// Host -> device copy ordered on `st` and complete on return.  The handles'
// streams are created non-blocking, so a cudaMemcpy / cudaMemset on the
// legacy stream is NOT ordered before their kernels (a pageable cudaMemcpy may
// return before its DMA lands, and cudaMemset of device memory is
// asynchronous): every upload a handle's kernels read goes through here.
inline cudaError_t upload_sync(cudaStream_t st, void* dst, const void* src, size_t bytes)
{
    if (bytes == 0) return cudaSuccess;
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    return e != cudaSuccess ? e : cudaStreamSynchronize(st);  // the host buffer may go out of scope
}

}  // namespace mqv
