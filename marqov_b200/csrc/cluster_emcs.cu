// Elementary Monte Carlo steps of mid-size int8 lattices held in the
// distributed shared memory of a thread-block cluster, for sm_100a.
//
// A lattice of up to kClMaxCTAs x kClSlab sites (the 384^2 and 512^2 members
// of a farm) does not fit one CTA's shared memory, but it fits the shared
// memory of a cluster of CTAs on neighbouring SMs: rank r keeps sites
// [r kClSlab, (r + 1) kClSlab) -- their spins, 32-bit union-find parents and
// candidate bits -- and reaches the other ranks' sites through distributed
// shared memory (loads, stores and compare-and-swap on addresses mapped with
// map_shared_rank).  The chunk of EMCS then runs as in the one-CTA resident
// kernel (smem_emcs.cu): clusters by labelling (the seed's component of the
// bonds activated on their keyed draws, the breadth-first kernel's cluster),
// sweeps on the same keyed words with the warps' shared acceptance bytes,
// the measurement accumulators -- with cluster barriers between the phases
// instead of CTA barriers.  Every CTA of a cluster passes the same sequence
// of cluster barriers, and the last barrier keeps every CTA resident until
// no rank reads its shared memory any more.  Results equal the other paths
// bit for bit.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "batch.h"
#include "int8_site.cuh"
#include "wolff_int8.cuh"

namespace cg = cooperative_groups;

namespace mqv {

constexpr int kClThreads = 512;
constexpr int kClWarps = kClThreads / 32;
constexpr int kClSlabLog = 15;
constexpr int64_t kClSlab = (int64_t)1 << kClSlabLog;  // sites per CTA
constexpr int kClMaxCTAs = 8;                          // portable cluster size
constexpr int kClRuns = kAccRuns;

__host__ __device__ inline size_t cluster_smem_bytes()
{
    return (size_t)kClWarps * kAccTab * 16 + (size_t)kClSlab * 4 + (size_t)kClSlab / 8 + (size_t)kClSlab;
}

// A per-site array spread over the cluster: site j lives in rank j >> 15.
template <class T>
struct Dist {
    T* base;  // this rank's slab
    unsigned me;
    __device__ __forceinline__ T* ptr(int64_t j) const
    {
        const unsigned r = (unsigned)(j >> kClSlabLog);
        T* b = r == me ? base : cg::this_cluster().map_shared_rank(base, r);
        return b + (j & (kClSlab - 1));
    }
    __device__ __forceinline__ T& operator[](int64_t j) const { return *ptr(j); }
};

__device__ __forceinline__ int dfind(const Dist<int>& p, int x)
{
    while (true) {
        const int px = *(volatile int*)p.ptr(x);
        if (px == x) return x;
        const int gp = *(volatile int*)p.ptr(px);
        if (gp != px) *(volatile int*)p.ptr(x) = gp;
        x = gp;
    }
}
__device__ __forceinline__ void dunite(const Dist<int>& p, int a, int b)
{
    while (true) {
        a = dfind(p, a);
        b = dfind(p, b);
        if (a == b) return;
        if (uf_prio((uint32_t)a) > uf_prio((uint32_t)b)) {  // the root of lower priority hangs below
            const int t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(p.ptr(a), a, b) == a) return;
    }
}
// candidate bit of site j (word (j mod kClSlab) / 32 of rank j / kClSlab)
__device__ __forceinline__ bool dcand(const Dist<uint32_t>& c, int64_t j)
{
    const unsigned r = (unsigned)(j >> kClSlabLog);
    const uint32_t* b = r == c.me ? c.base : cg::this_cluster().map_shared_rank(c.base, r);
    const uint32_t w = *(volatile const uint32_t*)(b + ((j & (kClSlab - 1)) >> 5));
    return (w >> (j & 31)) & 1u;
}

// One cluster per member of `order`: EMCS e0 .. e0 + count - 1 of the run,
// measurement slots from slot0.  The cluster has ceil(n / kClSlab) CTAs.
__global__ void __launch_bounds__(kClThreads, 1)
    batch_resident_cluster(const BatchRep* __restrict__ reps, const int32_t* __restrict__ order, int nrep,
                           uint32_t e0, int slot0, int count, int ncluster, int nmetro, long long* __restrict__ acc,
                           int32_t* __restrict__ csize)
{
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_rsite, s_val, s_newq, s_root, s_size;  // meaningful on rank 0
    __shared__ long long red[3][kClWarps];
    __shared__ int hist[64];
    const unsigned me = cl.block_rank(), C = cl.num_blocks();
    const int r = order[blockIdx.x / C];
    const BatchRep& B = reps[r];
    StencilDev lst = B.st;
    lst.split = 0;
    const int64_t n = lst.n, lo = (int64_t)me * kClSlab, hi = lo + kClSlab < n ? lo + kClSlab : n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint4* tab = reinterpret_cast<uint4*>(smem) + warp * kAccTab;
    unsigned char* p = smem + (size_t)kClWarps * kAccTab * 16;
    int* par = reinterpret_cast<int*>(p);
    p += (size_t)kClSlab * 4;
    uint32_t* cand = reinterpret_cast<uint32_t*>(p);
    p += (size_t)kClSlab / 8;
    int8_t* st = reinterpret_cast<int8_t*>(p);
    const Dist<int8_t> ds{st, me};
    const Dist<int> dp{par, me};
    const Dist<uint32_t> dc{cand, me};
    const int8_t* gstate = (const int8_t*)B.s;
    for (int64_t i = lo + tid; i < hi; i += kClThreads) st[i - lo] = gstate[B.st.addr(i)];
    cl.sync();
    const uint32_t tgs = tag(kWolffSeed, B.replica), tgb = tag(kWolffBond, B.replica);
    const uint32_t sweep0 = B.sweep0 + e0 * (uint32_t)nmetro, cluster0 = B.cluster0 + e0 * (uint32_t)ncluster;
    const bool potts = B.md.kind == MQV_MODEL_POTTS;
    for (int e = 0; e < count; ++e) {
        for (int c = 0; c < ncluster; ++c) {
            const uint32_t serial = cluster0 + (uint32_t)(e * ncluster + c);
            if (me == 0 && tid == 0) {
                int val, newq;
                s_rsite = (int)wolff_int8_seed(B.w, lst, ds, B.key, serial, tgs, val, newq);
                s_val = val;
                s_newq = newq;
                s_size = 0;
            }
            cl.sync();
            const int val = *cl.map_shared_rank(&s_val, 0);
            const int rsite = *cl.map_shared_rank(&s_rsite, 0);
            const int8_t nv = (int8_t)*cl.map_shared_rank(&s_newq, 0);
            for (int64_t wd = tid; wd < kClSlab / 32; wd += kClThreads) {
                uint32_t bits = 0;
                for (int b = 0; b < 32; ++b) {
                    const int64_t i = lo + wd * 32 + b;
                    if (i < hi && st[i - lo] == val) {
                        bits |= 1u << b;
                        par[i - lo] = (int)i;
                    }
                }
                cand[wd] = bits;
            }
            cl.sync();
            for (int64_t i = lo + tid; i < hi; i += kClThreads) {
                if (!((cand[(i - lo) >> 5] >> (i & 31)) & 1u)) continue;
                for (int d = 0; d < lst.dim; ++d) {
                    const int64_t j = lst.nbr(i, 2 * d);
                    if (dcand(dc, j) && wolff_int8_active(B.w, (uint32_t)i, (uint32_t)j, serial, tgb, B.key))
                        dunite(dp, (int)i, (int)j);
                }
            }
            cl.sync();
            // every candidate's path halved once, all side by side (the
            // one-CTA kernel's compression pass): the walks after it are short
            for (int64_t i = lo + tid; i < hi; i += kClThreads)
                if ((cand[(i - lo) >> 5] >> (i & 31)) & 1u) dfind(dp, (int)i);
            cl.sync();
            if (me == 0 && tid == 0) s_root = dfind(dp, rsite);
            cl.sync();
            const int root = *cl.map_shared_rank(&s_root, 0);
            int cnt = 0;
            for (int64_t i = lo + tid; i < hi; i += kClThreads) {
                if (!((cand[(i - lo) >> 5] >> (i & 31)) & 1u)) continue;
                int x = (int)i, px;
                while ((px = *(volatile int*)dp.ptr(x)) != x) x = px;  // read-only walks
                if (x == root) {
                    st[i - lo] = nv;
                    ++cnt;
                }
            }
            cnt = __reduce_add_sync(0xffffffffu, cnt);
            if (lane == 0 && cnt) atomicAdd(cl.map_shared_rank(&s_size, 0), cnt);
            cl.sync();
            if (me == 0 && tid == 0) csize[((size_t)(slot0 + e) * ncluster + c) * nrep + r] = s_size;
        }
        for (int j = 0; j < nmetro; ++j) {
            const uint32_t sweep = sweep0 + (uint32_t)(e * nmetro + j);
            const int64_t t_lo = lo / 2, t_hi = hi / 2, bs = 32 * (int64_t)kClRuns;
            for (int colour = 0; colour < 2; ++colour) {
                for (int64_t t0 = t_lo + (int64_t)warp * bs; t0 < t_hi; t0 += (int64_t)kClWarps * bs) {
                    const uint32_t run0 = (uint32_t)(t0 / 32);
                    accept_tab_fill(tab, run0, B.key, sweep, B.replica);
                    for (int k = 0; k < kClRuns; ++k) {
                        const int64_t t = t0 + k * 32 + lane;
                        const bool live = t < t_hi;
                        int8_site(B.md, lst, ds, live ? parity_site(lst, t, colour) : 0, B.key, sweep, B.replica,
                                  B.cuts, B.D, live, colour, tab, run0);
                    }
                }
                cl.sync();
            }
        }
        // measurement of this rank's sites (forward neighbours may be remote)
        if (!acc) {
            cl.sync();
            continue;
        }
        if (potts)
            for (int k = tid; k < 64; k += kClThreads) hist[k] = 0;
        __syncthreads();
        long long es = 0, ms = 0, sq = 0;
        for (int64_t i0 = lo + (tid & ~31); i0 < hi; i0 += kClThreads) {
            const int64_t i = i0 + lane;
            const bool live = i < hi;
            int si = 0;
            if (live) {
                si = st[i - lo];
                es += int8_bond_sum_stencil(lst, ds, i, si, potts);
                ms += si;
                sq += si * si;
            }
            if (potts) {
                const unsigned peers = __match_any_sync(0xffffffffu, live ? (si & 63) : 64);
                if (live && lane == (__ffs(peers) - 1)) atomicAdd(&hist[si & 63], __popc(peers));
            }
        }
        es = warp_sum_ll(es);
        ms = warp_sum_ll(ms);
        sq = warp_sum_ll(sq);
        if (lane == 0) {
            red[0][warp] = es;
            red[1][warp] = ms;
            red[2][warp] = sq;
        }
        __syncthreads();
        long long* a = acc + ((size_t)(slot0 + e) * nrep + r) * kAccStride;
        if (tid == 0) {
            long long x = 0, y = 0, z = 0;
            for (int k = 0; k < kClWarps; ++k) {
                x += red[0][k];
                y += red[1][k];
                z += red[2][k];
            }
            atomicAdd(reinterpret_cast<unsigned long long*>(a + kAccEne), (unsigned long long)x);
            atomicAdd(reinterpret_cast<unsigned long long*>(a + kAccMag), (unsigned long long)y);
            atomicAdd(reinterpret_cast<unsigned long long*>(a + kAccSq), (unsigned long long)z);
        }
        if (potts)
            for (int k = tid; k < B.md.q; k += kClThreads)
                if (hist[k]) atomicAdd(reinterpret_cast<unsigned long long*>(a + kAccPotts + k), (unsigned long long)hist[k]);
        cl.sync();  // every rank's reads of this EMCS are done before the next one writes
    }
    int8_t* gout = (int8_t*)B.s;
    for (int64_t i = lo + tid; i < hi; i += kClThreads) gout[B.st.addr(i)] = st[i - lo];
    cl.sync();  // no rank leaves while another may still read its shared memory
}

// CTAs of the cluster that holds an n-site lattice (0: does not fit).
int cluster_ctas(int64_t n)
{
    const int64_t c = (n + kClSlab - 1) / kClSlab;
    return c >= 1 && c <= kClMaxCTAs ? (int)c : 0;
}

// Can the device co-schedule a cluster of `ctas` CTAs of this kernel?
bool cluster_launchable(int ctas)
{
    if (cudaFuncSetAttribute(batch_resident_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)cluster_smem_bytes()) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = cluster_smem_bytes();
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, batch_resident_cluster, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return nclusters > 0;
}

// The batch's cluster-resident members with `ctas` CTAs each (order: member
// ids), EMCS e0 .. e0 + count - 1, measurement slots from slot0.
cudaError_t batch_launch_cluster(const BatchLaunch& b, cudaStream_t st, const int32_t* order, int nmem, int ctas,
                                 uint32_t e0, int slot0, int count, int ncluster, int nmetro)
{
    if (nmem <= 0 || count <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(batch_resident_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)cluster_smem_bytes());
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(ctas * nmem));
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = cluster_smem_bytes();
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, batch_resident_cluster, b.reps, order, b.nrep, e0, slot0, count, ncluster, nmetro,
                              b.acc, b.csize);
}

}  // namespace mqv
