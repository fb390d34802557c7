// Wolff clusters by connected-component labelling, for the batched path.
//
// With bond draws keyed by the undirected bond (lower id, cluster serial,
// upper id), the Wolff cluster is the seed's connected component of the
// activated bonds, whatever the visiting order.  A breadth-first growth from
// one CTA needs one step per level of the cluster; this variant labels every
// component of the activated-bond graph of every member in a fixed number of
// whole-lattice passes -- lock-free union-find: each undirected bond once,
// roots hooked by compare-and-swap in a fixed pseudo-random order (uf_prio),
// paths halved on the way -- and flips the
// seed's component:
//   ccl_seed      one thread per member: seed site, old/new state or the
//                 reflection vector (the same substream draws as the BFS);
//   ccl_local     per CTA of 256 consecutive sites: candidates (int8: state
//                 equal to the seed's old state; float: every site, whose
//                 projections on the reflection vector go to shared memory)
//                 get labels, and activated bonds with both ends in the CTA's
//                 sites are united in shared memory first; each candidate's
//                 label becomes its local root, non-candidates get -1;
//   ccl_hook      the other activated bonds between candidates are united;
//   ccl_halve     every candidate's path to its root halved;
//   ccl_flip      members of the seed's component (read-only walks to the
//                 roots) are flipped / reflected and counted into the cluster
//                 size.
// The label array is the member's BFS queue (n int32); the visited bitmap is
// not touched.
#pragma once
#include "batch.h"
#include "f32_site.cuh"
#include "wolff_int8.cuh"

namespace mqv {

struct CclSeed {
    int64_t rsite;
    int val, newq;  // int8
    float r[3];     // float
};

// member and local site of flattened site g
__device__ __forceinline__ int ccl_member(int64_t g, const int64_t* __restrict__ prefix,
                                          const int32_t* __restrict__ block_rep, int64_t& i)
{
    int r = block_rep[blockIdx.x];
    while (g >= prefix[r + 1]) ++r;
    i = g - prefix[r];
    return r;
}

// Position <-> site of a member in its labelling order (BatchRep::tile): the
// labelling kernels give CTA block b the positions [256 b, 256 b + 256) of
// the concatenated members, so that with tiles a block holds a 16 x 16 (2D)
// or 8 x 8 x 4 (3D) tile and most bonds join two sites of one block.
__device__ __forceinline__ int64_t ccl_site(const BatchRep& R, int64_t pos)
{
    if (R.tile == 0) return pos;
    const uint32_t L = (uint32_t)R.st.len, t = (uint32_t)(pos >> 8), o = (uint32_t)pos & 255u;
    if (R.tile == 2) {
        const uint32_t nx = L >> 4, ty = t / nx, tx = t - ty * nx;
        return (int64_t)((ty << 4) + (o >> 4)) * L + (tx << 4) + (o & 15u);
    }
    const uint32_t nx = L >> 3, ny = L >> 3, tyz = t / nx, tx = t - tyz * nx, tz = tyz / ny, ty = tyz - tz * ny;
    const uint32_t x = (tx << 3) + (o & 7u), y = (ty << 3) + ((o >> 3) & 7u), z = (tz << 2) + (o >> 6);
    return ((int64_t)z * L + y) * L + x;
}
__device__ __forceinline__ int64_t ccl_pos(const BatchRep& R, int64_t site)
{
    if (R.tile == 0) return site;
    const uint32_t L = (uint32_t)R.st.len, u = (uint32_t)site;
    if (R.tile == 2) {
        const uint32_t y = u / L, x = u - y * L;
        return (int64_t)(((y >> 4) * (L >> 4) + (x >> 4)) << 8) + ((y & 15u) << 4) + (x & 15u);
    }
    const uint32_t yz = u / L, x = u - yz * L, z = yz / L, y = yz - z * L;
    const uint32_t t = ((z >> 2) * (L >> 3) + (y >> 3)) * (L >> 3) + (x >> 3);
    return (int64_t)(t << 8) + ((z & 3u) << 6) + ((y & 7u) << 3) + (x & 7u);
}

__device__ __forceinline__ int ccl_find(int* __restrict__ p, int x)
{
    while (true) {
        const int px = __ldcg(p + x);
        if (px == x) return x;
        const int gp = __ldcg(p + px);
        if (gp != px) p[x] = gp;  // path halving (races only shorten paths)
        x = gp;
    }
}

__device__ __forceinline__ void ccl_unite(int* __restrict__ p, int a, int b)
{
    while (true) {
        a = ccl_find(p, a);
        b = ccl_find(p, b);
        if (a == b) return;
        if (uf_prio((uint32_t)a) > uf_prio((uint32_t)b)) {  // the root of lower priority hangs below
            const int t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(p + a, a, b) == a) return;
    }
}

__device__ __forceinline__ int64_t rep_n(const BatchRep& R)
{
    return R.lat_kind == MQV_LATTICE_HYPERCUBIC ? R.st.n : R.csr.n;
}

template <bool F32>
__global__ void ccl_seed(const BatchRep* __restrict__ reps, const BatchCtr* __restrict__ ctr, int ncluster, int c,
                         CclSeed* __restrict__ seeds, int32_t* __restrict__ csize, int nrep)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrep) return;
    const BatchRep& R = reps[r];
    if (R.resident) return;  // clusters grown by batch_resident
    const uint32_t e = ctr->e, slot = e - ctr->ebase;
    const uint32_t serial = R.cluster0 + e * (uint32_t)ncluster + (uint32_t)c;
    const uint32_t tgs = tag(kWolffSeed, R.replica);
    CclSeed sd{};
    if (F32) {
        sd.rsite = embed_seed(R.md, rep_n(R), R.key, serial, tgs, sd.r);
    } else if (R.lat_kind == MQV_LATTICE_HYPERCUBIC) {
        sd.rsite = wolff_int8_seed(R.w, R.st, (const int8_t*)R.s, R.key, serial, tgs, sd.val, sd.newq);
    } else {
        sd.rsite = wolff_int8_seed(R.w, R.csr, (const int8_t*)R.s, R.key, serial, tgs, sd.val, sd.newq);
    }
    seeds[r] = sd;
    csize[((size_t)slot * ncluster + c) * nrep + r] = 0;
}

// activation of the bond (i, j) between two candidate sites of member R, on
// the bond's keyed draw (the breadth-first growth's rule)
template <bool F32>
__device__ __forceinline__ bool ccl_active(const BatchRep& R, const CclSeed& sd, uint32_t serial, int64_t i, int64_t j)
{
    const uint32_t tgb = tag(kWolffBond, R.replica);
    if (F32) {
        const int64_t lo = i < j ? i : j, hi = i < j ? j : i;
        const float* s = (const float*)R.s;
        const int64_t n = rep_sites(R);
        const double cpl = embed_cpl(R.md.J, embed_proj(R.md.symd, s, n, lo, sd.r[0], sd.r[1], sd.r[2]),
                                     embed_proj(R.md.symd, s, n, hi, sd.r[0], sd.r[1], sd.r[2]));
        return cpl > 0 &&
               !update_accepted(2, cpl, R.md.beta, lo64(philox((uint32_t)lo, serial, (uint32_t)hi, tgb, R.key)));
    }
    return wolff_int8_active(R.w, (uint32_t)i, (uint32_t)j, serial, tgb, R.key);
}

// the forward bonds (i, j) of site i, each undirected bond once: +x, +y, ...
// on stencils, j > i on CSR graphs
template <class F>
__device__ __forceinline__ void ccl_forward_bonds(const BatchRep& R, int64_t i, F&& f)
{
    if (R.lat_kind == MQV_LATTICE_HYPERCUBIC) {
        for (int d = 0; d < R.st.dim; ++d) f(R.st.nbr(i, 2 * d));
    } else {
        for (int t = R.csr.rp[i]; t < R.csr.rp[i + 1]; ++t) {
            const int64_t j = R.csr.ci[t];
            if (j > i) f(j);
        }
    }
}

// union-find on the CTA's shared labels (the same scheme as ccl_find /
// ccl_unite on shared memory)
__device__ __forceinline__ int ccl_lfind(volatile int* p, int x)
{
    while (true) {
        const int px = p[x];
        if (px == x) return x;
        const int gp = p[px];
        if (gp != px) p[x] = gp;
        x = gp;
    }
}
__device__ __forceinline__ void ccl_lunite(volatile int* p, int a, int b)
{
    while (true) {
        a = ccl_lfind(p, a);
        b = ccl_lfind(p, b);
        if (a == b) return;
        if (uf_prio((uint32_t)a) > uf_prio((uint32_t)b)) {  // the root of lower priority hangs below
            const int t = a;
            a = b;
            b = t;
        }
        if (atomicCAS((int*)p + a, a, b) == a) return;
    }
}

// flattened site g and g2 in the same CTA block of kBatchMetroThreads sites
__device__ __forceinline__ bool ccl_same_block(int64_t g, int64_t g2)
{
    return g / kBatchMetroThreads == g2 / kBatchMetroThreads;
}

// Lattice coordinates of position `pos` of a tiled member (BatchRep::tile 2:
// 16 x 16 tiles, 3: 8 x 8 x 4 tiles, tile t = pos >> 8, offset o = pos & 255),
// by shifts where the side is a power of two.
struct TileSite {
    uint32_t x, y, z;
};
__device__ __forceinline__ TileSite ccl_tile_coords(const BatchRep& R, uint32_t pos)
{
    const uint32_t L = (uint32_t)R.st.len, t = pos >> 8, o = pos & 255u;
    const int lg = R.st.lg;
    TileSite c;
    if (R.tile == 2) {
        uint32_t ty, tx;
        if (lg >= 0) {
            ty = t >> (lg - 4);
            tx = t & ((L >> 4) - 1u);
        } else {
            ty = t / (L >> 4);
            tx = t - ty * (L >> 4);
        }
        c.x = (tx << 4) + (o & 15u);
        c.y = (ty << 4) + (o >> 4);
        c.z = 0;
    } else {
        uint32_t tz, ty, tx;
        if (lg >= 0) {
            tx = t & ((L >> 3) - 1u);
            ty = (t >> (lg - 3)) & ((L >> 3) - 1u);
            tz = t >> (2 * (lg - 3));
        } else {
            const uint32_t tyz = t / (L >> 3);
            tx = t - tyz * (L >> 3);
            tz = tyz / (L >> 3);
            ty = tyz - tz * (L >> 3);
        }
        c.x = (tx << 3) + (o & 7u);
        c.y = (ty << 3) + ((o >> 3) & 7u);
        c.z = (tz << 2) + (o >> 6);
    }
    return c;
}
__device__ __forceinline__ int64_t ccl_tile_index(const BatchRep& R, const TileSite& c)
{
    const int64_t L = R.st.len;
    return (R.tile == 2 ? 0 : (int64_t)c.z * L * L) + (int64_t)c.y * L + c.x;
}
// The forward neighbour in dimension d (+x, +y, +z, periodic) of a tiled
// member's site: its coordinates, whether it lies in the same tile (the same
// CTA block), and then its offset in the tile.
__device__ __forceinline__ TileSite ccl_tile_fwd(const BatchRep& R, TileSite c, int d, bool& same, int& k)
{
    const uint32_t L = (uint32_t)R.st.len;
    if (R.tile == 2) {
        if (d == 0) {
            const uint32_t xn = c.x + 1u == L ? 0u : c.x + 1u;
            same = (xn >> 4) == (c.x >> 4);
            c.x = xn;
        } else {
            const uint32_t yn = c.y + 1u == L ? 0u : c.y + 1u;
            same = (yn >> 4) == (c.y >> 4);
            c.y = yn;
        }
        k = (int)(((c.y & 15u) << 4) | (c.x & 15u));
    } else {
        if (d == 0) {
            const uint32_t xn = c.x + 1u == L ? 0u : c.x + 1u;
            same = (xn >> 3) == (c.x >> 3);
            c.x = xn;
        } else if (d == 1) {
            const uint32_t yn = c.y + 1u == L ? 0u : c.y + 1u;
            same = (yn >> 3) == (c.y >> 3);
            c.y = yn;
        } else {
            const uint32_t zn = c.z + 1u == L ? 0u : c.z + 1u;
            same = (zn >> 2) == (c.z >> 2);
            c.z = zn;
        }
        k = (int)(((c.z & 3u) << 6) | ((c.y & 7u) << 3) | (c.x & 7u));
    }
    return c;
}

// activation of the bond (lo, hi) of a float member given both ends'
// projections on the reflection vector (ccl_active's rule and order)
__device__ __forceinline__ bool ccl_active_f32(const BatchRep& R, uint32_t serial, int64_t lo, int64_t hi, double alo,
                                               double ahi)
{
    const double cpl = embed_cpl(R.md.J, alo, ahi);
    return cpl > 0 && !update_accepted(2, cpl, R.md.beta,
                                       lo64(philox((uint32_t)lo, serial, (uint32_t)hi, tag(kWolffBond, R.replica), R.key)));
}

template <bool F32>
__global__ void __launch_bounds__(kBatchMetroThreads)
    ccl_local(const BatchRep* __restrict__ reps, const int64_t* __restrict__ prefix,
              const int32_t* __restrict__ block_rep, int64_t total, const CclSeed* __restrict__ seeds,
              const BatchCtr* __restrict__ ctr, int ncluster, int c)
{
    __shared__ int slab[kBatchMetroThreads];
    __shared__ double sproj[F32 ? kBatchMetroThreads : 1];
    const int64_t base = (int64_t)blockIdx.x * kBatchMetroThreads;
    const int64_t g = base + threadIdx.x;
    int r = 0;
    int64_t i = 0;  // this thread's site (position g in the labelling order)
    bool cand = false;
    TileSite tc{0, 0, 0};
    double ai = 0.0;  // float: the site's projection on the reflection vector
    bool tiled = false;  // the CTA block is one tile of the member
    if (g < total) {
        r = ccl_member(g, prefix, block_rep, i);
        const BatchRep& R = reps[r];
        tiled = R.tile && (prefix[r] & 255) == 0;
        if (tiled) {
            tc = ccl_tile_coords(R, (uint32_t)i);
            i = ccl_tile_index(R, tc);
        } else {
            i = ccl_site(R, i);
        }
        cand = true;
        if (F32) {
            const CclSeed& sd = seeds[r];
            ai = embed_proj(R.md.symd, (const float*)R.s, rep_sites(R), i, sd.r[0], sd.r[1], sd.r[2]);
        } else {
            const int64_t a = R.lat_kind == MQV_LATTICE_HYPERCUBIC ? R.st.addr(i) : i;
            cand = ((const int8_t*)R.s)[a] == seeds[r].val;
        }
    }
    slab[threadIdx.x] = cand ? (int)threadIdx.x : -1;
    if (F32) sproj[threadIdx.x] = ai;
    __syncthreads();
    if (cand) {
        const BatchRep& R = reps[r];
        const uint32_t serial = R.cluster0 + ctr->e * (uint32_t)ncluster + (uint32_t)c;
        const CclSeed sd = seeds[r];
        volatile int* vl = slab;
        if (tiled) {
            // neighbours in the same tile, their offsets from the coordinates
            for (int d = 0; d < R.st.dim; ++d) {
                bool same;
                int k;
                const TileSite nc = ccl_tile_fwd(R, tc, d, same, k);
                if (!same || vl[k] < 0) continue;
                const int64_t j = ccl_tile_index(R, nc);
                bool act;
                if (F32) {
                    const double aj = sproj[k];
                    act = i < j ? ccl_active_f32(R, serial, i, j, ai, aj) : ccl_active_f32(R, serial, j, i, aj, ai);
                } else {
                    act = ccl_active<false>(R, sd, serial, i, j);
                }
                if (act) ccl_lunite(vl, (int)threadIdx.x, k);
            }
        } else {
            const int64_t off = prefix[r];
            ccl_forward_bonds(R, i, [&](int64_t j) {
                const int64_t gj = off + ccl_pos(R, j);
                if (!ccl_same_block(g, gj)) return;
                const int k = (int)(gj - base);
                if (vl[k] >= 0 && ccl_active<F32>(R, sd, serial, i, j)) ccl_lunite(vl, (int)threadIdx.x, k);
            });
        }
    }
    __syncthreads();
    if (cand) ccl_lfind(slab, (int)threadIdx.x);  // paths halved side by side first
    __syncthreads();
    if (g < total) {
        int lab = -1;
        if (cand) {
            // read-only walk to the local root (same member: bonds join only its sites)
            int x = (int)threadIdx.x, px;
            while ((px = ((volatile int*)slab)[x]) != x) x = px;
            const BatchRep& R = reps[r];
            const int64_t rpos = base + x - prefix[r];
            lab = (int)(tiled ? ccl_tile_index(R, ccl_tile_coords(R, (uint32_t)rpos)) : ccl_site(R, rpos));
        }
        reps[r].queue[i] = lab;
    }
}

template <bool F32>
__global__ void ccl_hook(const BatchRep* __restrict__ reps, const int64_t* __restrict__ prefix,
                         const int32_t* __restrict__ block_rep, int64_t total, const CclSeed* __restrict__ seeds,
                         const BatchCtr* __restrict__ ctr, int ncluster, int c)
{
    const int64_t base = (int64_t)blockIdx.x * blockDim.x, g = base + threadIdx.x;
    if (base >= total) return;
    {
        // A CTA block that is one tile of a member: its threads take the
        // bonds that leave the tile, one each (2D 16 x 16 tiles: the +x and +y
        // faces, 32 bonds; 3D 8 x 8 x 4 tiles: the +x, +y and +z faces, 128
        // bonds) -- the bonds inside the tile were united by ccl_local.
        int64_t p0;
        const int r = ccl_member(base, prefix, block_rep, p0);
        const BatchRep& R = reps[r];
        if (R.tile && (prefix[r] & 255) == 0) {  // the same member and test for the whole CTA
            const uint32_t t = threadIdx.x;
            if (t >= (R.tile == 2 ? 32u : 128u)) return;
            uint32_t o;
            int d;
            if (R.tile == 2) {
                d = t < 16u ? 0 : 1;
                o = d == 0 ? (t << 4) | 15u : (15u << 4) | (t - 16u);
            } else if (t < 32u) {
                d = 0;
                o = ((t >> 3) << 6) | ((t & 7u) << 3) | 7u;  // x = 7: (y, z) = (t & 7, t >> 3)
            } else if (t < 64u) {
                d = 1;
                o = (((t >> 3) & 3u) << 6) | (7u << 3) | (t & 7u);  // y = 7: (x, z) = (t & 7, (t >> 3) & 3)
            } else {
                d = 2;
                o = (3u << 6) | (((t >> 3) & 7u) << 3) | (t & 7u);  // z = 3: (x, y) = (t & 7, (t >> 3) & 7)
            }
            const TileSite tc = ccl_tile_coords(R, (uint32_t)p0 + o);
            bool same;
            int k;
            const TileSite nc = ccl_tile_fwd(R, tc, d, same, k);
            if (same) return;  // the periodic neighbour is in the same tile (side = tile width)
            int* lab = R.queue;
            const int64_t i = ccl_tile_index(R, tc), j = ccl_tile_index(R, nc);
            if (__ldcg(lab + i) < 0 || __ldcg(lab + j) < 0) return;
            const uint32_t serial = R.cluster0 + ctr->e * (uint32_t)ncluster + (uint32_t)c;
            bool act;
            if (F32) {
                const CclSeed& sd = seeds[r];
                const float* s = (const float*)R.s;
                const int64_t n = rep_sites(R);
                const double ai = embed_proj(R.md.symd, s, n, i, sd.r[0], sd.r[1], sd.r[2]);
                const double aj = embed_proj(R.md.symd, s, n, j, sd.r[0], sd.r[1], sd.r[2]);
                act = i < j ? ccl_active_f32(R, serial, i, j, ai, aj) : ccl_active_f32(R, serial, j, i, aj, ai);
            } else {
                act = ccl_active<false>(R, seeds[r], serial, i, j);
            }
            if (act) ccl_unite(lab, (int)i, (int)j);
            return;
        }
    }
    if (g >= total) return;
    int64_t i;
    const int r = ccl_member(g, prefix, block_rep, i);
    const BatchRep& R = reps[r];
    int* lab = R.queue;
    if (R.tile && (prefix[r] & 255) == 0) return;  // taken by its tile's face threads
    i = ccl_site(R, i);
    if (__ldcg(lab + i) < 0) return;
    const uint32_t serial = R.cluster0 + ctr->e * (uint32_t)ncluster + (uint32_t)c;
    const CclSeed sd = seeds[r];
    const int64_t off = prefix[r];
    // bonds within the CTA block were united by ccl_local
    ccl_forward_bonds(R, i, [&](int64_t j) {
        if (ccl_same_block(g, off + ccl_pos(R, j)) || __ldcg(lab + j) < 0) return;
        if (ccl_active<F32>(R, sd, serial, i, j)) ccl_unite(lab, (int)i, (int)j);
    });
}

// Every candidate's path halved, all side by side (a write only ever points
// a site to an ancestor, so the forest stays valid while others walk it), so
// that ccl_flip's walks are short.
static __global__ void ccl_halve(const BatchRep* __restrict__ reps, const int64_t* __restrict__ prefix,
                                 const int32_t* __restrict__ block_rep, int64_t total)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int64_t i;
    const int r = ccl_member(g, prefix, block_rep, i);
    int* lab = reps[r].queue;
    if (__ldcg(lab + i) < 0) return;
    ccl_find(lab, (int)i);
}

template <bool F32>
__global__ void ccl_flip(const BatchRep* __restrict__ reps, const int64_t* __restrict__ prefix,
                         const int32_t* __restrict__ block_rep, int64_t total, const CclSeed* __restrict__ seeds,
                         const BatchCtr* __restrict__ ctr, int ncluster, int c, int32_t* __restrict__ csize, int nrep)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool in = false;
    int r = 0;
    if (g < total) {
        int64_t i;
        r = ccl_member(g, prefix, block_rep, i);
        const BatchRep& R = reps[r];
        const CclSeed& sd = seeds[r];
        // read-only walks to the roots (short after ccl_halve)
        const int* lab = R.queue;
        int root = __ldcg(lab + sd.rsite), x = __ldcg(lab + i);
        if (root >= 0 && x >= 0) {
            int p;
            while ((p = __ldcg(lab + root)) != root) root = p;
            while ((p = __ldcg(lab + x)) != x) x = p;
            in = x == root;
        }
        if (in) {
            if (F32) {
                embed_reflect(R.md.symd, (float*)R.s, rep_sites(R), i, sd.r[0], sd.r[1], sd.r[2]);
            } else {
                const int64_t a = R.lat_kind == MQV_LATTICE_HYPERCUBIC ? R.st.addr(i) : i;
                ((int8_t*)R.s)[a] = (int8_t)sd.newq;
            }
        }
    }
    // count per member: lanes of one member aggregate their adds
    const unsigned lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(0xffffffffu, r);
    const unsigned cnt = __popc(__ballot_sync(0xffffffffu, in) & peers);
    if (cnt && lane == (unsigned)(__ffs(peers) - 1)) {
        const uint32_t slot = ctr->e - ctr->ebase;
        atomicAdd(csize + ((size_t)slot * ncluster + c) * nrep + r, (int)cnt);
    }
}

}  // namespace mqv
