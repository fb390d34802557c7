// The int8 Wolff cluster update as a device function, shared by the per-handle
// kernel (wolff.cu) and the batched kernel (batch.cu).  Reference semantics:
// src/libmarqov/wolff.h:72-126, src/hamiltonian/Ising.h:126-168,
// src/hamiltonian/Potts.h:220-320 (draws keyed by the undirected bond).
#pragma once
#include "engine.h"

namespace mqv {


// Seed site, its state and the cluster's new state from the WOLFF_SEED
// substream (Ising: the flipped spin; Potts: Embedder<Potts<Q>>::draw, a new
// state different from the old one).
template <class Lat, class SP>
__device__ __forceinline__ int64_t wolff_int8_seed(const WolffDev& w, const Lat& lat, SP s, Key key, uint32_t serial,
                                                   uint32_t tg_seed, int& val, int& newq)
{
    SubStream rng(key, 0u, serial, tg_seed);
    const int64_t rsite = (int64_t)(rng.next() % (uint64_t)lat.n);
    val = s[lat.addr(rsite)];
    newq = -val;
    if (w.mode == 2) {
        int tries = 0;
        do {
            newq = (int)(rng.next() % (uint64_t)w.q);
        } while (newq == val && ++tries < 256);
        if (newq == val) newq = (val + 1) % w.q;
    }
    return rsite;
}

// Union-find linking order of the labelling kernels: of two roots, the one
// of lower priority hangs below the other.  Priorities are a fixed
// pseudo-random permutation of the site index (multiplication by an odd
// constant is a bijection modulo 2^32 and modulo 2^16), so the trees stay
// O(log n) deep in expectation whatever order the bonds are united in --
// hooking by index chains up sites that are united side by side.
__device__ __forceinline__ uint32_t uf_prio(uint32_t i) { return i * 0x9E3779B1u; }
__device__ __forceinline__ uint32_t uf_prio16(uint32_t i) { return (i * 0x9E37u) & 0xFFFFu; }

// Bond activation of the int8 rules on the bond's keyed word
__device__ __forceinline__ bool wolff_int8_active(const WolffDev& w, uint32_t a, uint32_t b, uint32_t serial,
                                                  uint32_t tg_bond, Key key)
{
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    const unsigned long long u53 = lo64(philox(lo, serial, hi, tg_bond, key)) >> 11;
    return w.mode == 0 ? u53 < w.thr : u53 >= w.thr;
}

// One cluster grown and flipped by the calling CTA (any block size that is a
// multiple of 32); the visited bits of its members are cleared before return.
// A level's work items are (frontier site, neighbour lane) pairs, so the
// neighbours of a site are examined side by side rather than one after the
// other (the cluster is the same in any visiting order).
template <class Lat>
__device__ __forceinline__ void wolff_int8_cluster(const WolffDev& w, const Lat& lat, int8_t* __restrict__ s,
                                                   uint32_t* __restrict__ visited, int32_t* __restrict__ queue,
                                                   int32_t* __restrict__ out_size, Key key, uint32_t serial,
                                                   uint32_t tg_seed, uint32_t tg_bond, int max_degree,
                                                   int32_t* __restrict__ fbuf)
{
    __shared__ int s_head, s_tail, s_next;
    __shared__ int s_val, s_newq;
    constexpr int CAP = kWolffCap8;
    if (threadIdx.x == 0) {
        int val, newq;
        const int64_t rsite = wolff_int8_seed(w, lat, s, key, serial, tg_seed, val, newq);
        s_val = val;
        s_newq = newq;
        queue[0] = (int32_t)rsite;
        fbuf[0] = (int32_t)rsite;
        atomicOr(&visited[rsite >> 5], 1u << (rsite & 31));
        s_head = 0;
        s_tail = 1;
        s_next = 1;
    }
    __syncthreads();
    const int val = s_val;
    const int lanes = wolff_lanes(lat, max_degree);
    const unsigned lane = threadIdx.x & 31;
    for (int lvl = 0;; ++lvl) {
        const int head = s_head, tail = s_tail;
        if (head >= tail) break;
        // the level's sites: fbuf[(lvl & 1) * CAP ...] when they fit, else the queue
        const bool fits = tail - head <= CAP;
        const int32_t* fcur = fbuf + (lvl & 1) * CAP;
        int32_t* fnext = fbuf + ((lvl + 1) & 1) * CAP;
        const int64_t items = (int64_t)(tail - head) * lanes;
        for (int64_t base = 0; base < items; base += blockDim.x) {
            const int64_t k = base + threadIdx.x;
            int64_t cur = 0;
            int t0 = 0, deg = 0;
            if (k < items) {
                const int64_t q = k / lanes;
                t0 = (int)(k - q * lanes);
                cur = fits ? fcur[q] : queue[head + q];
                deg = lat.degree(cur);
            }
            const int rounds = __reduce_max_sync(0xffffffffu, deg > t0 ? (deg - t0 + lanes - 1) / lanes : 0);
            for (int rr = 0; rr < rounds; ++rr) {
                const int t = t0 + rr * lanes;
                bool add = false;
                int64_t j = 0;
                if (t < deg) {
                    j = lat.nbr(cur, t);
                    // both loads issued before either is tested
                    const int sj = s[lat.addr(j)];
                    const uint32_t vw = visited[j >> 5];
                    if (sj == val && !(vw & (1u << (j & 31)))) {
                        if (wolff_int8_active(w, (uint32_t)cur, (uint32_t)j, serial, tg_bond, key)) {
                            const uint32_t old = atomicOr(&visited[j >> 5], 1u << (j & 31));
                            add = !(old & (1u << (j & 31)));
                        }
                    }
                }
                const unsigned mask = __ballot_sync(0xffffffffu, add);
                if (mask) {
                    int pos = 0;
                    if (lane == 0) pos = atomicAdd(&s_next, __popc(mask));
                    pos = __shfl_sync(0xffffffffu, pos, 0);
                    if (add) {
                        const int at = pos + __popc(mask & ((1u << lane) - 1));
                        queue[at] = (int32_t)j;
                        if (at - tail < CAP) fnext[at - tail] = (int32_t)j;
                    }
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_head = tail;
            s_tail = s_next;
        }
        __syncthreads();
    }
    const int size = s_tail;
    const int8_t nv = (int8_t)s_newq;
    for (int k = threadIdx.x; k < size; k += blockDim.x) {
        const int32_t i = queue[k];
        s[lat.addr(i)] = nv;
        atomicAnd(&visited[i >> 5], ~(1u << (i & 31)));
    }
    if (threadIdx.x == 0) *out_size = size;
}

}  // namespace mqv
