// Device building blocks of the int8 models shared by the per-handle kernels
// (metropolis_int8.cu) and the batched kernels (batch.cu): the per-site
// Metropolis update, the checkerboard site map, the observable accumulation
// and its finalisation.
#pragma once
#include "engine.h"

namespace mqv {

// ---------------------------------------------------------------------------
// generic per-site update (Metropolis<H,L>::move, src/libmarqov/metropolis.h:88-126)

// `cuts`: the u53 cut of every dE the model can produce, indexed as
// int8_cut_index (host table int8_cut_table); the decision equals
// update_accepted<1>(dE, beta, word) on the site's acceptance word.  `sub`:
// the site's sublattice (checkerboard colour) where the lattice has a
// termselector.  Lanes with live == false touch no memory.
template <class Lat, class SP>
__device__ __forceinline__ void int8_site(const ModelDev& m, const Lat& lat, SP s, int64_t i,
                                          Key key, uint32_t sweep, uint32_t replica,
                                          const unsigned long long* __restrict__ cuts, int D, bool live, int sub = 0,
                                          const uint4* tab = nullptr, uint32_t run0 = 0)
{
    int64_t ai = 0;
    int nw = 0;
    uint64_t cut = 0;
    if (live) {
        SubStream rng(key, (uint32_t)i, sweep, tag(kMetro, replica));
        ai = lat.addr(i);
        const int old = s[ai];
        const int deg = lat.degree(i);
        int k;
        if (m.kind == MQV_MODEL_POTTS) {
            // Initializer<Potts<Q>>::newsv (src/hamiltonian/Potts.h:170-177) and
            // PottsInteraction::diff (src/hamiltonian/Potts.h:86-107)
            nw = (int)mod_small(rng.next(), (uint32_t)m.q);
            int eo = 0, en = 0;
            for (int t = 0; t < deg; ++t) {
                const int v = s[lat.addr(lat.nbr(i, t))];
                eo += (v == old);
                en += (v == nw);
            }
            k = en - eo + D;
        } else if (m.kind == MQV_MODEL_BLUME_CAPEL) {
            // Spin1_Initializer::newsv (src/hamiltonian/util/initializers.h:99-118)
            int st = old;
            if (st == 0) st = rng.real() < 0.5 ? -1 : 1;
            else st = rng.real() < 0.5 ? -st : 0;
            nw = st;
            int sum = 0;
            for (int t = 0; t < deg; ++t) sum += s[lat.addr(lat.nbr(i, t))];
            k = (((nw - old) + 2) * (2 * D + 1) + (sum + D)) * 3 + (nw * nw - old * old + 1);
            if (m.termsel && sub) k += 15 * (2 * D + 1);  // the sublattice-B table
        } else {
            // spin flip (src/hamiltonian/util/initializers.h:52-58), neighbourhood
            // sum with optional bonds (src/libmarqov/metropolishelpers.h:456-537)
            nw = -old;
            int sum = 0;
            for (int t = 0; t < deg; ++t) sum += lat.bond(i, t) * s[lat.addr(lat.nbr(i, t))];
            k = old * sum + D;
        }
        cut = cuts[k];
    }
    // metro_update_accepted (src/libmarqov/metropolis.h:61-64,120-124) on the
    // site's acceptance word, its top byte from the warp's shared table when
    // `tab` is given (accept_tab_fill)
    bool acc;
    if (tab) {
        const uint32_t top = live ? accept_top8_tab(tab, run0, (uint32_t)i) : 0u;
        acc = live && accept_top_or_fine(cut, top, key, (uint32_t)i, sweep, replica);
    } else {
        acc = live && accept_below(cut, key, (uint32_t)i, sweep, replica);
    }
    if (acc) s[ai] = (int8_t)nw;
}

// Site of colour `colour` in pair t of a parity-coloured hypercubic lattice
// with even side: sites 2t and 2t+1 differ only in x, so they have opposite
// colours.
template <class ST>
__device__ __forceinline__ int64_t parity_site(const ST& st, int64_t t, int colour)
{
    const int64_t i0 = 2 * t;
    int par = 0;
    for (int j = 1; j < st.degree(0) / 2; ++j) par += st.coord(i0, j);
    return i0 + (((par & 1) != colour) ? 1 : 0);
}

__device__ __forceinline__ long long warp_sum_ll(long long v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// measurement: InteractionEnergy / SelfEnergy / Magnetization / PottsMagnetization
// accumulators (src/hamiltonian/util/observables.h:47-65,186-217,251-268,
// src/hamiltonian/Potts.h:46-61), exact in int64.

// Neighbour sum of the interaction energy of site i: sum over nbrs(i) of
// s_i s_j (bonds) or [s_i == s_j] (Potts).  On stencils, where every bond
// appears in both endpoints' lists, twice the sum over the forward
// neighbours (+x, +y, ...) gives the same total with half the loads.
template <class Lat>
__device__ __forceinline__ int int8_bond_sum(const ModelDev& m, const Lat& lat, const int8_t* __restrict__ s,
                                             int64_t i, int si, bool potts)
{
    const int deg = lat.degree(i);
    int loc = 0;
    if (potts)
        for (int t = 0; t < deg; ++t) loc += (s[lat.addr(lat.nbr(i, t))] == si);
    else {
        for (int t = 0; t < deg; ++t) loc += lat.bond(i, t) * s[lat.addr(lat.nbr(i, t))];
        loc *= si;
    }
    return loc;
}
template <class ST, class SP>
__device__ __forceinline__ int int8_bond_sum_stencil(const ST& st, SP s, int64_t i, int si, bool potts)
{
    int loc = 0;
    for (int d = 0; d < st.degree(i) / 2; ++d) {
        const int v = s[st.addr(st.nbr(i, 2 * d))];
        loc += potts ? (v == si) : st.bond(i, 2 * d) * v;
    }
    return 2 * (potts ? loc : loc * si);
}
__device__ __forceinline__ int int8_bond_sum(const ModelDev&, const StencilDev& st, const int8_t* __restrict__ s,
                                             int64_t i, int si, bool potts)
{
    return int8_bond_sum_stencil(st, s, i, si, potts);
}
template <int D, bool P2, bool SPLIT>
__device__ __forceinline__ int int8_bond_sum(const ModelDev&, const StencilDim<D, P2, SPLIT>& st, const int8_t* __restrict__ s,
                                             int64_t i, int si, bool potts)
{
    return int8_bond_sum_stencil(st, s, i, si, potts);
}

// Part `part` of `nparts` of the accumulation (a grid-stride share per CTA;
// the CTA's totals go to acc with atomics).  Potts state counts are
// aggregated per warp (lanes with equal states add once) before the shared
// histogram.
template <class Lat>
__device__ __forceinline__ void measure_int8_part(const ModelDev& m, const Lat& lat, const int8_t* __restrict__ s,
                                                  long long* __restrict__ acc, int64_t part, int64_t nparts)
{
    __shared__ int hist[64];
    __shared__ long long red[3][32];
    const bool potts = m.kind == MQV_MODEL_POTTS;
    if (potts)
        for (int k = threadIdx.x; k < 64; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    long long e = 0, mg = 0, sq = 0;
    const unsigned lane = threadIdx.x & 31;
    // warp-uniform trip count: every lane takes part in the warp's votes
    const int64_t stride = nparts * blockDim.x;
    for (int64_t i0 = part * (int64_t)blockDim.x + (threadIdx.x & ~31u); i0 < lat.n; i0 += stride) {
        const int64_t i = i0 + lane;
        const bool live = i < lat.n;
        int si = 0;
        if (live) {
            si = s[lat.addr(i)];
            e += int8_bond_sum(m, lat, s, i, si, potts);
            mg += si;
            sq += si * si;
        }
        if (potts) {
            const unsigned peers = __match_any_sync(0xffffffffu, live ? (si & 63) : 64);
            if (live && lane == (unsigned)(__ffs(peers) - 1)) atomicAdd(&hist[si & 63], __popc(peers));
        }
    }
    e = warp_sum_ll(e);
    mg = warp_sum_ll(mg);
    sq = warp_sum_ll(sq);
    const int wid = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][wid] = e;
        red[1][wid] = mg;
        red[2][wid] = sq;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long a = 0, b = 0, c = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            a += red[0][k];
            b += red[1][k];
            c += red[2][k];
        }
        atomicAdd(reinterpret_cast<unsigned long long*>(acc + kAccEne), (unsigned long long)a);
        atomicAdd(reinterpret_cast<unsigned long long*>(acc + kAccMag), (unsigned long long)b);
        atomicAdd(reinterpret_cast<unsigned long long*>(acc + kAccSq), (unsigned long long)c);
    }
    if (potts)
        for (int k = threadIdx.x; k < m.q; k += blockDim.x)
            if (hist[k]) atomicAdd(reinterpret_cast<unsigned long long*>(acc + kAccPotts + k), (unsigned long long)hist[k]);
}

// Accumulators of one measurement -> (e, |m|, m^2, m^4), in the reference's
// order of operations.
__device__ __forceinline__ void finalize_int8_one(const ModelDev& m, int64_t n, const long long* __restrict__ a,
                                                  double* __restrict__ o)
{
    double e, mm;
    if (m.kind == MQV_MODEL_POTTS) {
        long long mx = 0;
        for (int j = 0; j < m.q; ++j) mx = a[kAccPotts + j] > mx ? a[kAccPotts + j] : mx;
        mm = (double)((long long)m.q * mx - n) / (double)(n * (long long)(m.q - 1));
        e = MQV_DMUL(m.k, (double)a[kAccEne]) / (double)(2 * n);
    } else {
        const double mag = (double)a[kAccMag];
        mm = sqrt(MQV_DMUL(mag, mag)) / (double)n;
        e = MQV_DMUL(m.J, (double)a[kAccEne]) / (double)(2 * n);
        // SelfEnergy sums every onsite term over every site, whatever the
        // termselector (observables.h:251-268): (h + h2 terms) / N
        if (m.kind == MQV_MODEL_BLUME_CAPEL)
            e = MQV_DADD(e, MQV_DADD(MQV_DMUL(m.h, (double)a[kAccSq]), MQV_DMUL(m.h2, (double)a[kAccSq])) / (double)n);
    }
    const double m2 = MQV_DMUL(mm, mm);
    o[0] = e;
    o[1] = mm;
    o[2] = m2;
    o[3] = MQV_DMUL(m2, m2);
}

}  // namespace mqv
