// Metropolis sweeps over int8 states (Ising, Potts, Blume-Capel, Edwards-
// Anderson) on any lattice, and their measurements, for sm_100a.
//
// Update order: colour classes in turn (checkerboard parity on hypercubic
// lattices, greedy colours on general graphs), one launch per colour.  Sites
// of one colour have no common bonds, so within a colour the order is
// irrelevant, and each site's random words are keyed by (seed, replica, site,
// sweep): the final state does not depend on the launch geometry.  The 2D
// Ising model on lattices with len % 32 == 0 takes the fused two-colour path
// of ising2d.cu instead; its state is stored in split rows, which the
// lattice's addr() maps for every other kernel.
#include <cuda_runtime.h>

#include "engine.h"

namespace mqv {

// ---------------------------------------------------------------------------
// generic per-site update (Metropolis<H,L>::move, src/libmarqov/metropolis.h:88-126)

template <class Lat>
__device__ __forceinline__ void int8_site(const ModelDev& m, const Lat& lat, int8_t* __restrict__ s, int64_t i,
                                          Key key, uint32_t sweep, uint32_t replica)
{
    SubStream rng(key, (uint32_t)i, sweep, tag(kMetro, replica));
    const int64_t ai = lat.addr(i);
    const int old = s[ai];
    const int deg = lat.degree(i);
    int nw;
    double dE;
    if (m.kind == MQV_MODEL_POTTS) {
        // Initializer<Potts<Q>>::newsv (src/hamiltonian/Potts.h:170-177) and
        // PottsInteraction::diff (src/hamiltonian/Potts.h:86-107)
        nw = (int)(rng.next() % (uint64_t)m.q);
        int eo = 0, en = 0;
        for (int t = 0; t < deg; ++t) {
            const int v = s[lat.addr(lat.nbr(i, t))];
            eo += (v == old);
            en += (v == nw);
        }
        dE = MQV_DMUL(m.k, (double)(en - eo));
    } else if (m.kind == MQV_MODEL_BLUME_CAPEL) {
        // Spin1_Initializer::newsv (src/hamiltonian/util/initializers.h:99-118)
        int st = old;
        if (st == 0) st = rng.real() < 0.5 ? -1 : 1;
        else st = rng.real() < 0.5 ? -st : 0;
        nw = st;
        int sum = 0;
        for (int t = 0; t < deg; ++t) sum += s[lat.addr(lat.nbr(i, t))];
        dE = MQV_DADD(MQV_DMUL(m.J, (double)((nw - old) * sum)), MQV_DMUL(m.h, (double)(nw * nw - old * old)));
    } else {
        // spin flip (src/hamiltonian/util/initializers.h:52-58), neighbourhood
        // sum with optional bonds (src/libmarqov/metropolishelpers.h:456-537)
        nw = -old;
        int sum = 0;
        for (int t = 0; t < deg; ++t) sum += lat.bond(i, t) * s[lat.addr(lat.nbr(i, t))];
        dE = MQV_DMUL(m.J, (double)((nw - old) * sum));
    }
    // metro_update_accepted (src/libmarqov/metropolis.h:61-64,120-124) on the
    // site's acceptance word
    if (dE <= 0 || update_accepted(1, dE, m.beta, accept_word(key, (uint32_t)i, sweep, replica))) s[ai] = (int8_t)nw;
}

// Site of colour `colour` in pair t of a parity-coloured hypercubic lattice
// with even side: sites 2t and 2t+1 differ only in x, so they have opposite
// colours.
__device__ __forceinline__ int64_t parity_site(const StencilDev& st, int64_t t, int colour)
{
    const int64_t i0 = 2 * t;
    int par = 0;
    for (int j = 1; j < st.dim; ++j) par += (int)((i0 / st.pows[j]) % st.len);
    return i0 + (((par & 1) != colour) ? 1 : 0);
}

__global__ void metro_int8_stencil(ModelDev m, StencilDev st, int8_t* __restrict__ s, int colour, Key key,
                                   uint32_t sweep, uint32_t replica)
{
    const int64_t half = st.n / 2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < half; t += (int64_t)gridDim.x * blockDim.x)
        int8_site(m, st, s, parity_site(st, t, colour), key, sweep, replica);
}

__global__ void metro_int8_csr(ModelDev m, CSRDev g, int8_t* __restrict__ s, const int32_t* __restrict__ order,
                               int64_t begin, int64_t count, Key key, uint32_t sweep, uint32_t replica)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x)
        int8_site(m, g, s, order[begin + t], key, sweep, replica);
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

template <class Lat>
__global__ void measure_int8(ModelDev m, Lat lat, const int8_t* __restrict__ s, long long* __restrict__ acc)
{
    __shared__ int hist[64];
    __shared__ long long red[3][32];
    const bool potts = m.kind == MQV_MODEL_POTTS;
    if (potts)
        for (int k = threadIdx.x; k < 64; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    long long e = 0, mg = 0, sq = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < lat.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int si = s[lat.addr(i)];
        const int deg = lat.degree(i);
        int loc = 0;
        if (potts) {
            for (int t = 0; t < deg; ++t) loc += (s[lat.addr(lat.nbr(i, t))] == si);
            atomicAdd(&hist[si & 63], 1);
        } else {
            for (int t = 0; t < deg; ++t) loc += lat.bond(i, t) * s[lat.addr(lat.nbr(i, t))];
            loc *= si;
        }
        e += loc;
        mg += si;
        sq += si * si;
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

// Accumulators -> observables, in the reference's order of operations.
__global__ void finalize_int8(ModelDev m, int64_t n, const long long* __restrict__ acc, int nslots,
                              double* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nslots) return;
    const long long* a = acc + (size_t)k * kAccStride;
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
        if (m.kind == MQV_MODEL_BLUME_CAPEL) e = MQV_DADD(e, MQV_DMUL(m.h, (double)a[kAccSq]) / (double)n);
    }
    const double m2 = MQV_DMUL(mm, mm);
    out[4 * k + 0] = e;
    out[4 * k + 1] = mm;
    out[4 * k + 2] = m2;
    out[4 * k + 3] = MQV_DMUL(m2, m2);
}

// ---------------------------------------------------------------------------
// initial state (Ising.h:99-107, Potts.h:149-156 rules on the INIT stream)

template <class Lat>
__global__ void init_int8(ModelDev m, Lat lat, int64_t n, int8_t* __restrict__ s, Key key, uint32_t tg)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t w = lo64(philox((uint32_t)i, 0u, 0u, tg, key));
        int v;
        if (m.kind == MQV_MODEL_POTTS) v = (int)(w % (uint64_t)m.q);
        else if (m.kind == MQV_MODEL_BLUME_CAPEL) v = (int)(w % 3ull) - 1;
        else v = real01(w) > 0.5 ? 1 : -1;
        s[lat.addr(i)] = (int8_t)v;
    }
}

// ---------------------------------------------------------------------------
// launchers

static int grid_for(int64_t work, int threads)
{
    int64_t b = (work + threads - 1) / threads;
    const int64_t cap = 148 * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

cudaError_t launch_init_int8(Sim* s)
{
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC)
        init_int8<<<grid_for(s->n, 256), 256, 0, s->stream>>>(s->md, s->sten, s->n, (int8_t*)s->state[s->cur],
                                                               make_key(s->seed), tag(kInit, s->replica));
    else
        init_int8<<<grid_for(s->n, 256), 256, 0, s->stream>>>(s->md, s->csr, s->n, (int8_t*)s->state[s->cur],
                                                               make_key(s->seed), tag(kInit, s->replica));
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_measure_int8(Sim* s, int slot)
{
    long long* acc = s->d_acc + (size_t)slot * kAccStride;
    const int8_t* st = (const int8_t*)s->state[s->cur];
    const int g = grid_for(s->n, 256);
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC) measure_int8<<<g, 256, 0, s->stream>>>(s->md, s->sten, st, acc);
    else measure_int8<<<g, 256, 0, s->stream>>>(s->md, s->csr, st, acc);
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_finalize_int8(Sim* s, int nslots, double* d_out)
{
    finalize_int8<<<(nslots + 127) / 128, 128, 0, s->stream>>>(s->md, s->n, s->d_acc, nslots, d_out);
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_ising2d_sweep(Sim* s, long long* acc);

// One Metropolis sweep; when slot >= 0 the new state's observables are
// accumulated into that slot.
cudaError_t launch_metropolis_int8(Sim* s, int slot)
{
    const Key key = make_key(s->seed);
    cudaError_t err = cudaSuccess;
    if (s->fused_ising2d) {
        long long* acc = slot >= 0 ? s->d_acc + (size_t)slot * kAccStride : nullptr;
        err = launch_ising2d_sweep(s, acc);
        s->launches++;
        s->cur ^= 1;
        s->sweep++;
        return err;
    }
    int8_t* st = (int8_t*)s->state[s->cur];
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC) {
        const int g = grid_for(s->n / 2, 256);
        for (int c = 0; c < 2; ++c) {
            metro_int8_stencil<<<g, 256, 0, s->stream>>>(s->md, s->sten, st, c, key, (uint32_t)s->sweep, s->replica);
            s->launches++;
        }
    } else {
        for (size_t c = 0; c + 1 < s->colour_ptr.size(); ++c) {
            const int64_t b = s->colour_ptr[c], cnt = s->colour_ptr[c + 1] - b;
            if (cnt == 0) continue;
            metro_int8_csr<<<grid_for(cnt, 256), 256, 0, s->stream>>>(s->md, s->csr, st, s->d_order, b, cnt, key,
                                                                       (uint32_t)s->sweep, s->replica);
            s->launches++;
        }
    }
    err = cudaGetLastError();
    s->sweep++;
    if (err == cudaSuccess && slot >= 0) err = launch_measure_int8(s, slot);
    return err;
}

}  // namespace mqv
