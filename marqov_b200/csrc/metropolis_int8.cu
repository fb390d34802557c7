// Metropolis sweeps over int8 states (Ising, Potts, Blume-Capel, Edwards-
// Anderson) and their measurements, for sm_100a.
//
// Update order: colour classes in turn (checkerboard parity on hypercubic
// lattices, greedy colours on general graphs).  Sites of one colour have no
// common bonds, so within a colour the order is irrelevant, and each site's
// random words are keyed by (seed, replica, site, sweep): the final state is
// independent of the launch geometry.
//
// Fast path (2D hypercubic Ising, len % 16 == 0): one kernel performs both
// colours.  A CTA stages its tile plus a two-row / one-word halo of the old
// state in shared memory, updates colour 0 on the tile and its one-site ring
// (recomputing the neighbours' updates, which are deterministic), then
// colour 1 on the tile, and writes the tile to the other state buffer.  Every
// site is read once and written once per sweep: 2 bytes of HBM traffic per
// site update.  The bond energy and magnetisation of the new state are
// reduced in the same pass.
#include <cuda_runtime.h>

#include "engine.h"

namespace mqv {

// ---------------------------------------------------------------------------
// generic per-site update (Metropolis<H,L>::move, src/libmarqov/metropolis.h:88-126)

template <class Lat>
__device__ __forceinline__ void int8_site(const ModelDev& m, const Lat& lat, int8_t* __restrict__ s,
                                          int64_t i, Key key, uint32_t sweep, uint32_t tg)
{
    SubStream rng(key, (uint32_t)i, sweep, tg);
    const int old = s[i];
    const int deg = lat.degree(i);
    int nw;
    double dE;
    if (m.kind == MQV_MODEL_POTTS) {
        // Initializer<Potts<Q>>::newsv (src/hamiltonian/Potts.h:170-177) and
        // PottsInteraction::diff (src/hamiltonian/Potts.h:86-107)
        nw = (int)(rng.next() % (uint64_t)m.q);
        int eo = 0, en = 0;
        for (int t = 0; t < deg; ++t) {
            const int v = s[lat.nbr(i, t)];
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
        for (int t = 0; t < deg; ++t) sum += s[lat.nbr(i, t)];
        dE = MQV_DADD(MQV_DMUL(m.J, (double)((nw - old) * sum)), MQV_DMUL(m.h, (double)(nw * nw - old * old)));
    } else {
        // spin flip (src/hamiltonian/util/initializers.h:52-58), neighbourhood
        // sum with optional bonds (src/libmarqov/metropolishelpers.h:456-537)
        nw = -old;
        int sum = 0;
        for (int t = 0; t < deg; ++t) sum += lat.bond(i, t) * s[lat.nbr(i, t)];
        dE = MQV_DMUL(m.J, (double)((nw - old) * sum));
    }
    if (dE <= 0 || update_accepted(1, dE, m.beta, rng.next())) s[i] = (int8_t)nw;
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
                                   uint32_t sweep, uint32_t tg)
{
    const int64_t half = st.n / 2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < half; t += (int64_t)gridDim.x * blockDim.x)
        int8_site(m, st, s, parity_site(st, t, colour), key, sweep, tg);
}

__global__ void metro_int8_csr(ModelDev m, CSRDev g, int8_t* __restrict__ s, const int32_t* __restrict__ order,
                               int64_t begin, int64_t count, Key key, uint32_t sweep, uint32_t tg)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x)
        int8_site(m, g, s, order[begin + t], key, sweep, tg);
}

// ---------------------------------------------------------------------------
// fused two-colour 2D Ising tile kernel

struct Thr2D {
    unsigned long long t[10];  // index 5*(self is -1) + (number of -1 neighbours)
};

__device__ __forceinline__ long long warp_sum_ll(long long v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One colour phase over rows [r0, r1) and words [w0, w1) of the tile.
// bytes of words w0 / w1-1 outside [c0, c1) columns are left alone.
template <int W, int COL, bool MEAS>
__device__ __forceinline__ void ising2d_phase(uint32_t* tile, int r0, int r1, int w0, int w1, int c0, int c1,
                                              int x0, int y0, int L, const unsigned long long* thr, Key key,
                                              uint32_t sweep, uint32_t tg, int& esum)
{
    const int nw = w1 - w0;
    const int tot = (r1 - r0) * nw;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int r = r0 + t / nw;
        const int w = w0 + t % nw;
        uint32_t C = tile[r * W + w];
        const uint32_t U = tile[(r - 1) * W + w];
        const uint32_t D = tile[(r + 1) * W + w];
        const uint32_t Lw = __funnelshift_l(tile[r * W + w - 1], C, 8);
        const uint32_t Rw = __funnelshift_r(C, tile[r * W + w + 1], 8);
        const uint32_t mC = (C >> 1) & 0x01010101u;
        const uint32_t M = ((U >> 1) & 0x01010101u) + ((D >> 1) & 0x01010101u) + ((Lw >> 1) & 0x01010101u) +
                           ((Rw >> 1) & 0x01010101u);
        const int p = (COL + r) & 1;
        uint32_t flip = 0;
#pragma unroll
        for (int bb = 0; bb < 2; ++bb) {
            const int b = p + 2 * bb;
            const int col = 4 * w + b;
            if (col < c0 || col >= c1) continue;
            const int mc = (mC >> (8 * b)) & 1;
            const int Mb = (M >> (8 * b)) & 0xFF;
            const unsigned long long T = thr[mc * 5 + Mb];
            bool acc;
            if (T >= (1ull << 53)) {
                acc = true;
            } else if (T == 0) {
                acc = false;
            } else {
                int gx = x0 + col - 16;
                gx += gx < 0 ? L : 0;
                gx -= gx >= L ? L : 0;
                int gy = y0 + r - 2;
                gy += gy < 0 ? L : 0;
                gy -= gy >= L ? L : 0;
                const uint32_t site = (uint32_t)gy * (uint32_t)L + (uint32_t)gx;
                const uint4 v = philox(site, sweep, 0u, tg, key);
                acc = (lo64(v) >> 11) < T;
            }
            if (acc) flip |= 0xFEu << (8 * b);
            if (MEAS) {
                const int sf = acc ? (mc ? 1 : -1) : (mc ? -1 : 1);
                esum += sf * (4 - 2 * Mb);
            }
        }
        if (flip) tile[r * W + w] = C ^ flip;
    }
}

template <int TX, int TY, bool MEAS>
__global__ void __launch_bounds__(256) ising2d_fused(const int8_t* __restrict__ src, int8_t* __restrict__ dst, int L,
                                                     Thr2D thr, Key key, uint32_t sweep, uint32_t tg,
                                                     long long* __restrict__ acc)
{
    constexpr int P = TX + 32;  // pitch in bytes: 16 pad/halo + TX + 16 halo/pad
    constexpr int W = P / 4;
    constexpr int R = TY + 4;
    constexpr int NV = TX / 16;
    __shared__ __align__(16) uint32_t tile[R * W];
    __shared__ unsigned long long sthr[10];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 10; ++k) sthr[k] = thr.t[k];
    }
    const int x0 = blockIdx.x * TX;
    const int y0 = blockIdx.y * TY;

    // stage old state: rows y0-2 .. y0+TY+1, columns x0-4 .. x0+TX+3 (wrapped)
    for (int t = threadIdx.x; t < R * (NV + 2); t += blockDim.x) {
        const int r = t / (NV + 2);
        const int c = t - r * (NV + 2);
        int gy = y0 - 2 + r;
        gy += gy < 0 ? L : 0;
        gy -= gy >= L ? L : 0;
        const int8_t* row = src + (size_t)gy * L;
        if (c < NV) {
            const uint4 v = __ldcs(reinterpret_cast<const uint4*>(row + x0) + c);
            *reinterpret_cast<uint4*>(&tile[r * W + 4 + 4 * c]) = v;
        } else if (c == NV) {
            const int gx = x0 == 0 ? L - 4 : x0 - 4;
            tile[r * W + 3] = *reinterpret_cast<const uint32_t*>(row + gx);
        } else {
            const int gx = x0 + TX >= L ? 0 : x0 + TX;
            tile[r * W + 4 + TX / 4] = *reinterpret_cast<const uint32_t*>(row + gx);
        }
    }
    __syncthreads();
    int esum = 0;
    // colour 0 on the tile and its one-site ring: rows 1..TY+2, cols 15..TX+16
    ising2d_phase<W, 0, false>(tile, 1, TY + 3, 3, 5 + TX / 4, 15, TX + 17, x0, y0, L, sthr, key, sweep, tg, esum);
    __syncthreads();
    // colour 1 on the tile: rows 2..TY+1, cols 16..TX+15
    ising2d_phase<W, 1, MEAS>(tile, 2, TY + 2, 4, 4 + TX / 4, 16, TX + 16, x0, y0, L, sthr, key, sweep, tg, esum);
    __syncthreads();
    int msum = 0;
    for (int t = threadIdx.x; t < TY * NV; t += blockDim.x) {
        const int r = t / NV;
        const int c = t - r * NV;
        const uint4 v = *reinterpret_cast<const uint4*>(&tile[(r + 2) * W + 4 + 4 * c]);
        __stcs(reinterpret_cast<uint4*>(dst + (size_t)(y0 + r) * L + x0) + c, v);
        if (MEAS) {
            msum = __dp4a((int)v.x, 0x01010101, msum);
            msum = __dp4a((int)v.y, 0x01010101, msum);
            msum = __dp4a((int)v.z, 0x01010101, msum);
            msum = __dp4a((int)v.w, 0x01010101, msum);
        }
    }
    if (MEAS) {
        __shared__ long long red[2][8];
        long long e = warp_sum_ll((long long)esum);
        long long mg = warp_sum_ll((long long)msum);
        const int wid = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) {
            red[0][wid] = e;
            red[1][wid] = mg;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            long long es = 0, ms = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
                es += red[0][k];
                ms += red[1][k];
            }
            // enepart = sum_i sum_{j in nbrs(i)} s_i s_j counts every bond twice
            atomicAdd(reinterpret_cast<unsigned long long*>(acc + kAccEne), (unsigned long long)(2 * es));
            atomicAdd(reinterpret_cast<unsigned long long*>(acc + kAccMag), (unsigned long long)ms);
        }
    }
}

template <int TX, int TY>
static cudaError_t launch_fused_t(Sim* s, bool meas, long long* acc)
{
    dim3 grid(s->len / TX, s->len / TY);
    const int8_t* src = (const int8_t*)s->state[s->cur];
    int8_t* dst = (int8_t*)s->state[s->cur ^ 1];
    Thr2D thr;
    for (int k = 0; k < 10; ++k) thr.t[k] = s->thr2d[k];
    const Key key = make_key(s->seed);
    const uint32_t tg = tag(kMetro, s->replica);
    if (meas)
        ising2d_fused<TX, TY, true><<<grid, 256, 0, s->stream>>>(src, dst, s->len, thr, key, (uint32_t)s->sweep, tg, acc);
    else
        ising2d_fused<TX, TY, false><<<grid, 256, 0, s->stream>>>(src, dst, s->len, thr, key, (uint32_t)s->sweep, tg, acc);
    return cudaGetLastError();
}

template <int TX>
static cudaError_t launch_fused_ty(Sim* s, bool meas, long long* acc)
{
    const int L = s->len;
    if (L % 32 == 0) return launch_fused_t<TX, 32>(s, meas, acc);
    if (L % 16 == 0) return launch_fused_t<TX, 16>(s, meas, acc);
    return cudaErrorInvalidValue;
}

static cudaError_t launch_fused(Sim* s, bool meas, long long* acc)
{
    const int L = s->len;
    if (L % 256 == 0) return launch_fused_ty<256>(s, meas, acc);
    if (L % 128 == 0) return launch_fused_ty<128>(s, meas, acc);
    if (L % 64 == 0) return launch_fused_ty<64>(s, meas, acc);
    if (L % 32 == 0) return launch_fused_ty<32>(s, meas, acc);
    return launch_fused_ty<16>(s, meas, acc);
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
        const int si = s[i];
        const int deg = lat.degree(i);
        int loc = 0;
        if (potts) {
            for (int t = 0; t < deg; ++t) loc += (s[lat.nbr(i, t)] == si);
            atomicAdd(&hist[si & 63], 1);
        } else {
            for (int t = 0; t < deg; ++t) loc += lat.bond(i, t) * s[lat.nbr(i, t)];
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

__global__ void init_int8(ModelDev m, int64_t n, int8_t* __restrict__ s, Key key, uint32_t tg)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t w = lo64(philox((uint32_t)i, 0u, 0u, tg, key));
        int v;
        if (m.kind == MQV_MODEL_POTTS) v = (int)(w % (uint64_t)m.q);
        else if (m.kind == MQV_MODEL_BLUME_CAPEL) v = (int)(w % 3ull) - 1;
        else v = real01(w) > 0.5 ? 1 : -1;
        s[i] = (int8_t)v;
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
    init_int8<<<grid_for(s->n, 256), 256, 0, s->stream>>>(s->md, s->n, (int8_t*)s->state[s->cur], make_key(s->seed),
                                                           tag(kInit, s->replica));
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

// One Metropolis sweep; when slot >= 0 the new state's observables are
// accumulated into that slot.
cudaError_t launch_metropolis_int8(Sim* s, int slot)
{
    const Key key = make_key(s->seed);
    const uint32_t tg = tag(kMetro, s->replica);
    cudaError_t err = cudaSuccess;
    if (s->fused_ising2d) {
        long long* acc = slot >= 0 ? s->d_acc + (size_t)slot * kAccStride : nullptr;
        err = launch_fused(s, slot >= 0, acc);
        s->launches++;
        s->cur ^= 1;
        s->sweep++;
        return err;
    }
    int8_t* st = (int8_t*)s->state[s->cur];
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC) {
        const int g = grid_for(s->n / 2, 256);
        for (int c = 0; c < 2; ++c) {
            metro_int8_stencil<<<g, 256, 0, s->stream>>>(s->md, s->sten, st, c, key, (uint32_t)s->sweep, tg);
            s->launches++;
        }
    } else {
        for (size_t c = 0; c + 1 < s->colour_ptr.size(); ++c) {
            const int64_t b = s->colour_ptr[c], cnt = s->colour_ptr[c + 1] - b;
            if (cnt == 0) continue;
            metro_int8_csr<<<grid_for(cnt, 256), 256, 0, s->stream>>>(s->md, s->csr, st, s->d_order, b, cnt, key,
                                                                       (uint32_t)s->sweep, tg);
            s->launches++;
        }
    }
    err = cudaGetLastError();
    s->sweep++;
    if (err == cudaSuccess && slot >= 0) err = launch_measure_int8(s, slot);
    return err;
}

}  // namespace mqv
