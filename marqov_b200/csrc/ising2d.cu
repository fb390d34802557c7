// Fused checkerboard Metropolis sweep for the 2D Ising model on sm_100a.
//
// Layout in HBM ("split rows"): row y of the L x L lattice is stored as its
// L/2 even-x sites followed by its L/2 odd-x sites.  In a colour phase every
// byte of a 32-bit word of the active half is a site of the active colour, and
// its four neighbours are the same word of the rows above and below plus the
// same (or the one-site shifted) word of the other half of its own row.
//
// One persistent CTA per SM slot loops over TY x TX tiles with a two-stage
// pipeline: while it updates tile n, the bulk-copy engine (cp.async.bulk,
// completion on an mbarrier) stages tile n+1 with a two-row / 32-column halo
// of the old state, and updated tiles leave shared memory by bulk stores.  In
// shared memory the CTA updates colour 0 on the tile plus its one-site ring
// (re-deriving the neighbouring tiles' updates, which are deterministic), then
// colour 1 on the tile, and writes the tile to the other state buffer: one HBM
// read and one write per site update.
//
// Randomness: a site's acceptance word has its top byte in a Philox block
// shared by 16 consecutive sites (see accept_word in common.cuh).  The CTA
// fills a shared-memory tile of those bytes -- one Philox4x32-10 per 16 sites --
// while the bulk copies are in flight.  A decision compares the byte with the
// top byte of the u53 threshold of the site's class (number of aligned
// neighbours); only on a tie (1/256) is the second block evaluated.  The
// decision equals update_accepted<1>(dE, beta, word) for the full word.
//
// Per word of 4 sites: neighbour minus-counts by byte-wise adds, the aligned
// count by a byte select, thresholds by byte-permute lookups, decisions by
// byte-wise compares, flips by one XOR.  Energy (sum over bonds, each bond
// seen once from its colour-1 end) and magnetisation are reduced in phase 2.
#include <cuda_runtime.h>

#include "engine.h"

namespace mqv {

struct Ising2DArgs {
    const int8_t* src;
    int8_t* dst;
    int L;
    int ntx;
    int ntiles;
    Key key;
    uint32_t sweep;
    uint32_t replica;
    uint32_t t8lo, t8hi;    // top byte of the threshold per aligned count a = 0..4 (clamped to 255)
    uint32_t alwlo, alwhi;  // 0xFF where class a always accepts
    uint32_t ztlo, ztlhi;   // 0xFF where a top-byte tie rejects without the low bits
    unsigned long long thr[5];
    long long* acc;
    int* status;
};

#define MQV_ISING_THREADS 256

template <int TX, int TY>
struct TileGeom {
    static constexpr int H2 = TX / 2;      // interior bytes of a half row
    static constexpr int PH = H2 + 32;     // half pitch: 16 halo + interior + 16 halo
    static constexpr int P = 2 * PH;       // row pitch
    static constexpr int R = TY + 4;       // staged rows: y0-2 .. y0+TY+1
    static constexpr int RR = TY + 2;      // rows with random bytes: y0-1 .. y0+TY
    static constexpr int NG = TX / 16 + 2; // 16-site Philox groups per random row
    static constexpr int STAGE = R * P;
    static constexpr int RND = RR * P;
    static constexpr uint32_t TX_BYTES = (uint32_t)(R * P);
    static constexpr int SMEM = 2 * STAGE + RND + 64;
};

__device__ __forceinline__ int wrapi(int v, int L)
{
    v += v < 0 ? L : 0;
    return v >= L ? v - L : v;
}

// Resolve the tie bytes of one word with the fine block.
__device__ __noinline__ uint32_t resolve_ties(uint32_t tie, uint32_t cbw, uint32_t aw, int j0, int half, int y, int x0,
                                              int L, Key key, uint32_t sweep, uint32_t replica,
                                              const unsigned long long* thr)
{
    uint32_t accm = 0;
    for (int b = 0; b < 4; ++b) {
        if (!((tie >> (8 * b)) & 0xFFu)) continue;
        const int x = wrapi(x0 - 32 + 2 * (j0 + b) + half, L);
        const uint32_t site = (uint32_t)y * (uint32_t)L + (uint32_t)x;
        const uint64_t cb = (cbw >> (8 * b)) & 0xFFu;
        const uint64_t u53 = ((cb << 56) | accept_fine56(key, site, sweep, replica)) >> 11;
        const int cls = (aw >> (8 * b)) & 0xFF;
        if (u53 < thr[cls]) accm |= 0xFFu << (8 * b);
    }
    return accm;
}

// One colour phase over rows [r0, r0 + NR) and words [w0, w0 + NW) of the
// active half of each row.
template <int TX, int TY, int COL, int NR, int NW, bool MEAS>
__device__ __forceinline__ void phase(uint8_t* st, const uint8_t* rnd, int r0, int w0, int x0, int y0,
                                      const Ising2DArgs& a, const unsigned long long* sthr, int& esum, int& msum)
{
    using G = TileGeom<TX, TY>;
    for (int t = threadIdx.x; t < NR * NW; t += MQV_ISING_THREADS) {
        const int r = r0 + t / NW;
        const int w = w0 + t % NW;
        const int p = (COL + r) & 1;  // active half: x parity of colour COL in this row
        uint32_t* H = reinterpret_cast<uint32_t*>(st + r * G::P + p * G::PH);
        const uint32_t* Gr = reinterpret_cast<const uint32_t*>(st + r * G::P + (1 - p) * G::PH);
        const uint32_t A = H[w];
        const uint32_t U = reinterpret_cast<const uint32_t*>(st + (r - 1) * G::P + p * G::PH)[w];
        const uint32_t D = reinterpret_cast<const uint32_t*>(st + (r + 1) * G::P + p * G::PH)[w];
        const uint32_t G0 = Gr[w];
        uint32_t Lw, Rw;
        if (p == 0) {
            Lw = __funnelshift_l(Gr[w - 1], G0, 8);
            Rw = G0;
        } else {
            Lw = G0;
            Rw = __funnelshift_r(G0, Gr[w + 1], 8);
        }
        const uint32_t m1 = 0x01010101u;
        const uint32_t mA = (A >> 1) & m1;
        const uint32_t M = ((U >> 1) & m1) + ((D >> 1) & m1) + ((Lw >> 1) & m1) + ((Rw >> 1) & m1);
        const uint32_t sel = mA * 0xFFu;
        const uint32_t aw = (M & sel) | ((0x04040404u - M) & ~sel);  // aligned neighbours per byte
        const uint32_t tt = aw | (aw >> 4);
        const uint32_t nib = (tt & 0xFFu) | ((tt >> 8) & 0xFF00u);
        const uint32_t T8 = __byte_perm(a.t8lo, a.t8hi, nib);
        const uint32_t ALW = __byte_perm(a.alwlo, a.alwhi, nib);
        const uint32_t cbw = reinterpret_cast<const uint32_t*>(rnd + (r - 1) * G::P + p * G::PH)[w];
        uint32_t accm = __vcmpltu4(cbw, T8) | ALW;
        const uint32_t tie = __vcmpeq4(cbw, T8) & ~ALW & ~__byte_perm(a.ztlo, a.ztlhi, nib);
        if (tie)
            accm |= resolve_ties(tie, cbw, aw, 4 * w, p, wrapi(y0 - 2 + r, a.L), x0, a.L, a.key, a.sweep, a.replica, sthr);
        const uint32_t An = A ^ (accm & 0xFEFEFEFEu);
        if (accm) H[w] = An;
        if (MEAS) {
            // bond sum seen from the colour-1 end, and both colours' spins
            esum = __dp4a((int)An, (int)__vsub4(0x04040404u, M + M), esum);
            msum = __dp4a((int)An, 0x01010101, msum);
            msum = __dp4a((int)G0, 0x01010101, msum);
        }
    }
}

template <int TX, int TY, bool MEAS>
__global__ void __launch_bounds__(MQV_ISING_THREADS, 4) ising2d_sweep(const __grid_constant__ Ising2DArgs a)
{
    using G = TileGeom<TX, TY>;
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* stage0 = smem;
    uint8_t* rnd = smem + 2 * G::STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * G::STAGE + G::RND);
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int L = a.L;
    const int Lh = L >> 1;
    const uint32_t tg_acc = tag(kAccept, a.replica);
    __shared__ unsigned long long sthr[5];
    if (tid == 0) {
        mbar_init(smem_addr(&bars[0]), 1);
        mbar_init(smem_addr(&bars[1]), 1);
        mbar_fence_init();
#pragma unroll
        for (int k = 0; k < 5; ++k) sthr[k] = a.thr[k];
    }
    __syncthreads();

    auto issue_load = [&](int tile, int stg) {
        // warp 0: stage rows y0-2 .. y0+TY+1 of both halves, columns x0-32 .. x0+TX+31
        const int tx = tile % a.ntx, ty = tile / a.ntx;
        const int x0 = tx * TX, y0 = ty * TY;
        uint8_t* sb = stage0 + stg * G::STAGE;
        const uint32_t bar = smem_addr(&bars[stg]);
        if (lane == 0) mbar_expect_tx(bar, G::TX_BYTES);
        __syncwarp();
        const bool inner = x0 > 0 && x0 + TX < L;
        for (int task = lane; task < 2 * G::R; task += 32) {
            const int r = task >> 1, h = task & 1;
            const int gy = wrapi(y0 - 2 + r, L);
            const int8_t* row = a.src + (size_t)gy * L + (size_t)h * Lh;
            const uint32_t d = smem_addr(sb + r * G::P + h * G::PH);
            const int j0 = (x0 >> 1) - 16;
            if (inner) {
                bulk_g2s(d, row + j0, G::PH, bar);
            } else {
                bulk_g2s(d, row + (j0 < 0 ? j0 + Lh : j0), 16, bar);
                bulk_g2s(d + 16, row + (x0 >> 1), G::H2, bar);
                const int jr = (x0 >> 1) + G::H2;
                bulk_g2s(d + 16 + G::H2, row + (jr >= Lh ? jr - Lh : jr), 16, bar);
            }
        }
    };

    int esum = 0, msum = 0;
    int tile = blockIdx.x;
    if (tile < a.ntiles && warp == 0) issue_load(tile, 0);
    for (int it = 0; tile < a.ntiles; ++it, tile += gridDim.x) {
        const int stg = it & 1;
        uint8_t* sb = stage0 + stg * G::STAGE;
        const int tx = tile % a.ntx, ty = tile / a.ntx;
        const int x0 = tx * TX, y0 = ty * TY;
        // prefetch the next tile into the other stage once its stores have read it
        const int next = tile + gridDim.x;
        if (warp == 0 && next < a.ntiles) {
            bulk_wait_read0();
            __syncwarp();
            issue_load(next, stg ^ 1);
        }
        // random top bytes of this tile's updated sites, split by x parity
        for (int task = tid; task < G::RR * G::NG; task += MQV_ISING_THREADS) {
            const int rr = task / G::NG, g = task % G::NG;
            const int gy = wrapi(y0 - 1 + rr, L);
            const int gx = wrapi(x0 - 16 + 16 * g, L);
            const uint32_t site0 = (uint32_t)gy * (uint32_t)L + (uint32_t)gx;
            const uint4 v = philox(site0 >> 4, a.sweep, 0u, tg_acc, a.key);
            uint8_t* rrow = rnd + rr * G::P + 8 * g + 8;
            *reinterpret_cast<uint2*>(rrow) = make_uint2(__byte_perm(v.x, v.y, 0x6420), __byte_perm(v.z, v.w, 0x6420));
            *reinterpret_cast<uint2*>(rrow + G::PH) =
                make_uint2(__byte_perm(v.x, v.y, 0x7531), __byte_perm(v.z, v.w, 0x7531));
        }
        // wait for the staged tile (bounded: a stuck copy sets an error status)
        {
            const uint32_t bar = smem_addr(&bars[stg]);
            const uint32_t par = (uint32_t)(it >> 1) & 1u;
            int timed_out = 0;
            if (!mbar_try_wait(bar, par)) {
                const uint64_t t0 = global_timer_ns();
                for (uint32_t k = 1;; ++k) {
                    if (mbar_try_wait(bar, par)) break;
                    if ((k & 63u) == 0 && global_timer_ns() - t0 > 2000000000ull) {
                        timed_out = 1;
                        break;
                    }
                }
            }
            if (__syncthreads_or(timed_out)) {
                if (tid == 0) atomicExch(a.status, MQV_ERR_TIMEOUT);
                break;
            }
        }
        // colour 0 on the tile and its ring (rows 1..TY+2), then colour 1 on the tile
        phase<TX, TY, 0, TY + 2, TX / 8 + 2, false>(sb, rnd, 1, 3, x0, y0, a, sthr, esum, msum);
        __syncthreads();
        phase<TX, TY, 1, TY, TX / 8, MEAS>(sb, rnd, 2, 4, x0, y0, a, sthr, esum, msum);
        fence_proxy_async_smem();
        __syncthreads();
        if (warp == 0) {
            for (int task = lane; task < 2 * TY; task += 32) {
                const int r = 2 + (task >> 1), h = task & 1;
                int8_t* drow = a.dst + (size_t)(y0 + r - 2) * L + (size_t)h * Lh + (x0 >> 1);
                bulk_s2g(drow, smem_addr(sb + r * G::P + h * G::PH + 16), G::H2);
            }
            bulk_commit();
        }
    }
    if (warp == 0) bulk_wait0();
    if (MEAS) {
        __shared__ long long red[2][MQV_ISING_THREADS / 32];
        long long e = esum, m = msum;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, o);
            m += __shfl_xor_sync(0xffffffffu, m, o);
        }
        if (lane == 0) {
            red[0][warp] = e;
            red[1][warp] = m;
        }
        __syncthreads();
        if (tid == 0) {
            long long es = 0, ms = 0;
            for (int k = 0; k < MQV_ISING_THREADS / 32; ++k) {
                es += red[0][k];
                ms += red[1][k];
            }
            // enepart = sum_i sum_{j in nbrs(i)} s_i s_j counts every bond twice
            atomicAdd(reinterpret_cast<unsigned long long*>(a.acc + kAccEne), (unsigned long long)(2 * es));
            atomicAdd(reinterpret_cast<unsigned long long*>(a.acc + kAccMag), (unsigned long long)ms);
        }
    }
}

// ---- layout conversion: row-major <-> split rows -----------------------------

__global__ void split_rows(const int8_t* __restrict__ in, int8_t* __restrict__ out, int L)
{
    const int64_t n = (int64_t)L * L;
    const int Lh = L >> 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t y = i / L;
        const int x = (int)(i - y * L);
        out[y * L + (x & 1) * Lh + (x >> 1)] = in[i];
    }
}

__global__ void merge_rows(const int8_t* __restrict__ in, int8_t* __restrict__ out, int L)
{
    const int64_t n = (int64_t)L * L;
    const int Lh = L >> 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t y = i / L;
        const int x = (int)(i - y * L);
        out[i] = in[y * L + (x & 1) * Lh + (x >> 1)];
    }
}

// ---- host side ------------------------------------------------------------------

constexpr int kIsingTY = 32;

static int tile_width(int L)
{
    for (int tx : {256, 128, 64, 32})
        if (L % tx == 0) return tx;
    return 0;
}

bool ising2d_supported(int L) { return L >= 32 && L % 32 == 0 && tile_width(L) > 0; }

template <int TX, bool MEAS>
static cudaError_t launch_t(const Ising2DArgs& a, int nsm, cudaStream_t stream)
{
    using G = TileGeom<TX, kIsingTY>;
    auto kern = ising2d_sweep<TX, kIsingTY, MEAS>;
    static int cps = 0;  // resident CTAs per SM for this instantiation
    if (cps == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
        if (e != cudaSuccess) return e;
        int c = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, kern, MQV_ISING_THREADS, G::SMEM);
        if (e != cudaSuccess) return e;
        cps = c < 1 ? 1 : c;
    }
    int grid = nsm * cps;
    if (grid > a.ntiles) grid = a.ntiles;
    kern<<<grid, MQV_ISING_THREADS, G::SMEM, stream>>>(a);
    return cudaGetLastError();
}

template <int TX>
static cudaError_t launch_tx(const Ising2DArgs& a, int nsm, cudaStream_t stream)
{
    return a.acc ? launch_t<TX, true>(a, nsm, stream) : launch_t<TX, false>(a, nsm, stream);
}

// Thresholds per aligned-neighbour count a: dE = J (s_new - s_old) sum_nbrs =
// J (8 - 4a), the cut of update_accepted<1> on u53, its top byte and flags.
void ising2d_thresholds(double J, double beta, unsigned long long thr[5], uint32_t pools[6])
{
    uint32_t t8[2] = {0, 0}, alw[2] = {0, 0}, zt[2] = {0, 0};
    for (int k = 0; k < 5; ++k) {
        const double dE = J * (double)(8 - 4 * k);
        const unsigned long long T = accept_cut(1, dE, beta);
        thr[k] = T;
        const unsigned long long hi = T >> 45;
        const uint32_t c = hi > 255 ? 255u : (uint32_t)hi;
        const int wd = k >> 2, sh = 8 * (k & 3);
        t8[wd] |= c << sh;
        if (T >= (1ull << 53)) alw[wd] |= 0xFFu << sh;
        if ((T & ((1ull << 45) - 1)) == 0) zt[wd] |= 0xFFu << sh;
    }
    pools[0] = t8[0];
    pools[1] = t8[1];
    pools[2] = alw[0];
    pools[3] = alw[1];
    pools[4] = zt[0];
    pools[5] = zt[1];
}

cudaError_t launch_ising2d_sweep(Sim* s, long long* acc)
{
    const int TX = tile_width(s->len);
    Ising2DArgs a{};
    a.src = (const int8_t*)s->state[s->cur];
    a.dst = (int8_t*)s->state[s->cur ^ 1];
    a.L = s->len;
    a.ntx = s->len / TX;
    a.ntiles = a.ntx * (s->len / kIsingTY);
    a.key = make_key(s->seed);
    a.sweep = (uint32_t)s->sweep;
    a.replica = s->replica;
    if (s->thr_J != s->md.J || s->thr_beta != s->md.beta) {
        ising2d_thresholds(s->md.J, s->md.beta, s->thr_cut, s->thr_pools);
        s->thr_J = s->md.J;
        s->thr_beta = s->md.beta;
    }
    const uint32_t* pools = s->thr_pools;
    for (int k = 0; k < 5; ++k) a.thr[k] = s->thr_cut[k];
    a.t8lo = pools[0];
    a.t8hi = pools[1];
    a.alwlo = pools[2];
    a.alwhi = pools[3];
    a.ztlo = pools[4];
    a.ztlhi = pools[5];
    a.acc = acc;
    a.status = s->d_status;
    const int nsm = s->num_sms;
    switch (TX) {
    case 256: return launch_tx<256>(a, nsm, s->stream);
    case 128: return launch_tx<128>(a, nsm, s->stream);
    case 64: return launch_tx<64>(a, nsm, s->stream);
    default: return launch_tx<32>(a, nsm, s->stream);
    }
}

cudaError_t launch_split_rows(Sim* s, const void* rowmajor, void* split)
{
    split_rows<<<148 * 8, 256, 0, s->stream>>>((const int8_t*)rowmajor, (int8_t*)split, s->len);
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_merge_rows(Sim* s, const void* split, void* rowmajor)
{
    merge_rows<<<148 * 8, 256, 0, s->stream>>>((const int8_t*)split, (int8_t*)rowmajor, s->len);
    s->launches++;
    return cudaGetLastError();
}

}  // namespace mqv
