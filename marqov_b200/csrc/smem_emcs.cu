// Elementary Monte Carlo steps of small int8 lattices held in the shared
// memory of one CTA each, for sm_100a.
//
// On a lattice of a few thousand sites (the 2D Ising L = 64 parity run) a
// launch per cluster, per colour and per measurement costs more than the
// work, and a breadth-first cluster pays a CTA barrier per level of its
// depth.  Here one CTA loads a lattice's state once and runs a whole chunk of
// EMCS (EMCS<H,L>::move, src/libmarqov/emcs.h:69-109: ncluster Wolff
// clusters, then nmetro sweeps, then the measurement) before writing it back:
//   * each cluster as the seed's component of the activated bonds: the seed
//     and its new state from the WOLFF_SEED substream (the breadth-first
//     kernel's draws), every bond between two sites in the seed's old state
//     tested once on its keyed draw (lower id, cluster serial, upper id) --
//     the same cluster as the breadth-first growth, whatever the order.  On
//     lattices of two or more dimensions the component is found by a
//     bit-parallel flood fill (resident_cluster_bits): candidate and
//     active-bond bit planes from warp ballots, then rows closed along x by
//     prefix scans on 32-site words and joined across rows by prefix scans
//     over a warp's lanes, repeated until nothing changes -- no atomics, and
//     a cost of a few passes over n / 32 words.  One-dimensional chains
//     take union-find on 16-bit parent indices instead;
//   * each sweep as the per-colour kernels do it (int8_site on the same
//     keyed words, the warps' acceptance bytes shared per block of runs);
//   * the measurement accumulators of every EMCS, as measure_int8.
// Results equal the per-launch path bit for bit.  A single handle runs one
// CTA (emcs_resident); a batch runs one CTA per small member
// (batch_resident), members being independent.
#include <cuda_runtime.h>

#include <atomic>
#include <type_traits>

#include "batch.h"
#include "int8_site.cuh"
#include "wolff_int8.cuh"

namespace mqv {

constexpr int kResThreads = 512;
constexpr int kResWarps = kResThreads / 32;
constexpr int kResBatch = 4;  // plane words a warp handles side by side

struct ResidentRun {
    ModelDev m;
    StencilDev st;  // the lattice in its global layout (split rows or not)
    WolffDev w;
    Key key;
    uint32_t replica, sweep0, cluster0;  // counters of the chunk's first EMCS
    int n_emcs, ncluster, nmetro, D, runs;
    const unsigned long long* cuts;
    int8_t* state;      // global state, read at the start and written at the end
    long long* acc;     // measurement accumulators of the first EMCS (zeroed), or NULL
    int64_t acc_e;      // stride between EMCS (long longs)
    int32_t* csize;     // cluster size of the first cluster
    int64_t csize_e;    // stride between EMCS
    int64_t csize_c;    // stride between the clusters of one EMCS
};

// Bit planes of the flood-fill cluster: rows are the x-lines of the lattice
// (n / len of them), each padded to kRowWords(len) 32-site words.
__host__ __device__ inline int res_row_words(int len) { return (len + 31) / 32; }
// the flood fill applies to lattices of >= 2 dimensions with rows of <= 8 words
__host__ __device__ inline bool res_bits_ok(int dim, int len) { return dim >= 2 && res_row_words(len) <= 8; }
// planes: candidates, flood, x bonds, one per other dimension
__host__ __device__ inline size_t res_bits_bytes(int64_t n, int dim, int len)
{
    return (size_t)(2 + dim) * (size_t)(n / len) * (size_t)res_row_words(len) * 4;
}
// union-find layout: 16-bit parents, candidate bits
__host__ __device__ inline size_t res_uf_bytes(int64_t n)
{
    return (size_t)((2 * n + 15) & ~15ll) + (size_t)((n + 31) / 32) * 4;
}
// shared memory: the warps' acceptance tables, the cluster's work area (bit
// planes or union-find arrays), the state
__host__ __device__ inline size_t resident_smem_bytes(int64_t n, int dim, int len)
{
    const size_t work = res_bits_ok(dim, len) ? res_bits_bytes(n, dim, len) : res_uf_bytes(n);
    return (size_t)kResWarps * kAccTab * 16 + ((work + 15) & ~(size_t)15) + (size_t)((n + 15) & ~15ll);
}
// the largest of any lattice on this path
__host__ __device__ inline size_t resident_smem_max()
{
    return (size_t)kResWarps * kAccTab * 16 + res_uf_bytes(kResidentMaxSites) + (size_t)kResidentMaxSites;
}
size_t resident_smem_for(const StencilDev& st) { return resident_smem_bytes(st.n, st.dim, st.len); }

// union-find on 16-bit parent indices (path halving; hooks by CAS, linking by uf_prio16)
__device__ __forceinline__ int rfind(volatile unsigned short* p, int x)
{
    while (true) {
        const int px = p[x];
        if (px == x) return x;
        const int gp = p[px];
        if (gp != px) p[x] = (unsigned short)gp;
        x = gp;
    }
}
__device__ __forceinline__ void runite(volatile unsigned short* p, int a, int b)
{
    while (true) {
        a = rfind(p, a);
        b = rfind(p, b);
        if (a == b) return;
        if (uf_prio16((uint32_t)a) > uf_prio16((uint32_t)b)) {  // the root of lower priority hangs below
            const int t = a;
            a = b;
            b = t;
        }
        if (atomicCAS((unsigned short*)p + a, (unsigned short)a, (unsigned short)b) == (unsigned short)a) return;
    }
}

// rows (x-lines) of a stencil: the row of site index i = r len, and the row
// one step up / down in dimension d >= 1, periodic
__device__ __forceinline__ uint32_t res_row_of(const StencilDev& st, uint32_t i)
{
    return st.lg >= 0 ? i >> st.lg : st.divlen(i);
}
__device__ __forceinline__ uint32_t res_row_step(const StencilDev& st, uint32_t r, int d, int dir)
{
    return res_row_of(st, (uint32_t)st.nbr((int64_t)r * st.len, 2 * d + (dir < 0 ? 1 : 0)));
}

// Rows of up to 64 sites as one integer (bit x = site x): the closure of a
// set S along a line through the bonds A (bit x set: site x joined to site
// x - 1) towards higher x, by one addition -- an entry bit just above a
// flooded site ripples its carry through the run of joined sites above it
// ((A + E) ^ A marks the bits it passes); an entry bit that the carry of a
// lower one reaches keeps its value, so the entries are added back.  Towards
// lower x: the same on the bit-reversed row.
template <class T>
__device__ __forceinline__ T row_brev(T x);
template <>
__device__ __forceinline__ uint32_t row_brev<uint32_t>(uint32_t x) { return __brev(x); }
template <>
__device__ __forceinline__ unsigned long long row_brev<unsigned long long>(unsigned long long x) { return __brevll(x); }
template <class T>
__device__ __forceinline__ T row_close_up(T S, T A)
{
    const T E = (S << 1) & A;
    return S | E | (((A + E) ^ A) & A);
}
template <class T>
__device__ __forceinline__ T row_close(T S, T Aup, T Adn)
{
    return row_brev(row_close_up(row_brev(row_close_up(S, Aup)), Adn));
}
__device__ __forceinline__ uint32_t fold32(uint32_t x) { return x; }
__device__ __forceinline__ uint32_t fold32(unsigned long long x) { return (uint32_t)x | (uint32_t)(x >> 32); }

// One warp closes the flood of a 2D lattice of at most 64 rows of at most 64
// sites on its own (two rows per lane: rows 2 lane and 2 lane + 1), so the
// fill needs no CTA barrier and no shared-memory round trip until it is
// closed.  Planes as resident_cluster_bits: F (in: the seed, out: the
// component), Bx the +x bonds, By the +y bonds (row r to row r + 1, periodic).
// Each pass: along y, prefix scans over the lanes upwards and downwards side
// by side from the same start (a column's vertical closure is what reaches up
// plus what reaches down; a lane block passes the flood between its rows
// through its inner bond), then the periodic bond of row R - 1 to row 0;
// along x, each row closed as a line by additions, joined through its
// periodic bond, closed again.  Until a pass adds no site.
template <int WR>  // words per row (1 or 2)
__device__ void resident_fill_warp2(uint32_t* F, const uint32_t* Bx, const uint32_t* By, int R, int len)
{
    using T = typename std::conditional<WR == 1, uint32_t, unsigned long long>::type;
    const unsigned lane = threadIdx.x & 31u;
    const int ra = (R - 1) >> 1, ka = (R - 1) & 1;  // lane and slot of the last row
    const T top = (T)1 << (len - 1), ends = top | (T)1;
    T G[2], Aup[2], Adn[2];
    uint32_t up[2][2];
    bool wrap[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int r = 2 * (int)lane + k;
        const bool live = r < R;
        T g = 0, b = 0;
#pragma unroll
        for (int q = 0; q < WR; ++q)
            if (live) {
                g |= (T)F[r * WR + q] << (32 * q);
                b |= (T)Bx[r * WR + q] << (32 * q);
            }
        wrap[k] = (b & top) != 0;  // the periodic x bond of the row, carried apart
        b &= ~top;
        G[k] = g;
        Aup[k] = b << 1;
        Adn[k] = row_brev(b);
#pragma unroll
        for (int q = 0; q < 2; ++q)
            // the +y bond of the row, except the periodic one of the last row
            up[k][q] = (live && q < WR && r < R - 1) ? By[r * WR + q] : 0u;
    }
    // the periodic y bond (row R - 1 to row 0), on every lane
    uint32_t wb[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const uint32_t own = (2 * (int)lane + ka == R - 1 && q < WR) ? By[(R - 1) * WR + q] : 0u;
        wb[q] = __shfl_sync(0xffffffffu, own, ra);
    }
    // The bonds do not change during the fill: the bond from the lane below
    // into each lane's row 0 (pin) and the propagate masks of every step of
    // the lane scans (upwards: into row 0, on through the lane's inner bond;
    // downwards: into row 1 through b1n, on through the inner bond) are
    // computed once, so that a scan step is one shuffle and one logic op.
    uint32_t pin[2], Pu[2][5], Pd[2][5];
#pragma unroll
    for (int q = 0; q < WR; ++q) {
        pin[q] = __shfl_up_sync(0xffffffffu, up[1][q], 1);
        if (lane == 0) pin[q] = 0u;
        uint32_t P = pin[q] & up[0][q];
#pragma unroll
        for (int s = 0, o = 1; s < 5; ++s, o <<= 1) {
            Pu[q][s] = P;
            const uint32_t Po = __shfl_up_sync(0xffffffffu, P, o);
            if ((int)lane >= o) P &= Po;
        }
        P = up[1][q] & up[0][q];
#pragma unroll
        for (int s = 0, o = 1; s < 5; ++s, o <<= 1) {
            Pd[q][s] = P;
            const uint32_t Po = __shfl_down_sync(0xffffffffu, P, o);
            if ((int)lane + o < 32) P &= Po;
        }
    }
    for (;;) {
        uint32_t moved = 0u;
        T Y[2] = {0, 0};
#pragma unroll
        for (int q = 0; q < WR; ++q) {
            const uint32_t g0 = (uint32_t)(G[0] >> (32 * q)), g1 = (uint32_t)(G[1] >> (32 * q));
            const uint32_t b01 = up[0][q], b1n = up[1][q];
            // within the lane first
            const uint32_t x0 = g0 | (g1 & b01), x1 = g1 | (g0 & b01);
            // upwards from each lane block's top row, downwards from its bottom row
            uint32_t Xu = x1, Xd = x0;
#pragma unroll
            for (int s = 0, o = 1; s < 5; ++s, o <<= 1) {
                const uint32_t Uo = __shfl_up_sync(0xffffffffu, Xu, o), Do = __shfl_down_sync(0xffffffffu, Xd, o);
                if ((int)lane >= o) Xu |= Pu[q][s] & Uo;
                if ((int)lane + o < 32) Xd |= Pd[q][s] & Do;
            }
            uint32_t below = __shfl_up_sync(0xffffffffu, Xu, 1), above = __shfl_down_sync(0xffffffffu, Xd, 1);
            if (lane == 0) below = 0u;
            if (lane == 31) above = 0u;
            const uint32_t n0 = x0 | (below & pin[q]), n1 = x1 | (above & b1n);
            uint32_t y0 = n0 | (n1 & b01), y1 = n1 | (n0 & b01);
            // the periodic bond between row R - 1 and row 0
            const uint32_t last = __shfl_sync(0xffffffffu, ka ? y1 : y0, ra), first = __shfl_sync(0xffffffffu, y0, 0);
            if (lane == 0) y0 |= last & wb[q];
            if ((int)lane == ra) {
                if (ka) y1 |= first & wb[q];
                else y0 |= first & wb[q];
            }
            moved |= (y0 ^ g0) | (y1 ^ g1);
            Y[0] |= (T)y0 << (32 * q);
            Y[1] |= (T)y1 << (32 * q);
        }
        // along x: each row as a line, then through its periodic bond
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            T X = row_close(Y[k], Aup[k], Adn[k]);
            if (wrap[k] && (X & ends)) X |= ends;
            X = row_close(X, Aup[k], Adn[k]);
            moved |= fold32(X ^ Y[k]);
            G[k] = X;
        }
        if (!__any_sync(0xffffffffu, moved != 0u)) break;
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int r = 2 * (int)lane + k;
#pragma unroll
        for (int q = 0; q < WR; ++q)
            if (r < R) F[r * WR + q] = (uint32_t)(G[k] >> (32 * q));
    }
}

// The seed's component of the activated bonds as the bit plane F, by flood
// fill (every thread of the CTA calls it).  Planes of NW = rows x WR words:
// C candidates (sites in the seed's old state), Bx the +x bond of each site
// (periodic; bit len-1 of a row is the bond to its site 0), Bd + (d-1) NW the
// +d bond of each site for d = 1 .. dim-1; a bond is set when both ends are
// candidates and its keyed draw activates it (wolff_int8_active, the other
// paths' rule).  The fill repeats, until no word changes: every row takes the
// flood of its neighbouring rows through their bonds (every dimension >= 1);
// then each warp, whose lanes hold consecutive rows, alternates spreading
// the flood along dimension 1 over its lanes (prefix scans over the lanes,
// down and up) with closing it along each row's x-line (prefix scans over the
// bits of the row's words, forward and backward, with the periodic carry)
// until neither adds a site.  Every step only adds sites joined to the flood
// by an active bond, and the fill stops when the flood is closed: F is the
// component.
__device__ void resident_cluster_bits(const StencilDev& lst, const WolffDev& w, const int8_t* s, int val,
                                      uint32_t rsite, uint32_t serial, uint32_t tgb, Key key, uint32_t* C,
                                      uint32_t* F, uint32_t* Bx, uint32_t* Bd)
{
    const int len = lst.len, WR = res_row_words(len), D = lst.dim;
    const uint32_t R = (uint32_t)(lst.n / len), NW = R * (uint32_t)WR;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // row of word wi: a shift when the words per row are a power of two
    const int wsh = (WR & (WR - 1)) == 0 ? __ffs(WR) - 1 : -1;
    auto row_of_word = [&](uint32_t wi) { return wsh >= 0 ? wi >> wsh : wi / (uint32_t)WR; };
    // Candidates, the flood cleared; then the active bonds.  A warp takes
    // kResBatch words at a time and computes all of them before it stores
    // any (a store to a plane would order the next word's loads behind it),
    // so its loads and its bond draws run side by side.
    for (uint32_t w0 = warp; w0 < NW; w0 += kResBatch * kResWarps) {
        uint32_t cb[kResBatch];
#pragma unroll
        for (int k = 0; k < kResBatch; ++k) {
            const uint32_t wi = w0 + (uint32_t)(k * kResWarps);
            const uint32_t r = row_of_word(wi);
            const int x = (int)(wi - r * (uint32_t)WR) * 32 + lane;
            const bool c = wi < NW && x < len && s[(int64_t)r * len + x] == val;
            cb[k] = __ballot_sync(0xffffffffu, c);
        }
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < kResBatch; ++k) {
                const uint32_t wi = w0 + (uint32_t)(k * kResWarps);
                if (wi < NW) {
                    C[wi] = cb[k];
                    F[wi] = 0u;
                }
            }
    }
    __syncthreads();
    // a bond is tested when both ends are candidates; its draw is made on
    // every lane (the lanes of a warp issue it once either way), so the
    // draws of a batch form straight-line code
    for (uint32_t w0 = warp; w0 < NW; w0 += kResBatch * kResWarps) {
        uint32_t ax[kResBatch], ad[2][kResBatch];
#pragma unroll
        for (int k = 0; k < kResBatch; ++k) {
            const uint32_t wi = w0 + (uint32_t)(k * kResWarps);
            const bool inw = wi < NW;  // uniform over the warp
            const uint32_t r = row_of_word(wi);
            const int wx = (int)(wi - r * (uint32_t)WR);
            const int x = wx * 32 + lane;  // C bits of x >= len are clear
            const bool ci = inw && ((C[inw ? wi : 0] >> lane) & 1u) != 0;
            const uint32_t i = r * (uint32_t)len + (uint32_t)x;
            const int xj = x + 1 == len ? 0 : x + 1;
            const bool cx = ci && ((C[r * WR + (xj >> 5)] >> (xj & 31)) & 1u);
            const bool dx = wolff_int8_active(w, i, r * (uint32_t)len + (uint32_t)xj, serial, tgb, key);
            ax[k] = __ballot_sync(0xffffffffu, cx & dx);
#pragma unroll
            for (int d = 1; d < 3; ++d) {
                ad[d - 1][k] = 0u;
                if (d < D) {
                    const uint32_t rp = res_row_step(lst, inw ? r : 0u, d, +1);
                    const bool cj = ci && ((C[rp * WR + wx] >> lane) & 1u);
                    const bool dj = wolff_int8_active(w, i, rp * (uint32_t)len + (uint32_t)x, serial, tgb, key);
                    ad[d - 1][k] = __ballot_sync(0xffffffffu, cj & dj);
                }
            }
        }
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < kResBatch; ++k) {
                const uint32_t wi = w0 + (uint32_t)(k * kResWarps);
                if (wi < NW) {
                    Bx[wi] = ax[k];
                    if (D > 1) Bd[wi] = ad[0][k];
                    if (D > 2) Bd[(size_t)NW + wi] = ad[1][k];
                }
            }
    }
    if (tid == 0) {
        const uint32_t rr = res_row_of(lst, rsite), xx = rsite - rr * (uint32_t)len;
        F[rr * WR + (xx >> 5)] = 1u << (xx & 31);
    }
    __syncthreads();
    if (D == 2 && R <= 64 && WR <= 2) {  // one warp holds the whole lattice
        if (warp == 0) {
            if (WR == 1) resident_fill_warp2<1>(F, Bx, Bd, (int)R, len);
            else resident_fill_warp2<2>(F, Bx, Bd, (int)R, len);
        }
        __syncthreads();
        return;
    }
    const int lb = (len - 1) & 31, lw = WR - 1;
    const uint32_t rounds = (R + kResThreads - 1) / kResThreads;
    for (uint32_t it = 0; it <= NW * 32u; ++it) {  // each pass adds a site or ends the fill
        int changed = 0;
        for (uint32_t k = 0; k < rounds; ++k) {
            if (k * kResThreads + (uint32_t)warp * 32u >= R) break;  // this warp holds no rows (uniform)
            const uint32_t r = k * kResThreads + (uint32_t)tid;  // a warp's lanes: consecutive rows
            const bool live = r < R;
            uint32_t G[8], old[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) old[q] = G[q] = (live && q < WR) ? F[r * WR + q] : 0u;
            int y = 0;
            if (live) {
                y = lst.coord((int64_t)r * len, 1);
                for (int d = 1; d < D; ++d) {
                    const uint32_t rp = res_row_step(lst, r, d, +1), rm = res_row_step(lst, r, d, -1);
                    const uint32_t* B = Bd + (size_t)(d - 1) * NW;
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        if (q < WR) G[q] |= (F[rp * WR + q] & B[r * WR + q]) | (F[rm * WR + q] & B[rm * WR + q]);
                }
            }
            // Warp-local fixpoint: alternate the spread along dimension 1
            // over the warp's lanes (rows r - 1, r + 1 when they are this
            // row's neighbours without the periodic wrap) with the closure
            // along each row's x-line, until no lane changes; the other
            // warps' rows and the periodic wraps come in through the
            // neighbour rows at the next pass.
            const bool hasprev = live && y != 0, hasnext = live && y != len - 1;
            uint32_t bx[8], pb[8], qb[8], wrap = 0u;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                bx[q] = (live && q < WR) ? Bx[r * WR + q] : 0u;
                pb[q] = (hasprev && q < WR) ? Bd[(r - 1) * WR + q] : 0u;
                qb[q] = (hasnext && q < WR) ? Bd[r * WR + q] : 0u;
                if (q == lw) {  // constant indices only: the arrays stay in registers
                    wrap = (bx[q] >> lb) & 1u;
                    bx[q] &= ~(1u << lb);
                }
            }
            for (;;) {
                uint32_t moved = 0u;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (q >= WR) break;
                    uint32_t X = G[q], P = pb[q], Q = qb[q];
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t Xo = __shfl_up_sync(0xffffffffu, X, o), Po = __shfl_up_sync(0xffffffffu, P, o);
                        if (lane >= o) {
                            X |= P & Xo;
                            P &= Po;
                        }
                    }
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t Xo = __shfl_down_sync(0xffffffffu, X, o), Qo = __shfl_down_sync(0xffffffffu, Q, o);
                        if (lane + o < 32) {
                            X |= Q & Xo;
                            Q &= Qo;
                        }
                    }
                    moved |= X ^ G[q];
                    G[q] = X;
                }
                // along the row's x-line (the periodic bond, bit lb of the
                // last word, carried explicitly)
                uint32_t glast = 0u;
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (q == lw) glast = G[q];
                uint32_t cin = (glast >> lb) & wrap;  // site len-1 -> site 0
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (q >= WR) break;
                    uint32_t X = G[q] | cin, p = bx[q] << 1;
                    X |= (X << 1) & p;
                    p &= p << 1;
                    X |= (X << 2) & p;
                    p &= p << 2;
                    X |= (X << 4) & p;
                    p &= p << 4;
                    X |= (X << 8) & p;
                    p &= p << 8;
                    X |= (X << 16) & p;
                    moved |= X ^ G[q];
                    G[q] = X;
                    cin = (X >> 31) & (bx[q] >> 31);
                }
                cin = G[0] & 1u & wrap;  // site 0 -> site len-1
#pragma unroll
                for (int q = 7; q >= 0; --q) {
                    if (q > lw) continue;
                    uint32_t X = G[q] | (cin << (q == lw ? lb : 31)), p = bx[q];
                    X |= (X >> 1) & p;
                    p &= p >> 1;
                    X |= (X >> 2) & p;
                    p &= p >> 2;
                    X |= (X >> 4) & p;
                    p &= p >> 4;
                    X |= (X >> 8) & p;
                    p &= p >> 8;
                    X |= (X >> 16) & p;
                    moved |= X ^ G[q];
                    G[q] = X;
                    cin = q > 0 ? (X & 1u) & (bx[q - 1] >> 31) : 0u;
                }
                if (!__any_sync(0xffffffffu, moved != 0u)) break;
            }
            if (live) {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (q < WR && G[q] != old[q]) {
                        F[r * WR + q] = G[q];
                        changed = 1;
                    }
            }
        }
        if (!__syncthreads_or(changed)) break;
    }
}

__device__ void resident_run(const ResidentRun& R, unsigned char* smem)
{
    __shared__ int s_rsite, s_val, s_newq, s_root, s_size;
    const int64_t n = R.st.n;
    const int64_t words = (n + 31) / 32;
    uint4* tab = reinterpret_cast<uint4*>(smem) + (threadIdx.x >> 5) * kAccTab;
    // the cluster's work area (bit planes, or union-find parents and
    // candidate bits on one-dimensional chains), then the state
    const bool bits_mode = res_bits_ok(R.st.dim, R.st.len);
    const size_t work = bits_mode ? res_bits_bytes(n, R.st.dim, R.st.len) : res_uf_bytes(n);
    unsigned char* wk = smem + (size_t)kResWarps * kAccTab * 16;
    volatile unsigned short* par = reinterpret_cast<unsigned short*>(wk);
    uint32_t* cand = reinterpret_cast<uint32_t*>(wk + (size_t)((2 * n + 15) & ~15ll));
    const uint32_t NW = (uint32_t)(n / R.st.len) * (uint32_t)res_row_words(R.st.len);
    uint32_t* bC = reinterpret_cast<uint32_t*>(wk);
    uint32_t* bF = bC + NW;
    uint32_t* bX = bF + NW;
    uint32_t* bD = bX + NW;
    int8_t* s = reinterpret_cast<int8_t*>(wk + ((work + 15) & ~(size_t)15));
    StencilDev lst = R.st;
    lst.split = 0;  // site order in shared memory
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int64_t i = tid; i < n; i += kResThreads) s[i] = R.state[R.st.addr(i)];
    __syncthreads();
    const uint32_t tgs = tag(kWolffSeed, R.replica), tgb = tag(kWolffBond, R.replica);
    for (int e = 0; e < R.n_emcs; ++e) {
        for (int c = 0; c < R.ncluster; ++c) {
            const uint32_t serial = R.cluster0 + (uint32_t)(e * R.ncluster + c);
            if (tid == 0) {
                int val, newq;
                s_rsite = (int)wolff_int8_seed(R.w, lst, s, R.key, serial, tgs, val, newq);
                s_val = val;
                s_newq = newq;
                s_size = 0;
            }
            __syncthreads();
            const int val = s_val;
            if (bits_mode) {
                resident_cluster_bits(lst, R.w, s, val, (uint32_t)s_rsite, serial, tgb, R.key, bC, bF, bX, bD);
                // flip the component and count it
                const int8_t nv = (int8_t)s_newq;
                const int len = lst.len, WR = res_row_words(len);
                int cnt = 0;
                for (uint32_t w0 = warp; w0 < NW; w0 += kResBatch * kResWarps) {
                    uint32_t fb[kResBatch];
#pragma unroll
                    for (int k = 0; k < kResBatch; ++k) {
                        const uint32_t wi = w0 + (uint32_t)(k * kResWarps);
                        fb[k] = wi < NW ? bF[wi] : 0u;
                    }
#pragma unroll
                    for (int k = 0; k < kResBatch; ++k) {
                        const uint32_t b = fb[k];
                        if (b) {
                            const uint32_t wi = w0 + (uint32_t)(k * kResWarps);
                            const uint32_t r = wi / (uint32_t)WR;
                            const int x = (int)(wi - r * (uint32_t)WR) * 32 + lane;
                            if ((b >> lane) & 1u) s[(int64_t)r * len + x] = nv;
                            if (lane == 0) cnt += __popc(b);
                        }
                    }
                }
                if (lane == 0 && cnt) atomicAdd(&s_size, cnt);
                __syncthreads();
                if (tid == 0) R.csize[e * R.csize_e + c * R.csize_c] = s_size;
                continue;
            }
            // candidates: sites in the seed's old state, each its own root
            for (int64_t wd = warp; wd < words; wd += kResWarps) {
                const int64_t i = wd * 32 + lane;
                const bool c = i < n && s[i] == val;
                const uint32_t bits = __ballot_sync(0xffffffffu, c);
                if (c) par[i] = (unsigned short)i;
                if (lane == 0) cand[wd] = bits;
            }
            __syncthreads();
            for (int64_t i = tid; i < n; i += kResThreads) {
                if (!((cand[i >> 5] >> (i & 31)) & 1u)) continue;
                for (int d = 0; d < lst.dim; ++d) {
                    const int64_t j = lst.nbr(i, 2 * d);
                    if (((cand[j >> 5] >> (j & 31)) & 1u) &&
                        wolff_int8_active(R.w, (uint32_t)i, (uint32_t)j, serial, tgb, R.key))
                        runite(par, (int)i, (int)j);
                }
            }
            __syncthreads();
            // Hooks made side by side chain up (a warp hooks 32 consecutive
            // sites one under the next), so the trees can be as deep as a
            // row.  Every candidate's path is halved once, all at the same
            // time (a write only ever points a site to an ancestor, so the
            // forest stays valid while other walks read it); the walks after
            // this are short.
            for (int64_t i = tid; i < n; i += kResThreads)
                if ((cand[i >> 5] >> (i & 31)) & 1u) rfind(par, (int)i);
            __syncthreads();
            if (tid == 0) s_root = rfind(par, s_rsite);
            __syncthreads();
            const int root = s_root;
            const int8_t nv = (int8_t)s_newq;
            int cnt = 0;
            for (int64_t i = tid; i < n; i += kResThreads) {
                if (!((cand[i >> 5] >> (i & 31)) & 1u)) continue;
                int x = (int)i, px;
                while ((px = par[x]) != x) x = px;  // read-only walks
                if (x == root) {
                    s[i] = nv;
                    ++cnt;
                }
            }
            cnt = __reduce_add_sync(0xffffffffu, cnt);
            if (lane == 0 && cnt) atomicAdd(&s_size, cnt);
            __syncthreads();
            if (tid == 0) R.csize[e * R.csize_e + c * R.csize_c] = s_size;
        }
        for (int j = 0; j < R.nmetro; ++j) {
            const uint32_t sweep = R.sweep0 + (uint32_t)(e * R.nmetro + j);
            const int64_t half = n / 2, bs = 32 * (int64_t)R.runs, nblk = (half + bs - 1) / bs;
            for (int colour = 0; colour < 2; ++colour) {
                for (int64_t b = warp; b < nblk; b += kResWarps) {
                    const uint32_t run0 = (uint32_t)(b * R.runs);
                    accept_tab_fill(tab, run0, R.key, sweep, R.replica, (uint32_t)R.runs);
                    for (int k = 0; k < R.runs; ++k) {
                        const int64_t t = b * bs + k * 32 + lane;
                        const bool live = t < half;
                        with_dim(lst, [&](const auto& lt) {
                            int8_site(R.m, lt, s, live ? parity_site(lt, t, colour) : 0, R.key, sweep, R.replica,
                                      R.cuts, R.D, live, colour, tab, run0);
                        });
                    }
                }
                __syncthreads();
            }
        }
        if (R.acc) with_dim(lst, [&](const auto& lt) { measure_int8_part(R.m, lt, s, R.acc + e * R.acc_e, 0, 1); });
        __syncthreads();
    }
    for (int64_t i = tid; i < n; i += kResThreads) R.state[R.st.addr(i)] = s[i];
}

// acceptance blocks of `runs` 64-site runs: enough blocks per colour for every warp
__host__ __device__ inline int resident_runs(int64_t n)
{
    int runs = 1;
    while (runs < kAccRuns && (n / 2) / (32 * (int64_t)runs * 2) >= kResWarps) runs *= 2;
    return runs;
}

__global__ void __launch_bounds__(kResThreads, 1) emcs_resident(ResidentRun R)
{
    extern __shared__ __align__(16) unsigned char smem[];
    resident_run(R, smem);
}

// One CTA per member of `order` (the batch's resident members, largest
// first): EMCS e0 .. e0 + count - 1 of the run, measurement slots slot0 ..
__global__ void __launch_bounds__(kResThreads, 1)
    batch_resident(const BatchRep* __restrict__ reps, const int32_t* __restrict__ order, int nrep, uint32_t e0,
                   int slot0, int count, int ncluster, int nmetro, long long* __restrict__ acc,
                   int32_t* __restrict__ csize)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int r = order[blockIdx.x];
    const BatchRep& B = reps[r];
    ResidentRun R;
    R.m = B.md;
    R.st = B.st;
    R.w = B.w;
    R.key = B.key;
    R.replica = B.replica;
    R.sweep0 = B.sweep0 + e0 * (uint32_t)nmetro;
    R.cluster0 = B.cluster0 + e0 * (uint32_t)ncluster;
    R.n_emcs = count;
    R.ncluster = ncluster;
    R.nmetro = nmetro;
    R.D = B.D;
    R.runs = resident_runs(B.st.n);
    R.cuts = B.cuts;
    R.state = (int8_t*)B.s;
    R.acc = acc + ((size_t)slot0 * nrep + r) * kAccStride;
    R.acc_e = (int64_t)nrep * kAccStride;
    R.csize = csize + (size_t)slot0 * ncluster * nrep + r;
    R.csize_e = (int64_t)ncluster * nrep;
    R.csize_c = nrep;
    resident_run(R, smem);
}

// Lattices this path takes: int8 models on hypercubic stencils of at most
// kResidentMaxSites sites.
bool resident_fits(const Sim* s)
{
    return !s->is_f32 && s->lat_kind == MQV_LATTICE_HYPERCUBIC && s->n <= kResidentMaxSites && s->n >= 2;
}

static cudaError_t resident_attr(int device)
{
    static std::atomic<bool> done[64] = {};  // host threads share it
    if (device >= 0 && device < 64 && done[device]) return cudaSuccess;
    const int bytes = (int)resident_smem_max();
    cudaError_t e = cudaFuncSetAttribute(emcs_resident, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(batch_resident, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && device >= 0 && device < 64) done[device] = true;
    return e;
}

// n_emcs EMCS (clusters, sweeps, the measurement into acc slots 0 ..
// n_emcs - 1 when acc is given, cluster sizes into csize) in one launch;
// advances the counters.
cudaError_t launch_emcs_resident(Sim* s, int n_emcs, int ncluster, int nmetro, bool measure, long long* acc,
                                 int32_t* csize)
{
    cudaError_t e = resident_attr(s->device);
    if (e != cudaSuccess) return e;
    ResidentRun R{};
    R.m = s->md;
    R.st = s->sten;
    if (ncluster > 0) R.w = wolff_int8_params(s->md);
    R.key = make_key(s->seed);
    R.replica = s->replica;
    R.sweep0 = (uint32_t)s->sweep;
    R.cluster0 = (uint32_t)s->cluster;
    R.n_emcs = n_emcs;
    R.ncluster = ncluster;
    R.nmetro = nmetro;
    R.D = s->max_degree;
    R.runs = resident_runs(s->n);
    R.cuts = s->d_cuts;
    R.state = (int8_t*)s->state[s->cur];
    R.acc = measure ? acc : nullptr;
    R.acc_e = kAccStride;
    R.csize = csize;
    R.csize_e = ncluster;
    R.csize_c = 1;
    emcs_resident<<<1, kResThreads, resident_smem_for(s->sten), s->stream>>>(R);
    s->launches++;
    s->sweep += (uint64_t)n_emcs * (uint64_t)nmetro;
    s->cluster += (uint64_t)n_emcs * (uint64_t)ncluster;
    return cudaGetLastError();
}

// The batch's resident members (order: member ids, largest first; nres of
// them, smem: the largest shared-memory layout among them), EMCS e0 .. e0 + count - 1.
cudaError_t batch_launch_resident(const BatchLaunch& b, cudaStream_t st, const int32_t* order, int nres, size_t smem,
                                  uint32_t e0, int slot0, int count, int ncluster, int nmetro, int device)
{
    if (nres <= 0 || count <= 0) return cudaSuccess;
    cudaError_t e = resident_attr(device);
    if (e != cudaSuccess) return e;
    batch_resident<<<nres, kResThreads, smem, st>>>(b.reps, order, b.nrep, e0, slot0, count,
                                                                          ncluster, nmetro, b.acc, b.csize);
    return cudaGetLastError();
}

}  // namespace mqv
