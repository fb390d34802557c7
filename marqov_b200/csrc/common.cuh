// Shared device/host pieces of the MARQOV update engine for sm_100a.
//
// * Philox4x32-10 counter-based generator keyed by (seed, replica) and counted
//   by (site, sweep, block, stream): the random word a site update consumes
//   does not depend on which thread or tile performs it.
// * The reference acceptance rule update_accepted<pref>
//   (src/libmarqov/metropolishelpers.h:109-142) in FP64 with every operation
//   rounded separately (no contraction), so host and device agree bit for bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define MQV_HD __host__ __device__ __forceinline__

namespace mqv {

// Stream tags, counter word 3 bits 24..31 (replica id in bits 0..23).
enum Stream : uint32_t { kMetro = 1, kInit = 2, kWolffSeed = 3, kWolffBond = 4, kAccept = 5, kAcceptFine = 6, kTemper = 7 };

struct Key {
    uint32_t k0, k1;
};

MQV_HD Key make_key(uint64_t seed) { return Key{(uint32_t)seed, (uint32_t)(seed >> 32)}; }

MQV_HD uint32_t tag(uint32_t stream, uint32_t replica) { return (stream << 24) | (replica & 0xFFFFFFu); }

// 32 x 32 -> 64-bit product (one wide multiply-add on the GPU)
MQV_HD void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo)
{
    const uint64_t p = (uint64_t)a * b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

// Philox4x32-10 (Salmon et al., SC'11): 10 rounds, multipliers 0xD2511F53 /
// 0xCD9E8D57, Weyl key increments 0x9E3779B9 / 0xBB67AE85.
MQV_HD uint4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, Key k)
{
    uint32_t k0 = k.k0, k1 = k.k1;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(0xD2511F53u, c0, hi0, lo0);
        mulhilo(0xCD9E8D57u, c2, hi1, lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    return make_uint4(c0, c1, c2, c3);
}

MQV_HD uint64_t lo64(uint4 v) { return (uint64_t)v.x | ((uint64_t)v.y << 32); }
MQV_HD uint64_t hi64(uint4 v) { return (uint64_t)v.z | ((uint64_t)v.w << 32); }

// The Metropolis acceptance word of a site.  Top byte, bit-sliced: sites are
// grouped by G(i) = ((i >> 6) << 1) | (i & 1) (32 sites of equal parity in an
// aligned run of 64); bit b of the byte is bit ((i >> 1) & 31) of plane b,
// planes 0..3 = Philox(G, sweep, 0, ACCEPT), planes 4..7 = Philox(G, sweep, 1,
// ACCEPT).  Low 56 bits: low 56 bits of half (i & 1) of Philox(i >> 1, sweep,
// 0, ACCEPT_FINE).  A threshold test on real() is decided by the top byte
// except on a tie with the threshold's top byte (probability 1/256), so
// kernels draw two Philox blocks per 32 sites and the fine block rarely.
MQV_HD uint32_t accept_group(uint32_t site) { return ((site >> 6) << 1) | (site & 1u); }
MQV_HD uint64_t accept_fine56(Key key, uint32_t site, uint32_t sweep, uint32_t replica)
{
    const uint4 f = philox(site >> 1, sweep, 0u, (kAcceptFine << 24) | (replica & 0xFFFFFFu), key);
    return ((site & 1u) ? hi64(f) : lo64(f)) & 0x00FFFFFFFFFFFFFFull;
}
MQV_HD uint32_t accept_top8(Key key, uint32_t site, uint32_t sweep, uint32_t replica)
{
    const uint32_t g = accept_group(site), q = (site >> 1) & 31u;
    const uint32_t c3 = (kAccept << 24) | (replica & 0xFFFFFFu);
    const uint4 a = philox(g, sweep, 0u, c3, key);
    const uint4 b = philox(g, sweep, 1u, c3, key);
    return ((a.x >> q) & 1u) | (((a.y >> q) & 1u) << 1) | (((a.z >> q) & 1u) << 2) | (((a.w >> q) & 1u) << 3) |
           (((b.x >> q) & 1u) << 4) | (((b.y >> q) & 1u) << 5) | (((b.z >> q) & 1u) << 6) | (((b.w >> q) & 1u) << 7);
}
MQV_HD uint64_t accept_word(Key key, uint32_t site, uint32_t sweep, uint32_t replica)
{
    return ((uint64_t)accept_top8(key, site, sweep, replica) << 56) | accept_fine56(key, site, sweep, replica);
}
// u53 < cut on the site's acceptance word given its top byte: the fine half
// is drawn only when the top byte ties the cut's
MQV_HD bool accept_with_top(uint64_t cut, uint32_t top, Key key, uint32_t site, uint32_t sweep, uint32_t replica)
{
    if (cut >= (1ull << 53)) return true;
    if (cut == 0) return false;
    const uint32_t t8 = (uint32_t)(cut >> 45);
    if (top != t8) return top < t8;
    return (((uint64_t)top << 45) | (accept_fine56(key, site, sweep, replica) >> 11)) < cut;
}
// u53 < cut on the site's acceptance word (cut = accept_cut of the move's dE)
MQV_HD bool accept_below(uint64_t cut, Key key, uint32_t site, uint32_t sweep, uint32_t replica)
{
    if (cut >= (1ull << 53) || cut == 0) return cut != 0;
    return accept_with_top(cut, accept_top8(key, site, sweep, replica), key, site, sweep, replica);
}

// u53 < cut given the site's top byte, for per-site kernels that share the
// ACCEPT blocks (accept_tab_fill): dE <= 0 cuts accept without a draw.
MQV_HD bool accept_top_or_fine(uint64_t cut, uint32_t top, Key key, uint32_t site, uint32_t sweep, uint32_t replica)
{
    if (cut >= (1ull << 53) || cut == 0) return cut != 0;
    return accept_with_top(cut, top, key, site, sweep, replica);
}

#ifdef __CUDACC__
// Warp-shared acceptance bytes.  A warp that updates sites of an aligned
// block of kAccRuns 64-site runs (sites [64 run0, 64 (run0 + kAccRuns)))
// draws the two ACCEPT blocks of each of the block's 2 kAccRuns groups once,
// one per lane -- lane L draws half (L & 1) of parity (L >> 1) & 1 of run
// run0 + (L >> 2) into `tab` (kAccTab uint4 of warp-private shared memory) --
// and every site of the block then reads its eight planes from there: one
// Philox block per lane per 512 sites instead of two per site.  Same bits as
// accept_top8.
constexpr int kAccRuns = 8;
constexpr int kAccTab = 4 * kAccRuns;  // uint4 per warp: [run][parity][half]
constexpr int kAccSites = 32 * kAccRuns;  // sites of one colour in a block (checkerboard)
// (nruns < kAccRuns: a block of nruns runs, drawn by the first 4 nruns lanes.)
__device__ __forceinline__ void accept_tab_fill(uint4* tab, uint32_t run0, Key key, uint32_t sweep, uint32_t replica,
                                                uint32_t nruns = kAccRuns)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t c3 = (kAccept << 24) | (replica & 0xFFFFFFu);
    __syncwarp();  // the previous block's readers are done
    if (lane < 4u * nruns)
        tab[lane] = philox(((run0 + (lane >> 2)) << 1) | ((lane >> 1) & 1u), sweep, lane & 1u, c3, key);
    __syncwarp();
}
__device__ __forceinline__ uint32_t accept_top8_tab(const uint4* tab, uint32_t run0, uint32_t site)
{
    const uint32_t k = (site >> 6) - run0, p = site & 1u, q = (site >> 1) & 31u;
    const uint4 a = tab[(k * 2 + p) * 2], b = tab[(k * 2 + p) * 2 + 1];
    return ((a.x >> q) & 1u) | (((a.y >> q) & 1u) << 1) | (((a.z >> q) & 1u) << 2) | (((a.w >> q) & 1u) << 3) |
           (((b.x >> q) & 1u) << 4) | (((b.y >> q) & 1u) << 5) | (((b.z >> q) & 1u) << 6) | (((b.w >> q) & 1u) << 7);
}
#endif

// x % q for the small ranges of state draws (q <= 65535): constant divisors
// for the common q, else three 32-bit remainders of x = hi 2^32 + lo.
MQV_HD uint32_t mod_small(uint64_t x, uint32_t q)
{
    switch (q) {
        case 2: return (uint32_t)(x % 2ull);
        case 3: return (uint32_t)(x % 3ull);
        case 4: return (uint32_t)(x % 4ull);
        default: break;
    }
    const uint32_t p32 = (0xFFFFFFFFu % q + 1u) % q;  // 2^32 mod q
    return ((((uint32_t)(x >> 32)) % q) * p32 + ((uint32_t)x) % q) % q;
}

// real() of RNGCache: (word >> 11) * 2^-53 (src/libmarqov/rngcache.h:202-206).
MQV_HD double real01(uint64_t w) { return (double)(w >> 11) * 0x1.0p-53; }

// Sequential words of one (stream, c0, c1) substream: word k sits in block
// c2 = k/2, half k%2.  Blocks are computed on demand.
struct SubStream {
    Key key;
    uint32_t c0, c1, c3;
    uint32_t k;
    uint4 blk;
    MQV_HD SubStream(Key key_, uint32_t c0_, uint32_t c1_, uint32_t c3_)
        : key(key_), c0(c0_), c1(c1_), c3(c3_), k(0), blk(make_uint4(0, 0, 0, 0)) {}
    MQV_HD uint64_t next()
    {
        if ((k & 1u) == 0) blk = philox(c0, c1, k >> 1, c3, key);
        uint64_t w = (k & 1u) ? hi64(blk) : lo64(blk);
        ++k;
        return w;
    }
    MQV_HD double real() { return real01(next()); }
};

// ---- acceptance rule -------------------------------------------------------

#ifdef __CUDA_ARCH__
#define MQV_DMUL(a, b) __dmul_rn((a), (b))
#define MQV_DADD(a, b) __dadd_rn((a), (b))
#define MQV_DSUB(a, b) __dsub_rn((a), (b))
#else
#define MQV_DMUL(a, b) ((a) * (b))
#define MQV_DADD(a, b) ((a) + (b))
#define MQV_DSUB(a, b) ((a) - (b))
#endif

// 2^x on [-1, 0]: the reference's sixth-order polynomial, Horner order
// (src/libmarqov/metropolishelpers.h:39-48).
MQV_HD double exp2app6(double x)
{
    double u = 1.0944614513161076e-4;
    u = MQV_DADD(MQV_DMUL(u, x), 1.2758920456516547e-3);
    u = MQV_DADD(MQV_DMUL(u, x), 9.5802562122641916e-3);
    u = MQV_DADD(MQV_DMUL(u, x), 5.5491137793956362e-2);
    u = MQV_DADD(MQV_DMUL(u, x), 2.4022437948159954e-1);
    u = MQV_DADD(MQV_DMUL(u, x), 6.9314704935511511e-1);
    return MQV_DADD(MQV_DMUL(u, x), 9.9999999867786389e-1);
}

// cvttsd2si: truncation toward zero, INT64_MIN for NaN / out of range
// (src/libmarqov/metropolishelpers.h:59-70).
MQV_HD int64_t trunc_i64(double f)
{
    if (!(f > -9223372036854775808.0 && f < 9223372036854775808.0)) return INT64_MIN;
    return (int64_t)f;
}

MQV_HD int64_t bits_of(double d)
{
#ifdef __CUDA_ARCH__
    return __double_as_longlong(d);
#else
    int64_t i;
    __builtin_memcpy(&i, &d, 8);
    return i;
#endif
}
MQV_HD double double_of(int64_t i)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double(i);
#else
    double d;
    __builtin_memcpy(&d, &i, 8);
    return d;
#endif
}

// update_accepted<pref>(dE, beta, rng) with the word the reference would
// draw: accept when dE <= 0; otherwise compare the binary exponent of
// u = real(word) with trunc(pref log2(e) (-beta dE)) and, on a tie, the
// mantissa in [0.5, 1) with exp2app6 of the fractional part.
MQV_HD bool update_accepted(int pref, double dE, double beta, uint64_t word)
{
    if (dE <= 0) return true;
    const double plog2e = (double)pref * 1.4426950408889634074;
    double rngnum = real01(word);
    double action = MQV_DMUL(-beta, dE);
    double action2 = MQV_DMUL(plog2e, action);
    int64_t i64 = bits_of(rngnum);
    int64_t t = trunc_i64(action2);
    int64_t e = (i64 >> 52) - 1022;
    if (e != t) return e < t;
    i64 = (i64 & ~(int64_t)0xFFF0000000000000LL) | 0x3FE0000000000000LL;
    double remainder = MQV_DSUB(action2, trunc(action2));
    return double_of(i64) < exp2app6(remainder);
}

// The cut of update_accepted<pref>(dE, beta, .) in closed form: the smallest
// u53 = word >> 11 it rejects (2^53: it accepts every word), so that the rule
// is u53 < cut.  With t = trunc(pref log2(e) (-beta dE)) and X the exp2app6
// of the fractional part: u = u53 2^-53 lies in binade e (u53 in
// [2^(52+e), 2^(53+e)); u53 = 0 has e = -1022); a smaller binade than t is
// accepted, binade t when its mantissa u53 / 2^(53+t) < X, that is
// u53 < X 2^(53+t) (a power-of-two scaling, exact).
MQV_HD uint64_t accept_cut_direct(int pref, double dE, double beta)
{
    if (dE <= 0) return 1ull << 53;
    const double plog2e = (double)pref * 1.4426950408889634074;
    const double action2 = MQV_DMUL(plog2e, MQV_DMUL(-beta, dE));
    const int64_t t = trunc_i64(action2);
    if (t > 0) return 1ull << 53;  // every binade of u is below t
    if (t < -1022) return 0;       // even u53 = 0 lies above t (also NaN)
    const double x = exp2app6(MQV_DSUB(action2, trunc(action2)));
    if (t == -1022) return 0.5 < x ? 1 : 0;  // only u53 = 0 ties; its mantissa reads 0.5
    if (t < -52) return 1;                    // only u53 = 0 lies below t
    const uint64_t lo = 1ull << (52 + t);
    const double p2 = double_of((int64_t)(1023 + 53 + t) << 52);  // 2^(53 + t), t in [-52, 0]
    const uint64_t c = (uint64_t)ceil(MQV_DMUL(x, p2));
    return c < lo ? lo : c;
}

// ---- Blackwell async copies (bulk copy engine) and mbarriers -----------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ uint64_t global_timer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// global -> shared bulk copy completing on an mbarrier (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
// shared -> global bulk copy in the issuing thread's bulk group
__device__ __forceinline__ void bulk_s2g(void* dst, uint32_t src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace mqv
