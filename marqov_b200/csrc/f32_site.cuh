// Device building blocks of the float models shared by the per-handle kernels
// (metropolis_f32.cu) and the batched kernels (batch.cu): proposals, the
// per-site Metropolis update, the embedded Wolff cluster, the observable
// accumulation and its finalisation.  Storage is FP32 in structure-of-arrays
// layout (component c of site i at s[c n + i]); proposals, onsite terms and
// acceptance are FP64, like the reference's double arithmetic
// (src/libmarqov/metropolishelpers.h:598-738).
#pragma once
#include "engine.h"

namespace mqv {

// set_to_rnddir for SymD = 3 (src/hamiltonian/util/randomdir.h:45-64): two
// reals -> (1 - a0, sqrt(a0 (2 - a0)) sin(pi a1), sqrt(a0 (2 - a0)) cos(pi a1)).
__device__ __forceinline__ void rnddir3(SubStream& rng, double v[3])
{
    const double a0 = 2.0 * rng.real(), a1 = 2.0 * rng.real();
    const double r1 = sqrt(a0 * (2.0 - a0));
    double sn, cs;
    sincospi(a1, &sn, &cs);
    v[0] = 1.0 - a0;
    v[1] = r1 * sn;
    v[2] = r1 * cs;
}

// Small-cap proposal: uniform on the cap cos(angle to old) >= cap, built in
// the frame that rotates +z onto the old spin (mirrored in z on the southern
// hemisphere), then normalised.
__device__ __forceinline__ void smallcap3(SubStream& rng, const float o[3], double cap, double v[3])
{
    const double u0 = rng.real(), u1 = rng.real();
    const double ca = 1.0 - u0 * (1.0 - cap);
    const double sa = sqrt(fmax(0.0, 1.0 - ca * ca));
    double sn, cs;
    sincospi(2.0 * u1, &sn, &cs);
    const double dx = sa * cs, dy = sa * sn, dz = ca;
    const double x = o[0], y = o[1], z = o[2];
    const double sg = z < 0 ? -1.0 : 1.0;
    const double a = 1.0 / (1.0 + sg * z);
    const double bxy = -x * y * a;
    const double e1[3] = {1.0 - x * x * a, bxy, -x * sg};
    const double e2[3] = {bxy, 1.0 - y * y * a, -y * sg};
    double nv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) nv[c] = dx * e1[c] + dy * e2[c] + dz * (double)o[c];
    const double nn = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = nv[c] / nn;
}

// Component c of site i of a float state: structure of arrays, s[c n + i]
// (n = the lattice's sites), so that the lanes of a warp, which update
// neighbouring sites of one colour, read each component in one coalesced run.
__device__ __forceinline__ float f32_get(const float* __restrict__ s, int64_t n, int c, int64_t i)
{
    return s[(int64_t)c * n + i];
}

// One Metropolis move (Metropolis<H,L>::move, src/libmarqov/metropolis.h:88-126)
// of a float model.  The neighbourhood sums are FP32 like the reference's
// float state vectors (nbrhoodloop, src/libmarqov/metropolishelpers.h:456-537:
// neighbourhood = neighbourhood + get(s_j) in the state's type), the
// interaction difference J dot(s_new - s_old, neighbourhood) takes FP32
// products summed in FP64 (svmath.h dot: inner_product with a double
// initial value), the onsite terms and the acceptance are FP64.  The
// decision is u53 < accept_cut_direct(1, dE, beta), which equals
// update_accepted<1> on the site's acceptance word; its top byte comes from
// the warp's shared table when `tab` is given (accept_tab_fill), else from
// the site's own two ACCEPT blocks.  `sub`: the site's sublattice
// (checkerboard colour) where the lattice has a termselector.  Lanes with
// live == false touch no memory.
template <class Lat>
__device__ __forceinline__ void f32_site(const ModelDev& m, const Lat& lat, float* __restrict__ s, int64_t i,
                                         Key key, uint32_t sweep, uint32_t replica, bool live, int sub = 0,
                                         const uint4* tab = nullptr, uint32_t run0 = 0)
{
    const int64_t n = lat.n;
    uint64_t cut = 0;
    float nf[3] = {0.f, 0.f, 0.f};
    if (live) {
        SubStream rng(key, (uint32_t)i, sweep, tag(kMetro, replica));
        const int deg = lat.degree(i);
        double dE;
        if (m.symd == 1) {
            // shift proposal old + amp * real(-1, 1) (Phi4_Initializer_Cartesian,
            // src/hamiltonian/Phi4.h:44-57); interaction + Onsite_Quadratic +
            // Onsite_Fourth_Minus_One (src/hamiltonian/Phi4.h:63-74,103-121)
            const double r = 1.0 + (-1.0 - 1.0) * real01(rng.next());
            const float of = s[i];
            const double old = of;
            nf[0] = (float)(old + m.cap * r);
            const double nw = nf[0];
            float sum = 0.f;
            for (int t = 0; t < deg; ++t) sum += s[lat.nbr(i, t)];
            const double o2 = old * old, n2 = nw * nw;
            dE = m.J * (double)((nf[0] - of) * sum) + onsite_w0(m, sub) * m.h * (n2 - o2) +
                 onsite_w1(m, sub) * m.h2 * ((n2 - 1.0) * (n2 - 1.0) - (o2 - 1.0) * (o2 - 1.0));
        } else {
            const float o[3] = {f32_get(s, n, 0, i), f32_get(s, n, 1, i), f32_get(s, n, 2, i)};
            double v[3];
            if (m.proposal == MQV_PROPOSAL_SMALL_CAP) smallcap3(rng, o, m.cap, v);
            else rnddir3(rng, v);  // SVInitializer for float vectors (initializers.h:74-80)
            nf[0] = (float)v[0];
            nf[1] = (float)v[1];
            nf[2] = (float)v[2];
            float nb[3] = {0.f, 0.f, 0.f};
            for (int t = 0; t < deg; ++t) {
                const int64_t j = lat.nbr(i, t);
                nb[0] += f32_get(s, n, 0, j);
                nb[1] += f32_get(s, n, 1, j);
                nb[2] += f32_get(s, n, 2, j);
            }
            // XXZAntiferro_interaction::get (src/hamiltonian/XXZAntiferro.h:135-150)
            // weights x and y by delta; Heisenberg's is the identity
            const double dxy = (double)((nf[0] - o[0]) * nb[0]) + (double)((nf[1] - o[1]) * nb[1]);
            const double dz = (double)((nf[2] - o[2]) * nb[2]);
            dE = m.J * (m.kind == MQV_MODEL_XXZ ? m.delta * dxy + dz : dxy + dz);
            if (m.kind == MQV_MODEL_XXZ) {
                // XXZAntiferro_extfield H s_z and XXZAntiferro_onsiteaniso D s_z^2
                // (XXZAntiferro.h:162-170, XXZAntiferroSingleAniso.h:31-44)
                const double zn = nf[2], zo = o[2];
                dE += onsite_w0(m, sub) * m.h * (zn - zo) + onsite_w1(m, sub) * m.h2 * (zn * zn - zo * zo);
            }
        }
        cut = accept_cut_direct(1, dE, m.beta);
    }
    bool acc;
    if (tab) {
        const uint32_t top = live ? accept_top8_tab(tab, run0, (uint32_t)i) : 0u;
        acc = live && accept_top_or_fine(cut, top, key, (uint32_t)i, sweep, replica);
    } else {
        acc = live && accept_below(cut, key, (uint32_t)i, sweep, replica);
    }
    if (acc) {
        s[i] = nf[0];
        if (m.symd != 1) {
            s[n + i] = nf[1];
            s[2 * n + i] = nf[2];
        }
    }
}

template <class ST>
__device__ __forceinline__ int64_t parity_site_f(const ST& st, int64_t t, int colour)
{
    const int64_t i0 = 2 * t;
    int par = 0;
    for (int j = 1; j < st.degree(0) / 2; ++j) par += st.coord(i0, j);
    return i0 + (((par & 1) != colour) ? 1 : 0);
}

// ---- measurement (FP64) ---------------------------------------------------------

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Part `part` of `nparts` of the accumulation (grid-stride share of a CTA;
// the CTA's totals go to acc with atomics).
template <class Lat>
__device__ __forceinline__ void measure_f32_part(const ModelDev& m, const Lat& lat, const float* __restrict__ s,
                                                 double* __restrict__ acc, int64_t part, int64_t nparts)
{
    __shared__ double red[6][32];
    double e = 0, mx = 0, my = 0, mz = 0, q2 = 0, q4 = 0;
    // InteractionEnergy applies the interaction's get() to both ends
    // (observables.h:186-217): XXZ weights x x' and y y' by delta^2
    const double wxy = m.kind == MQV_MODEL_XXZ ? m.delta * m.delta : 1.0;
    const bool xxz = m.kind == MQV_MODEL_XXZ;
    for (int64_t i = part * (int64_t)blockDim.x + threadIdx.x; i < lat.n; i += nparts * blockDim.x) {
        const int deg = lat.degree(i);
        if (m.symd == 1) {
            const double si = s[i];
            double nb = 0;
            for (int t = 0; t < deg; ++t) nb += (double)s[lat.nbr(i, t)];
            e += si * nb;
            mx += si;
            const double p2 = si * si;
            q2 += p2;
            q4 += (p2 - 1.0) * (p2 - 1.0);
        } else {
            const int64_t n = lat.n;
            const double a = f32_get(s, n, 0, i), b = f32_get(s, n, 1, i), c = f32_get(s, n, 2, i);
            double na = 0, nb = 0, nc = 0;
            for (int t = 0; t < deg; ++t) {
                const int64_t j = lat.nbr(i, t);
                na += (double)f32_get(s, n, 0, j);
                nb += (double)f32_get(s, n, 1, j);
                nc += (double)f32_get(s, n, 2, j);
            }
            e += wxy * (a * na + b * nb) + c * nc;
            mx += a;
            my += b;
            mz += c;
            if (xxz) {
                q2 += c * c;  // the single-ion term's sum of s_z^2
            } else {
                const double p2 = a * a + b * b + c * c;
                q2 += p2;
                q4 += (p2 - 1.0) * (p2 - 1.0);
            }
        }
    }
    double v[6] = {e, mx, my, mz, q2, q4};
    const int wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        v[k] = warp_sum_d(v[k]);
        if ((threadIdx.x & 31) == 0) red[k][wid] = v[k];
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double a = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) a += red[threadIdx.x][k];
        const int idx[6] = {kAccEne, kAccMag, kAccMagY, kAccMagZ, kAccSq, kAccQ4};
        atomicAdd(acc + idx[threadIdx.x], a);
    }
}

// Accumulators of one measurement -> (e, |m|, m^2, m^4).
__device__ __forceinline__ void finalize_f32_one(const ModelDev& m, int64_t n, const double* __restrict__ a,
                                                 double* __restrict__ o)
{
    const double mag = a[kAccMag] * a[kAccMag] + a[kAccMagY] * a[kAccMagY] + a[kAccMagZ] * a[kAccMagZ];
    const double mm = sqrt(mag) / (double)n;
    double e = m.J * a[kAccEne] / (double)(2 * n);
    // SelfEnergy: every onsite term over every site (observables.h:251-268)
    if (m.kind == MQV_MODEL_PHI4) e += (m.h * a[kAccSq] + m.h2 * a[kAccQ4]) / (double)n;
    if (m.kind == MQV_MODEL_XXZ) e += (m.h * a[kAccMagZ] + m.h2 * a[kAccSq]) / (double)n;
    const double m2 = mm * mm;
    o[0] = e;
    o[1] = mm;
    o[2] = m2;
    o[3] = m2 * m2;
}

// ---- embedded Wolff for float states ----------------------------------------------
// Generic Wolff (src/libmarqov/wolff.h:72-126) with Embedder<Heisenberg>
// (src/hamiltonian/Heisenberg.h:158-185: random unit r, reflection about the
// plane normal to r) or Embedder<Phi4> for one component
// (src/hamiltonian/Phi4.h:217-243: r = +-1, phi -> -phi).  A neighbour joins
// when cpl = J (-a_cur) a_nbr > 0 (a = s.r before any flip) and
// !update_accepted<2>(cpl) on the bond's keyed word.

// One cluster grown and reflected by the calling CTA (block size a multiple of
// 32); the visited bits of its members are cleared before return.
// The embedding arithmetic shared by the breadth-first and the labelling
// cluster kernels, rounded as written (no contraction), as the reference's
// double code: a = s . r, cpl = J (-a_i) a_j, and the reflection
// s -> (s - 2 (s.r) r) / |s - 2 (s.r) r|.
__device__ __forceinline__ double embed_proj(int symd, const float* __restrict__ s, int64_t n, int64_t i, float r0,
                                             float r1, float r2)
{
    if (symd == 3)
        return __dadd_rn(__dadd_rn(__dmul_rn((double)f32_get(s, n, 0, i), (double)r0),
                                   __dmul_rn((double)f32_get(s, n, 1, i), (double)r1)),
                         __dmul_rn((double)f32_get(s, n, 2, i), (double)r2));
    return __dmul_rn((double)s[i], (double)r0);
}
__device__ __forceinline__ double embed_cpl(double J, double ai, double aj) { return __dmul_rn(__dmul_rn(J, -ai), aj); }
__device__ __forceinline__ void embed_reflect(int symd, float* __restrict__ s, int64_t n, int64_t i, float r0, float r1,
                                              float r2)
{
    if (symd != 3) {
        s[i] = -s[i];
        return;
    }
    const double x = f32_get(s, n, 0, i), y = f32_get(s, n, 1, i), z = f32_get(s, n, 2, i);
    const double d = __dadd_rn(__dadd_rn(__dmul_rn(x, (double)r0), __dmul_rn(y, (double)r1)), __dmul_rn(z, (double)r2));
    const double d2 = __dmul_rn(2.0, d);
    const double w0 = __dsub_rn(x, __dmul_rn(d2, (double)r0)), w1 = __dsub_rn(y, __dmul_rn(d2, (double)r1)),
                 w2 = __dsub_rn(z, __dmul_rn(d2, (double)r2));
    const double nn = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(w0, w0), __dmul_rn(w1, w1)), __dmul_rn(w2, w2)));
    s[i] = (float)__ddiv_rn(w0, nn);
    s[n + i] = (float)__ddiv_rn(w1, nn);
    s[2 * n + i] = (float)__ddiv_rn(w2, nn);
}

// The embedding of a cluster: seed site and reflection vector r (plane
// reflections of O(3) spins, sign flips of scalars) from the WOLFF_SEED
// substream.
__device__ __forceinline__ int64_t embed_seed(const ModelDev& m, int64_t n, Key key, uint32_t serial, uint32_t tg_seed,
                                              float r[3])
{
    SubStream rng(key, 0u, serial, tg_seed);
    const int64_t rsite = (int64_t)(rng.next() % (uint64_t)n);
    double v[3] = {1.0, 0.0, 0.0};
    if (m.symd == 3) rnddir3(rng, v);
    else if (rng.real() < 0.5) v[0] = -1.0;
    r[0] = (float)v[0];
    r[1] = (float)v[1];
    r[2] = (float)v[2];
    return rsite;
}

template <class Lat>
__device__ __forceinline__ void wolff_f32_cluster(const ModelDev& m, const Lat& lat, float* __restrict__ s,
                                                  uint32_t* __restrict__ visited, int32_t* __restrict__ queue,
                                                  int32_t* __restrict__ out_size, Key key, uint32_t serial,
                                                  uint32_t tg_seed, uint32_t tg_bond, int max_degree,
                                                  int32_t* __restrict__ fbuf, double* __restrict__ fproj)
{
    __shared__ int s_head, s_tail, s_next;
    __shared__ float s_r[3];
    constexpr int CAP = kWolffCapF;
    const int64_t n = lat.n;
    const int symd = m.symd;
    if (threadIdx.x == 0) {
        float r[3];
        const int64_t rsite = embed_seed(m, n, key, serial, tg_seed, r);
        s_r[0] = r[0];
        s_r[1] = r[1];
        s_r[2] = r[2];
        queue[0] = (int32_t)rsite;
        fbuf[0] = (int32_t)rsite;
        fproj[0] = embed_proj(symd, s, n, rsite, r[0], r[1], r[2]);
        atomicOr(&visited[rsite >> 5], 1u << (rsite & 31));
        s_head = 0;
        s_tail = 1;
        s_next = 1;
    }
    __syncthreads();
    const float r0 = s_r[0], r1 = s_r[1], r2 = s_r[2];
    auto proj = [&](int64_t i) -> double { return embed_proj(symd, s, n, i, r0, r1, r2); };
    const int lanes = wolff_lanes(lat, max_degree);
    const unsigned lane = threadIdx.x & 31;
    for (int lvl = 0;; ++lvl) {
        const int head = s_head, tail = s_tail;
        if (head >= tail) break;
        // (frontier site, neighbour lane) items, as in wolff_int8_cluster; the
        // level's sites and projections from shared memory when they fit
        const bool fits = tail - head <= CAP;
        const int32_t* fcur = fbuf + (lvl & 1) * CAP;
        const double* pcur = fproj + (lvl & 1) * CAP;
        int32_t* fnext = fbuf + ((lvl + 1) & 1) * CAP;
        double* pnext = fproj + ((lvl + 1) & 1) * CAP;
        const int64_t items = (int64_t)(tail - head) * lanes;
        for (int64_t base = 0; base < items; base += blockDim.x) {
            const int64_t k = base + threadIdx.x;
            int64_t cur = 0;
            int t0 = 0, deg = 0;
            double ac = 0.0;
            if (k < items) {
                const int64_t q = k / lanes;
                t0 = (int)(k - q * lanes);
                if (fits) {
                    cur = fcur[q];
                    ac = pcur[q];
                } else {
                    cur = queue[head + q];
                    ac = proj(cur);
                }
                deg = lat.degree(cur);
            }
            const int rounds = __reduce_max_sync(0xffffffffu, deg > t0 ? (deg - t0 + lanes - 1) / lanes : 0);
            for (int rr = 0; rr < rounds; ++rr) {
                const int t = t0 + rr * lanes;
                bool add = false;
                int64_t j = 0;
                double aj = 0.0;
                if (t < deg) {
                    j = lat.nbr(cur, t);
                    // both loads issued before either is tested
                    const uint32_t vw = visited[j >> 5];
                    aj = proj(j);
                    if (!(vw & (1u << (j & 31)))) {
                        const double cpl = embed_cpl(m.J, ac, aj);
                        if (cpl > 0) {
                            const uint32_t lo = (uint32_t)(cur < j ? cur : j), hi = (uint32_t)(cur < j ? j : cur);
                            const uint64_t wd = lo64(philox(lo, serial, hi, tg_bond, key));
                            if (!update_accepted(2, cpl, m.beta, wd)) {
                                const uint32_t old = atomicOr(&visited[j >> 5], 1u << (j & 31));
                                add = !(old & (1u << (j & 31)));
                            }
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
                        if (at - tail < CAP) {
                            fnext[at - tail] = (int32_t)j;
                            pnext[at - tail] = aj;
                        }
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
    for (int k = threadIdx.x; k < size; k += blockDim.x) {
        const int32_t i = queue[k];
        embed_reflect(symd, s, n, i, r0, r1, r2);
        atomicAnd(&visited[i >> 5], ~(1u << (i & 31)));
    }
    if (threadIdx.x == 0) *out_size = size;
}

}  // namespace mqv
