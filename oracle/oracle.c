/*
 * CPU oracle for the MARQOV Monte Carlo update hot path -- TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of the reference algorithm, used only as the checker
 * of the CUDA engine (tests, smoke check, bench CPU-baseline leg).  Every
 * function cites the reference file:line it restates.  See oracle.h for how
 * the restatement itself is pinned to the reference.
 *
 * Random numbers: the reference draws from one sequential RNGCache stream
 * (src/libmarqov/rngcache.h:156-206).  The oracle keeps the RNGCache
 * interface semantics -- integer() is a 64-bit word, integer(r) = word % r,
 * real() = (word >> 11) * 2^-53 -- but the words come from Philox4x32-10
 * keyed by (seed, replica) and counted by (stream, site, sweep, block), so
 * results do not depend on the order in which sites or bonds are visited.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Stream tags (counter word 3, bits 24..31). */
enum { ST_METRO = 1, ST_INIT = 2, ST_WOLFF_SEED = 3, ST_WOLFF_BOND = 4, ST_ACCEPT = 5, ST_ACCEPT_FINE = 6 };

/* Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw, "Parallel
 * random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two 32x32->64
 * multiplies with a Weyl key schedule. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0; c1 = (uint32_t)p1; c2 = n2; c3 = (uint32_t)p0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

uint64_t orc_draw_c2(uint64_t seed, uint32_t replica, uint32_t stream, uint32_t c0,
                     uint32_t c1, uint32_t c2)
{
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t ctr[4] = {c0, c1, c2, (stream << 24) | (replica & 0xFFFFFFu)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    return (uint64_t)o[0] | ((uint64_t)o[1] << 32);
}

uint64_t orc_draw(uint64_t seed, uint32_t replica, uint32_t stream, uint32_t c0,
                  uint32_t c1, uint32_t k)
{
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t ctr[4] = {c0, c1, k >> 1, (stream << 24) | (replica & 0xFFFFFFu)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    if (k & 1u) return (uint64_t)o[2] | ((uint64_t)o[3] << 32);
    return (uint64_t)o[0] | ((uint64_t)o[1] << 32);
}

/* The acceptance word of site i in sweep t.  Its top byte is bit-sliced:
 * sites are grouped by G(i) = ((i >> 6) << 1) | (i & 1) -- 32 sites of equal
 * index parity in an aligned run of 64 -- and bit b of the byte is bit
 * ((i >> 1) & 31) of plane b, where planes 0..3 are the Philox block
 * (c0 = G(i), c1 = t, c2 = 0, ACCEPT stream) and planes 4..7 the block with
 * c2 = 1.  Its low 56 bits are the low 56 bits of half (i & 1) of the block
 * (c0 = i >> 1, c1 = t, c2 = 0, ACCEPT_FINE stream).  A comparison of real()
 * against a threshold is decided by the top byte unless it ties with the
 * threshold's top byte. */
uint64_t orc_accept_word(uint64_t seed, uint32_t replica, uint32_t site, uint32_t sweep)
{
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const uint32_t g = ((site >> 6) << 1) | (site & 1u), q = (site >> 1) & 31u;
    uint32_t p0[4], p1[4];
    uint32_t ctr0[4] = {g, sweep, 0, (ST_ACCEPT << 24) | (replica & 0xFFFFFFu)};
    uint32_t ctr1[4] = {g, sweep, 1, (ST_ACCEPT << 24) | (replica & 0xFFFFFFu)};
    orc_philox4x32_10(ctr0, key, p0);
    orc_philox4x32_10(ctr1, key, p1);
    uint64_t cb = 0;
    for (int b = 0; b < 8; ++b) {
        const uint32_t plane = b < 4 ? p0[b] : p1[b - 4];
        cb |= (uint64_t)((plane >> q) & 1u) << b;
    }
    uint32_t o[4];
    uint32_t ctrf[4] = {site >> 1, sweep, 0, (ST_ACCEPT_FINE << 24) | (replica & 0xFFFFFFu)};
    orc_philox4x32_10(ctrf, key, o);
    const uint64_t f = (site & 1u) ? ((uint64_t)o[2] | ((uint64_t)o[3] << 32)) : ((uint64_t)o[0] | ((uint64_t)o[1] << 32));
    return (cb << 56) | (f & 0x00FFFFFFFFFFFFFFULL);
}

/* RNGCache::real(max, min) = min + (max-min) * (word >> 11) * 2^-53
 * (src/libmarqov/rngcache.h:202-206). */
static double real_of(uint64_t w, double max, double min)
{
    double r = (double)(w >> 11) * 0x1.0p-53;
    return min + (max - min) * r;
}

/* Sequential draws of one (stream, c0, c1) substream, RNGCache-like. */
typedef struct { uint64_t seed; uint32_t replica, stream, c0, c1, k; } orc_rng;
static uint64_t rng_integer(orc_rng* r)
{
    return orc_draw(r->seed, r->replica, r->stream, r->c0, r->c1, r->k++);
}
static uint64_t rng_integer_r(orc_rng* r, uint64_t range) { return rng_integer(r) % range; }
static double rng_real(orc_rng* r) { return real_of(rng_integer(r), 1.0, 0.0); }

/* ---- acceptance rule ---------------------------------------------------- */

/* 2^x polynomial, src/libmarqov/metropolishelpers.h:39-48 (Horner order kept). */
double orc_exp2app6(double x)
{
    double u = 1.0944614513161076e-4;
    u = u * x + 1.2758920456516547e-3;
    u = u * x + 9.5802562122641916e-3;
    u = u * x + 5.5491137793956362e-2;
    u = u * x + 2.4022437948159954e-1;
    u = u * x + 6.9314704935511511e-1;
    return u * x + 9.9999999867786389e-1;
}

/* cvttsd2si semantics, src/libmarqov/metropolishelpers.h:59-70: truncation,
 * with the "integer indefinite" INT64_MIN for NaN and out-of-range inputs. */
int64_t orc_trunctoi64(double f)
{
    if (!(f > -9223372036854775808.0 && f < 9223372036854775808.0)) return INT64_MIN;
    return (int64_t)f;
}

/* update_accepted<pref>, src/libmarqov/metropolishelpers.h:109-142. */
int orc_update_accepted(int pref, double dE, double beta, uint64_t draw)
{
    if (dE <= 0) return 1;
    double rngnum = (double)(draw >> 11) * 0x1.0p-53;
    double action = -beta * dE;
    double action2 = (double)pref * 1.4426950408889634074 * action;
    int64_t i64;
    memcpy(&i64, &rngnum, 8);
    int64_t t = orc_trunctoi64(action2);
    if ((i64 >> 52) - 1022 != t) return ((i64 >> 52) - 1022) < t;
    i64 = (i64 & ~(int64_t)0xFFF0000000000000LL) | 0x3FE0000000000000LL;
    double remainder = action2 - trunc(action2);
    memcpy(&rngnum, &i64, 8);
    return rngnum < orc_exp2app6(remainder);
}

/* For fixed (pref, dE, beta) the rule accepts exactly the draws whose 53-bit
 * mantissa source u53 = draw >> 11 lies below a cut: the exponent test is
 * monotone in u53 and, at equal exponent, so is the mantissa test.  The cut
 * is found by bisection on the rule itself. */
uint64_t orc_accept_threshold(int pref, double dE, double beta)
{
    if (dE <= 0) return (uint64_t)1 << 53;
    uint64_t lo = 0, hi = (uint64_t)1 << 53; /* invariant: accepted(<lo), rejected(>=hi) */
    if (!orc_update_accepted(pref, dE, beta, 0)) return 0;
    lo = 1;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (orc_update_accepted(pref, dE, beta, mid << 11)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* ---- lattices ----------------------------------------------------------- */

/* Neighbours of src/lattice/regular_hypercubic.h:31-66 (order +x,-x,+y,-y,..). */
void orc_hypercubic_csr(int dim, int len, int32_t* row_ptr, int32_t* col_idx)
{
    int64_t n = 1;
    int64_t pows[8];
    for (int j = 0; j < dim; ++j) { pows[j] = n; n *= len; }
    for (int64_t i = 0; i < n; ++i) {
        row_ptr[i] = (int32_t)(i * 2 * dim);
        for (int j = 0; j < dim; ++j) {
            int64_t pl = pows[j] * len;
            int64_t base = (i / pl) * pl;
            col_idx[i * 2 * dim + 2 * j] = (int32_t)(base + (i + pows[j]) % pl);
            int64_t c = i - pows[j];
            col_idx[i * 2 * dim + 2 * j + 1] =
                (int32_t)(c < base ? base + (c + pl) % pl : c);
        }
    }
    row_ptr[n] = (int32_t)(n * 2 * dim);
}

void orc_parity_colours(int dim, int len, int32_t* colour_ptr, int32_t* order)
{
    int64_t n = 1;
    for (int j = 0; j < dim; ++j) n *= len;
    int64_t a = 0, b = 0;
    int64_t nb = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t k = i, p = 0;
        for (int j = 0; j < dim; ++j) { p += k % len; k /= len; }
        if ((p & 1) == 0) ++nb;
    }
    for (int64_t i = 0; i < n; ++i) {
        int64_t k = i, p = 0;
        for (int j = 0; j < dim; ++j) { p += k % len; k /= len; }
        if ((p & 1) == 0) order[a++] = (int32_t)i;
        else order[nb + b++] = (int32_t)i;
    }
    colour_ptr[0] = 0; colour_ptr[1] = (int32_t)nb; colour_ptr[2] = (int32_t)n;
}

/* ---- int8 models: Metropolis --------------------------------------------- */

/* Weights of onsite terms 0 / 1 at a site of sublattice `sub` (the parity
 * colour): every term acts unless the lattice has SimpleBipartite's
 * termselector (src/lattice/simple_bipartite.h:22-41, read by get_terms,
 * src/libmarqov/metropolishelpers.h:402-430), which gives sublattice p term p. */
static int ons0(const orc_model* m, int sub) { return !(m->termsel && sub); }
static int ons1(const orc_model* m, int sub) { return !(m->termsel && !sub); }

/* One Metropolis::move (src/libmarqov/metropolis.h:88-126) at site i. */
static void metro_int8_site(const orc_model* m, const orc_lattice* g, int8_t* s, double beta,
                            orc_rng* rng, int32_t i, int sub)
{
    const int32_t b = g->row_ptr[i], e = g->row_ptr[i + 1];
    int old = s[i], nw;
    double dE;
    switch (m->kind) {
    case ORC_POTTS: {
        /* Initializer<Potts<Q>>::newsv, src/hamiltonian/Potts.h:170-177 */
        nw = (int)rng_integer_r(rng, (uint64_t)m->q);
        /* PottsInteraction::diff, src/hamiltonian/Potts.h:86-107 */
        int eo = 0, en = 0;
        for (int32_t p = b; p < e; ++p) {
            int nb = s[g->col_idx[p]];
            eo += (old == nb);
            en += (nw == nb);
        }
        dE = m->k * (double)(en - eo);
        break;
    }
    case ORC_BLUME_CAPEL: {
        /* Spin1_Initializer::newsv, src/hamiltonian/util/initializers.h:99-118 */
        int st = old;
        if (st == 0) st = rng_real(rng) < 0.5 ? -1 : +1;
        else st = rng_real(rng) < 0.5 ? -st : 0;
        nw = st;
        int sum = 0;
        for (int32_t p = b; p < e; ++p) sum += s[g->col_idx[p]];
        /* compute_onsiteenergydiff (metropolishelpers.h:651-683): the site's
         * terms in order, each h_b (get(new) - get(old)), get = s^2 */
        const double dq = (double)(nw * nw - old * old);
        double ons = 0.0;
        if (ons0(m, sub)) ons += m->h * dq;
        if (ons1(m, sub) && (m->termsel || m->h2 != 0.0)) ons += m->h2 * dq;
        dE = m->J * (double)((nw - old) * sum) + ons;
        break;
    }
    default: {
        /* SVInitializer<array<int,1>>: spin flip, initializers.h:52-58;
         * nbrhoodloop with/without bonds, metropolishelpers.h:456-537;
         * compute_interactionenergydiff, metropolishelpers.h:598-623 */
        nw = -old;
        int sum = 0;
        if (g->bonds)
            for (int32_t p = b; p < e; ++p) sum += g->bonds[p] * s[g->col_idx[p]];
        else
            for (int32_t p = b; p < e; ++p) sum += s[g->col_idx[p]];
        dE = m->J * (double)((nw - old) * sum);
        break;
    }
    }
    /* metro_update_accepted, metropolis.h:61-64,120-124: the draw after the
     * proposal draws is the site's acceptance word */
    if (dE <= 0 || orc_update_accepted(1, dE, beta, orc_accept_word(rng->seed, rng->replica, rng->c0, rng->c1)))
        s[i] = (int8_t)nw;
}

void orc_sweep_int8(const orc_model* m, const orc_lattice* g, int8_t* s, double beta,
                    uint64_t seed, uint32_t replica, uint32_t sweep)
{
    for (int c = 0; c < g->ncolours; ++c)
        for (int32_t p = g->colour_ptr[c]; p < g->colour_ptr[c + 1]; ++p) {
            int32_t i = g->order[p];
            orc_rng rng = {seed, replica, ST_METRO, (uint32_t)i, sweep, 0};
            metro_int8_site(m, g, s, beta, &rng, i, c);
        }
}

/* One colour-order sweep of Ising<int> on FixedDimRegularHypercubic<2>(L)
 * without a materialised neighbour list: the neighbours of
 * src/lattice/regular_hypercubic.h:31-66 computed per site.  State in the
 * reference layout (site = x + L y). */
void orc_ising2d_sweep(int32_t L, double J, int8_t* s, double beta, uint64_t seed, uint32_t replica,
                       uint32_t sweep)
{
    for (int c = 0; c < 2; ++c)
        for (int64_t y = 0; y < L; ++y) {
            const int64_t yu = (y + 1) % L, yd = (y + L - 1) % L;
            for (int64_t x = (y + c) & 1; x < L; x += 2) {
                const int64_t i = y * L + x;
                const int64_t xr = (x + 1) % L, xl = (x + L - 1) % L;
                const int old = s[i];
                const int sum = s[y * L + xr] + s[y * L + xl] + s[yu * L + x] + s[yd * L + x];
                const double dE = J * (double)((-2 * old) * sum);
                if (dE <= 0 || orc_update_accepted(1, dE, beta, orc_accept_word(seed, replica, (uint32_t)i, sweep)))
                    s[i] = (int8_t)-old;
            }
        }
}

/* Initial states: Ising::initstatespace (src/hamiltonian/Ising.h:99-107),
 * Potts::initstatespace (src/hamiltonian/Potts.h:149-156); Blume-Capel has
 * none and gets Core::init_hot (src/libmarqov/core.h:773-782): the
 * one-component random direction of set_to_rnddir, +1 turned to -1 when
 * real() < 0.5 (src/hamiltonian/util/randomdir.h:84-90,102-106).  One INIT
 * substream per site. */
void orc_init_int8(const orc_model* m, int32_t n, int8_t* s, uint64_t seed, uint32_t replica)
{
    for (int32_t i = 0; i < n; ++i) {
        orc_rng rng = {seed, replica, ST_INIT, (uint32_t)i, 0, 0};
        if (m->kind == ORC_POTTS) s[i] = (int8_t)rng_integer_r(&rng, (uint64_t)m->q);
        else if (m->kind == ORC_BLUME_CAPEL) s[i] = rng_real(&rng) < 0.5 ? -1 : 1;
        else s[i] = rng_real(&rng) > 0.5 ? 1 : -1;
    }
}

/* ---- float models --------------------------------------------------------- */

/* set_to_rnddir for SymD = 3, src/hamiltonian/util/randomdir.h:45-64,102-106 */
static void rnddir3(orc_rng* rng, double v[3])
{
    double a0 = 2.0 * rng_real(rng), a1 = 2.0 * rng_real(rng);
    double r0 = 1.0;
    double r1 = r0 * a0 * (2.0 - a0);
    r0 = sqrt(r0) * (1.0 - a0);
    r1 = sqrt(r1);
    double r2 = r1 * cos(M_PI * a1);
    r1 = r1 * sin(M_PI * a1);
    v[0] = r0; v[1] = r1; v[2] = r2;
}

/* Small-cap proposal (an Initializer<Heisenberg> plugin): a direction drawn
 * uniformly from the spherical cap {cos(angle to old) >= cap} around the old
 * spin.  Frame: the rotation taking +z to the old spin, mirrored in z for
 * old spins on the southern hemisphere. */
static void smallcap3(orc_rng* rng, const float* o, double cap, double v[3])
{
    double u0 = rng_real(rng), u1 = rng_real(rng);
    double ca = 1.0 - u0 * (1.0 - cap);
    double sa = sqrt(fmax(0.0, 1.0 - ca * ca));
    double ph = 2.0 * M_PI * u1;
    double dx = sa * cos(ph), dy = sa * sin(ph), dz = ca;
    double x = o[0], y = o[1], z = o[2];
    double sg = z < 0 ? -1.0 : 1.0;
    double zz = sg * z;
    double a = 1.0 / (1.0 + zz);
    double bxy = -x * y * a;
    double e1[3] = {1.0 - x * x * a, bxy, -x};
    double e2[3] = {bxy, 1.0 - y * y * a, -y};
    e1[2] *= sg; e2[2] *= sg;
    double nv[3];
    for (int c = 0; c < 3; ++c) nv[c] = dx * e1[c] + dy * e2[c] + dz * (double)o[c];
    double nn = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    for (int c = 0; c < 3; ++c) v[c] = nv[c] / nn;
}

static void metro_f32_site(const orc_model* m, const orc_lattice* g, float* s, int symd,
                           double beta, orc_rng* rng, int32_t i, int sub)
{
    const int32_t b = g->row_ptr[i], e = g->row_ptr[i + 1];
    float* so = s + (size_t)i * symd;
    double nw[3] = {0, 0, 0};
    double dE;
    if (symd == 1) {
        /* scalar phi^4: shift proposal old + amp * real(-1, 1) as
         * Phi4_Initializer_Cartesian, src/hamiltonian/Phi4.h:44-57 */
        double r = real_of(rng_integer(rng), -1.0, 1.0);
        double old = so[0];
        nw[0] = (double)(float)(old + m->cap * r);
        /* the neighbourhood is summed in the state's float type (nbrhoodloop,
         * metropolishelpers.h:456-537) and dot() multiplies float components */
        float sum = 0.f;
        for (int32_t p = b; p < e; ++p) sum += s[g->col_idx[p]];
        double o2 = old * old, n2 = nw[0] * nw[0];
        /* interaction + Onsite_Quadratic + Onsite_Fourth_Minus_One,
         * src/hamiltonian/Phi4.h:63-74,103-121 */
        dE = m->J * (double)(((float)nw[0] - so[0]) * sum) + ons0(m, sub) * m->h * (n2 - o2) +
             ons1(m, sub) * m->h2 * ((n2 - 1.0) * (n2 - 1.0) - (o2 - 1.0) * (o2 - 1.0));
    } else {
        double v[3];
        if (m->proposal == 1) smallcap3(rng, so, m->cap, v);
        else rnddir3(rng, v); /* SVInitializer<float>, initializers.h:74-80 */
        for (int c = 0; c < 3; ++c) nw[c] = (double)(float)v[c];
        /* float neighbourhood sums and float component products summed in
         * double (nbrhoodloop and svmath.h dot on float state vectors) */
        float nb[3] = {0.f, 0.f, 0.f};
        for (int32_t p = b; p < e; ++p) {
            const float* sj = s + (size_t)g->col_idx[p] * 3;
            for (int c = 0; c < 3; ++c) nb[c] += sj[c];
        }
        double pr[3];
        for (int c = 0; c < 3; ++c) pr[c] = (double)(((float)nw[c] - so[c]) * nb[c]);
        /* the interaction's get(): XXZAntiferro_interaction weights x and y
         * by Delta (src/hamiltonian/XXZAntiferro.h:135-150), Heisenberg none */
        double dxy = pr[0] + pr[1];
        dE = m->J * ((m->kind == ORC_XXZ ? m->delta * dxy : dxy) + pr[2]);
        if (m->kind == ORC_XXZ) {
            /* XXZAntiferro_extfield H s_z (XXZAntiferro.h:162-170) and
             * XXZAntiferro_onsiteaniso D s_z^2 (XXZAntiferroSingleAniso.h:31-44) */
            double zn = nw[2], zo = so[2];
            dE += ons0(m, sub) * m->h * (zn - zo) + ons1(m, sub) * m->h2 * (zn * zn - zo * zo);
        }
    }
    if (dE <= 0 || orc_update_accepted(1, dE, beta, orc_accept_word(rng->seed, rng->replica, rng->c0, rng->c1)))
        for (int c = 0; c < symd; ++c) so[c] = (float)nw[c];
}

void orc_sweep_f32(const orc_model* m, const orc_lattice* g, float* s, int symd,
                   double beta, uint64_t seed, uint32_t replica, uint32_t sweep)
{
    for (int c = 0; c < g->ncolours; ++c)
        for (int32_t p = g->colour_ptr[c]; p < g->colour_ptr[c + 1]; ++p) {
            int32_t i = g->order[p];
            orc_rng rng = {seed, replica, ST_METRO, (uint32_t)i, sweep, 0};
            metro_f32_site(m, g, s, symd, beta, &rng, i, c);
        }
}

/* Heisenberg::initstatespace (src/hamiltonian/Heisenberg.h:97-104): random
 * directions; scalar fields start from a standard normal (Box-Muller). */
void orc_init_f32(const orc_model* m, int32_t n, float* s, int symd, uint64_t seed,
                  uint32_t replica)
{
    (void)m;
    for (int32_t i = 0; i < n; ++i) {
        orc_rng rng = {seed, replica, ST_INIT, (uint32_t)i, 0, 0};
        if (symd == 3) {
            double v[3];
            rnddir3(&rng, v);
            for (int c = 0; c < 3; ++c) s[(size_t)i * 3 + c] = (float)v[c];
        } else {
            double u0 = rng_real(&rng), u1 = rng_real(&rng);
            s[i] = (float)(sqrt(-2.0 * log(1.0 - u0)) * cos(2.0 * M_PI * u1));
        }
    }
}

/* ---- Wolff ------------------------------------------------------------------ */

static uint64_t bond_draw(uint64_t seed, uint32_t replica, uint32_t serial, int32_t a, int32_t c)
{
    uint32_t lo = (uint32_t)(a < c ? a : c), hi = (uint32_t)(a < c ? c : a);
    return orc_draw_c2(seed, replica, ST_WOLFF_BOND, lo, serial, hi);
}

/* Wolff cluster, int8 models.
 *  ORC_ISING:       Wolff<Ising<int>>, src/hamiltonian/Ising.h:126-168
 *  ORC_ISING_EMBED: Wolff<H,L> + Embedder<H,L>, src/libmarqov/wolff.h:72-126,
 *                   src/libmarqov/embedder.h:66-93
 *  ORC_POTTS:       Wolff<Potts<Q>> + Embedder<Potts<Q>>, src/hamiltonian/Potts.h:220-320
 * The seed site is integer(N) of the cluster's WOLFF_SEED substream
 * (src/libmarqov/emcs.h:85); embedder draws follow in that substream.  Each
 * bond test uses the draw keyed by the undirected bond, so the cluster is the
 * seed's component of activated bonds whatever the visiting order. */
int32_t orc_wolff_int8(const orc_model* m, const orc_lattice* g, int8_t* s, double beta,
                       uint64_t seed, uint32_t replica, uint32_t serial, int32_t* work)
{
    const int32_t n = g->n;
    orc_rng rng = {seed, replica, ST_WOLFF_SEED, 0, serial, 0};
    int32_t rsite = (int32_t)rng_integer_r(&rng, (uint64_t)n);
    int32_t* stack = work;
    int32_t q = 0, size = 1;
    stack[0] = rsite;
    if (m->kind == ORC_ISING) {
        const int val = s[rsite];
        s[rsite] = (int8_t)-val;
        const double prob = -expm1(2.0 * beta * m->J);
        while (q >= 0) {
            int32_t cur = stack[q--];
            for (int32_t p = g->row_ptr[cur]; p < g->row_ptr[cur + 1]; ++p) {
                int32_t nb = g->col_idx[p];
                if (s[nb] != val) continue;
                double u = real_of(bond_draw(seed, replica, serial, cur, nb), 1.0, 0.0);
                if (u < prob) { stack[++q] = nb; ++size; s[nb] = (int8_t)-val; }
            }
        }
    } else if (m->kind == ORC_POTTS) {
        const int oldq = s[rsite];
        int newq = oldq, tries = 0;
        do { newq = (int)rng_integer_r(&rng, (uint64_t)m->q); } while (newq == oldq && ++tries < 256);
        if (newq == oldq) newq = (oldq + 1) % m->q;
        s[rsite] = (int8_t)newq;
        while (q >= 0) {
            int32_t cur = stack[q--];
            for (int32_t p = g->row_ptr[cur]; p < g->row_ptr[cur + 1]; ++p) {
                int32_t nb = g->col_idx[p];
                double cpl = m->k * (s[nb] != oldq ? 0.0 : -0.5);
                if (cpl <= 0) continue;
                if (!orc_update_accepted(2, cpl, beta, bond_draw(seed, replica, serial, cur, nb))) {
                    stack[++q] = nb; ++size; s[nb] = (int8_t)newq;
                }
            }
        }
    } else {
        (void)rng_integer_r(&rng, 1); /* Embedder::draw: rdir = integer(SymD) */
        s[rsite] = (int8_t)-s[rsite];
        while (q >= 0) {
            int32_t cur = stack[q--];
            for (int32_t p = g->row_ptr[cur]; p < g->row_ptr[cur + 1]; ++p) {
                int32_t nb = g->col_idx[p];
                double cpl = m->J * (double)(s[cur] * s[nb]);
                if (cpl <= 0) continue;
                if (!orc_update_accepted(2, cpl, beta, bond_draw(seed, replica, serial, cur, nb))) {
                    stack[++q] = nb; ++size; s[nb] = (int8_t)-s[nb];
                }
            }
        }
    }
    return size;
}

/* Wolff cluster, float models, through the generic Wolff
 * (src/libmarqov/wolff.h:72-126) with reflection embedders:
 *  symd 3: Embedder<Heisenberg> (src/hamiltonian/Heisenberg.h:158-185):
 *          random unit r, coupling (s1.r)(s2.r), flip s -= 2(s.r)r + normalize
 *  symd 1: Embedder<Phi4> (src/hamiltonian/Phi4.h:217-243) for one component:
 *          r = +-1, coupling s1 s2, flip s = -s (no normalisation).
 * The coupling of a bond is evaluated from the projections before either
 * end is flipped: (-a_cur)(a_nbr) J with a = s.r, as the reference computes it
 * after the current site's flip. */
int32_t orc_wolff_f32(const orc_model* m, const orc_lattice* g, float* s, int symd,
                      double beta, uint64_t seed, uint32_t replica, uint32_t serial,
                      int32_t* work)
{
    const int32_t n = g->n;
    orc_rng rng = {seed, replica, ST_WOLFF_SEED, 0, serial, 0};
    int32_t rsite = (int32_t)rng_integer_r(&rng, (uint64_t)n);
    double r[3] = {1.0, 0.0, 0.0};
    if (symd == 3) rnddir3(&rng, r);
    else if (rng_real(&rng) < 0.5) r[0] = -1.0;
    float rf[3] = {(float)r[0], (float)r[1], (float)r[2]};
    int32_t* stack = work;
    uint8_t* inc = (uint8_t*)(work + n); /* n bytes: membership marks */
    memset(inc, 0, (size_t)n);
    int32_t q = 0, size = 1;
    stack[0] = rsite;
    inc[rsite] = 1;
    /* projections before flipping */
    #define PROJ(i) (symd == 3 ? ((double)s[(size_t)(i) * 3] * rf[0] + (double)s[(size_t)(i) * 3 + 1] * rf[1] + (double)s[(size_t)(i) * 3 + 2] * rf[2]) : (double)s[i] * rf[0])
    int32_t nmem = 0;
    int32_t* members = work + n + (n + 3) / 4;
    members[nmem++] = rsite;
    while (q >= 0) {
        int32_t cur = stack[q--];
        double ac = PROJ(cur);
        for (int32_t p = g->row_ptr[cur]; p < g->row_ptr[cur + 1]; ++p) {
            int32_t nb = g->col_idx[p];
            if (inc[nb]) continue;
            double cpl = m->J * (-ac) * PROJ(nb);
            if (cpl <= 0) continue;
            if (!orc_update_accepted(2, cpl, beta, bond_draw(seed, replica, serial, cur, nb))) {
                stack[++q] = nb; ++size; inc[nb] = 1; members[nmem++] = nb;
            }
        }
    }
    #undef PROJ
    for (int32_t t = 0; t < nmem; ++t) {
        int32_t i = members[t];
        if (symd == 3) {
            float* v = s + (size_t)i * 3;
            double d = (double)v[0] * rf[0] + (double)v[1] * rf[1] + (double)v[2] * rf[2];
            double w[3];
            for (int c = 0; c < 3; ++c) w[c] = (double)v[c] - 2.0 * d * rf[c];
            double nn = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
            for (int c = 0; c < 3; ++c) v[c] = (float)(w[c] / nn);
        } else {
            s[i] = -s[i];
        }
    }
    return size;
}

/* ---- observables ---------------------------------------------------------- */

/* Magnetization::measure (src/hamiltonian/util/observables.h:47-65),
 * InteractionEnergy (observables.h:186-217), SelfEnergy (observables.h:251-268),
 * PottsMagnetization (src/hamiltonian/Potts.h:46-61). */
void orc_measure_int8(const orc_model* m, const orc_lattice* g, const int8_t* s, orc_obs* out)
{
    const int32_t n = g->n;
    double mm, e;
    if (m->kind == ORC_POTTS) {
        int64_t cnt[128] = {0};
        for (int32_t i = 0; i < n; ++i) cnt[(int)s[i]]++;
        int64_t mx = 0;
        for (int a = 0; a < m->q; ++a) if (cnt[a] > mx) mx = cnt[a];
        mm = (double)(m->q * mx - n) / (double)((int64_t)n * (m->q - 1));
        int64_t same = 0;
        for (int32_t i = 0; i < n; ++i)
            for (int32_t p = g->row_ptr[i]; p < g->row_ptr[i + 1]; ++p) same += (s[i] == s[g->col_idx[p]]);
        e = m->k * (double)same / (double)(2 * (int64_t)n);
    } else {
        double mag = 0;
        for (int32_t i = 0; i < n; ++i) mag += s[i];
        mm = sqrt(mag * mag) / (double)n;
        double enepart = 0;
        for (int32_t i = 0; i < n; ++i) {
            for (int32_t p = g->row_ptr[i]; p < g->row_ptr[i + 1]; ++p) {
                int w = g->bonds ? g->bonds[p] : 1;
                enepart += (double)(w * s[i] * s[g->col_idx[p]]);
            }
        }
        e = m->J * enepart / (double)(2 * (int64_t)n);
        if (m->kind == ORC_BLUME_CAPEL) {
            /* SelfEnergy: every onsite term over every site (observables.h:251-268) */
            double sq = 0;
            for (int32_t i = 0; i < n; ++i) sq += (double)(s[i] * s[i]);
            e += (m->h * sq + m->h2 * sq) / (double)n;
        }
    }
    out->e = e; out->m = mm; out->m2 = mm * mm; out->m4 = out->m2 * out->m2;
}

void orc_measure_f32(const orc_model* m, const orc_lattice* g, const float* s, int symd,
                     orc_obs* out)
{
    const int32_t n = g->n;
    double mag[3] = {0, 0, 0};
    for (int32_t i = 0; i < n; ++i)
        for (int c = 0; c < symd; ++c) mag[c] += s[(size_t)i * symd + c];
    double r = 0;
    for (int c = 0; c < symd; ++c) r += mag[c] * mag[c];
    double mm = sqrt(r) / (double)n;
    /* InteractionEnergy applies get() to both ends (observables.h:186-217):
     * XXZ weights x x' and y y' by Delta^2 */
    const double d2 = m->kind == ORC_XXZ ? m->delta * m->delta : 1.0;
    double w[3] = {d2, d2, 1.0};
    double enepart = 0, q2 = 0, q4 = 0, sz = 0, szz = 0;
    for (int32_t i = 0; i < n; ++i) {
        const float* si = s + (size_t)i * symd;
        for (int32_t p = g->row_ptr[i]; p < g->row_ptr[i + 1]; ++p) {
            const float* sj = s + (size_t)g->col_idx[p] * symd;
            for (int c = 0; c < symd; ++c) enepart += w[c] * (double)si[c] * (double)sj[c];
        }
        double p2 = 0;
        for (int c = 0; c < symd; ++c) p2 += (double)si[c] * (double)si[c];
        q2 += p2;
        q4 += (p2 - 1.0) * (p2 - 1.0);
        if (symd == 3) {
            sz += (double)si[2];
            szz += (double)si[2] * (double)si[2];
        }
    }
    double e = m->J * enepart / (double)(2 * (int64_t)n);
    /* SelfEnergy: every onsite term over every site (observables.h:251-268) */
    if (m->kind == ORC_PHI4) e += (m->h * q2 + m->h2 * q4) / (double)n;
    if (m->kind == ORC_XXZ) e += (m->h * sz + m->h2 * szz) / (double)n;
    out->e = e; out->m = mm; out->m2 = mm * mm; out->m4 = out->m2 * out->m2;
}

/* ---- known-answer test of the acceptance rule ----------------------------- */

/* 64-bit Mersenne Twister (Matsumoto & Nishimura, MT19937-64 with the
 * parameters of std::mt19937_64), the engine of the reference's acceptance
 * test testsuite/components/5-metro_exp.cpp. */
typedef struct { uint64_t mt[312]; int idx; } orc_mt64;
static void mt64_seed(orc_mt64* g, uint64_t seed)
{
    g->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->idx = 312;
}
static uint64_t mt64_next(orc_mt64* g)
{
    if (g->idx >= 312) {
        for (int i = 0; i < 312; ++i) {
            uint64_t x = (g->mt[i] & 0xFFFFFFFF80000000ULL) | (g->mt[(i + 1) % 312] & 0x7FFFFFFFULL);
            uint64_t xa = x >> 1;
            if (x & 1ULL) xa ^= 0xB5026F5AA96619E9ULL;
            g->mt[i] = g->mt[(i + 156) % 312] ^ xa;
        }
        g->idx = 0;
    }
    uint64_t y = g->mt[g->idx++];
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= y >> 43;
    return y;
}

void orc_mt19937_64_words(uint64_t seed, int64_t n, uint64_t* out)
{
    orc_mt64 g;
    mt64_seed(&g, seed);
    for (int64_t i = 0; i < n; ++i) out[i] = mt64_next(&g);
}

/* testsuite/components/5-metro_exp.cpp:41-51 with the restated rule: dE = 10
 * real() for N words of mt19937_64(0), then `reps` passes of the rule at
 * beta, one word per decision with dE > 0.  Returns the accept count and the
 * decisions (when non-NULL). */
int64_t orc_metro_exp(int32_t N, int32_t reps, double beta, uint8_t* decisions)
{
    orc_mt64 g;
    mt64_seed(&g, 0);
    double* dE = (double*)malloc(sizeof(double) * (size_t)N);
    for (int32_t i = 0; i < N; ++i) dE[i] = 10.0 * real_of(mt64_next(&g), 1.0, 0.0);
    int64_t acc = 0;
    for (int32_t r = 0; r < reps; ++r)
        for (int32_t i = 0; i < N; ++i) {
            int a = dE[i] <= 0 ? 1 : orc_update_accepted(1, dE[i], beta, mt64_next(&g));
            acc += a;
            if (decisions) decisions[(size_t)r * N + i] = (uint8_t)a;
        }
    free(dE);
    return acc;
}
