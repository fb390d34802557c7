/*
 * CPU oracle for the MARQOV Monte Carlo update hot path -- TEST INFRASTRUCTURE.
 *
 * This is a plain-C restatement of the reference algorithm (MARQOV,
 * src/libmarqov/{metropolis,metropolishelpers,wolff,embedder,rngcache}.h and
 * src/hamiltonian/*.h), driven in colour order with the counter-based Philox
 * stream that the CUDA engine uses.  It is the checker for the engine's
 * parity tests, the CPU baseline leg of bench.py and nothing else: the engine
 * never links, loads or calls it.
 *
 * Pinned against: (1) the reference's own templates compiled from its sources
 * by oracle/ref_harness.cpp (oracle/_ref), through the golden fixtures in
 * tests/golden; (2) the reference acceptance known-answer test
 * (testsuite/components/5-metro_exp.cpp); (3) the Random123 Philox4x32-10
 * known-answer vectors.
 */
#ifndef MQV_ORACLE_H
#define MQV_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- random numbers ---------------------------------------------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* k-th 64-bit draw of the stream (seed, replica, stream, c0, c1); draws 2b and
 * 2b+1 are the two halves of the Philox block with c2 = b. */
uint64_t orc_draw(uint64_t seed, uint32_t replica, uint32_t stream, uint32_t c0,
                  uint32_t c1, uint32_t k);
/* The Metropolis acceptance word of `site` in `sweep` (top byte bit-sliced
 * from two Philox blocks shared by 32 sites, low 56 bits from a block shared
 * by 2 sites). */
uint64_t orc_accept_word(uint64_t seed, uint32_t replica, uint32_t site, uint32_t sweep);
/* single draw keyed fully by the counter words (used for Wolff bonds) */
uint64_t orc_draw_c2(uint64_t seed, uint32_t replica, uint32_t stream, uint32_t c0,
                     uint32_t c1, uint32_t c2);

/* ---- acceptance rule ---------------------------------------------------- */
double orc_exp2app6(double x);
int64_t orc_trunctoi64(double f);
int orc_update_accepted(int pref, double dE, double beta, uint64_t draw);
/* smallest u53 that is rejected (2^53 when every u53 is accepted) */
uint64_t orc_accept_threshold(int pref, double dE, double beta);

/* ---- models -------------------------------------------------------------- */
enum {
    ORC_ISING = 1,        /* Ising<int>: flip proposal, Wolff<Ising<int>> exact-expm1 */
    ORC_ISING_EMBED = 2,  /* Ising<int8_t>: flip proposal, generic Wolff + Embedder */
    ORC_POTTS = 3,        /* Potts<Q>: flex delta term, Embedder<Potts<Q>> */
    ORC_BLUME_CAPEL = 4,  /* BlumeCapel: Spin1 proposal, onsite D s^2 */
    ORC_EA = 5,           /* EdwardsAndersonIsing with lattice bonds */
    ORC_HEISENBERG = 6,   /* O(3), fresh-direction or small-cap proposals */
    ORC_PHI4 = 7,         /* scalar phi^4, Cartesian shift proposal */
    ORC_XXZ = 8           /* XXZAntiferro(SingleAniso): (Delta x, Delta y, z) interaction, H s_z, D s_z^2 */
};

typedef struct orc_model {
    int kind;
    int q;           /* Potts states */
    int proposal;    /* 0 = model default, 1 = small-cap (Heisenberg/XXZ) */
    double J;        /* interaction prefactor, reference sign: dE = J dot(dS, sum nbrs) */
    double h;        /* onsite term 0 (Blume-Capel D or DA; phi^4 mass/beta; XXZ field H) */
    double h2;       /* onsite term 1 (Blume-Capel DB; phi^4 lambda/beta; XXZ single-ion D) */
    double k;        /* flex prefactor (Potts) */
    double delta;    /* XXZ anisotropy (weight of the x and y components) */
    double cap;      /* proposal width: small-cap cos(theta_max) or phi^4 shift amplitude */
    int termsel;     /* 1: SimpleBipartite termselector -- onsite term p only on the sites of
                        colour p (the lattice's colouring must be the coordinate parity) */
} orc_model;

typedef struct orc_lattice {
    int32_t n;               /* sites */
    const int32_t* row_ptr;  /* n+1 */
    const int32_t* col_idx;  /* row_ptr[n] */
    const int8_t* bonds;     /* optional, per CSR entry */
    int32_t ncolours;
    const int32_t* colour_ptr;  /* ncolours+1 offsets into order */
    const int32_t* order;       /* sites grouped by colour */
} orc_lattice;

/* One Metropolis sweep in colour order over an int8 state (Ising/Potts/BC/EA). */
void orc_sweep_int8(const orc_model* m, const orc_lattice* g, int8_t* s, double beta,
                    uint64_t seed, uint32_t replica, uint32_t sweep);
/* One Metropolis sweep over float state vectors (symd components AoS). */
void orc_sweep_f32(const orc_model* m, const orc_lattice* g, float* s, int symd,
                   double beta, uint64_t seed, uint32_t replica, uint32_t sweep);

/* Colour-order sweep of 2D Ising<int> on an L x L periodic lattice, neighbours
 * computed on the fly (for lattices too large for a neighbour list). */
void orc_ising2d_sweep(int32_t L, double J, int8_t* s, double beta, uint64_t seed, uint32_t replica,
                       uint32_t sweep);

/* Initial states from the INIT stream (reference initstatespace rules). */
void orc_init_int8(const orc_model* m, int32_t n, int8_t* s, uint64_t seed, uint32_t replica);
void orc_init_f32(const orc_model* m, int32_t n, float* s, int symd, uint64_t seed,
                  uint32_t replica);

/* One Wolff cluster with bond-keyed draws; returns cluster size. `serial` is
 * the global cluster counter. `work` must hold 2n int32. */
int32_t orc_wolff_int8(const orc_model* m, const orc_lattice* g, int8_t* s, double beta,
                       uint64_t seed, uint32_t replica, uint32_t serial, int32_t* work);
int32_t orc_wolff_f32(const orc_model* m, const orc_lattice* g, float* s, int symd,
                      double beta, uint64_t seed, uint32_t replica, uint32_t serial,
                      int32_t* work);

/* Observables of the reference (energy per site, |m|) plus m^2 and m^4 moments. */
typedef struct orc_obs { double e, m, m2, m4; } orc_obs;
void orc_measure_int8(const orc_model* m, const orc_lattice* g, const int8_t* s, orc_obs* out);
void orc_measure_f32(const orc_model* m, const orc_lattice* g, const float* s, int symd,
                     orc_obs* out);

/* Hypercubic lattice helpers: neighbour order +x,-x,+y,-y,... as the
 * reference's FixedDimRegularHypercubic::nbrs; colours by coordinate parity. */
void orc_hypercubic_csr(int dim, int len, int32_t* row_ptr, int32_t* col_idx);
void orc_parity_colours(int dim, int len, int32_t* colour_ptr, int32_t* order);

/* Known-answer test support: std::mt19937_64 words and the reference
 * acceptance test (testsuite/components/5-metro_exp.cpp) on the restated rule. */
void orc_mt19937_64_words(uint64_t seed, int64_t n, uint64_t* out);
int64_t orc_metro_exp(int32_t N, int32_t reps, double beta, uint8_t* decisions);

#ifdef __cplusplus
}
#endif
#endif
