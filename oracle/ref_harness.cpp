// Reference harness -- TEST INFRASTRUCTURE (builds oracle/_ref/libmarqov_ref.so).
//
// Compiles MARQOV's own hot-path templates from the reference source tree
// (include path given at build time) and drives them:
//   * MARQOV::Metropolis<H,L>::move (src/libmarqov/metropolis.h:88-126) over
//     the engine's colour order, with an RNGCache specialisation whose words
//     come from the keyed Philox stream (one substream per site and sweep);
//   * MARQOV::Wolff<H,L>::move (src/libmarqov/wolff.h:72-126 and the model
//     specialisations) on one sequential Philox substream per cluster, for
//     statistical comparison;
//   * the reference observables Energy / Magnetization / PottsMagnetization;
//   * the reference acceptance known-answer test
//     (testsuite/components/5-metro_exp.cpp) on RNGCache<std::mt19937_64>{0};
//   * the reference EMCS in its own random-site order on RNGCache<mt19937_64>
//     (src/libmarqov/emcs.h:69-109), single thread or one replica per thread,
//     as the CPU baseline.
// Nothing here is part of the engine; only tests and bench.py's reference
// arm load it.
#define CACHECONTAINER_H 1
#include <algorithm>
#include <array>
#include <chrono>
#include <numeric>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <thread>
#include <vector>

namespace H5 { struct Group {}; }
template <class... T> inline void dumpscalartoH5(T&&...) {}

namespace MARQOV {
// Minimal stand-in for MARQOV::Space (src/libmarqov/core.h:249-330): the
// embedders only need the type name and operator[].
template <class SV, class Grid>
class Space {
public:
    typedef Grid Lattice;
    typedef SV StateVector;
    using value_type = SV;
    explicit Space(std::size_t n) : v(n) {}
    SV& operator[](int j) { return v[j]; }
    const SV& operator[](int j) const { return v[j]; }
    std::size_t size() const { return v.size(); }
    std::vector<SV> v;
};
}  // namespace MARQOV

#include "libmarqov/rngcache.h"
#include "libmarqov/util/svmath.h"

extern "C" uint64_t orc_draw(uint64_t seed, uint32_t replica, uint32_t stream, uint32_t c0,
                             uint32_t c1, uint32_t k);

// Tag type: the keyed Philox stream.
struct PhiloxSite {};

extern "C" uint64_t orc_accept_word(uint64_t seed, uint32_t replica, uint32_t site, uint32_t sweep);

// RNGCache over the keyed Philox stream, with the interface and semantics of
// src/libmarqov/rngcache.h:156-206 (integer, integer(range), real(max,min)).
// In a Metropolis move the first `nprop` words are the proposal words of the
// site's substream and the next word is its acceptance word.
template <>
class RNGCache<PhiloxSite> {
public:
    uint64_t seed = 0;
    uint32_t replica = 0, stream = 0, c0 = 0, c1 = 0, k = 0;
    int nprop = -1;  // < 0: plain substream (no acceptance word)
    void rekey(uint32_t st, uint32_t a, uint32_t b, int np = -1) { stream = st; c0 = a; c1 = b; k = 0; nprop = np; }
    inline uint64_t integer() noexcept
    {
        if (nprop >= 0 && (int)k == nprop) {
            ++k;
            return orc_accept_word(seed, replica, c0, c1);
        }
        return orc_draw(seed, replica, stream, c0, c1, k++);
    }
    inline uint64_t integer(uint64_t range) noexcept { return integer() % range; }
    inline double real(double max = 1.0, double min = 0.0) noexcept
    {
        double ret = (integer() >> 11) * 0x1.0p-53;
        return min + (max - min) * ret;
    }
};

#include "libmarqov/metropolis.h"
#include "libmarqov/wolff.h"
#include "hamiltonian/Ising.h"
#include "hamiltonian/Potts.h"
#include "hamiltonian/Heisenberg.h"
#include "hamiltonian/Phi4.h"
#include "hamiltonian/BlumeCapel.h"
#include "hamiltonian/BlumeCapelBipartite.h"
#include "hamiltonian/XXZAntiferro.h"
#include "hamiltonian/XXZAntiferroSingleAniso.h"
#include "lattice/regular_hypercubic.h"

enum { ST_METRO = 1, ST_INIT = 2, ST_WOLFF_SEED = 3 };

// ---------------------------------------------------------------------------
// User-side plugins written in the reference API.

// A lattice given as CSR with optional per-bond weights: nbrs(a,i) and
// bnds(a,i) as the reference lattice concept (src/lattice/regular_random_bond.h:58-67).
struct CSRLattice {
    int n;
    const int32_t* rp;
    const int32_t* ci;
    std::vector<int> nb(int i) const { return std::vector<int>(ci + rp[i], ci + rp[i + 1]); }
    std::vector<int> nbrs(int, int i) const { return nb(i); }
    std::vector<int> flexnbrs(int, int i) const { return nb(i); }
    std::size_t size() const { return n; }
    std::vector<double> crds(int) const { return {0.0}; }
};
struct CSRBondLattice : CSRLattice {
    const int8_t* bd;
    std::vector<int> bnds(int, int i) const { return std::vector<int>(bd + rp[i], bd + rp[i + 1]); }
};

// Heisenberg with small-cap proposals: an Initializer specialisation.
struct HeisenbergCap : public Heisenberg<float, double> {
    explicit HeisenbergCap(double J) : Heisenberg<float, double>(J) {}
    static double cap;
};
double HeisenbergCap::cap = 0.9;
template <>
class Initializer<HeisenbergCap> {
public:
    template <class R>
    static std::array<float, 3> newsv(const std::array<float, 3>& o, R& rng)
    {
        double u0 = rng.real(), u1 = rng.real();
        double ca = 1.0 - u0 * (1.0 - HeisenbergCap::cap);
        double sa = std::sqrt(std::fmax(0.0, 1.0 - ca * ca));
        double ph = 2.0 * M_PI * u1;
        double dx = sa * std::cos(ph), dy = sa * std::sin(ph), dz = ca;
        double x = o[0], y = o[1], z = o[2];
        double sg = z < 0 ? -1.0 : 1.0;
        double a = 1.0 / (1.0 + sg * z);
        double bxy = -x * y * a;
        double e1[3] = {1.0 - x * x * a, bxy, -x * sg};
        double e2[3] = {bxy, 1.0 - y * y * a, -y * sg};
        double nv[3];
        for (int c = 0; c < 3; ++c) nv[c] = dx * e1[c] + dy * e2[c] + dz * (double)o[c];
        double nn = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
        return {(float)(nv[0] / nn), (float)(nv[1] / nn), (float)(nv[2] / nn)};
    }
};

// Scalar phi^4 (one component) in the reference's Phi4 form
// (src/hamiltonian/Phi4.h:84-121): J = -1, onsite mass/beta phi^2 and
// lambda/beta (phi^2-1)^2, shift proposal old + amp * real(-1,1).
struct Phi4Scalar {
    static constexpr int SymD = 1;
    typedef std::array<float, 1> StateVector;
    const double J = -1;
    double beta, lambda, mass;
    static double amp;
    Standard_Interaction<StateVector> inter{-1.0};
    Onsite_Quadratic<StateVector> q2;
    Onsite_Fourth_Minus_One<StateVector> q4;
    std::array<Standard_Interaction<StateVector>*, 1> interactions{&inter};
    std::vector<OnSite<StateVector, double>*> onsite;
    Phi4Scalar(double b, double l, double m) : beta(b), lambda(l), mass(m), q2(m / b), q4(l / b)
    {
        onsite.push_back(&q2);
        onsite.push_back(&q4);
    }
};
double Phi4Scalar::amp = 0.5;
template <>
class Initializer<Phi4Scalar> {
public:
    template <class R>
    static std::array<float, 1> newsv(const std::array<float, 1>& o, R& rng)
    {
        double r = rng.real(-1.0, 1.0);
        return {(float)((double)o[0] + Phi4Scalar::amp * r)};
    }
};

// Heisenberg whose clusters are the reference's generic Wolff<H,L>::move
// (src/libmarqov/wolff.h:72-126) driven by the reference's own
// Embedder<Heisenberg> (src/hamiltonian/Heisenberg.h:123-186: random unit
// rdir, coupling (s_i.r)(s_j.r), reflection about the plane normal to r,
// normalised).  The derived type only keeps the reference's Wolff<Heisenberg>
// specialisation (random Cartesian axis, Heisenberg.h:191-243) out of the
// way, and forwards the two-argument draw() the generic Wolff calls to the
// embedder's one-argument draw().
struct HeisenbergPlane : public Heisenberg<float, double> {
    explicit HeisenbergPlane(double J) : Heisenberg<float, double>(J) {}
};
namespace MARQOV {
template <class Lattice>
class Embedder<HeisenbergPlane, Lattice> : public Embedder<Heisenberg<float, double>, Lattice> {
    typedef Embedder<Heisenberg<float, double>, Lattice> Base;

public:
    Embedder(const HeisenbergPlane& h, const Lattice& l, Space<std::array<float, 3>, Lattice>& s) : Base(h, l, s) {}
    template <class RNG>
    void draw(RNG& rng, std::array<float, 3>&) { Base::draw(rng); }
};
// The scalar field's embedder, Embedder<Phi4> (src/hamiltonian/Phi4.h:182-244)
// for one component: rdir = set_to_rnddir of a one-component vector (+-1),
// coupling (s_i r)(s_j r), flip s -> s - 2 (s r) r, no normalisation.
template <class Lattice>
class Embedder<Phi4Scalar, Lattice> {
    typedef std::array<float, 1> SV;
    const Space<SV, Lattice>& ss;
    SV rdir;

public:
    Embedder(const Phi4Scalar&, const Lattice&, Space<SV, Lattice>& s) : ss(s) {}
    template <class RNG>
    void draw(RNG& rng, SV&) { set_to_rnddir(rng, rdir); }
    double coupling(int a, int b) const { return dot(ss[a], rdir) * dot(ss[b], rdir); }
    void flip(SV& sv)
    {
        const double d = dot(sv, rdir);
        sv[0] -= 2 * d * rdir[0];
    }
};
}  // namespace MARQOV

// ---------------------------------------------------------------------------
// Colour-order Metropolis through the reference templates.

// Proposal words drawn by Initializer<H>::newsv before the acceptance word.
template <class H> struct NProp { static constexpr int value = 0; };
template <> struct NProp<Potts<3>> { static constexpr int value = 1; };
template <> struct NProp<BlumeCapel<int>> { static constexpr int value = 1; };
template <> struct NProp<Heisenberg<float, double>> { static constexpr int value = 2; };
template <> struct NProp<Phi4Scalar> { static constexpr int value = 1; };

template <class H, class L, class SS>
static void colour_sweep(const H& ham, const L& grid, SS& ss, RNGCache<PhiloxSite>& rng, double beta,
                         uint32_t sweep, int ncol, const int32_t* cptr, const int32_t* order, int nprop)
{
    for (int c = 0; c < ncol; ++c)
        for (int32_t p = cptr[c]; p < cptr[c + 1]; ++p) {
            const int i = order[p];
            rng.rekey(ST_METRO, (uint32_t)i, sweep, nprop);
            MARQOV::Metropolis<H, L>::move(ham, grid, ss, rng, beta, i);
        }
}

// A lattice with SimpleBipartite's termselector (src/lattice/simple_bipartite.h:38-41):
// site i takes only onsite term sub[i] (its sublattice).
struct CSRTermLattice : CSRLattice {
    const uint8_t* sub;
    std::vector<int> termselector(int i) const { return {(int)sub[i]}; }
};
struct CSRBondTermLattice : CSRBondLattice {
    const uint8_t* sub;
    std::vector<int> termselector(int i) const { return {(int)sub[i]}; }
};

// Energy per site as the reference's Metropolis moves see it, through the
// reference's own helpers: J/(2N) sum_i dot(get(s_i), nbrhoodloop(i)), with
// the lattice's bonds when it has them (src/libmarqov/metropolishelpers.h:
// 456-537), plus the SelfEnergy observable.  It equals Energy<H> on lattices
// without bonds; Energy<H> itself never reads bnds() (observables.h:186-217).
template <class H, class L, class SS>
static double nbrhood_energy(const H& ham, const L& lat, const SS& ss)
{
    typedef typename MARQOV::has_bnds<L>::type HB;
    const int n = (int)lat.size();
    double part = 0.0;
    for (int i = 0; i < n; ++i) {
        auto nb = MARQOV::nbrhoodloop<L, H, SS>(lat, ham, ss, 0, i, std::true_type(), HB());
        part += dot(ham.interactions[0]->get(ss[i]), nb);
    }
    SelfEnergy<H> se(ham);
    return ham.interactions[0]->J * part / double(2 * n) + se.measure(ss, lat);
}

// Potts energy as its Metropolis moves see it: k/(2N) sum_i #{j in nbrs(i):
// s_j = s_i}, each count taken from the reference's PottsInteraction::diff
// with an old state no neighbour holds (src/hamiltonian/Potts.h:86-107).
// Energy<Potts<Q>> reads 0: PottsInteraction::energy is a stub (Potts.h:108-109).
template <class L, class SS>
static double potts_energy(const Potts<3>& ham, const L& lat, SS& ss)
{
    const int n = (int)lat.size();
    double cnt = 0.0;
    std::array<int, 1> none{{-1}};
    for (int i = 0; i < n; ++i)
        cnt += const_cast<Potts<3>&>(ham).potts_interaction.diff(i, none, ss[i], lat.nbrs(0, i), ss);
    return ham.potts_interaction.k * cnt / double(2 * n);
}

// Runs nsweeps colour-ordered sweeps of the reference Metropolis on ss and
// writes per sweep (e, m, e_obs): e the energy per site the moves see, m the
// model's magnetization observable, e_obs the reference's Energy<H> observable.
template <class H, class L, class SS, class EFn, class MFn>
static void run_sweeps(const H& ham, const L& lat, SS& ss, RNGCache<PhiloxSite>& rng, double beta, uint32_t sweep0,
                       int nsweeps, int ncol, const int32_t* cptr, const int32_t* order, int nprop, EFn efn,
                       MFn mfn, double* obs)
{
    for (int t = 0; t < nsweeps; ++t) {
        colour_sweep(ham, lat, ss, rng, beta, sweep0 + t, ncol, cptr, order, nprop);
        if (obs) {
            Energy<H> eo(ham);
            obs[3 * t] = efn(ss);
            obs[3 * t + 1] = mfn(ss);
            obs[3 * t + 2] = eo.measure(ss, lat);
        }
    }
}

template <class SV, class L, class T>
static void load_state(MARQOV::Space<SV, L>& ss, const T* s, int n)
{
    constexpr int D = std::tuple_size<SV>::value;
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < D; ++c) ss[i][c] = s[(size_t)i * D + c];
}
template <class SV, class L, class T>
static void store_state(const MARQOV::Space<SV, L>& ss, T* s, int n)
{
    constexpr int D = std::tuple_size<SV>::value;
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < D; ++c) s[(size_t)i * D + c] = (T)ss[i][c];
}

template <class H, class L>
static void int_model(const H& ham, const L& lat, int8_t* spins, RNGCache<PhiloxSite>& rng, double beta,
                      uint32_t sweep0, int nsweeps, int ncol, const int32_t* cptr, const int32_t* order, int nprop,
                      double* obs)
{
    const int n = (int)lat.size();
    MARQOV::Space<std::array<int, 1>, L> ss(n);
    load_state(ss, spins, n);
    auto ef = [&](const MARQOV::Space<std::array<int, 1>, L>& x) { return nbrhood_energy(ham, lat, x); };
    auto mf = [&](const MARQOV::Space<std::array<int, 1>, L>& x) { return Magnetization().measure(x, lat); };
    run_sweeps(ham, lat, ss, rng, beta, sweep0, nsweeps, ncol, cptr, order, nprop, ef, mf, obs);
    store_state(ss, spins, n);
}

template <class H, class L>
static void f32_model(const H& ham, const L& lat, float* s, RNGCache<PhiloxSite>& rng, double beta,
                      uint32_t sweep0, int nsweeps, int ncol, const int32_t* cptr, const int32_t* order, int nprop,
                      double* obs)
{
    typedef typename H::StateVector SV;
    const int n = (int)lat.size();
    MARQOV::Space<SV, L> ss(n);
    load_state(ss, s, n);
    auto ef = [&](const MARQOV::Space<SV, L>& x) { return nbrhood_energy(ham, lat, x); };
    auto mf = [&](const MARQOV::Space<SV, L>& x) { return Magnetization().measure(x, lat); };
    run_sweeps(ham, lat, ss, rng, beta, sweep0, nsweeps, ncol, cptr, order, nprop, ef, mf, obs);
    store_state(ss, s, n);
}

extern "C" {

// Metropolis sweeps for int8-state models.  kind: 1 Ising<int>, 3 Potts<3>,
// 4 BlumeCapel<int>(J, D), 5 Ising with bonds (EdwardsAndersonIsing form),
// 11 BlumeCapelBipartite<int>(J, D, D2).  sub (optional): per-site
// sublattice, giving the lattice SimpleBipartite's termselector.  obs
// (optional): per sweep (e, m, e_obs) as run_sweeps.
int ref_sweeps_int(int kind, int n, const int32_t* rp, const int32_t* ci, const int8_t* bonds, const uint8_t* sub,
                   int ncol, const int32_t* cptr, const int32_t* order, int8_t* spins,
                   double J, double D, double D2, double beta, uint64_t seed, uint32_t replica,
                   uint32_t sweep0, int nsweeps, double* obs)
{
    RNGCache<PhiloxSite> rng;
    rng.seed = seed;
    rng.replica = replica;
    CSRLattice lat{n, rp, ci};
    CSRTermLattice tlat;
    tlat.n = n; tlat.rp = rp; tlat.ci = ci; tlat.sub = sub;
    if (kind == 1) {
        Ising<int> ham(J);
        int_model(ham, lat, spins, rng, beta, sweep0, nsweeps, ncol, cptr, order, 0, obs);
    } else if (kind == 3) {
        Potts<3> ham(J);
        MARQOV::Space<std::array<int, 1>, CSRLattice> ss(n);
        load_state(ss, spins, n);
        auto ef = [&](MARQOV::Space<std::array<int, 1>, CSRLattice>& x) { return potts_energy(ham, lat, x); };
        auto mf = [&](MARQOV::Space<std::array<int, 1>, CSRLattice>& x) { return PottsMagnetization<3>().measure(x, lat); };
        run_sweeps(ham, lat, ss, rng, beta, sweep0, nsweeps, ncol, cptr, order, NProp<Potts<3>>::value, ef, mf, obs);
        store_state(ss, spins, n);
    } else if (kind == 4) {
        BlumeCapel<int> ham(J, D);
        if (sub) int_model(ham, tlat, spins, rng, beta, sweep0, nsweeps, ncol, cptr, order, 1, obs);
        else int_model(ham, lat, spins, rng, beta, sweep0, nsweeps, ncol, cptr, order, 1, obs);
    } else if (kind == 11) {
        BlumeCapelBipartite<int> ham(J, D, D2);
        if (sub) int_model(ham, tlat, spins, rng, beta, sweep0, nsweeps, ncol, cptr, order, 1, obs);
        else int_model(ham, lat, spins, rng, beta, sweep0, nsweeps, ncol, cptr, order, 1, obs);
    } else if (kind == 5) {
        CSRBondLattice blat;
        blat.n = n; blat.rp = rp; blat.ci = ci; blat.bd = bonds;
        Ising<int> ham(J);
        int_model(ham, blat, spins, rng, beta, sweep0, nsweeps, ncol, cptr, order, 0, obs);
    } else {
        return -1;
    }
    return 0;
}

// Initial state by the reference's own rules, one INIT substream per site:
// Ising::initstatespace (src/hamiltonian/Ising.h:99-107) for kind 1,
// Potts<3>::initstatespace (src/hamiltonian/Potts.h:149-156) for 3, and for
// 4 (BlumeCapel, which has no initstatespace) Core::init_hot's
// set_to_rnddir of a one-component integer state (src/libmarqov/core.h:773-782).
int ref_init_int(int kind, int n, uint64_t seed, uint32_t replica, int8_t* out)
{
    RNGCache<PhiloxSite> rng;
    rng.seed = seed;
    rng.replica = replica;
    FixedDimRegularHypercubic<1> one(1);
    for (int i = 0; i < n; ++i) {
        rng.rekey(ST_INIT, (uint32_t)i, 0);
        MARQOV::Space<std::array<int, 1>, FixedDimRegularHypercubic<1>> ss(1);
        if (kind == 1) Ising<int>(-1.0).initstatespace(ss, one, rng);
        else if (kind == 3) Potts<3>(-1.0).initstatespace(ss, one, rng);
        else if (kind == 4) set_to_rnddir(rng, ss[0]);
        else return -1;
        out[i] = (int8_t)ss[0][0];
    }
    return 0;
}

// Metropolis sweeps for float-state models. kind: 6 Heisenberg<float> with
// the reference's fresh-direction proposal, 7 Heisenberg small-cap (cap =
// cos of the cap half-angle), 8 scalar phi^4 (p0 = lambda, p1 = mass,
// cap = shift amplitude), 9 XXZAntiferro<float>(Delta = p0, H = p1),
// 10 XXZAntiferroSingleAniso<float>(H = p1, Delta = p0, D = p2).  sub
// (optional): per-site sublattice (SimpleBipartite's termselector).  obs
// (optional): per sweep (e, m, e_obs) as run_sweeps.
int ref_sweeps_f32(int kind, int n, const int32_t* rp, const int32_t* ci, const uint8_t* sub, int ncol,
                   const int32_t* cptr, const int32_t* order, float* s, double J, double p0,
                   double p1, double p2, double cap, double beta, uint64_t seed, uint32_t replica,
                   uint32_t sweep0, int nsweeps, double* obs)
{
    RNGCache<PhiloxSite> rng;
    rng.seed = seed;
    rng.replica = replica;
    CSRLattice lat{n, rp, ci};
    CSRTermLattice tlat;
    tlat.n = n; tlat.rp = rp; tlat.ci = ci; tlat.sub = sub;
    if (kind == 6) {
        Heisenberg<float, double> ham(J);
        f32_model(ham, lat, s, rng, beta, sweep0, nsweeps, ncol, cptr, order, 2, obs);
    } else if (kind == 7) {
        HeisenbergCap::cap = cap;
        HeisenbergCap ham(J);
        f32_model(ham, lat, s, rng, beta, sweep0, nsweeps, ncol, cptr, order, 2, obs);
    } else if (kind == 8) {
        Phi4Scalar::amp = cap;
        Phi4Scalar ham(beta, p0, p1);
        if (sub) f32_model(ham, tlat, s, rng, beta, sweep0, nsweeps, ncol, cptr, order, 1, obs);
        else f32_model(ham, lat, s, rng, beta, sweep0, nsweeps, ncol, cptr, order, 1, obs);
    } else if (kind == 9) {
        XXZAntiferro<float> ham(p0, p1);
        if (sub) f32_model(ham, tlat, s, rng, beta, sweep0, nsweeps, ncol, cptr, order, 2, obs);
        else f32_model(ham, lat, s, rng, beta, sweep0, nsweeps, ncol, cptr, order, 2, obs);
    } else if (kind == 10) {
        XXZAntiferroSingleAniso<float> ham(p1, p0, p2);
        if (sub) f32_model(ham, tlat, s, rng, beta, sweep0, nsweeps, ncol, cptr, order, 2, obs);
        else f32_model(ham, lat, s, rng, beta, sweep0, nsweeps, ncol, cptr, order, 2, obs);
    } else {
        return -1;
    }
    return 0;
}

// Unmodified reference Wolff clusters (Wolff<Ising<int>> and Wolff<Potts<3>>)
// on a sequential Philox substream per cluster. Returns the cluster sizes.
int ref_wolff_int(int kind, int n, const int32_t* rp, const int32_t* ci, int8_t* spins, double J,
                  double beta, uint64_t seed, uint32_t replica, uint32_t serial0, int nclusters,
                  int32_t* sizes)
{
    RNGCache<PhiloxSite> rng;
    rng.seed = seed;
    rng.replica = replica;
    CSRLattice lat{n, rp, ci};
    MARQOV::Space<std::array<int, 1>, CSRLattice> ss(n);
    for (int i = 0; i < n; ++i) ss[i][0] = spins[i];
    if (kind == 1) {
        Ising<int> ham(J);
        MARQOV::Wolff<Ising<int>, CSRLattice> w;
        for (int c = 0; c < nclusters; ++c) {
            rng.rekey(ST_WOLFF_SEED, 0, serial0 + c);
            int site = (int)rng.integer(n);
            sizes[c] = w.move(ham, lat, ss, rng, beta, site);
        }
    } else if (kind == 3) {
        Potts<3> ham(J);
        MARQOV::Wolff<Potts<3>, CSRLattice> w;
        for (int c = 0; c < nclusters; ++c) {
            rng.rekey(ST_WOLFF_SEED, 0, serial0 + c);
            int site = (int)rng.integer(n);
            sizes[c] = w.move(ham, lat, ss, rng, beta, site);
        }
    } else {
        return -1;
    }
    for (int i = 0; i < n; ++i) spins[i] = (int8_t)ss[i][0];
    return 0;
}

// Unmodified generic Wolff<H,L>::move (src/libmarqov/wolff.h:72-126) for the
// float models on a sequential Philox substream per cluster: kind 6 with the
// reference's Embedder<Heisenberg> (HeisenbergPlane), kind 8 with the scalar
// Embedder<Phi4> (p0 = lambda, p1 = mass: they do not enter the clusters).
// s: site-major float state, updated in place; sizes: the cluster sizes.
int ref_wolff_f32(int kind, int n, const int32_t* rp, const int32_t* ci, float* s, double J, double p0, double p1,
                  double beta, uint64_t seed, uint32_t replica, uint32_t serial0, int nclusters, int32_t* sizes)
{
    RNGCache<PhiloxSite> rng;
    rng.seed = seed;
    rng.replica = replica;
    CSRLattice lat{n, rp, ci};
    if (kind == 6) {
        HeisenbergPlane ham(J);
        MARQOV::Space<std::array<float, 3>, CSRLattice> ss(n);
        load_state(ss, s, n);
        MARQOV::Wolff<HeisenbergPlane, CSRLattice> w;
        for (int c = 0; c < nclusters; ++c) {
            rng.rekey(ST_WOLFF_SEED, 0, serial0 + c);
            const int site = (int)rng.integer(n);
            sizes[c] = w.move(ham, lat, ss, rng, beta, site);
        }
        store_state(ss, s, n);
    } else if (kind == 8) {
        Phi4Scalar ham(beta, p0, p1);
        MARQOV::Space<std::array<float, 1>, CSRLattice> ss(n);
        load_state(ss, s, n);
        MARQOV::Wolff<Phi4Scalar, CSRLattice> w;
        for (int c = 0; c < nclusters; ++c) {
            rng.rekey(ST_WOLFF_SEED, 0, serial0 + c);
            const int site = (int)rng.integer(n);
            sizes[c] = w.move(ham, lat, ss, rng, beta, site);
        }
        store_state(ss, s, n);
    } else {
        return -1;
    }
    return 0;
}

// testsuite/components/5-metro_exp.cpp, decision by decision: dE = 10 real()
// for N words of RNGCache<std::mt19937_64>{0}, then `reps` passes of
// MARQOV::metro_update_accepted at beta.  decisions[r*N+i] receives each
// accept bit (when non-NULL); the return value is the accept count.
long long ref_metro_exp(int N, int reps, double beta, double* dE, uint8_t* decisions)
{
    RNGCache<std::mt19937_64> rc{0};
    for (int i = 0; i < N; ++i) dE[i] = 10.0 * rc.real();
    long long acc = 0;
    for (int r = 0; r < reps; ++r)
        for (int i = 0; i < N; ++i) {
            bool a = MARQOV::metro_update_accepted(dE[i], beta, rc);
            acc += a;
            if (decisions) decisions[(size_t)r * N + i] = a;
        }
    return acc;
}

// The first n words of RNGCache<std::mt19937_64>{0}.
void ref_mt_words(long long n, uint64_t* out)
{
    RNGCache<std::mt19937_64> rc{0};
    for (long long i = 0; i < n; ++i) out[i] = rc.integer();
}

// Plain-exp count of the same test (the "OLD" branch of 5-metro_exp.cpp).
long long ref_metro_exp_plain(int N, int reps, double beta)
{
    RNGCache<std::mt19937_64> rc{0};
    std::vector<double> dE(N);
    for (int i = 0; i < N; ++i) dE[i] = 10.0 * rc.real();
    long long acc = 0;
    for (int r = 0; r < reps; ++r)
        for (int i = 0; i < N; ++i) acc += (dE[i] <= 0) || (rc.real() < std::exp(-beta * dE[i]));
    return acc;
}

}  // extern "C"

// The reference rule evaluated on one explicit word (the template reads one
// word from an RNGCache; a one-word cache supplies it).
struct OneWordEngine {};

template <>
class RNGCache<OneWordEngine> {
public:
    uint64_t w = 0;
    inline uint64_t integer() noexcept { return w; }
    inline uint64_t integer(uint64_t r) noexcept { return w % r; }
    inline double real(double max = 1.0, double min = 0.0) noexcept
    {
        double ret = (w >> 11) * 0x1.0p-53;
        return min + (max - min) * ret;
    }
};

extern "C" {
int ref_update_accepted(int pref, double dE, double beta, uint64_t word)
{
    RNGCache<OneWordEngine> r;
    r.w = word;
    if (pref == 1) return MARQOV::update_accepted<1>(dE, beta, r) ? 1 : 0;
    return MARQOV::update_accepted<2>(dE, beta, r) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// CPU baseline: the reference EMCS Metropolis loop (src/libmarqov/emcs.h:93-105)
// in its own random-site order on RNGCache<std::mt19937_64>, 2D Ising<int8_t>
// on FixedDimRegularHypercubic<2>.  A farm holds nthreads independent
// replicas, one per thread, as CXX11Scheduler farms simulations
// (src/libmarqov/marqovscheduler.h:281-285); one farm step runs `nupdates`
// random-site updates on every replica in parallel.

struct Farm {
    typedef FixedDimRegularHypercubic<2> G;
    typedef MARQOV::Space<std::array<int8_t, 1>, G> SS;
    int len;
    double beta;
    G grid;
    Ising<int8_t> ham{-1.0};
    std::vector<std::unique_ptr<SS>> states;
    std::vector<std::unique_ptr<RNGCache<std::mt19937_64>>> rngs;
    Farm(int l, double b) : len(l), beta(b), grid(l) {}
};

static void farm_run(Farm* f, int t, long long nupdates)
{
    auto& ss = *f->states[t];
    auto& rng = *f->rngs[t];
    const int N = (int)f->grid.size();
    for (long long i = 0; i < nupdates; ++i) {
        const int rsite = rng.integer(N);
        MARQOV::Metropolis<Ising<int8_t>, Farm::G>::move(f->ham, f->grid, ss, rng, f->beta, rsite);
    }
}

void* ref_farm_create(int len, double beta, int nthreads, uint64_t seed)
{
    Farm* f = new Farm(len, beta);
    f->states.resize(nthreads);
    f->rngs.resize(nthreads);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([f, t, seed]() {
            f->states[t].reset(new Farm::SS(f->grid.size()));
            f->rngs[t].reset(new RNGCache<std::mt19937_64>(seed + 7919u * (unsigned)t));
            f->ham.initstatespace(*f->states[t], f->grid, *f->rngs[t]);
        });
    for (auto& x : th) x.join();
    return f;
}

// Runs one step; returns its wall time in seconds.
double ref_farm_step(void* h, long long nupdates)
{
    Farm* f = (Farm*)h;
    const int n = (int)f->states.size();
    auto t0 = std::chrono::steady_clock::now();
    if (n == 1) {
        farm_run(f, 0, nupdates);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < n; ++t) th.emplace_back(farm_run, f, t, nupdates);
        for (auto& x : th) x.join();
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Magnetisation sum of replica t (keeps the work observable).
long long ref_farm_magnetisation(void* h, int t)
{
    Farm* f = (Farm*)h;
    long long m = 0;
    for (auto& v : f->states[t]->v) m += v[0];
    return m;
}

void ref_farm_destroy(void* h) { delete (Farm*)h; }

// The reference's own EMCS (the loop of src/libmarqov/emcs.h:69-109: ncluster
// Wolff<Ising<int>> clusters seeded at rng.integer(N), then N random-site
// Metropolis<Ising<int>> moves per sweep) for the 2D Ising model on
// FixedDimRegularHypercubic<2> with RNGCache<mt19937_64>, from the
// reference's initstatespace; obs receives (Energy, Magnetization) after each
// of the nmeas measured EMCS, mean_cluster the mean cluster size per EMCS.
int ref_emcs_ising2d(int len, double J, double beta, uint64_t seed, int ncluster, int nmetro, int ntherm,
                     int nmeas, double* obs, double* mean_cluster)
{
    typedef FixedDimRegularHypercubic<2> G;
    G grid(len);
    Ising<int> ham(J);
    MARQOV::Space<std::array<int, 1>, G> ss(grid.size());
    RNGCache<std::mt19937_64> rng(seed);
    ham.initstatespace(ss, grid, rng);
    MARQOV::Wolff<Ising<int>, G> wolff;
    const int N = (int)grid.size();
    for (int t = 0; t < ntherm + nmeas; ++t) {
        double avg = 0;
        for (int c = 0; c < ncluster; ++c) {
            const int site = rng.integer(N);
            avg += (double)wolff.move(ham, grid, ss, rng, beta, site);
        }
        for (int j = 0; j < nmetro; ++j)
            for (int i = 0; i < N; ++i) {
                const int rsite = rng.integer(N);
                MARQOV::Metropolis<Ising<int>, G>::move(ham, grid, ss, rng, beta, rsite);
            }
        if (t >= ntherm) {
            const int k = t - ntherm;
            Magnetization mo;
            Energy<Ising<int>> eo(ham);
            obs[2 * k] = eo.measure(ss, grid);
            obs[2 * k + 1] = mo.measure(ss, grid);
            if (mean_cluster) mean_cluster[k] = ncluster ? avg / ncluster : 0.0;
        }
    }
    return 0;
}

}  // extern "C"

// The reference's own EMCS loop (src/libmarqov/emcs.h:69-109: ncluster
// Wolff clusters seeded at rng.integer(N), then nmetro x N random-site
// Metropolis moves) on RegularHypercubic(len, dim) with
// RNGCache<mt19937_64>, for the models other than Ising:
//   kind 3: Potts<3>(J), Wolff<Potts<3>>, initstatespace of Potts<3>;
//   kind 6: Heisenberg<float> (J) with fresh-direction proposals and the
//           generic Wolff over Embedder<Heisenberg> (HeisenbergPlane),
//           Heisenberg::initstatespace;
//   kind 8: scalar phi^4 (p0 = lambda, p1 = mass, p2 = shift amplitude) with
//           its embedder, phi_i started from N(0, 1) (Box-Muller on real()).
// obs receives per measured EMCS (e, |m|): the energy the moves see
// (potts_energy / nbrhood_energy) and the magnetization observable;
// mean_cluster the mean cluster size per EMCS.
template <class H, class G, class SS, class EFn, class MFn>
static void generic_emcs(const H& ham, const G& grid, SS& ss, RNGCache<std::mt19937_64>& rng, double beta, int ncluster,
                         int nmetro, int ntherm, int nmeas, EFn efn, MFn mfn, double* obs, double* mean_cluster)
{
    MARQOV::Wolff<H, G> wolff;
    const int N = (int)grid.size();
    for (int t = 0; t < ntherm + nmeas; ++t) {
        double avg = 0;
        for (int c = 0; c < ncluster; ++c) {
            const int site = rng.integer(N);
            avg += (double)wolff.move(ham, grid, ss, rng, beta, site);
        }
        for (int j = 0; j < nmetro; ++j)
            for (int i = 0; i < N; ++i) {
                const int rsite = rng.integer(N);
                MARQOV::Metropolis<H, G>::move(ham, grid, ss, rng, beta, rsite);
            }
        if (t >= ntherm) {
            const int k = t - ntherm;
            obs[2 * k] = efn(ss);
            obs[2 * k + 1] = mfn(ss);
            if (mean_cluster) mean_cluster[k] = ncluster ? avg / ncluster : 0.0;
        }
    }
}

extern "C" int ref_emcs_generic(int kind, int len, int dim, double J, double p0, double p1, double p2, double beta,
                                uint64_t seed, int ncluster, int nmetro, int ntherm, int nmeas, double* obs,
                                double* mean_cluster)
{
    typedef RegularHypercubic G;
    G grid(len, dim);
    const int N = (int)grid.size();
    RNGCache<std::mt19937_64> rng(seed);
    if (kind == 3) {
        Potts<3> ham(J);
        MARQOV::Space<std::array<int, 1>, G> ss(N);
        ham.initstatespace(ss, grid, rng);
        auto ef = [&](MARQOV::Space<std::array<int, 1>, G>& x) { return potts_energy(ham, grid, x); };
        auto mf = [&](MARQOV::Space<std::array<int, 1>, G>& x) { return PottsMagnetization<3>().measure(x, grid); };
        generic_emcs(ham, grid, ss, rng, beta, ncluster, nmetro, ntherm, nmeas, ef, mf, obs, mean_cluster);
    } else if (kind == 6) {
        HeisenbergPlane ham(J);
        MARQOV::Space<std::array<float, 3>, G> ss(N);
        ham.initstatespace(ss, grid, rng);
        auto ef = [&](MARQOV::Space<std::array<float, 3>, G>& x) { return nbrhood_energy(ham, grid, x); };
        auto mf = [&](MARQOV::Space<std::array<float, 3>, G>& x) { return Magnetization().measure(x, grid); };
        generic_emcs(ham, grid, ss, rng, beta, ncluster, nmetro, ntherm, nmeas, ef, mf, obs, mean_cluster);
    } else if (kind == 8) {
        Phi4Scalar::amp = p2;
        Phi4Scalar ham(beta, p0, p1);
        MARQOV::Space<std::array<float, 1>, G> ss(N);
        for (int i = 0; i < N; ++i) {
            const double u0 = rng.real(), u1 = rng.real();
            ss[i][0] = (float)(std::sqrt(-2.0 * std::log(1.0 - u0)) * std::cos(2.0 * M_PI * u1));
        }
        auto ef = [&](MARQOV::Space<std::array<float, 1>, G>& x) { return nbrhood_energy(ham, grid, x); };
        auto mf = [&](MARQOV::Space<std::array<float, 1>, G>& x) { return Magnetization().measure(x, grid); };
        generic_emcs(ham, grid, ss, rng, beta, ncluster, nmetro, ntherm, nmeas, ef, mf, obs, mean_cluster);
    } else {
        return -1;
    }
    return 0;
}

// The reference's Wolff<Ising<int>> (src/hamiltonian/Ising.h:122-169) on
// FixedDimRegularHypercubic<2>(len) with RNGCache<mt19937_64>: ntherm EMCS of
// one cluster + one random-site sweep from initstatespace, then nclusters
// clusters alone, timed.  Writes the seconds and the summed cluster size.
extern "C" int ref_wolff_ising2d(int len, double beta, uint64_t seed, int ntherm, int nclusters, double* seconds,
                                 double* total)
{
    typedef FixedDimRegularHypercubic<2> G;
    G grid(len);
    Ising<int> ham(-1.0);
    MARQOV::Space<std::array<int, 1>, G> ss(grid.size());
    RNGCache<std::mt19937_64> rng(seed);
    ham.initstatespace(ss, grid, rng);
    MARQOV::Wolff<Ising<int>, G> wolff;
    const int N = (int)grid.size();
    for (int t = 0; t < ntherm; ++t) {
        wolff.move(ham, grid, ss, rng, beta, rng.integer(N));
        for (int i = 0; i < N; ++i) MARQOV::Metropolis<Ising<int>, G>::move(ham, grid, ss, rng, beta, rng.integer(N));
    }
    double tot = 0;
    const auto t0 = std::chrono::steady_clock::now();
    for (int c = 0; c < nclusters; ++c) tot += wolff.move(ham, grid, ss, rng, beta, rng.integer(N));
    const auto t1 = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(t1 - t0).count();
    *total = tot;
    return 0;
}
