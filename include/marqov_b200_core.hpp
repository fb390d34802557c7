/*
 * marqov_b200 -- header-only C++ host layer over the C ABI.
 *
 * Mirrors the public face of MARQOV's Core so that a program built on the
 * reference switches by replacing makeCore with makeGPUCore:
 *   makeCore<L,H>(std::tuple<L&, Config, std::tuple<beta, HArgs...>>)
 *                                            src/libmarqov/core.h:1223-1229
 *   Core::init / wrmploop / gameloop / elementaryMCstep
 *                                            src/libmarqov/core.h:829-834,1001-1050
 *   CXX11Scheduler::createSimfromParameter / start
 *                                            src/libmarqov/marqovscheduler.h:75-144,223-273
 * A Hamiltonian reaches the engine through ModelLowering<H> and a lattice
 * through LatticeLowering<L>: hypercubic lattices (HypercubicShape<L>) take
 * the stencil path, any other lattice with nbrs() is lowered to CSR once (with
 * its bnds() when it has them).  marqov_b200_marqov.hpp provides the
 * specialisations for MARQOV's own classes; user classes add their own.
 * The Config type is any type with MARQOV::Config's fields (seed, repid,
 * ncluster, nmetro, warmupsteps, gameloopsteps).
 */
#ifndef MARQOV_B200_CORE_HPP
#define MARQOV_B200_CORE_HPP

#include <cstddef>
#include <cstdint>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "marqov_b200.h"

namespace marqov_b200 {

// Every failing C-ABI call becomes this exception (status + message).
struct Error : std::runtime_error {
    mqv_status status;
    Error(mqv_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(mqv_status s)
{
    if (s == MQV_OK) return;
    char m[512];
    mqv_last_error(m, sizeof m);
    throw Error(s, std::string("[marqov_b200] ") + m);
}

// ---- generic lowering of a Hamiltonian by its term objects -----------------
//
// A Hamiltonian written against MARQOV's term API (interactions / onsite /
// multisite containers of term objects with get(), J, h, k;
// src/hamiltonian/util/hamparts.h:27-104) is lowered without a
// specialisation: the containers are found with the reference's detection
// rules (HasInteractions / HasOnsite / HasFlexTerms,
// src/libmarqov/metropolishelpers.h:203-288), and each term is recognised by
// probing its get() -- a linear interaction diagonal in the components
// (weights (1, ..., 1): the standard interaction; (Delta, Delta, 1): XXZ),
// onsite terms s^2, (s^2 - 1)^2, s_z or s_z^2.  A term of any other shape
// gives kind 0, which mqv_create refuses with MQV_ERR_UNSUPPORTED_TERM (no CPU
// fallback).  The Metropolis proposal is the model's Initializer<H>
// (ProposalOf<H>; the default of its state type unless specialised).
namespace detail {
template <class T, class = int>
struct has_interactions : std::false_type {};
template <class T>
struct has_interactions<T, decltype((void)T::interactions, 0)> : std::true_type {};
template <class T, class = int>
struct has_onsite : std::false_type {};
template <class T>
struct has_onsite<T, decltype((void)T::onsite, 0)> : std::true_type {};
template <class T, class = int>
struct has_multisite : std::false_type {};
template <class T>
struct has_multisite<T, decltype((void)T::multisite, 0)> : std::true_type {};
template <class T, class = int>
struct has_q : std::false_type {};
template <class T>
struct has_q<T, decltype((void)T::q, 0)> : std::true_type {};

template <class SV>
SV unit(int c, double v)
{
    SV x{};
    x[c] = (typename SV::value_type)v;
    return x;
}

// weights of an interaction term whose get() is linear and diagonal in the
// components; false for any other shape
template <class SV, class T>
bool diagonal_weights(T* t, double* w)
{
    constexpr int D = (int)std::tuple_size<SV>::value;
    for (int c = 0; c < D; ++c) {
        const SV g1 = t->get(unit<SV>(c, 1.0)), g2 = t->get(unit<SV>(c, 2.0));
        for (int d = 0; d < D; ++d)
            if (d != c && ((double)g1[d] != 0.0 || (double)g2[d] != 0.0)) return false;
        w[c] = (double)g1[c];
        if ((double)g2[c] != 2.0 * w[c]) return false;
    }
    return true;
}

enum OnsiteShape { kOnsiteOther = 0, kOnsiteSq, kOnsiteQuartic, kOnsiteZ, kOnsiteZ2 };

// shape of an onsite term from its values at a few states
template <class SV, class T>
int onsite_shape(T* t)
{
    constexpr int D = (int)std::tuple_size<SV>::value;
    auto f = [&](const SV& v) { return (double)t->get(v); };
    if (D == 1) {
        const double a = f(unit<SV>(0, 0.0)), b = f(unit<SV>(0, 1.0)), c = f(unit<SV>(0, -1.0)), d = f(unit<SV>(0, 2.0));
        if (a == 0 && b == 1 && c == 1 && d == 4) return kOnsiteSq;
        if (a == 1 && b == 0 && c == 0 && d == 9) return kOnsiteQuartic;
        return kOnsiteOther;
    }
    if (D == 3) {
        const double x = f(unit<SV>(0, 1.0)), y = f(unit<SV>(1, 1.0)), z = f(unit<SV>(2, 1.0)), z2 = f(unit<SV>(2, 2.0)),
                     zm = f(unit<SV>(2, -1.0)), o = f(SV{});
        if (o == 0 && x == 0 && y == 0 && z == 1 && z2 == 2 && zm == -1) return kOnsiteZ;
        if (o == 0 && x == 0 && y == 0 && z == 1 && z2 == 4 && zm == 1) return kOnsiteZ2;
    }
    return kOnsiteOther;
}

template <class C>
std::size_t size_of(const C& c)
{
    return c.size();
}
}  // namespace detail

// The Metropolis proposal of Initializer<H>: specialise value for models
// whose Initializer is not the default of their state type
// (marqov_b200_marqov.hpp does so from the reference's initializer classes).
enum { kProposalDefault = 0, kProposalSpin1 = 1, kProposalPottsQ = 2, kProposalShift = 3 };
template <class H, class Enable = void>
struct ProposalOf {
    static constexpr int value = kProposalDefault;
};

template <class H>
void lower_inter(const H& h, double& J, double* w, int& n, bool& ok, std::true_type)
{
    typedef typename H::StateVector SV;
    n = (int)detail::size_of(h.interactions);
    if (n >= 1) {
        J = (double)h.interactions[0]->J;
        ok = detail::diagonal_weights<SV>(h.interactions[0], w);
    }
}
template <class H>
void lower_inter(const H&, double&, double*, int& n, bool&, std::false_type)
{
    n = 0;
}
template <class H>
bool lower_onsite(const H& h, int* shapes, double* coef, int& n, std::true_type)
{
    typedef typename H::StateVector SV;
    n = (int)detail::size_of(h.onsite);
    if (n > 2) return false;
    for (int k = 0; k < n; ++k) {
        shapes[k] = detail::onsite_shape<SV>(h.onsite[k]);
        coef[k] = (double)h.onsite[k]->h;
        if (shapes[k] == detail::kOnsiteOther) return false;
    }
    return true;
}
template <class H>
bool lower_onsite(const H&, int*, double*, int& n, std::false_type)
{
    n = 0;
    return true;
}
template <class H>
void lower_potts(const H& h, mqv_model_desc& d, std::true_type)
{
    if (detail::size_of(h.multisite) != 1 || ProposalOf<H>::value != kProposalPottsQ) return;
    d.kind = MQV_MODEL_POTTS;
    d.q = H::q;
    d.k = (double)h.multisite[0]->k;
}
template <class H>
void lower_potts(const H&, mqv_model_desc&, std::false_type)
{
}

template <class H>
mqv_model_desc lower_by_terms(const H& h)
{
    typedef typename H::StateVector SV;
    typedef typename SV::value_type T;
    constexpr int D = (int)std::tuple_size<SV>::value;
    mqv_model_desc d{};
    d.kind = 0;  // unsupported unless recognised below
    double J = 0, w[3] = {1, 1, 1};
    int ninter = 0;
    bool inter_ok = true;
    lower_inter(h, J, w, ninter, inter_ok, detail::has_interactions<H>{});
    if (!inter_ok || ninter > 1) return d;
    int shapes[2] = {0, 0};
    double coef[2] = {0, 0};
    int nons = 0;
    if (!lower_onsite(h, shapes, coef, nons, detail::has_onsite<H>{})) return d;
    const bool flex = detail::has_multisite<H>::value;
    if (std::is_integral<T>::value && D == 1) {
        if (flex) {
            lower_potts(h, d, std::integral_constant<bool, detail::has_q<H>::value && detail::has_multisite<H>::value>{});
            return d;
        }
        if (ninter != 1 || w[0] != 1.0) return d;
        d.J = J;
        if (nons == 0 && ProposalOf<H>::value == kProposalDefault) {
            d.kind = MQV_MODEL_ISING_EMBED;  // the generic Wolff + Embedder of a user Ising
            return d;
        }
        if (ProposalOf<H>::value == kProposalSpin1 && nons >= 1 && shapes[0] == detail::kOnsiteSq &&
            (nons == 1 || shapes[1] == detail::kOnsiteSq)) {
            d.kind = MQV_MODEL_BLUME_CAPEL;
            d.h = coef[0];
            d.h2 = nons > 1 ? coef[1] : 0.0;
        }
        return d;
    }
    if (!std::is_floating_point<T>::value || flex || ninter != 1) return d;
    d.J = J;
    if (D == 3 && ProposalOf<H>::value == kProposalDefault && w[0] == w[1] && w[2] == 1.0) {
        bool ok = true;
        for (int k = 0; k < nons; ++k) ok = ok && shapes[k] == (k == 0 ? detail::kOnsiteZ : detail::kOnsiteZ2);
        if (!ok) return d;
        if (nons == 0 && w[0] == 1.0) {
            d.kind = MQV_MODEL_HEISENBERG;
            return d;
        }
        d.kind = MQV_MODEL_XXZ;
        d.delta = w[0];
        d.h = nons > 0 ? coef[0] : 0.0;
        d.h2 = nons > 1 ? coef[1] : 0.0;
        return d;
    }
    if (D == 1 && w[0] == 1.0 && ProposalOf<H>::value == kProposalShift) {
        for (int k = 0; k < nons; ++k)
            if (shapes[k] != (k == 0 ? detail::kOnsiteSq : detail::kOnsiteQuartic)) return d;
        d.kind = MQV_MODEL_PHI4;
        d.h = nons > 0 ? coef[0] : 0.0;
        d.h2 = nons > 1 ? coef[1] : 0.0;
        d.cap = 0.5;  // Phi4_Initializer_Cartesian's amplitude (src/hamiltonian/Phi4.h:47)
    }
    return d;
}

// Hamiltonian -> model descriptor.  The primary template lowers by term
// probing (lower_by_terms); specialise lower(const H&, double beta) for a
// model whose terms are not of the recognised shapes.
template <class H, class Enable = void>
struct ModelLowering {
    static mqv_model_desc lower(const H& h, double) { return lower_by_terms(h); }
};

// Hypercubic lattices: specialise get() to return true with (dim, len).
template <class L, class Enable = void>
struct HypercubicShape {
    static bool get(const L&, int&, int&) { return false; }
};

// Lattices with SimpleBipartite's termselector (sublattice by coordinate
// parity): specialise get() to return true with (dim, len).
template <class L, class Enable = void>
struct BipartiteShape {
    static bool get(const L&, int&, int&) { return false; }
};

template <class L, class = void>
struct has_bnds : std::false_type {};
template <class L>
struct has_bnds<L, decltype((void)std::declval<const L&>().bnds(0, 0), void())> : std::true_type {};

// Lattice -> lattice descriptor; the CSR arrays live as long as this object.
template <class L>
class LatticeLowering {
public:
    mqv_lattice_desc lower(const L& g)
    {
        mqv_lattice_desc d{};
        int dim = 0, len = 0;
        if (BipartiteShape<L>::get(g, dim, len)) {
            d.kind = MQV_LATTICE_BIPARTITE;
            d.dim = dim;
            d.len = len;
            return d;
        }
        if (HypercubicShape<L>::get(g, dim, len)) {
            d.kind = MQV_LATTICE_HYPERCUBIC;
            d.dim = dim;
            d.len = len;
            return d;
        }
        const std::size_t n = g.size();
        rp_.assign(1, 0);
        ci_.clear();
        bd_.clear();
        for (std::size_t i = 0; i < n; ++i) {
            const auto nb = g.nbrs(0, (int)i);
            for (std::size_t k = 0; k < nb.size(); ++k) ci_.push_back((int32_t)nb[k]);
            add_bonds(g, (int)i, nb.size(), has_bnds<L>{});
            rp_.push_back((int32_t)ci_.size());
        }
        d.kind = MQV_LATTICE_CSR;
        d.n = (int32_t)n;
        d.row_ptr = rp_.data();
        d.col_idx = ci_.data();
        d.bonds = bd_.empty() ? nullptr : bd_.data();
        return d;
    }

private:
    void add_bonds(const L&, int, std::size_t, std::false_type) {}
    void add_bonds(const L& g, int i, std::size_t deg, std::true_type)
    {
        const auto b = g.bnds(0, i);
        for (std::size_t k = 0; k < deg; ++k) bd_.push_back((int8_t)b[k]);
    }
    std::vector<int32_t> rp_, ci_;
    std::vector<int8_t> bd_;
};

// One simulation on the GPU with Core's public face.  H is constructed from
// the Hamiltonian arguments, as Core does (core.h:469).
template <class L, class H, class ConfigT>
class GPUCore {
public:
    template <class... HArgs>
    GPUCore(L& lat, const ConfigT& c, double beta, HArgs&&... hargs)
        : ham_(std::forward<HArgs>(hargs)...), beta_(beta), ncluster_(c.ncluster), nmetro_(c.nmetro),
          warmup_(c.warmupsteps), gameloop_(c.gameloopsteps)
    {
        const mqv_model_desc md = ModelLowering<H>::lower(ham_, beta);
        const mqv_lattice_desc ld = lowering_.lower(lat);
        mqv_run_params rp{};
        rp.beta = beta;
        rp.seed = (uint64_t)(int64_t)c.seed;
        rp.replica = (uint32_t)c.repid;
        check(mqv_create(&md, &ld, &rp, &sim_));
    }
    ~GPUCore()
    {
        if (sim_) mqv_destroy(sim_);
    }
    GPUCore(const GPUCore&) = delete;
    GPUCore& operator=(const GPUCore&) = delete;

    void init() { check(mqv_init_state(sim_)); }  // Core::init (core.h:829-834)
    double elementaryMCstep()                      // core.h:1001-1028, emcs.h:69-109
    {
        double mc = 0;
        check(mqv_emcs(sim_, 1, ncluster_, nmetro_, nullptr, &mc));
        return mc;
    }
    void wrmploop() { check(mqv_emcs(sim_, warmup_, ncluster_, nmetro_, nullptr, nullptr)); }
    void gameloop()
    {
        const std::size_t old = obs_.size();
        obs_.resize(old + (std::size_t)gameloop_);
        cluster_.resize(old + (std::size_t)gameloop_);
        check(mqv_emcs(sim_, gameloop_, ncluster_, nmetro_, obs_.data() + old, cluster_.data() + old));
    }
    // per-EMCS energy per site, |m|, m^2, m^4 of the game loops so far
    const std::vector<mqv_obs>& observables() const { return obs_; }
    const std::vector<double>& cluster_sizes() const { return cluster_; }
    // state in the reference layout: int8 for integer models, float otherwise
    template <class T>
    std::vector<T> state() const
    {
        size_t b = 0;
        check(mqv_state_bytes(sim_, &b));
        std::vector<T> v(b / sizeof(T));
        check(mqv_get_state(sim_, v.data(), b));
        return v;
    }
    const H& hamiltonian() const { return ham_; }
    mqv_sim* handle() const { return sim_; }

private:
    H ham_;
    double beta_;
    int ncluster_, nmetro_, warmup_, gameloop_;
    LatticeLowering<L> lowering_;
    mqv_sim* sim_ = nullptr;
    std::vector<mqv_obs> obs_;
    std::vector<double> cluster_;
};

namespace detail {
template <class L, class H, class ConfigT, class Tuple, std::size_t... I>
std::unique_ptr<GPUCore<L, H, ConfigT>> make(L& lat, const ConfigT& c, const Tuple& h, std::index_sequence<I...>)
{
    return std::unique_ptr<GPUCore<L, H, ConfigT>>(
        new GPUCore<L, H, ConfigT>(lat, c, (double)std::get<0>(h), std::get<I + 1>(h)...));
}
}  // namespace detail

// makeCore's tuple convention: (lattice&, Config, (beta, hamiltonian args...))
template <class L, class H, class ConfigT, class... HArgs>
std::unique_ptr<GPUCore<L, H, ConfigT>> makeGPUCore(const std::tuple<L&, ConfigT, std::tuple<HArgs...>>& t)
{
    static_assert(sizeof...(HArgs) >= 1, "the Hamiltonian arguments start with beta");
    return detail::make<L, H, ConfigT>(std::get<0>(t), std::get<1>(t), std::get<2>(t),
                                       std::make_index_sequence<sizeof...(HArgs) - 1>());
}

// The farm: parameter sets collected with createSimfromParameter (the
// CXX11Scheduler's interface), run together by start() as one batch on the
// GPU -- warm-up, then maxptsteps game loops with per-EMCS observables.
// With maxptsteps > 1 the members exchange states between game loops as the
// reference's parallel tempering does (CXX11Scheduler::start / ptstep,
// src/libmarqov/marqovscheduler.h:223-273,374-413): a plan of maxptsteps
// random pairs (x % len, y % len) from a 64-bit Mersenne twister
// (createPTplan, :203-210), the pair of step t >= 1 attempting its exchange
// after the t-th game loop, self pairs skipped.  The reference seeds that
// generator from the clock; here it is ptseed.  The exchanges run on the
// device (mqv_batch_tempering).  Partners must differ in beta only.
template <class L, class H, class ConfigT>
class GPUScheduler {
public:
    // CXX11Scheduler(int maxptsteps = 1, uint nthreads = 0, int mid = 0)
    // (marqovscheduler.h:280-284); nthreads and mid have no meaning here.
    explicit GPUScheduler(int maxptsteps = 1, unsigned nthreads = 0, int mid = 0, uint64_t ptseed = 0)
        : maxpt_(maxptsteps < 1 ? 1 : maxptsteps), ptseed_(ptseed)
    {
        (void)nthreads;
        (void)mid;
    }
    template <class... HArgs>
    void createSimfromParameter(const std::tuple<L&, ConfigT, std::tuple<HArgs...>>& t)
    {
        Member m;
        m.lowering.reset(new LatticeLowering<L>());
        create(m, std::get<0>(t), std::get<1>(t), std::get<2>(t), std::make_index_sequence<sizeof...(HArgs) - 1>());
        members_.push_back(std::move(m));
    }
    void start()
    {
        if (members_.empty()) return;
        std::vector<mqv_sim_spec> specs;
        for (auto& m : members_) specs.push_back(m.spec);
        if (batch_) mqv_batch_destroy(batch_);
        batch_ = nullptr;
        check(mqv_batch_create(specs.data(), (int32_t)specs.size(), &batch_));
        check(mqv_batch_init_state(batch_));
        const Member& f = members_.front();
        check(mqv_batch_emcs(batch_, f.warmup, f.ncluster, f.nmetro, nullptr, nullptr));
        obs_.resize((std::size_t)f.gameloop * (std::size_t)maxpt_ * members_.size());
        if (maxpt_ == 1) {
            check(mqv_batch_emcs(batch_, f.gameloop, f.ncluster, f.nmetro, obs_.data(), nullptr));
            return;
        }
        const uint64_t len = members_.size();
        std::mt19937_64 rng(ptseed_);
        std::vector<int32_t> plan(2 * (std::size_t)maxpt_, 0);  // the last step has no exchange
        for (int t = 0; t < maxpt_; ++t) {
            const int32_t a = (int32_t)(rng() % len), b = (int32_t)(rng() % len);
            if (t > 0) {
                plan[2 * (std::size_t)(t - 1)] = a;
                plan[2 * (std::size_t)(t - 1) + 1] = b;
            }
        }
        std::vector<int32_t> acc((std::size_t)maxpt_, 0);
        check(mqv_batch_tempering(batch_, maxpt_, f.gameloop, f.ncluster, f.nmetro, plan.data(), 1, ptseed_,
                                  obs_.data(), acc.data()));
        for (int32_t x : acc) acceptedmoves_ += x == 1;
    }
    // record e * size() + i: member i after game-loop EMCS e
    const std::vector<mqv_obs>& observables() const { return obs_; }
    std::size_t size() const { return members_.size(); }
    // accepted exchanges / maxptsteps, the figure the reference logs
    // ("PT acceptance", marqovscheduler.h:300)
    double pt_acceptance() const { return (double)acceptedmoves_ / (double)maxpt_; }
    ~GPUScheduler()
    {
        if (batch_) mqv_batch_destroy(batch_);
    }

private:
    struct Member {
        mqv_sim_spec spec{};
        std::unique_ptr<LatticeLowering<L>> lowering;
        int ncluster = 0, nmetro = 0, warmup = 0, gameloop = 0;
    };
    template <class Tuple, std::size_t... I>
    void create(Member& m, L& lat, const ConfigT& c, const Tuple& h, std::index_sequence<I...>)
    {
        const double beta = (double)std::get<0>(h);
        const H ham(std::get<I + 1>(h)...);
        m.spec.model = ModelLowering<H>::lower(ham, beta);
        m.spec.lattice = m.lowering->lower(lat);
        m.spec.params.beta = beta;
        m.spec.params.seed = (uint64_t)(int64_t)c.seed;
        m.spec.params.replica = (uint32_t)c.repid;
        m.ncluster = c.ncluster;
        m.nmetro = c.nmetro;
        m.warmup = c.warmupsteps;
        m.gameloop = c.gameloopsteps;
    }
    std::vector<Member> members_;
    mqv_batch* batch_ = nullptr;
    std::vector<mqv_obs> obs_;
    int maxpt_ = 1;
    uint64_t ptseed_ = 0;
    int acceptedmoves_ = 0;
};

}  // namespace marqov_b200

#endif /* MARQOV_B200_CORE_HPP */
