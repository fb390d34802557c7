// The C++ drop-in, as a MARQOV program uses it -- TEST PROGRAM.
//
// Built against the reference's own Hamiltonian and lattice headers and the
// engine's headers, linked against libmarqov_b200.so.  It runs, through
// makeGPUCore and GPUScheduler, what the reference's libshowcase.cpp runs
// through makeCore (src/libshowcase.cpp:40-58): init, wrmploop, gameloop.
// Output (one line each): "core <e> <|m|>" per game-loop EMCS of a 2D Ising
// run, then "farm <i> <e> <|m|>" for the last EMCS of each member of a
// three-member Potts farm, "pt <i> <e> <|m|>" for the last EMCS of each
// member of a four-member Ising ladder with parallel tempering and "ptacc
// <acceptance>", "ea <e> <|m|>" for a random-bond lattice, and "xxz <e>
// <|m|>" per game-loop EMCS of an XXZ model on SimpleBipartite.  With
// no GPU it prints "no device: <message>" and exits 0.
#define CACHECONTAINER_H 1
#include <cstdio>
#include <string>
#include <tuple>
#include <vector>

#include <algorithm>
#include <numeric>
#include <random>
#include <vector>

namespace H5 { struct Group {}; }
template <class... T> inline void dumpscalartoH5(T&&...) {}
namespace MARQOV {
// the state-space type the Hamiltonian headers name (src/libmarqov/core.h:249-330)
template <class SV, class Grid>
struct Space {
    typedef Grid Lattice;
    typedef SV StateVector;
    using value_type = SV;
    std::vector<SV> v;
    SV& operator[](int j) { return v[j]; }
    const SV& operator[](int j) const { return v[j]; }
};
}  // namespace MARQOV

// the Hamiltonian headers specialise MARQOV's update templates: those first
#include "libmarqov/rngcache.h"
#include "libmarqov/util/svmath.h"
#include "libmarqov/metropolis.h"
#include "libmarqov/wolff.h"
#include "hamiltonian/EdwardsAndersonIsing.h"
#include "hamiltonian/Ising.h"
#include "hamiltonian/Potts.h"
#include "hamiltonian/XXZAntiferroSingleAniso.h"
#include "lattice/regular_hypercubic.h"
#include "lattice/regular_random_bond.h"
#include "lattice/util/regular_lattice.h"
#include "lattice/simple_bipartite.h"

#include "marqov_b200_marqov.hpp"

// User Hamiltonians written against MARQOV's term API (hamparts.h), with no
// lowering of their own: the C++ layer recognises their terms.
struct MyIsing {
    static constexpr int SymD = 1;
    typedef std::array<int, 1> StateVector;
    Standard_Interaction<StateVector> inter;
    std::array<Standard_Interaction<StateVector>*, 1> interactions{{&inter}};
    explicit MyIsing(double J) : inter(J) {}
};
template <class SV>
struct MyXXZInteraction : public Interaction<SV> {
    double delta;
    MyXXZInteraction(double J, double d) : Interaction<SV>(J), delta(d) {}
    SV get(const SV& p) override { return {{delta * p[0], delta * p[1], p[2]}}; }
};
template <class SV>
struct MyFieldZ : public OnSite<SV, double> {
    explicit MyFieldZ(double h) : OnSite<SV, double>(h) {}
    double get(const SV& p) override { return p[2]; }
};
struct MyXXZ {
    static constexpr int SymD = 3;
    typedef std::array<double, 3> StateVector;
    MyXXZInteraction<StateVector> inter;
    MyFieldZ<StateVector> field;
    std::array<Interaction<StateVector>*, 1> interactions{{&inter}};
    std::array<OnSite<StateVector, double>*, 1> onsite{{&field}};
    MyXXZ(double delta, double h) : inter(1.0, delta), field(h) {}
};
// a term the engine does not lower: an interaction that mixes components
template <class SV>
struct SwapXY : public Interaction<SV> {
    explicit SwapXY(double J) : Interaction<SV>(J) {}
    SV get(const SV& p) override { return {{p[1], p[0], p[2]}}; }
};
struct MyOdd {
    static constexpr int SymD = 3;
    typedef std::array<double, 3> StateVector;
    SwapXY<StateVector> inter{-1.0};
    std::array<Interaction<StateVector>*, 1> interactions{{&inter}};
    explicit MyOdd(double) {}
};

// MARQOV::Config's fields (src/libmarqov/core.h:74-192); core.h itself needs HDF5
struct Config {
    std::string outpath;
    int id = 0, repid = 0, seed = 0, nsteps = 250, warmupsteps = 100, gameloopsteps = 200, ncluster = 20, nmetro = 10;
    explicit Config(std::string p) : outpath(std::move(p)) {}
};

int main()
{
    try {
        RegularHypercubic latt(32, 2);
        Config cfg("out");
        cfg.seed = 17;
        cfg.ncluster = 1;
        cfg.nmetro = 1;
        cfg.warmupsteps = 50;
        cfg.gameloopsteps = 5;
        auto sim = marqov_b200::makeGPUCore<RegularHypercubic, Ising<int>>(
            std::make_tuple(std::ref(latt), cfg, std::make_tuple(0.44068679, -1.0)));
        sim->init();
        sim->wrmploop();
        sim->gameloop();
        for (const auto& o : sim->observables()) std::printf("core %.17g %.17g\n", o.e, o.m);

        marqov_b200::GPUScheduler<RegularHypercubic, Potts<3>, Config> farm;
        std::vector<RegularHypercubic> lats{RegularHypercubic(16, 2), RegularHypercubic(24, 2), RegularHypercubic(32, 2)};
        for (int i = 0; i < 3; ++i) {
            Config c("out");
            c.seed = 5;
            c.repid = i;
            c.ncluster = 1;
            c.nmetro = 2;
            c.warmupsteps = 20;
            c.gameloopsteps = 4;
            farm.createSimfromParameter(std::make_tuple(std::ref(lats[i]), c, std::make_tuple(1.0 + 0.05 * i, -1.0)));
        }
        farm.start();
        const auto& fo = farm.observables();
        for (std::size_t i = 0; i < farm.size(); ++i) {
            const auto& o = fo[3 * farm.size() + i];
            std::printf("farm %zu %.17g %.17g\n", i, o.e, o.m);
        }

        // parallel tempering over an Ising ladder: CXX11Scheduler(maxptsteps)
        marqov_b200::GPUScheduler<RegularHypercubic, Ising<int>, Config> pt(6, 0, 0, 3);
        RegularHypercubic lpt(12, 2);
        for (int i = 0; i < 4; ++i) {
            Config c("out");
            c.seed = 21 + i;
            c.repid = i;
            c.ncluster = 1;
            c.nmetro = 1;
            c.warmupsteps = 10;
            c.gameloopsteps = 3;
            pt.createSimfromParameter(std::make_tuple(std::ref(lpt), c, std::make_tuple(0.38 + 0.04 * i, -1.0)));
        }
        pt.start();
        const auto& po = pt.observables();
        const std::size_t last = po.size() / pt.size() - 1;
        for (std::size_t i = 0; i < pt.size(); ++i)
            std::printf("pt %zu %.17g %.17g\n", i, po[last * pt.size() + i].e, po[last * pt.size() + i].m);
        std::printf("ptacc %.17g\n", pt.pt_acceptance());
        RegularRandomBond<BimodalPDF> rb(6, 3);
        Config ce("out");
        ce.seed = 9;
        ce.ncluster = 0;
        ce.nmetro = 1;
        ce.warmupsteps = 10;
        ce.gameloopsteps = 1;
        auto ea = marqov_b200::makeGPUCore<RegularRandomBond<BimodalPDF>, EdwardsAndersonIsing<int>>(
            std::make_tuple(std::ref(rb), ce, std::make_tuple(0.9, -1.0)));
        ea->init();
        ea->wrmploop();
        ea->gameloop();
        std::printf("ea %.17g %.17g\n", ea->observables().back().e, ea->observables().back().m);

        // XXZAntiferroSingleAniso(H, Delta, D) on SimpleBipartite: the
        // termselector gives sublattice A the field and B the anisotropy
        SimpleBipartite sb(6, 3);
        Config cx("out");
        cx.seed = 33;
        cx.ncluster = 0;
        cx.nmetro = 1;
        cx.warmupsteps = 4;
        cx.gameloopsteps = 3;
        auto xxz = marqov_b200::makeGPUCore<SimpleBipartite, XXZAntiferroSingleAniso<double>>(
            std::make_tuple(std::ref(sb), cx, std::make_tuple(0.8, 0.3, 1.2, 0.5)));
        xxz->init();
        xxz->wrmploop();
        xxz->gameloop();
        for (const auto& o : xxz->observables()) std::printf("xxz %.17g %.17g\n", o.e, o.m);

        // user term-API Hamiltonians, lowered by their terms
        RegularHypercubic lu(16, 2);
        Config cu("out");
        cu.seed = 44;
        cu.ncluster = 1;
        cu.nmetro = 1;
        cu.warmupsteps = 5;
        cu.gameloopsteps = 4;
        auto mi = marqov_b200::makeGPUCore<RegularHypercubic, MyIsing>(
            std::make_tuple(std::ref(lu), cu, std::make_tuple(0.44, -1.0)));
        mi->init();
        mi->wrmploop();
        mi->gameloop();
        for (const auto& o : mi->observables()) std::printf("myising %.17g %.17g\n", o.e, o.m);
        RegularHypercubic lx(6, 3);
        Config cxx("out");
        cxx.seed = 45;
        cxx.ncluster = 0;
        cxx.nmetro = 1;
        cxx.warmupsteps = 3;
        cxx.gameloopsteps = 3;
        auto mx = marqov_b200::makeGPUCore<RegularHypercubic, MyXXZ>(
            std::make_tuple(std::ref(lx), cxx, std::make_tuple(0.7, 0.6, 0.25)));
        mx->init();
        mx->wrmploop();
        mx->gameloop();
        for (const auto& o : mx->observables()) std::printf("myxxz %.17g %.17g\n", o.e, o.m);
        try {
            auto bad = marqov_b200::makeGPUCore<RegularHypercubic, MyOdd>(
                std::make_tuple(std::ref(lx), cxx, std::make_tuple(0.7, 1.0)));
            std::printf("unsupported none\n");
        } catch (const marqov_b200::Error& e) {
            std::printf("unsupported %d\n", (int)e.status);
        }
    } catch (const marqov_b200::Error& e) {
        if (e.status == MQV_ERR_NO_DEVICE) {
            std::printf("no device: %s\n", e.what());
            return 0;
        }
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
