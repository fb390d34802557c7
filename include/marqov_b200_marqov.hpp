/*
 * marqov_b200 -- lowering of MARQOV's own Hamiltonian and lattice classes.
 *
 * Include after the MARQOV headers of the classes you use; each block is
 * compiled only when its MARQOV header (by its include guard) is present.
 *   Ising<int>            Wolff<Ising<int>> specialisation   src/hamiltonian/Ising.h:62-169
 *   Ising<other spin>     generic Wolff + Embedder           src/libmarqov/wolff.h:72-126
 *   Potts<Q>              flex term k                         src/hamiltonian/Potts.h:80-156
 *   BlumeCapel<S>         J, onsite D                         src/hamiltonian/BlumeCapel.h:46-80
 *   BlumeCapelBipartite<S> J, onsite DA, DB                   src/hamiltonian/BlumeCapelBipartite.h:39-86
 *   Heisenberg<S, C>      J                                   src/hamiltonian/Heisenberg.h:62-105
 *   XXZAntiferro<S>       J = +1, Delta, field H              src/hamiltonian/XXZAntiferro.h:135-205
 *   XXZAntiferroSingleAniso<S>  ... and single-ion D          src/hamiltonian/XXZAntiferroSingleAniso.h:31-96
 *   EdwardsAndersonIsing  J with the lattice's bnds()         src/hamiltonian/EdwardsAndersonIsing.h:286-310
 *   RegularHypercubic, FixedDimRegularHypercubic<d>: stencil  src/lattice/regular_hypercubic.h
 *   SimpleBipartite: stencil + termselector by sublattice     src/lattice/simple_bipartite.h:8-58
 * Other lattices (RegularRandomBond, GraphFromCSV, ...) are lowered to CSR
 * from nbrs() / bnds() by LatticeLowering.  Hamiltonians without a block
 * here -- user classes written with MARQOV's term API -- are lowered by
 * probing their terms (lower_by_terms in marqov_b200_core.hpp); the
 * ProposalOf blocks below tell it their Initializer.  MARQOV's Phi4 is a
 * three-component field; the engine's phi^4 is the scalar form, and a
 * three-component Phi4 comes out of the term probe as unsupported.
 */
#ifndef MARQOV_B200_MARQOV_HPP
#define MARQOV_B200_MARQOV_HPP

#include <type_traits>

#include "marqov_b200_core.hpp"

namespace marqov_b200 {

#ifdef ISING_H
template <class S>
struct ModelLowering<Ising<S>> {
    static mqv_model_desc lower(const Ising<S>& h, double)
    {
        mqv_model_desc d{};
        d.kind = std::is_same<S, int>::value ? MQV_MODEL_ISING : MQV_MODEL_ISING_EMBED;
        d.J = h.J;
        return d;
    }
};
#endif

#ifdef POTTS_H
template <int Q>
struct ModelLowering<Potts<Q>> {
    static mqv_model_desc lower(const Potts<Q>& h, double)
    {
        mqv_model_desc d{};
        d.kind = MQV_MODEL_POTTS;
        d.q = Q;
        d.k = h.potts_interaction.k;
        return d;
    }
};
#endif

#ifdef BLUMECAPEL_H
template <class S>
struct ModelLowering<BlumeCapel<S>> {
    static mqv_model_desc lower(const BlumeCapel<S>& h, double)
    {
        mqv_model_desc d{};
        d.kind = MQV_MODEL_BLUME_CAPEL;
        d.J = h.J;
        d.h = h.D;
        return d;
    }
};
#endif

#ifdef BLUMECAPELBIPARTITE_H
template <class S>
struct ModelLowering<BlumeCapelBipartite<S>> {
    static mqv_model_desc lower(const BlumeCapelBipartite<S>& h, double)
    {
        mqv_model_desc d{};
        d.kind = MQV_MODEL_BLUME_CAPEL;
        d.J = h.J;
        d.h = h.DA;  // onsite term 0
        d.h2 = h.DB; // onsite term 1
        return d;
    }
};
#endif

#ifdef XXZANTIFERRO_H
template <class S>
struct ModelLowering<XXZAntiferro<S>> {
    static mqv_model_desc lower(const XXZAntiferro<S>& h, double)
    {
        mqv_model_desc d{};
        d.kind = MQV_MODEL_XXZ;
        d.J = XXZAntiferro_interaction<typename XXZAntiferro<S>::StateVector>::J;
        d.delta = h.Delta;
        d.h = h.H;
        return d;
    }
};
#endif

#ifdef XXZANTIFERROSINGLEANISO_H
template <class S>
struct ModelLowering<XXZAntiferroSingleAniso<S>> {
    static mqv_model_desc lower(const XXZAntiferroSingleAniso<S>& h, double)
    {
        mqv_model_desc d{};
        d.kind = MQV_MODEL_XXZ;
        d.J = XXZAntiferro_interaction<typename XXZAntiferroSingleAniso<S>::StateVector>::J;
        d.delta = h.Delta;
        d.h = h.H;   // onsite term 0: XXZAntiferro_extfield
        d.h2 = h.D;  // onsite term 1: XXZAntiferro_onsiteaniso
        return d;
    }
};
#endif

#ifdef HEISENBERG_H
template <class S, class C>
struct ModelLowering<Heisenberg<S, C>> {
    static mqv_model_desc lower(const Heisenberg<S, C>& h, double)
    {
        mqv_model_desc d{};
        d.kind = MQV_MODEL_HEISENBERG;
        d.J = h.J;
        return d;
    }
};
#endif

#ifdef EDWARDSANDERSONISING_H
template <class S>
struct ModelLowering<EdwardsAndersonIsing<S>> {
    static mqv_model_desc lower(const EdwardsAndersonIsing<S>& h, double)
    {
        mqv_model_desc d{};
        d.kind = MQV_MODEL_EA;
        d.J = h.J;
        return d;
    }
};
#endif

#ifdef REGULAR_HYPERCUBIC_H
template <>
struct HypercubicShape<RegularHypercubic> {
    static bool get(const RegularHypercubic& g, int& dim, int& len)
    {
        dim = g.dim;
        len = g.len;
        return true;
    }
};
template <int D>
struct HypercubicShape<FixedDimRegularHypercubic<D>> {
    static bool get(const FixedDimRegularHypercubic<D>& g, int& dim, int& len)
    {
        dim = D;
        len = g.len;
        return true;
    }
};
#endif

// Proposals of the generic lowering, from the reference's initializer
// classes (src/hamiltonian/util/initializers.h:87-119, src/hamiltonian/Phi4.h:37-58)
#ifdef INITIALIZERS_H
template <class H>
struct ProposalOf<H, typename std::enable_if<std::is_base_of<Spin1_Initializer<typename H::StateVector>,
                                                             Initializer<H>>::value>::type> {
    static constexpr int value = kProposalSpin1;
};
#endif
#ifdef PHI4_H
template <class H>
struct ProposalOf<H, typename std::enable_if<std::is_base_of<Phi4_Initializer_Cartesian<typename H::StateVector>,
                                                             Initializer<H>>::value>::type> {
    static constexpr int value = kProposalShift;
};
#endif

#ifdef SIMPLE_BIPARTITE_H
template <>
struct BipartiteShape<SimpleBipartite> {
    static bool get(const SimpleBipartite& g, int& dim, int& len)
    {
        dim = g.dim;
        len = g.len;
        return true;
    }
};
#endif

}  // namespace marqov_b200

#endif /* MARQOV_B200_MARQOV_HPP */
