// Metropolis sweeps over int8 states (Ising, Potts, Blume-Capel, Edwards-
// Anderson) on any lattice, and their measurements, for sm_100a.
//
// Update order: colour classes in turn (checkerboard parity on hypercubic
// lattices, greedy colours on general graphs), one launch per colour.  Sites
// of one colour have no common bonds, so within a colour the order is
// irrelevant, and each site's random words are keyed by (seed, replica, site,
// sweep): the final state does not depend on the launch geometry.  The 2D
// Ising model on lattices with len % 32 == 0 takes the fused two-colour path
// of ising2d.cu instead; its state is stored in split rows, which the
// lattice's addr() maps for every other kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "int8_site.cuh"

namespace mqv {

// One colour of a stencil sweep.  A CTA takes one aligned block of kAccSites
// sites of the colour (kAccRuns runs of 64 lattice sites), one site per
// thread: its first warp draws the block's acceptance bytes (accept_tab_fill,
// one Philox block per lane), a CTA barrier publishes them, and every thread
// updates its site.
constexpr int kMetroThreads = kAccSites;
__global__ void __launch_bounds__(kMetroThreads) metro_int8_stencil(ModelDev m, StencilDev st, int8_t* __restrict__ s,
                                                                    int colour, Key key, uint32_t sweep,
                                                                    uint32_t replica,
                                                                    const unsigned long long* __restrict__ cuts, int D)
{
    __shared__ uint4 tab[kAccTab];
    const int64_t half = st.n / 2, nblk = (half + kAccSites - 1) / kAccSites;
    for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x) {
        const uint32_t run0 = (uint32_t)(b * kAccRuns);
        if (threadIdx.x < 32) accept_tab_fill(tab, run0, key, sweep, replica);
        __syncthreads();
        const int64_t t = b * kAccSites + threadIdx.x;
        const bool live = t < half;
        with_dim(st, [&](const auto& lt) {
            int8_site(m, lt, s, live ? parity_site(lt, t, colour) : 0, key, sweep, replica, cuts, D, live, colour, tab,
                      run0);
        });
        __syncthreads();  // every thread has read the table before the next block's draw
    }
}

__global__ void metro_int8_csr(ModelDev m, CSRDev g, int8_t* __restrict__ s, const int32_t* __restrict__ order,
                               int64_t begin, int64_t count, Key key, uint32_t sweep, uint32_t replica,
                               const unsigned long long* __restrict__ cuts, int D)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t0 = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31u); t0 < count; t0 += stride) {
        const int64_t t = t0 + (threadIdx.x & 31u);
        const bool live = t < count;
        int8_site(m, g, s, live ? (int64_t)order[begin + t] : 0, key, sweep, replica, cuts, D, live);
    }
}

// dE of every move index of int8_site, with the kernel's own FP64 operations
std::vector<unsigned long long> int8_cut_table(const ModelDev& m, int D)
{
    std::vector<unsigned long long> t;
    if (m.kind == MQV_MODEL_BLUME_CAPEL) {
        // interaction J dn sum plus the onsite terms of the site, summed in
        // the reference's order (compute_onsiteenergydiff,
        // src/libmarqov/metropolishelpers.h:651-683): every term, or with a
        // termselector term 0 on sublattice A (table 0) and term 1 on B (table 1)
        const int per = 5 * (2 * D + 1) * 3;
        t.resize((size_t)per * (m.termsel ? 2 : 1));
        for (int sub = 0; sub < (m.termsel ? 2 : 1); ++sub)
            for (int dn = -2; dn <= 2; ++dn)
                for (int sum = -D; sum <= D; ++sum)
                    for (int dq = -1; dq <= 1; ++dq) {
                        double ons;
                        if (!m.termsel) ons = MQV_DADD(MQV_DMUL(m.h, (double)dq), MQV_DMUL(m.h2, (double)dq));
                        else ons = MQV_DMUL(sub ? m.h2 : m.h, (double)dq);
                        const double dE = MQV_DADD(MQV_DMUL(m.J, (double)(dn * sum)), ons);
                        t[(size_t)sub * per + (size_t)(((dn + 2) * (2 * D + 1) + (sum + D)) * 3 + (dq + 1))] =
                            accept_cut(1, dE, m.beta);
                    }
    } else {
        t.resize((size_t)2 * D + 1);
        for (int k = 0; k <= 2 * D; ++k) {
            const double dE = m.kind == MQV_MODEL_POTTS ? MQV_DMUL(m.k, (double)(k - D))
                                                        : MQV_DMUL(m.J, (double)(-2 * (k - D)));
            t[(size_t)k] = accept_cut(1, dE, m.beta);
        }
    }
    return t;
}

// the handle's cut table, rebuilt when the model or beta changed
cudaError_t ensure_cuts(Sim* s)
{
    const double key[7] = {s->md.J, s->md.h, s->md.k, s->md.beta, (double)s->md.kind, s->md.h2, (double)s->md.termsel};
    if (s->d_cuts && std::equal(key, key + 7, s->cuts_for)) return cudaSuccess;
    const std::vector<unsigned long long> t = int8_cut_table(s->md, s->max_degree);
    if ((int)t.size() > s->n_cuts) {
        if (s->d_cuts) cudaFree(s->d_cuts);
        s->d_cuts = nullptr;
        s->n_cuts = 0;
        const cudaError_t e = cudaMalloc(&s->d_cuts, sizeof(unsigned long long) * t.size());
        if (e != cudaSuccess) return e;
        s->n_cuts = (int)t.size();
    }
    // stream-ordered with the sweeps that read the previous table
    const cudaError_t e = cudaMemcpyAsync(s->d_cuts, t.data(), sizeof(unsigned long long) * t.size(),
                                          cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) return e;
    std::copy(key, key + 7, s->cuts_for);
    return cudaStreamSynchronize(s->stream);  // the host table goes out of scope
}

template <class Lat>
__global__ void measure_int8(ModelDev m, Lat lat, const int8_t* __restrict__ s, long long* __restrict__ acc)
{
    measure_int8_part(m, lat, s, acc, blockIdx.x, gridDim.x);
}
template <>
__global__ void measure_int8(ModelDev m, StencilDev st, const int8_t* __restrict__ s, long long* __restrict__ acc)
{
    with_dim(st, [&](const auto& lt) { measure_int8_part(m, lt, s, acc, blockIdx.x, gridDim.x); });
}

__global__ void finalize_int8(ModelDev m, int64_t n, const long long* __restrict__ acc, int nslots,
                              double* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nslots) finalize_int8_one(m, n, acc + (size_t)k * kAccStride, out + 4 * (size_t)k);
}

// ---------------------------------------------------------------------------
// initial state on the INIT stream: Ising::initstatespace (Ising.h:99-107),
// Potts<Q>::initstatespace (Potts.h:149-156); Blume-Capel has no
// initstatespace and takes Core::init_hot's random direction of a one-
// component integer state, +1 turned to -1 when real() < 0.5
// (src/libmarqov/core.h:773-782, src/hamiltonian/util/randomdir.h:84-90)

template <class Lat>
__global__ void init_int8(ModelDev m, Lat lat, int64_t n, int8_t* __restrict__ s, Key key, uint32_t tg)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t w = lo64(philox((uint32_t)i, 0u, 0u, tg, key));
        int v;
        if (m.kind == MQV_MODEL_POTTS) v = (int)(w % (uint64_t)m.q);
        else if (m.kind == MQV_MODEL_BLUME_CAPEL) v = real01(w) < 0.5 ? -1 : 1;
        else v = real01(w) > 0.5 ? 1 : -1;
        s[lat.addr(i)] = (int8_t)v;
    }
}

// ---------------------------------------------------------------------------
// launchers

static int grid_for(int64_t work, int threads)
{
    int64_t b = (work + threads - 1) / threads;
    const int64_t cap = 148 * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

cudaError_t launch_init_int8(Sim* s)
{
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC)
        init_int8<<<grid_for(s->n, 256), 256, 0, s->stream>>>(s->md, s->sten, s->n, (int8_t*)s->state[s->cur],
                                                               make_key(s->seed), tag(kInit, s->replica));
    else
        init_int8<<<grid_for(s->n, 256), 256, 0, s->stream>>>(s->md, s->csr, s->n, (int8_t*)s->state[s->cur],
                                                               make_key(s->seed), tag(kInit, s->replica));
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_measure_int8(Sim* s, int slot)
{
    long long* acc = s->d_acc + (size_t)slot * kAccStride;
    const int8_t* st = (const int8_t*)s->state[s->cur];
    const int g = grid_for(s->n, 256);
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC) measure_int8<<<g, 256, 0, s->stream>>>(s->md, s->sten, st, acc);
    else measure_int8<<<g, 256, 0, s->stream>>>(s->md, s->csr, st, acc);
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_finalize_int8(Sim* s, int nslots, double* d_out)
{
    finalize_int8<<<(nslots + 127) / 128, 128, 0, s->stream>>>(s->md, s->n, s->d_acc, nslots, d_out);
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_ising2d_sweep(Sim* s, long long* acc);
unsigned long long accept_cut(int pref, double dE, double beta);

// One Metropolis sweep; when slot >= 0 the new state's observables are
// accumulated into that slot.
cudaError_t launch_metropolis_int8(Sim* s, int slot)
{
    const Key key = make_key(s->seed);
    cudaError_t err = cudaSuccess;
    if (s->fused_ising2d) {
        long long* acc = slot >= 0 ? s->d_acc + (size_t)slot * kAccStride : nullptr;
        err = launch_ising2d_sweep(s, acc);
        s->launches++;
        s->cur ^= 1;
        s->sweep++;
        return err;
    }
    int8_t* st = (int8_t*)s->state[s->cur];
    err = ensure_cuts(s);
    if (err != cudaSuccess) return err;
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC) {
        // one CTA per block of kAccSites sites of a colour
        const int g = grid_for((s->n / 2 + kAccSites - 1) / kAccSites * kMetroThreads, kMetroThreads);
        for (int c = 0; c < 2; ++c) {
            metro_int8_stencil<<<g, kMetroThreads, 0, s->stream>>>(s->md, s->sten, st, c, key, (uint32_t)s->sweep,
                                                                   s->replica, s->d_cuts, s->max_degree);
            s->launches++;
        }
    } else {
        for (size_t c = 0; c + 1 < s->colour_ptr.size(); ++c) {
            const int64_t b = s->colour_ptr[c], cnt = s->colour_ptr[c + 1] - b;
            if (cnt == 0) continue;
            metro_int8_csr<<<grid_for(cnt, 256), 256, 0, s->stream>>>(s->md, s->csr, st, s->d_order, b, cnt, key,
                                                                       (uint32_t)s->sweep, s->replica, s->d_cuts,
                                                                       s->max_degree);
            s->launches++;
        }
    }
    err = cudaGetLastError();
    s->sweep++;
    if (err == cudaSuccess && slot >= 0) err = launch_measure_int8(s, slot);
    return err;
}

}  // namespace mqv
