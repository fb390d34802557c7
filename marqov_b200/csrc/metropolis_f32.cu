// Metropolis sweeps, measurements and embedded Wolff clusters for float
// states: O(3) Heisenberg / XXZ (3 x FP32 per site, site-major) and scalar
// phi^4 (FP32 per site), for sm_100a.
//
// Storage is FP32; the energy difference, proposals and acceptance are
// evaluated in FP64 so that they follow the reference's double arithmetic
// (src/libmarqov/metropolishelpers.h:598-738 with double couplings), and the
// lattice-wide reductions accumulate in FP64.
#include <cuda_runtime.h>

#include "f32_site.cuh"

namespace mqv {

unsigned long long accept_cut(int pref, double dE, double beta);

// One colour of a stencil sweep.  A CTA takes one aligned block of kAccSites
// sites of the colour (kAccRuns runs of 64 lattice sites), one site per
// thread: its first warp draws the block's acceptance bytes (accept_tab_fill,
// one Philox block per lane), a CTA barrier publishes them, and every thread
// updates its site.  One site per thread keeps enough warps in flight to
// cover the FP64 latency of the proposal and the acceptance.
constexpr int kMetroThreads = kAccSites;
__global__ void __launch_bounds__(kMetroThreads) metro_f32_stencil(ModelDev m, StencilDev st, float* __restrict__ s,
                                                                   int colour, Key key, uint32_t sweep, uint32_t replica)
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
            f32_site(m, lt, s, live ? parity_site_f(lt, t, colour) : 0, key, sweep, replica, live, colour, tab, run0);
        });
        __syncthreads();  // every thread has read the table before the next block's draw
    }
}

__global__ void metro_f32_csr(ModelDev m, CSRDev g, float* __restrict__ s, const int32_t* __restrict__ order,
                              int64_t begin, int64_t count, Key key, uint32_t sweep, uint32_t replica)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t0 = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31u); t0 < count; t0 += stride) {
        const int64_t t = t0 + (threadIdx.x & 31u);
        const bool live = t < count;
        f32_site(m, g, s, live ? (int64_t)order[begin + t] : 0, key, sweep, replica, live);
    }
}

template <class Lat>
__global__ void measure_f32(ModelDev m, Lat lat, const float* __restrict__ s, double* __restrict__ acc)
{
    measure_f32_part(m, lat, s, acc, blockIdx.x, gridDim.x);
}
template <>
__global__ void measure_f32(ModelDev m, StencilDev st, const float* __restrict__ s, double* __restrict__ acc)
{
    with_dim(st, [&](const auto& lt) { measure_f32_part(m, lt, s, acc, blockIdx.x, gridDim.x); });
}

__global__ void finalize_f32(ModelDev m, int64_t n, const double* __restrict__ acc, int nslots, double* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nslots) finalize_f32_one(m, n, acc + (size_t)k * kAccStride, out + 4 * (size_t)k);
}

// ---- initial state --------------------------------------------------------------

__global__ void init_f32(ModelDev m, int64_t n, float* __restrict__ s, Key key, uint32_t tg)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        SubStream rng(key, (uint32_t)i, 0u, tg);
        if (m.symd == 3) {
            double v[3];
            rnddir3(rng, v);
            s[i] = (float)v[0];
            s[n + i] = (float)v[1];
            s[2 * n + i] = (float)v[2];
        } else {
            // standard normal by Box-Muller
            const double u0 = rng.real(), u1 = rng.real();
            s[i] = (float)(sqrt(-2.0 * log(1.0 - u0)) * cospi(2.0 * u1));
        }
    }
}

template <class Lat>
__global__ void __launch_bounds__(1024) wolff_f32(ModelDev m, Lat lat, float* __restrict__ s,
                                                  uint32_t* __restrict__ visited, int32_t* __restrict__ queue,
                                                  int32_t* __restrict__ out_size, Key key, uint32_t serial,
                                                  uint32_t tg_seed, uint32_t tg_bond, int max_degree)
{
    __shared__ int32_t fbuf[2 * kWolffCapF];
    __shared__ double fproj[2 * kWolffCapF];
    wolff_f32_cluster(m, lat, s, visited, queue, out_size, key, serial, tg_seed, tg_bond, max_degree, fbuf, fproj);
}

// ---- launchers ------------------------------------------------------------------

static int grid_for_f(int64_t work, int threads)
{
    int64_t b = (work + threads - 1) / threads;
    const int64_t cap = 148 * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

cudaError_t launch_init_f32(Sim* s)
{
    init_f32<<<grid_for_f(s->n, 256), 256, 0, s->stream>>>(s->md, s->n, (float*)s->state[s->cur], make_key(s->seed),
                                                           tag(kInit, s->replica));
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_measure_f32(Sim* s, int slot)
{
    double* acc = reinterpret_cast<double*>(s->d_acc + (size_t)slot * kAccStride);
    const float* st = (const float*)s->state[s->cur];
    const int g = grid_for_f(s->n, 256);
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC) measure_f32<<<g, 256, 0, s->stream>>>(s->md, s->sten, st, acc);
    else measure_f32<<<g, 256, 0, s->stream>>>(s->md, s->csr, st, acc);
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_finalize_f32(Sim* s, int nslots, double* d_out)
{
    finalize_f32<<<(nslots + 127) / 128, 128, 0, s->stream>>>(s->md, s->n, reinterpret_cast<const double*>(s->d_acc),
                                                                nslots, d_out);
    s->launches++;
    return cudaGetLastError();
}

cudaError_t launch_metropolis_f32(Sim* s, int slot)
{
    const Key key = make_key(s->seed);
    float* st = (float*)s->state[s->cur];
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC) {
        // one CTA per block of kAccSites sites of a colour
        const int g = grid_for_f((s->n / 2 + kAccSites - 1) / kAccSites * kMetroThreads, kMetroThreads);
        for (int c = 0; c < 2; ++c) {
            metro_f32_stencil<<<g, kMetroThreads, 0, s->stream>>>(s->md, s->sten, st, c, key, (uint32_t)s->sweep,
                                                                  s->replica);
            s->launches++;
        }
    } else {
        for (size_t c = 0; c + 1 < s->colour_ptr.size(); ++c) {
            const int64_t b = s->colour_ptr[c], cnt = s->colour_ptr[c + 1] - b;
            if (cnt == 0) continue;
            metro_f32_csr<<<grid_for_f(cnt, 256), 256, 0, s->stream>>>(s->md, s->csr, st, s->d_order, b, cnt, key,
                                                                        (uint32_t)s->sweep, s->replica);
            s->launches++;
        }
    }
    cudaError_t err = cudaGetLastError();
    s->sweep++;
    if (err == cudaSuccess && slot >= 0) err = launch_measure_f32(s, slot);
    return err;
}

cudaError_t launch_wolff_f32(Sim* s, int slot)
{
    float* st = (float*)s->state[s->cur];
    const Key key = make_key(s->seed);
    const uint32_t serial = (uint32_t)s->cluster;
    int32_t* out = s->d_csize + slot;
    if (s->lat_kind == MQV_LATTICE_HYPERCUBIC)
        wolff_f32<<<1, 1024, 0, s->stream>>>(s->md, s->sten, st, s->d_visited, s->d_queue, out, key, serial,
                                             tag(kWolffSeed, s->replica), tag(kWolffBond, s->replica), s->max_degree);
    else
        wolff_f32<<<1, 1024, 0, s->stream>>>(s->md, s->csr, st, s->d_visited, s->d_queue, out, key, serial,
                                             tag(kWolffSeed, s->replica), tag(kWolffBond, s->replica), s->max_degree);
    s->launches++;
    s->cluster++;
    return cudaGetLastError();
}

}  // namespace mqv
