// Batched elementary Monte Carlo steps over many independent simulations
// (replicas, temperatures, disorder realisations, lattice sizes) on one GPU.
//
// MARQOV runs such a farm as one simulation per CPU thread
// (src/libmarqov/marqovscheduler.h:64-494); on the GPU the same farm is a
// handful of kernels per EMCS that each cover every member:
//   batch_wolff      one CTA per member grows and flips/reflects its cluster,
//   batch_metro      one launch per colour over the sites of that colour of
//                    all members (flattened, block -> first member table);
//                    members on hypercubic lattices use the checkerboard,
//                    CSR members their own colouring,
//   batch_measure    CTAs (part, member) accumulate each member's observables,
//   batch_tick       advances the EMCS counter.
// Every per-step number (sweep and cluster serials, measurement slot) is
// derived on the device from that counter, so the kernels of one EMCS form a
// fixed sequence: it is captured once into a CUDA graph and replayed.  The
// per-member arithmetic is that of the per-handle kernels, keyed by each
// member's (seed, replica id, sweep, site), so a batched run equals running
// every member handle on its own, bit for bit.  A batch holds either int8 or
// float members.
#include <cuda_runtime.h>

#include "batch.h"
#include "f32_site.cuh"
#include "int8_site.cuh"
#include "wolff_ccl.cuh"
#include "wolff_int8.cuh"

namespace mqv {

template <bool F32, class Lat>
__device__ __forceinline__ void batch_site(const BatchRep& R, const Lat& lat, int64_t i, uint32_t sweep, bool live,
                                           int sub, const uint4* tab, uint32_t run0)
{
    if (F32) f32_site(R.md, lat, (float*)R.s, i, R.key, sweep, R.replica, live, sub, tab, run0);
    else int8_site(R.md, lat, (int8_t*)R.s, i, R.key, sweep, R.replica, R.cuts, R.D, live, sub, tab, run0);
}

// One colour of a sweep over every member.  Each CTA takes one block of
// kAccSites consecutive positions of one member's colour-c sites, one
// position per thread (member counts are padded to whole blocks, positions
// past a member's count are idle threads): on hypercubic members the block's
// sites fill kAccRuns aligned 64-site runs, whose acceptance bytes the first
// warp draws once (accept_tab_fill) for the whole CTA; CSR members draw per
// site.
template <bool F32>
__global__ void __launch_bounds__(kBatchMetroThreads)
    batch_metro(const BatchRep* __restrict__ reps, const int64_t* __restrict__ prefix,
                const int32_t* __restrict__ block_rep, const int32_t* __restrict__ cbegin,
                const int32_t* __restrict__ ccount, int ncol, int64_t total, int colour,
                const BatchCtr* __restrict__ ctr, int nmetro, int j)
{
    static_assert(kBatchMetroThreads == kAccSites, "one position per thread");
    __shared__ uint4 tab[kAccTab];
    const int64_t g0 = (int64_t)blockIdx.x * kAccSites;
    if (g0 >= total) return;  // whole CTAs
    const int r = block_rep[blockIdx.x];
    const BatchRep& R = reps[r];
    const int64_t t0 = g0 - prefix[r];
    const int64_t cnt = ccount[(size_t)r * ncol + colour];
    const uint32_t sweep = R.sweep0 + ctr->e * (uint32_t)nmetro + (uint32_t)j;
    const int64_t t = t0 + threadIdx.x;
    const bool live = t < cnt;
    if (R.lat_kind == MQV_LATTICE_HYPERCUBIC) {
        const uint32_t run0 = (uint32_t)(t0 / 32);  // sites [2 t0, 2 t0 + 2 kAccSites)
        if (threadIdx.x < 32) accept_tab_fill(tab, run0, R.key, sweep, R.replica);
        __syncthreads();
        with_dim(R.st, [&](const auto& lt) {
            batch_site<F32>(R, lt, F32 ? parity_site_f(lt, t, colour) : parity_site(lt, t, colour), sweep, live,
                            colour, tab, run0);
        });
    } else {
        const int32_t* ord = R.order + cbegin[(size_t)r * ncol + colour];
        batch_site<F32>(R, R.csr, live ? (int64_t)ord[t] : 0, sweep, live, 0, nullptr, 0u);
    }
}

template <bool F32>
__global__ void __launch_bounds__(1024) batch_wolff(const BatchRep* __restrict__ reps,
                                                    const BatchCtr* __restrict__ ctr, int ncluster, int c,
                                                    int32_t* __restrict__ csize, int nrep)
{
    const BatchRep& R = reps[blockIdx.x];
    if (R.resident) return;  // its clusters are grown by batch_resident
    const uint32_t e = ctr->e, slot = e - ctr->ebase;
    const uint32_t serial = R.cluster0 + e * (uint32_t)ncluster + (uint32_t)c;
    int32_t* out = csize + ((size_t)slot * ncluster + c) * nrep + blockIdx.x;
    const uint32_t tgs = tag(kWolffSeed, R.replica), tgb = tag(kWolffBond, R.replica);
    // frontier buffers: int8 ids, or float ids followed by their projections
    __shared__ __align__(16) unsigned char wbuf[kWolffSmem];
    int32_t* fbuf = reinterpret_cast<int32_t*>(wbuf);
    double* fproj = reinterpret_cast<double*>(wbuf + 2 * kWolffCapF * sizeof(int32_t));
    if (F32) {
        if (R.lat_kind == MQV_LATTICE_HYPERCUBIC)
            wolff_f32_cluster(R.md, R.st, (float*)R.s, R.visited, R.queue, out, R.key, serial, tgs, tgb, R.D, fbuf,
                              fproj);
        else
            wolff_f32_cluster(R.md, R.csr, (float*)R.s, R.visited, R.queue, out, R.key, serial, tgs, tgb, R.D, fbuf,
                              fproj);
    } else {
        if (R.lat_kind == MQV_LATTICE_HYPERCUBIC)
            wolff_int8_cluster(R.w, R.st, (int8_t*)R.s, R.visited, R.queue, out, R.key, serial, tgs, tgb, R.D, fbuf);
        else
            wolff_int8_cluster(R.w, R.csr, (int8_t*)R.s, R.visited, R.queue, out, R.key, serial, tgs, tgb, R.D, fbuf);
    }
}

// One CTA per (member, part): member sizes set their number of parts.
template <bool F32>
__global__ void batch_measure(const BatchRep* __restrict__ reps, const BatchCtr* __restrict__ ctr,
                              long long* __restrict__ acc, int nrep, const int32_t* __restrict__ meas_prefix,
                              const int32_t* __restrict__ meas_rep)
{
    const int r = meas_rep[blockIdx.x];
    const int part = (int)blockIdx.x - meas_prefix[r], nparts = meas_prefix[r + 1] - meas_prefix[r];
    const BatchRep& R = reps[r];
    const uint32_t slot = ctr->e - ctr->ebase;
    long long* a = acc + ((size_t)slot * nrep + r) * kAccStride;
    if (F32) {
        if (R.lat_kind == MQV_LATTICE_HYPERCUBIC)
            with_dim(R.st, [&](const auto& lt) { measure_f32_part(R.md, lt, (const float*)R.s, (double*)a, part, nparts); });
        else
            measure_f32_part(R.md, R.csr, (const float*)R.s, (double*)a, part, nparts);
    } else {
        if (R.lat_kind == MQV_LATTICE_HYPERCUBIC)
            with_dim(R.st, [&](const auto& lt) { measure_int8_part(R.md, lt, (const int8_t*)R.s, a, part, nparts); });
        else
            measure_int8_part(R.md, R.csr, (const int8_t*)R.s, a, part, nparts);
    }
}

__global__ void batch_tick(BatchCtr* ctr) { ctr->e += 1u; }

__global__ void batch_chunk_start(BatchCtr* ctr, uint32_t e)
{
    ctr->e = e;
    ctr->ebase = e;
}

// acc/out: slot-major, entry k = slot * nrep + member
__global__ void batch_finalize(const BatchRep* __restrict__ reps, const long long* __restrict__ acc, int nslots,
                               int nrep, int f32, double* __restrict__ out)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)nslots * nrep) return;
    const BatchRep& R = reps[k % nrep];
    const int64_t n = R.lat_kind == MQV_LATTICE_HYPERCUBIC ? R.st.n : R.csr.n;
    if (f32) finalize_f32_one(R.md, n, (const double*)(acc + (size_t)k * kAccStride), out + 4 * (size_t)k);
    else finalize_int8_one(R.md, n, acc + (size_t)k * kAccStride, out + 4 * (size_t)k);
}

// raw sums (interaction, sum s, sum s^2, sum (s^2 - 1)^2) -> samples[r][e0 + slot][4]
__global__ void batch_samples(const long long* __restrict__ acc, int nslots, int nrep, int f32, int e0, int n_total,
                              double* __restrict__ out)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)nslots * nrep) return;
    const int slot = (int)(k / nrep), r = (int)(k % nrep);
    const long long* a = acc + (size_t)k * kAccStride;
    double* o = out + ((size_t)r * n_total + e0 + slot) * 4;
    if (f32) {
        const double* d = (const double*)a;
        o[0] = d[kAccEne];
        o[1] = d[kAccMag];
        o[2] = d[kAccSq];
        o[3] = d[kAccQ4];
    } else {
        o[0] = (double)a[kAccEne];
        o[1] = (double)a[kAccMag];
        o[2] = (double)a[kAccSq];
        o[3] = 0.0;
    }
}

// Replica exchange after the EMCS just done: one thread per pair of the step's
// plan, the pairs of a step disjoint (host-checked), a self pair skipped.
// CXX11Scheduler::calcprob / calcMHratio / exchange_statespace
// (src/libmarqov/marqovscheduler.h:44-57,445-470): action = beta * E_total
// (Core::calcAction, src/libmarqov/core.h:1145-1151) with E_total the
// measured energy per site times the sites; the two members share their
// Hamiltonian and lattice (host-checked), so each member's action of the
// partner's state is its beta times the partner's energy.  The exchange
// swaps the members' state pointers in the member table (the graphs read
// them there) and in the permutation the host applies to its handles.
template <bool F32>
__global__ void batch_temper(BatchRep* __restrict__ reps, const BatchCtr* __restrict__ ctr,
                             const long long* __restrict__ acc, int nrep, const int32_t* __restrict__ pairs,
                             int npairs, uint32_t step, Key key, double en_min, double en_max,
                             int32_t* __restrict__ perm, int32_t* __restrict__ flags)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int a = pairs[2 * p], b = pairs[2 * p + 1];
    if (a == b) {
        flags[p] = -1;
        return;
    }
    const uint32_t slot = ctr->e - 1u - ctr->ebase;
    double oa[4], ob[4];
    BatchRep& Ra = reps[a];
    BatchRep& Rb = reps[b];
    const int64_t n = Ra.lat_kind == MQV_LATTICE_HYPERCUBIC ? Ra.st.n : Ra.csr.n;
    const long long* acc_a = acc + ((size_t)slot * nrep + a) * kAccStride;
    const long long* acc_b = acc + ((size_t)slot * nrep + b) * kAccStride;
    if (F32) {
        finalize_f32_one(Ra.md, n, (const double*)acc_a, oa);
        finalize_f32_one(Rb.md, n, (const double*)acc_b, ob);
    } else {
        finalize_int8_one(Ra.md, n, acc_a, oa);
        finalize_int8_one(Rb.md, n, acc_b, ob);
    }
    const double Ea = MQV_DMUL(oa[0], (double)n), Eb = MQV_DMUL(ob[0], (double)n);
    const double aa = MQV_DMUL(Ra.md.beta, Ea), ab = MQV_DMUL(Ra.md.beta, Eb);
    const double bb = MQV_DMUL(Rb.md.beta, Eb), ba = MQV_DMUL(Rb.md.beta, Ea);
    const double en = MQV_DSUB(MQV_DADD(MQV_DSUB(aa, ab), bb), ba);
    double ratio = 0.0;
    if (en > en_min) ratio = en > en_max ? 1.7976931348623157e308 : exp(en);
    const double u = (double)(lo64(philox(step, (uint32_t)p, 0u, tag(kTemper, 0u), key)) >> 11) * 0x1.0p-53;
    const bool acc_ok = u < fmin(1.0, ratio);
    flags[p] = acc_ok ? 1 : 0;
    if (acc_ok) {
        void* t = Ra.s;
        Ra.s = Rb.s;
        Rb.s = t;
        const int32_t q = perm[a];
        perm[a] = perm[b];
        perm[b] = q;
    }
}

// ---- launchers (stream-ordered; all capturable) ------------------------------------

template <bool F32>
static void launch_emcs_t(const BatchLaunch& b, cudaStream_t st, int ncluster, int nmetro)
{
    for (int c = 0; c < ncluster; ++c) {
        if (b.wolff_ccl) {
            CclSeed* sd = (CclSeed*)b.ccl_seeds;
            const unsigned gb = (unsigned)b.site_blocks;
            if (b.site_blocks == 0) continue;  // every member is resident
            ccl_seed<F32><<<(b.nrep + 127) / 128, 128, 0, st>>>(b.reps, b.ctr, ncluster, c, sd, b.csize, b.nrep);
            ccl_local<F32><<<gb, kBatchMetroThreads, 0, st>>>(b.reps, b.site_prefix, b.site_block_rep, b.total_sites,
                                                              sd, b.ctr, ncluster, c);
            ccl_hook<F32><<<gb, kBatchMetroThreads, 0, st>>>(b.reps, b.site_prefix, b.site_block_rep, b.total_sites,
                                                             sd, b.ctr, ncluster, c);
            ccl_halve<<<gb, kBatchMetroThreads, 0, st>>>(b.reps, b.site_prefix, b.site_block_rep, b.total_sites);
            ccl_flip<F32><<<gb, kBatchMetroThreads, 0, st>>>(b.reps, b.site_prefix, b.site_block_rep, b.total_sites,
                                                             sd, b.ctr, ncluster, c, b.csize, b.nrep);
        } else {
            batch_wolff<F32><<<b.nrep, 1024, 0, st>>>(b.reps, b.ctr, ncluster, c, b.csize, b.nrep);
        }
    }
    for (int j = 0; j < nmetro; ++j)
        for (int colour = 0; colour < b.ncol; ++colour) {
            if (b.total[colour] == 0) continue;
            batch_metro<F32><<<b.blocks[colour], kBatchMetroThreads, 0, st>>>(
                b.reps, b.prefix + (size_t)colour * (b.nrep + 1), b.block_rep + b.block_off[colour], b.cbegin,
                b.ccount, b.ncol, b.total[colour], colour, b.ctr, nmetro, j);
        }
    if (b.meas_blocks > 0)
        batch_measure<F32><<<b.meas_blocks, 256, 0, st>>>(b.reps, b.ctr, b.acc, b.nrep, b.meas_prefix, b.meas_rep);
    batch_tick<<<1, 1, 0, st>>>(b.ctr);
}

cudaError_t batch_launch_emcs(const BatchLaunch& b, cudaStream_t st, int ncluster, int nmetro)
{
    if (b.f32) launch_emcs_t<true>(b, st, ncluster, nmetro);
    else launch_emcs_t<false>(b, st, ncluster, nmetro);
    return cudaGetLastError();
}

cudaError_t batch_launch_chunk_start(const BatchLaunch& b, cudaStream_t st, uint32_t e)
{
    batch_chunk_start<<<1, 1, 0, st>>>(b.ctr, e);
    return cudaGetLastError();
}

cudaError_t batch_launch_finalize(const BatchLaunch& b, cudaStream_t st, int nslots, double* out)
{
    const int64_t n = (int64_t)nslots * b.nrep;
    batch_finalize<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(b.reps, b.acc, nslots, b.nrep, b.f32, out);
    return cudaGetLastError();
}

cudaError_t batch_launch_temper(const BatchLaunch& b, cudaStream_t st, const int32_t* pairs, int npairs, uint32_t step,
                                uint64_t seed, double en_min, double en_max, int32_t* perm, int32_t* flags)
{
    if (npairs <= 0) return cudaSuccess;
    const unsigned g = (unsigned)((npairs + 127) / 128);
    if (b.f32)
        batch_temper<true><<<g, 128, 0, st>>>(const_cast<BatchRep*>(b.reps), b.ctr, b.acc, b.nrep, pairs, npairs, step,
                                               make_key(seed), en_min, en_max, perm, flags);
    else
        batch_temper<false><<<g, 128, 0, st>>>(const_cast<BatchRep*>(b.reps), b.ctr, b.acc, b.nrep, pairs, npairs,
                                                step, make_key(seed), en_min, en_max, perm, flags);
    return cudaGetLastError();
}

cudaError_t batch_launch_samples(const BatchLaunch& b, cudaStream_t st, int nslots, int e0, int n_total,
                                 double* samples)
{
    const int64_t n = (int64_t)nslots * b.nrep;
    batch_samples<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(b.acc, nslots, b.nrep, b.f32, e0, n_total, samples);
    return cudaGetLastError();
}

}  // namespace mqv
