// C ABI of the marqov_b200 engine: handle lifecycle, descriptor lowering and
// validation, the EMCS driver and state transfer.  No exception crosses the
// ABI; every entry point returns an mqv_status and leaves a message for
// mqv_last_error on failure.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "batch.h"
#include "engine.h"

namespace mqv {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }

// launchers implemented in the kernel files
cudaError_t launch_init_int8(Sim* s);
cudaError_t launch_metropolis_int8(Sim* s, int slot);
cudaError_t launch_measure_int8(Sim* s, int slot);
cudaError_t launch_finalize_int8(Sim* s, int nslots, double* d_out);
cudaError_t launch_wolff_int8(Sim* s, int slot);
cudaError_t ensure_cuts(Sim* s);
cudaError_t launch_init_f32(Sim* s);
cudaError_t launch_metropolis_f32(Sim* s, int slot);
cudaError_t launch_measure_f32(Sim* s, int slot);
cudaError_t launch_finalize_f32(Sim* s, int nslots, double* d_out);
cudaError_t launch_wolff_f32(Sim* s, int slot);
cudaError_t launch_wolff_label(Sim* s, int slot);
int64_t wolff_noalloc_max_sites();
int wolff_noalloc_max_clusters();
cudaError_t wolff_noalloc_scratch(int device, uint32_t** out);
cudaError_t launch_wolff_int8_noalloc(Sim* s, uint32_t* scratch, int slot);
const int32_t* wolff_noalloc_sizes(const uint32_t* scratch);
bool resident_fits(const Sim* s);
cudaError_t launch_emcs_cluster(Sim* s, int n_emcs, int ncluster, int nmetro, long long* acc, int32_t* csize);
cudaError_t launch_emcs_resident(Sim* s, int n_emcs, int ncluster, int nmetro, bool measure, long long* acc,
                                 int32_t* csize);
cudaError_t launch_acc_to_samples(const long long* acc, int is_f32, int nslots, double* out, cudaStream_t st);
cudaError_t launch_phi4_fdt(const double* samples, int nrep, int nsamp, double invN, const double* beta,
                            const double* lam, double mass, double* obs, double* jac, const double* gout,
                            double* grads, cudaStream_t st);

// Smallest u53 rejected by update_accepted<pref>(dE, beta, .), 2^53 when all
// are accepted: the rule accepts exactly the words with u53 below a cut.
unsigned long long accept_cut(int pref, double dE, double beta)
{
    if (dE <= 0) return 1ull << 53;
    if (!update_accepted(pref, dE, beta, 0)) return 0;
    unsigned long long lo = 1, hi = 1ull << 53;
    while (lo < hi) {
        const unsigned long long mid = lo + (hi - lo) / 2;
        if (update_accepted(pref, dE, beta, mid << 11)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static bool is_f32_kind(int k) { return k == MQV_MODEL_HEISENBERG || k == MQV_MODEL_PHI4 || k == MQV_MODEL_XXZ; }

bool ising2d_supported(int L);
int ising2d_band_config(const Sim* s);
const char* ising2d_config_name(Sim* s, char* buf, int len);
cudaError_t launch_split_rows(Sim* s, const void* rowmajor, void* split);
cudaError_t launch_merge_rows(Sim* s, const void* split, void* rowmajor);
cudaError_t launch_validate_int8(Sim* s, const void* rowmajor, int* flag);

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int now = -1;
        cudaGetDevice(&now);
        if (prev >= 0 && now != prev) cudaSetDevice(prev);
    }
};

#define MQV_CK(expr)                                                                         \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #expr); \
            return e_ == cudaErrorMemoryAllocation ? MQV_ERR_OUT_OF_MEMORY : MQV_ERR_CUDA;   \
        }                                                                                    \
    } while (0)

static mqv_status fail(mqv_status st, const std::string& msg)
{
    set_error(msg);
    return st;
}

static void free_sim(Sim* s)
{
    if (!s) return;
    DeviceGuard g(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (void* p : {s->state[0], s->state[1], (void*)s->d_rp, (void*)s->d_ci, (void*)s->d_bonds, (void*)s->d_order,
                    (void*)s->d_acc, (void*)s->d_obs, (void*)s->d_visited, (void*)s->d_queue, (void*)s->d_csize,
                    (void*)s->d_status, (void*)s->d_counter, (void*)s->d_cuts, (void*)s->d_rep1, (void*)s->d_ctr1,
                    s->d_seed1, (void*)s->d_sprefix1, (void*)s->d_sbrep1})
        if (p) cudaFree(p);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

static mqv_status ensure_slots(Sim* s, int nslots)
{
    if (nslots <= s->nslots) return MQV_OK;
    if (s->d_acc) cudaFree(s->d_acc);
    if (s->d_obs) cudaFree(s->d_obs);
    s->d_acc = nullptr;
    s->d_obs = nullptr;
    s->nslots = 0;
    MQV_CK(cudaMalloc(&s->d_acc, sizeof(long long) * kAccStride * (size_t)nslots));
    MQV_CK(cudaMalloc(&s->d_obs, sizeof(double) * 4 * (size_t)nslots));
    s->nslots = nslots;
    return MQV_OK;
}

static mqv_status ensure_cslots(Sim* s, int n)
{
    if (n <= s->nslots_c) return MQV_OK;
    if (s->d_csize) cudaFree(s->d_csize);
    s->d_csize = nullptr;
    s->nslots_c = 0;
    MQV_CK(cudaMalloc(&s->d_csize, sizeof(int32_t) * (size_t)n));
    s->nslots_c = n;
    return MQV_OK;
}

static mqv_status ensure_wolff(Sim* s)
{
    if (s->d_queue) return MQV_OK;
    MQV_CK(cudaMalloc(&s->d_queue, sizeof(int32_t) * (size_t)s->n));
    const size_t words = (size_t)((s->n + 31) / 32);
    MQV_CK(cudaMalloc(&s->d_visited, sizeof(uint32_t) * words));
    MQV_CK(cudaMemsetAsync(s->d_visited, 0, sizeof(uint32_t) * words, s->stream));
    return MQV_OK;
}

// Reads (and clears) the device error word that bounded waits set.
static mqv_status check_device_status(Sim* s)
{
    int st = 0;
    MQV_CK(cudaMemcpyAsync(&st, s->d_status, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    MQV_CK(cudaStreamSynchronize(s->stream));
    if (st != 0) {
        MQV_CK(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
        s->failed = true;
        return fail(st, "a device-side wait gave up (status " + std::to_string(st) +
                            "): the sweep in flight was abandoned and the state is incomplete; set the state "
                            "again (mqv_set_state or mqv_init_state) before the next run");
    }
    return MQV_OK;
}

// Compute on a handle whose last run timed out is refused until its state is set again.
static mqv_status check_runnable(const Sim* s)
{
    if (s->failed)
        return fail(MQV_ERR_STATE, "a device wait timed out in an earlier run; set the state again (mqv_set_state "
                                   "or mqv_init_state) first");
    if (!s->initialised) return fail(MQV_ERR_STATE, "state not initialised");
    return MQV_OK;
}

// ---- lattice lowering -----------------------------------------------------------

static mqv_status lower_csr(Sim* s, const mqv_lattice_desc* L)
{
    const int64_t n = L->n;
    if (n < 2 || n >= (int64_t)1 << 31) return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: n out of range");
    if (!L->row_ptr || !L->col_idx) return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: row_ptr/col_idx missing");
    const int32_t* rp = L->row_ptr;
    const int32_t* ci = L->col_idx;
    if (rp[0] != 0) return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: row_ptr[0] != 0");
    int maxdeg = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (rp[i + 1] < rp[i]) return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: row_ptr not monotone");
        maxdeg = std::max(maxdeg, rp[i + 1] - rp[i]);
    }
    const int64_t nnz = rp[n];
    // neighbour ids in range, no self bonds, symmetric adjacency with equal bond weights
    std::vector<std::pair<int64_t, int64_t>> e;
    e.reserve((size_t)nnz);
    for (int64_t i = 0; i < n; ++i)
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int64_t j = ci[p];
            if (j < 0 || j >= n) return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: neighbour id out of range");
            if (j == i) return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: self bond at site " + std::to_string(i));
            e.emplace_back(i, j);
        }
    {
        std::vector<std::pair<int64_t, int64_t>> a = e, b;
        b.reserve(a.size());
        for (auto& x : a) b.emplace_back(x.second, x.first);
        std::sort(a.begin(), a.end());
        std::sort(b.begin(), b.end());
        if (a != b) return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: adjacency is not symmetric");
        if (std::adjacent_find(a.begin(), a.end()) != a.end())
            return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: repeated bond");
    }
    if (L->bonds) {
        // bnds must be symmetric: the weight of (i,j) equals that of (j,i)
        std::vector<std::vector<std::pair<int32_t, int8_t>>> w((size_t)n);
        for (int64_t i = 0; i < n; ++i)
            for (int32_t p = rp[i]; p < rp[i + 1]; ++p) w[i].emplace_back(ci[p], L->bonds[p]);
        for (auto& v : w) std::sort(v.begin(), v.end());
        for (int64_t i = 0; i < n; ++i)
            for (auto& pr : w[i]) {
                auto& o = w[pr.first];
                auto it = std::lower_bound(o.begin(), o.end(), std::make_pair((int32_t)i, (int8_t)-128));
                if (it == o.end() || it->first != i || it->second != pr.second)
                    return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: bond weights are not symmetric");
            }
    }
    // colours: given (validated) or greedy in site order
    std::vector<int32_t> col((size_t)n, -1);
    int ncol = 0;
    if (L->colours) {
        for (int64_t i = 0; i < n; ++i) {
            if (L->colours[i] < 0 || L->colours[i] > 4096)
                return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: colour out of range");
            col[i] = L->colours[i];
            ncol = std::max(ncol, col[i] + 1);
        }
        for (int64_t i = 0; i < n; ++i)
            for (int32_t p = rp[i]; p < rp[i + 1]; ++p)
                if (col[ci[p]] == col[i]) return fail(MQV_ERR_BAD_DESCRIPTOR, "CSR lattice: colouring is not proper");
    } else {
        std::vector<int64_t> mark((size_t)maxdeg + 2, -1);
        for (int64_t i = 0; i < n; ++i) {
            for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
                const int c = col[ci[p]];
                if (c >= 0 && c <= maxdeg) mark[c] = i;
            }
            int c = 0;
            while (mark[c] == i) ++c;
            col[i] = c;
            ncol = std::max(ncol, c + 1);
        }
    }
    std::vector<int32_t> order((size_t)n);
    s->colour_ptr.assign((size_t)ncol + 1, 0);
    for (int64_t i = 0; i < n; ++i) s->colour_ptr[col[i] + 1]++;
    for (int c = 0; c < ncol; ++c) s->colour_ptr[c + 1] += s->colour_ptr[c];
    {
        std::vector<int32_t> fill(s->colour_ptr.begin(), s->colour_ptr.end() - 1);
        for (int64_t i = 0; i < n; ++i) order[fill[col[i]]++] = (int32_t)i;
    }
    MQV_CK(cudaMalloc(&s->d_rp, sizeof(int32_t) * (size_t)(n + 1)));
    MQV_CK(cudaMalloc(&s->d_ci, sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1)));
    MQV_CK(cudaMalloc(&s->d_order, sizeof(int32_t) * (size_t)n));
    MQV_CK(upload_sync(s->stream, s->d_rp, rp, sizeof(int32_t) * (size_t)(n + 1)));
    MQV_CK(upload_sync(s->stream, s->d_ci, ci, sizeof(int32_t) * (size_t)nnz));
    MQV_CK(upload_sync(s->stream, s->d_order, order.data(), sizeof(int32_t) * (size_t)n));
    if (L->bonds) {
        MQV_CK(cudaMalloc(&s->d_bonds, (size_t)std::max<int64_t>(nnz, 1)));
        MQV_CK(upload_sync(s->stream, s->d_bonds, L->bonds, (size_t)nnz));
    }
    s->n = n;
    s->max_degree = maxdeg;
    s->csr = CSRDev{n, s->d_rp, s->d_ci, s->d_bonds};
    uint64_t h = 1469598103934665603ull;
    auto mix = [&h](const void* p, size_t bytes) {
        const unsigned char* c = (const unsigned char*)p;
        for (size_t k = 0; k < bytes; ++k) h = (h ^ c[k]) * 1099511628211ull;
    };
    mix(rp, sizeof(int32_t) * (size_t)(n + 1));
    mix(ci, sizeof(int32_t) * (size_t)nnz);
    if (L->bonds) mix(L->bonds, (size_t)nnz);
    s->lat_hash = h;
    return MQV_OK;
}

static uint64_t fnv1a(const void* p, size_t bytes, uint64_t h = 1469598103934665603ull)
{
    const unsigned char* c = (const unsigned char*)p;
    for (size_t k = 0; k < bytes; ++k) h = (h ^ c[k]) * 1099511628211ull;
    return h;
}

// Bonds of a hypercubic lattice, given per neighbour entry in nbrs(0, i)
// order (+x, -x, +y, -y, ...; RegularRandomBond::bnds,
// src/lattice/regular_random_bond.h:58-67): checked symmetric and stored as
// one plane of +d bonds per dimension (StencilDev::fb), 1 byte per site and
// dimension.
static mqv_status lower_stencil_bonds(Sim* s, const int8_t* bonds)
{
    const int64_t n = s->n;
    const int dim = s->dim, deg = 2 * dim;
    std::vector<int8_t> fb((size_t)dim * (size_t)n);
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < dim; ++d) {
            const int8_t w = bonds[(size_t)i * deg + 2 * d];
            const int64_t j = s->sten.nbr(i, 2 * d);
            if (bonds[(size_t)j * deg + 2 * d + 1] != w)
                return fail(MQV_ERR_BAD_DESCRIPTOR, "hypercubic bonds are not symmetric at site " + std::to_string(i));
            fb[(size_t)d * n + i] = w;
        }
    MQV_CK(cudaMalloc(&s->d_bonds, fb.size()));
    MQV_CK(upload_sync(s->stream, s->d_bonds, fb.data(), fb.size()));
    s->sten.fb = s->d_bonds;
    s->lat_hash = fnv1a(fb.data(), fb.size());
    return MQV_OK;
}

static mqv_status lower_model(Sim* s, const mqv_model_desc* m, bool has_bonds)
{
    if (m->kind < MQV_MODEL_ISING || m->kind > MQV_MODEL_XXZ)
        return fail(MQV_ERR_UNSUPPORTED_TERM, "unsupported model kind " + std::to_string(m->kind));
    if (m->kind == MQV_MODEL_POTTS && (m->q < 2 || m->q > 64))
        return fail(MQV_ERR_UNSUPPORTED_TERM, "Potts q must be in [2, 64]");
    if (m->kind == MQV_MODEL_EA && !has_bonds)
        return fail(MQV_ERR_BAD_DESCRIPTOR, "EdwardsAndersonIsing needs a lattice with bonds");
    if (has_bonds && !(m->kind == MQV_MODEL_EA || m->kind == MQV_MODEL_ISING || m->kind == MQV_MODEL_ISING_EMBED))
        return fail(MQV_ERR_UNSUPPORTED_TERM, "lattice bonds are supported for Ising-type models only");
    if (m->proposal == MQV_PROPOSAL_SMALL_CAP &&
        !(m->kind == MQV_MODEL_HEISENBERG || m->kind == MQV_MODEL_XXZ))
        return fail(MQV_ERR_UNSUPPORTED_TERM, "small-cap proposals need an O(3) model");
    if (m->proposal == MQV_PROPOSAL_SMALL_CAP && !(m->cap >= -1.0 && m->cap < 1.0))
        return fail(MQV_ERR_INVALID_ARG, "small-cap proposal: cap must be cos(half-angle) in [-1, 1)");
    for (double v : {m->J, m->h, m->h2, m->k, m->delta, m->cap})
        if (!std::isfinite(v)) return fail(MQV_ERR_INVALID_ARG, "model coefficients must be finite");
    s->model = *m;
    s->md.kind = m->kind;
    s->md.q = m->q;
    s->md.proposal = m->proposal;
    s->md.J = m->J;
    s->md.h = m->h;
    s->md.h2 = m->h2;
    s->md.k = m->k;
    s->md.delta = m->delta;
    s->md.cap = m->cap;
    s->md.termsel = s->termsel;
    s->is_f32 = is_f32_kind(m->kind);
    s->symd = (m->kind == MQV_MODEL_HEISENBERG || m->kind == MQV_MODEL_XXZ) ? 3 : 1;
    s->md.symd = s->symd;
    return MQV_OK;
}

static mqv_status launch_measure(Sim* s, int slot)
{
    MQV_CK(s->is_f32 ? launch_measure_f32(s, slot) : launch_measure_int8(s, slot));
    return MQV_OK;
}
static mqv_status launch_finalize(Sim* s, int nslots)
{
    MQV_CK(s->is_f32 ? launch_finalize_f32(s, nslots, s->d_obs) : launch_finalize_int8(s, nslots, s->d_obs));
    return MQV_OK;
}
static mqv_status launch_sweep(Sim* s, int slot)
{
    MQV_CK(s->is_f32 ? launch_metropolis_f32(s, slot) : launch_metropolis_int8(s, slot));
    return MQV_OK;
}
// Clusters by labelling (a fixed number of whole-lattice passes) or by one
// CTA's breadth-first growth (one barrier per level of the cluster's depth):
// MQV_WOLFF_AUTO labels int8 lattices of at least kLabelMinSites sites, where
// critical clusters are thousands of levels deep; both give the same cluster.
constexpr int64_t kLabelMinSites = (int64_t)1 << 18;
static bool cluster_by_label(const Sim* s)
{
    if (s->wolff_algo == MQV_WOLFF_LABEL) return true;
    if (s->wolff_algo == MQV_WOLFF_BFS) return false;
    return !s->is_f32 && s->n >= kLabelMinSites;
}

static mqv_status launch_cluster(Sim* s, int slot)
{
    mqv_status st = ensure_wolff(s);
    if (st) return st;
    if (cluster_by_label(s)) MQV_CK(launch_wolff_label(s, slot));
    else MQV_CK(s->is_f32 ? launch_wolff_f32(s, slot) : launch_wolff_int8(s, slot));
    return MQV_OK;
}

static mqv_status check_wolff_supported(Sim* s)
{
    if (s->md.kind == MQV_MODEL_ISING_EMBED && s->md.J > 0)
        return fail(MQV_ERR_UNSUPPORTED_TERM, "embedded Wolff clusters need a ferromagnetic J < 0");
    if (s->md.kind == MQV_MODEL_BLUME_CAPEL || s->md.kind == MQV_MODEL_EA)
        return fail(MQV_ERR_UNSUPPORTED_TERM, "no Wolff embedding for this model");
    if (s->is_f32 && s->md.J > 0)
        return fail(MQV_ERR_UNSUPPORTED_TERM, "embedded Wolff clusters need a ferromagnetic J < 0");
    if (s->is_f32 && s->md.kind == MQV_MODEL_XXZ)
        return fail(MQV_ERR_UNSUPPORTED_TERM, "no Wolff embedding for XXZ");
    return MQV_OK;
}

// A single handle takes the resident path by default up to this many sites:
// one SM then beats a launch per cluster, colour and measurement (2D Ising
// at L = 128: 176 against 335 us per EMCS); above it the launches, which
// spread a sweep over every SM, win (L = 256: 678 against 646 us).
constexpr int64_t kResidentAutoSites = 16384;
// EMCS of this handle run on the resident path (smem_emcs.cu)?
static bool use_resident(const Sim* s)
{
    if ((s->flags & MQV_FLAG_NO_RESIDENT) || !resident_fits(s)) return false;
    return (s->flags & MQV_FLAG_RESIDENT) || s->n <= kResidentAutoSites;
}
// ... or on a thread-block cluster (cluster_emcs.cu), for int8 stencils of
// 65,537 .. 262,144 sites the device can co-schedule (when asked for)
static bool use_cluster(Sim* s)
{
    if (!(s->flags & MQV_FLAG_RESIDENT) || s->is_f32 || s->lat_kind != MQV_LATTICE_HYPERCUBIC || resident_fits(s))
        return false;
    const int c = cluster_ctas(s->n);
    if (c < 2) return false;
    if (s->cluster_ok < 0) s->cluster_ok = cluster_launchable(c) ? 1 : 0;
    return s->cluster_ok == 1;
}

}  // namespace mqv

using namespace mqv;

#define MQV_GUARD(sim)                                                      \
    if (!(sim)) return fail(MQV_ERR_INVALID_ARG, "null handle");            \
    DeviceGuard guard_((sim)->device)

extern "C" {

MQV_API const char* mqv_version(void) { return "marqov_b200 0.1 (sm_100a)"; }

MQV_API mqv_status mqv_device_count(int32_t* count)
{
    if (!count) return fail(MQV_ERR_INVALID_ARG, "null argument");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return MQV_OK;
}

MQV_API mqv_status mqv_last_error(char* buf, size_t len)
{
    if (!buf || len == 0) return MQV_ERR_INVALID_ARG;
    std::snprintf(buf, len, "%s", g_err.c_str());
    return MQV_OK;
}

MQV_API mqv_status mqv_create(const mqv_model_desc* model, const mqv_lattice_desc* lattice,
                              const mqv_run_params* params, mqv_sim** out)
{
    if (!model || !lattice || !params || !out) return fail(MQV_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(MQV_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (params->device < 0 || params->device >= ndev) return fail(MQV_ERR_INVALID_ARG, "device ordinal out of range");
    if (!(params->beta >= 0) || !std::isfinite(params->beta)) return fail(MQV_ERR_INVALID_ARG, "beta must be finite and >= 0");
    if (params->replica > 0xFFFFFFu) return fail(MQV_ERR_INVALID_ARG, "replica id must fit in 24 bits");
    Sim* s = new (std::nothrow) Sim();
    if (!s) return fail(MQV_ERR_OUT_OF_MEMORY, "host allocation failed");
    s->device = params->device;
    DeviceGuard g(s->device);
    auto bail = [&](mqv_status st) {
        free_sim(s);
        return st;
    };
    // SimpleBipartite: the hypercubic stencil plus its termselector
    s->termsel = lattice->kind == MQV_LATTICE_BIPARTITE ? 1 : 0;
    mqv_status st = lower_model(s, model, lattice->bonds != nullptr);
    if (st) return bail(st);
    s->md.beta = params->beta;
    s->flags = params->flags;
    s->seed = params->seed;
    s->replica = params->replica;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("cudaStreamCreate failed");
        return bail(MQV_ERR_CUDA);
    }
    s->own_stream = true;
    if (lattice->kind == MQV_LATTICE_HYPERCUBIC || lattice->kind == MQV_LATTICE_BIPARTITE) {
        if (lattice->dim < 1 || lattice->dim > 4) return bail(fail(MQV_ERR_BAD_DESCRIPTOR, "hypercubic dim must be 1..4"));
        if (lattice->len < 4 || (lattice->len & 1))
            return bail(fail(MQV_ERR_BAD_DESCRIPTOR,
                             "hypercubic checkerboard needs an even side >= 4 (use a CSR lattice otherwise)"));
        int64_t n = 1;
        for (int j = 0; j < lattice->dim; ++j) {
            s->sten.pows[j] = n;
            n *= lattice->len;
            if (n >= (int64_t)1 << 31) return bail(fail(MQV_ERR_BAD_DESCRIPTOR, "lattice too large (>= 2^31 sites)"));
        }
        s->lat_kind = MQV_LATTICE_HYPERCUBIC;
        s->dim = lattice->dim;
        s->len = lattice->len;
        s->n = n;
        s->sten.dim = lattice->dim;
        s->sten.len = lattice->len;
        s->sten.n = n;
        s->sten.lg = -1;
        for (int b = 0; b < 31; ++b)
            if ((1 << b) == lattice->len) s->sten.lg = b;
        s->sten.mlen = s->sten.lg >= 0 ? 0 : UINT64_MAX / (uint64_t)lattice->len + 1;
        s->max_degree = 2 * lattice->dim;
        s->colour_ptr = {0, (int32_t)(n / 2), (int32_t)n};
        if (lattice->bonds) {
            st = lower_stencil_bonds(s, lattice->bonds);
            if (st) return bail(st);
        }
    } else if (lattice->kind == MQV_LATTICE_CSR) {
        s->lat_kind = MQV_LATTICE_CSR;
        st = lower_csr(s, lattice);
        if (st) return bail(st);
    } else {
        return bail(fail(MQV_ERR_BAD_DESCRIPTOR, "unknown lattice kind"));
    }
    s->fused_ising2d = !(params->flags & MQV_FLAG_PER_COLOUR) && !s->is_f32 && s->lat_kind == MQV_LATTICE_HYPERCUBIC &&
                       !s->d_bonds &&
                       s->dim == 2 && ising2d_supported(s->len) &&
                       (s->md.kind == MQV_MODEL_ISING || s->md.kind == MQV_MODEL_ISING_EMBED);
    s->sten.split = s->fused_ising2d ? 1 : 0;
    cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device);
    if (cudaMalloc(&s->d_status, sizeof(int)) != cudaSuccess || cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream) != cudaSuccess ||
        cudaMalloc(&s->d_counter, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of the status word failed");
        return bail(MQV_ERR_OUT_OF_MEMORY);
    }
    s->state_bytes = (size_t)s->n * (s->is_f32 ? sizeof(float) * s->symd : 1);
    if (cudaMalloc(&s->state[0], s->state_bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of the state failed");
        return bail(MQV_ERR_OUT_OF_MEMORY);
    }
    if (s->fused_ising2d && cudaMalloc(&s->state[1], s->state_bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of the second state buffer failed");
        return bail(MQV_ERR_OUT_OF_MEMORY);
    }
    st = ensure_slots(s, 64);
    if (st) return bail(st);
    st = ensure_cslots(s, 256);
    if (st) return bail(st);
    *out = reinterpret_cast<mqv_sim*>(s);
    return MQV_OK;
}

MQV_API mqv_status mqv_destroy(mqv_sim* h)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s) return MQV_OK;
    free_sim(s);
    return MQV_OK;
}

MQV_API mqv_status mqv_set_stream(mqv_sim* h, void* stream)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    MQV_CK(cudaStreamSynchronize(s->stream));
    if (s->own_stream) cudaStreamDestroy(s->stream);
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
    return MQV_OK;
}

MQV_API mqv_status mqv_get_stream(mqv_sim* h, void** stream)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s || !stream) return fail(MQV_ERR_INVALID_ARG, "null argument");
    *stream = (void*)s->stream;
    return MQV_OK;
}

MQV_API mqv_status mqv_set_beta(mqv_sim* h, double beta)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (!(beta >= 0) || !std::isfinite(beta)) return fail(MQV_ERR_INVALID_ARG, "beta must be finite and >= 0");
    s->md.beta = beta;
    return MQV_OK;
}

MQV_API mqv_status mqv_set_model(mqv_sim* h, const mqv_model_desc* m)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (!m) return fail(MQV_ERR_INVALID_ARG, "null model");
    if (m->kind != s->model.kind) return fail(MQV_ERR_INVALID_ARG, "mqv_set_model cannot change the model kind");
    const double beta = s->md.beta;
    mqv_status st = lower_model(s, m, s->d_bonds != nullptr);
    if (st) return st;
    s->md.beta = beta;
    return MQV_OK;
}

MQV_API mqv_status mqv_init_state(mqv_sim* h)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    MQV_CK(s->is_f32 ? launch_init_f32(s) : launch_init_int8(s));
    s->initialised = true;
    s->failed = false;
    return MQV_OK;
}

MQV_API mqv_status mqv_state_bytes(mqv_sim* h, size_t* bytes)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s || !bytes) return fail(MQV_ERR_INVALID_ARG, "null argument");
    *bytes = s->state_bytes;
    return MQV_OK;
}

MQV_API mqv_status mqv_get_state(mqv_sim* h, void* host, size_t bytes)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (s->failed) return check_runnable(s);
    if (!host || bytes != s->state_bytes)
        return fail(MQV_ERR_INVALID_ARG, "state buffer size mismatch (expected " + std::to_string(s->state_bytes) + ")");
    if (s->fused_ising2d) {
        // the other buffer is free between sweeps: merge the split rows into it
        MQV_CK(launch_merge_rows(s, s->state[s->cur], s->state[s->cur ^ 1]));
        MQV_CK(cudaMemcpyAsync(host, s->state[s->cur ^ 1], bytes, cudaMemcpyDeviceToHost, s->stream));
    } else if (s->is_f32 && s->symd > 1) {
        // device: one array per component; host: the reference's site-major vectors
        std::vector<float> soa((size_t)s->n * s->symd);
        MQV_CK(cudaMemcpyAsync(soa.data(), s->state[s->cur], bytes, cudaMemcpyDeviceToHost, s->stream));
        MQV_CK(cudaStreamSynchronize(s->stream));
        float* out = (float*)host;
        for (int c = 0; c < s->symd; ++c)
            for (int64_t i = 0; i < s->n; ++i) out[(size_t)i * s->symd + c] = soa[(size_t)c * s->n + i];
    } else {
        MQV_CK(cudaMemcpyAsync(host, s->state[s->cur], bytes, cudaMemcpyDeviceToHost, s->stream));
    }
    MQV_CK(cudaStreamSynchronize(s->stream));
    return check_device_status(s);
}

MQV_API mqv_status mqv_set_state(mqv_sim* h, const void* host, size_t bytes)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (!host || bytes != s->state_bytes)
        return fail(MQV_ERR_INVALID_ARG, "state buffer size mismatch (expected " + std::to_string(s->state_bytes) + ")");
    if (s->fused_ising2d) {
        // upload into the spare buffer, check every spin on the device, then
        // convert into the current buffer (left untouched on an illegal spin)
        int bad = 0;
        MQV_CK(cudaMemcpyAsync(s->state[s->cur ^ 1], host, bytes, cudaMemcpyHostToDevice, s->stream));
        MQV_CK(cudaMemsetAsync(s->d_counter, 0, sizeof(int), s->stream));
        MQV_CK(launch_validate_int8(s, s->state[s->cur ^ 1], s->d_counter));
        MQV_CK(cudaMemcpyAsync(&bad, s->d_counter, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MQV_CK(cudaStreamSynchronize(s->stream));
        if (bad) return fail(MQV_ERR_INVALID_ARG, "illegal spin value in the state");
        MQV_CK(launch_split_rows(s, s->state[s->cur ^ 1], s->state[s->cur]));
        MQV_CK(cudaStreamSynchronize(s->stream));
        s->initialised = true;
        s->failed = false;
        return MQV_OK;
    }
    if (!s->is_f32) {
        // integer states must be legal values of the model (branch-free scan)
        const int8_t* v = (const int8_t*)host;
        const int kind = s->md.kind, q = s->md.q;
        int bad = 0;
        if (kind == MQV_MODEL_POTTS)
            for (int64_t i = 0; i < s->n; ++i) bad |= (v[i] < 0) | (v[i] >= q);
        else if (kind == MQV_MODEL_BLUME_CAPEL)
            for (int64_t i = 0; i < s->n; ++i) bad |= (v[i] < -1) | (v[i] > 1);
        else
            for (int64_t i = 0; i < s->n; ++i) bad |= (v[i] * v[i]) != 1;
        if (bad) return fail(MQV_ERR_INVALID_ARG, "illegal spin value in the state");
    }
    if (s->is_f32 && s->symd > 1) {
        std::vector<float> soa((size_t)s->n * s->symd);
        const float* in = (const float*)host;
        for (int c = 0; c < s->symd; ++c)
            for (int64_t i = 0; i < s->n; ++i) soa[(size_t)c * s->n + i] = in[(size_t)i * s->symd + c];
        MQV_CK(cudaMemcpyAsync(s->state[s->cur], soa.data(), bytes, cudaMemcpyHostToDevice, s->stream));
        MQV_CK(cudaStreamSynchronize(s->stream));
        s->initialised = true;
        s->failed = false;
        return MQV_OK;
    }
    MQV_CK(cudaMemcpyAsync(s->state[s->cur], host, bytes, cudaMemcpyHostToDevice, s->stream));
    MQV_CK(cudaStreamSynchronize(s->stream));
    s->initialised = true;
        s->failed = false;
    return MQV_OK;
}

MQV_API mqv_status mqv_state_device_ptr(mqv_sim* h, void** dev, size_t* bytes)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s || !dev) return fail(MQV_ERR_INVALID_ARG, "null argument");
    *dev = s->state[s->cur];
    if (bytes) *bytes = s->state_bytes;
    return MQV_OK;
}

MQV_API mqv_status mqv_get_counters(mqv_sim* h, uint64_t* sweep, uint64_t* cluster)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s) return fail(MQV_ERR_INVALID_ARG, "null handle");
    if (sweep) *sweep = s->sweep;
    if (cluster) *cluster = s->cluster;
    return MQV_OK;
}

MQV_API mqv_status mqv_set_counters(mqv_sim* h, uint64_t sweep, uint64_t cluster)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s) return fail(MQV_ERR_INVALID_ARG, "null handle");
    s->sweep = sweep;
    s->cluster = cluster;
    return MQV_OK;
}

MQV_API mqv_status mqv_metropolis(mqv_sim* h, int32_t nsweeps)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (nsweeps < 0) return fail(MQV_ERR_INVALID_ARG, "nsweeps < 0");
    {
        const mqv_status rs = check_runnable(s);
        if (rs) return rs;
    }
    for (int t = 0; t < nsweeps; ++t) {
        mqv_status st = launch_sweep(s, -1);
        if (st) return st;
    }
    return MQV_OK;
}

MQV_API mqv_status mqv_wolff(mqv_sim* h, int32_t nclusters, int32_t* sizes)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (nclusters < 0) return fail(MQV_ERR_INVALID_ARG, "nclusters < 0");
    {
        const mqv_status rs = check_runnable(s);
        if (rs) return rs;
    }
    mqv_status st = check_wolff_supported(s);
    if (st) return st;
    int done = 0;
    while (done < nclusters) {
        const int chunk = std::min(nclusters - done, 65536);
        st = ensure_cslots(s, chunk);
        if (st) return st;
        if (use_resident(s)) {
            MQV_CK(launch_emcs_resident(s, chunk, 1, 0, false, nullptr, s->d_csize));
        } else if (use_cluster(s)) {
            MQV_CK(launch_emcs_cluster(s, chunk, 1, 0, nullptr, s->d_csize));
        } else {
            for (int c = 0; c < chunk; ++c) {
                st = launch_cluster(s, c);
                if (st) return st;
            }
        }
        if (sizes) {
            MQV_CK(cudaMemcpyAsync(sizes + done, s->d_csize, sizeof(int32_t) * chunk, cudaMemcpyDeviceToHost, s->stream));
            MQV_CK(cudaStreamSynchronize(s->stream));
        }
        done += chunk;
    }
    return MQV_OK;
}

// mqv_wolff without any device allocation: the clusters run on the static
// scratch of wolff.cu (int8 models, lattices of up to 2^20 sites).
MQV_API mqv_status mqv_wolff_noalloc(mqv_sim* h, int32_t nclusters, int32_t* sizes)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (nclusters < 0) return fail(MQV_ERR_INVALID_ARG, "nclusters < 0");
    {
        const mqv_status rs = check_runnable(s);
        if (rs) return rs;
    }
    mqv_status st = check_wolff_supported(s);
    if (st) return st;
    if (s->is_f32)
        return fail(MQV_ERR_UNSUPPORTED_TERM, "mqv_wolff_noalloc: int8 models only (Ising, embedded Ising, Potts)");
    if (s->n > wolff_noalloc_max_sites())
        return fail(MQV_ERR_INVALID_ARG, "mqv_wolff_noalloc: lattice of " + std::to_string(s->n) +
                                             " sites exceeds the static scratch limit of " +
                                             std::to_string(wolff_noalloc_max_sites()) + " sites");
    uint32_t* scratch = nullptr;
    MQV_CK(wolff_noalloc_scratch(s->device, &scratch));
    int done = 0;
    while (done < nclusters) {
        const int chunk = std::min(nclusters - done, wolff_noalloc_max_clusters());
        for (int c = 0; c < chunk; ++c) MQV_CK(launch_wolff_int8_noalloc(s, scratch, c));
        if (sizes) {
            MQV_CK(cudaMemcpyAsync(sizes + done, wolff_noalloc_sizes(scratch), sizeof(int32_t) * chunk,
                                   cudaMemcpyDeviceToHost, s->stream));
            MQV_CK(cudaStreamSynchronize(s->stream));
        }
        done += chunk;
    }
    return MQV_OK;
}

MQV_API mqv_status mqv_emcs(mqv_sim* h, int32_t n_emcs, int32_t ncluster, int32_t nmetro, mqv_obs* obs,
                            double* mean_cluster)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (n_emcs < 0 || ncluster < 0 || nmetro < 0) return fail(MQV_ERR_INVALID_ARG, "negative count");
    {
        const mqv_status rs = check_runnable(s);
        if (rs) return rs;
    }
    if (ncluster > 0) {
        mqv_status st = check_wolff_supported(s);
        if (st) return st;
    }
    const int CH = 1024;
    std::vector<int32_t> csz;
    int done = 0;
    while (done < n_emcs) {
        const int ch = std::min(n_emcs - done, CH);
        mqv_status st = ensure_slots(s, ch);
        if (st) return st;
        if (ncluster > 0) {
            st = ensure_cslots(s, ch * ncluster);
            if (st) return st;
        }
        MQV_CK(cudaMemsetAsync(s->d_acc, 0, sizeof(long long) * kAccStride * (size_t)ch, s->stream));
        if (use_resident(s)) {
            MQV_CK(ensure_cuts(s));
            MQV_CK(launch_emcs_resident(s, ch, ncluster, nmetro, true, s->d_acc, s->d_csize));
        } else if (use_cluster(s)) {
            MQV_CK(ensure_cuts(s));
            MQV_CK(launch_emcs_cluster(s, ch, ncluster, nmetro, s->d_acc, s->d_csize));
        } else {
            for (int e = 0; e < ch; ++e) {
                for (int c = 0; c < ncluster; ++c) {
                    st = launch_cluster(s, e * ncluster + c);
                    if (st) return st;
                }
                for (int j = 0; j < nmetro; ++j) {
                    st = launch_sweep(s, j == nmetro - 1 ? e : -1);
                    if (st) return st;
                }
                if (nmetro == 0) {
                    st = launch_measure(s, e);
                    if (st) return st;
                }
            }
        }
        st = launch_finalize(s, ch);
        if (st) return st;
        if (obs) MQV_CK(cudaMemcpyAsync(obs + done, s->d_obs, sizeof(double) * 4 * ch, cudaMemcpyDeviceToHost, s->stream));
        if (mean_cluster && ncluster > 0) {
            csz.resize((size_t)ch * ncluster);
            MQV_CK(cudaMemcpyAsync(csz.data(), s->d_csize, sizeof(int32_t) * csz.size(), cudaMemcpyDeviceToHost, s->stream));
        }
        if (obs || mean_cluster) {
            st = check_device_status(s);
            if (st) return st;
        }
        if (mean_cluster) {
            for (int e = 0; e < ch; ++e) {
                double a = 0;
                for (int c = 0; c < ncluster; ++c) a += (double)csz[(size_t)e * ncluster + c];
                mean_cluster[done + e] = ncluster > 0 ? a / ncluster : 0.0;
            }
        }
        done += ch;
    }
    return MQV_OK;
}

MQV_API mqv_status mqv_emcs_samples(mqv_sim* h, int32_t n_emcs, int32_t ncluster, int32_t nmetro, double* d_samples)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (n_emcs < 0 || ncluster < 0 || nmetro < 0) return fail(MQV_ERR_INVALID_ARG, "negative count");
    if (n_emcs > 0 && !d_samples) return fail(MQV_ERR_INVALID_ARG, "null sample buffer");
    {
        const mqv_status rs = check_runnable(s);
        if (rs) return rs;
    }
    if (ncluster > 0) {
        mqv_status st = check_wolff_supported(s);
        if (st) return st;
    }
    const int CH = 1024;
    int done = 0;
    while (done < n_emcs) {
        const int ch = std::min(n_emcs - done, CH);
        mqv_status st = ensure_slots(s, ch);
        if (st) return st;
        if (ncluster > 0) {
            st = ensure_cslots(s, ch * ncluster);
            if (st) return st;
        }
        MQV_CK(cudaMemsetAsync(s->d_acc, 0, sizeof(long long) * kAccStride * (size_t)ch, s->stream));
        if (use_resident(s)) {
            MQV_CK(ensure_cuts(s));
            MQV_CK(launch_emcs_resident(s, ch, ncluster, nmetro, true, s->d_acc, s->d_csize));
        } else if (use_cluster(s)) {
            MQV_CK(ensure_cuts(s));
            MQV_CK(launch_emcs_cluster(s, ch, ncluster, nmetro, s->d_acc, s->d_csize));
        } else {
            for (int e = 0; e < ch; ++e) {
                for (int c = 0; c < ncluster; ++c) {
                    st = launch_cluster(s, e * ncluster + c);
                    if (st) return st;
                }
                for (int j = 0; j < nmetro; ++j) {
                    st = launch_sweep(s, j == nmetro - 1 ? e : -1);
                    if (st) return st;
                }
                if (nmetro == 0) {
                    st = launch_measure(s, e);
                    if (st) return st;
                }
            }
        }
        MQV_CK(launch_acc_to_samples(s->d_acc, s->is_f32 ? 1 : 0, ch, d_samples + 4 * (size_t)done, s->stream));
        s->launches++;
        done += ch;
    }
    return MQV_OK;
}

MQV_API mqv_status mqv_phi4_fdt(const double* d_samples, int32_t nrep, int32_t nsamp, int64_t nsites, double mass,
                                const double* d_beta, const double* d_lambda, double* d_obs, double* d_jac,
                                const double* d_gout, double* d_grads, void* stream)
{
    if (!d_samples || !d_beta || !d_lambda || !d_obs || !d_jac) return fail(MQV_ERR_INVALID_ARG, "null argument");
    if (nrep < 1 || nsamp < 2 || nsites < 1) return fail(MQV_ERR_INVALID_ARG, "need nrep >= 1, nsamp >= 2, nsites >= 1");
    if ((d_gout == nullptr) != (d_grads == nullptr)) return fail(MQV_ERR_INVALID_ARG, "gout and grads go together");
    MQV_CK(launch_phi4_fdt(d_samples, nrep, nsamp, 1.0 / (double)nsites, d_beta, d_lambda, mass, d_obs, d_jac, d_gout,
                           d_grads, (cudaStream_t)stream));
    return MQV_OK;
}

MQV_API mqv_status mqv_measure(mqv_sim* h, mqv_obs* out)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (!out) return fail(MQV_ERR_INVALID_ARG, "null output");
    {
        const mqv_status rs = check_runnable(s);
        if (rs) return rs;
    }
    MQV_CK(cudaMemsetAsync(s->d_acc, 0, sizeof(long long) * kAccStride, s->stream));
    mqv_status st = launch_measure(s, 0);
    if (st) return st;
    st = launch_finalize(s, 1);
    if (st) return st;
    MQV_CK(cudaMemcpyAsync(out, s->d_obs, sizeof(double) * 4, cudaMemcpyDeviceToHost, s->stream));
    MQV_CK(cudaStreamSynchronize(s->stream));
    return check_device_status(s);
}

MQV_API mqv_status mqv_synchronize(mqv_sim* h)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    MQV_CK(cudaStreamSynchronize(s->stream));
    return check_device_status(s);
}

MQV_API mqv_status mqv_describe(mqv_sim* h, char* buf, size_t len)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    MQV_GUARD(s);
    if (!s || !buf || len == 0) return fail(MQV_ERR_INVALID_ARG, "bad arguments");
    char cfg[96] = "";
    if (s->fused_ising2d) ising2d_config_name(s, cfg, sizeof(cfg));
    // the sweep kernel's name, when there is one, ends the line
    std::snprintf(buf, len, "model=%d lattice=%s n=%lld clusters=%s path=%s%s%s", s->md.kind,
                  s->lat_kind == MQV_LATTICE_HYPERCUBIC ? (s->termsel ? "bipartite" : "hypercubic") : "csr", (long long)s->n,
                  use_resident(s) ? "label-smem" : use_cluster(s) ? "label-dsmem" : (cluster_by_label(s) ? "label" : "bfs"),
                  use_resident(s) ? "resident-smem"
                  : use_cluster(s) ? "resident-cluster"
                                   : (s->fused_ising2d ? "fused-2d-bitsliced" : (s->is_f32 ? "per-colour-f32" : "per-colour-int8")),
                  cfg[0] ? " kernel=" : "", cfg);
    return MQV_OK;
}

static uint64_t state_hash(const void* p, size_t bytes) { return fnv1a(p, bytes); }

MQV_API mqv_status mqv_get_state_checked(mqv_sim* h, void* host, size_t bytes, uint64_t* hash)
{
    if (!hash) return fail(MQV_ERR_INVALID_ARG, "null hash");
    const mqv_status st = mqv_get_state(h, host, bytes);
    if (st) return st;
    *hash = state_hash(host, bytes);
    return MQV_OK;
}

MQV_API mqv_status mqv_set_state_checked(mqv_sim* h, const void* host, size_t bytes, uint64_t hash)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s || !host) return fail(MQV_ERR_INVALID_ARG, "null argument");
    if (bytes != s->state_bytes)
        return fail(MQV_ERR_INVALID_ARG, "state buffer size mismatch (expected " + std::to_string(s->state_bytes) + ")");
    if (state_hash(host, bytes) != hash)
        return fail(MQV_ERR_CHECKSUM, "state checksum mismatch: the stored state is corrupt");
    return mqv_set_state(h, host, bytes);
}

MQV_API mqv_status mqv_selftest_inject_timeout(mqv_sim* h, int32_t row, uint64_t wait_ns)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s) return fail(MQV_ERR_INVALID_ARG, "null handle");
    if (!s->fused_ising2d || ising2d_band_config(s) < 0)
        return fail(MQV_ERR_UNSUPPORTED_TERM, "timeout injection needs the fused 2D Ising band path (L = 8192 or 16384)");
    if (row < 2 || row > 64) return fail(MQV_ERR_INVALID_ARG, "withheld row must be in [2, 64]");
    s->inject_row = row;
    s->inject_wait_ns = wait_ns;
    return MQV_OK;
}

MQV_API mqv_status mqv_set_wolff(mqv_sim* h, int32_t algorithm)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s) return fail(MQV_ERR_INVALID_ARG, "null handle");
    if (algorithm < MQV_WOLFF_AUTO || algorithm > MQV_WOLFF_LABEL) return fail(MQV_ERR_INVALID_ARG, "unknown algorithm");
    s->wolff_algo = algorithm;
    return MQV_OK;
}

MQV_API mqv_status mqv_launch_count(mqv_sim* h, uint64_t* count)
{
    Sim* s = reinterpret_cast<Sim*>(h);
    if (!s || !count) return fail(MQV_ERR_INVALID_ARG, "null argument");
    *count = s->launches;
    return MQV_OK;
}

MQV_API mqv_status mqv_selftest_accept_cut(int32_t pref, int32_t n, const double* dE, const double* beta,
                                           uint64_t* cut)
{
    if (n < 0 || (n > 0 && (!dE || !beta || !cut)) || (pref != 1 && pref != 2))
        return fail(MQV_ERR_INVALID_ARG, "bad arguments");
    for (int32_t i = 0; i < n; ++i) cut[i] = accept_cut_direct(pref, dE[i], beta[i]);
    return MQV_OK;
}

MQV_API mqv_status mqv_selftest_philox(uint64_t seed, uint32_t c1, uint32_t c2, uint32_t c3, int32_t n,
                                       uint32_t* out_engine, uint32_t* out_curand)
{
    if (n <= 0 || !out_engine || !out_curand) return fail(MQV_ERR_INVALID_ARG, "bad arguments");
    uint32_t *de = nullptr, *dc = nullptr;
    MQV_CK(cudaMalloc(&de, sizeof(uint32_t) * 4 * (size_t)n));
    MQV_CK(cudaMalloc(&dc, sizeof(uint32_t) * 4 * (size_t)n));
    cudaError_t e = launch_selftest_philox(seed, c1, c2, c3, n, de, dc, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out_engine, de, sizeof(uint32_t) * 4 * (size_t)n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(out_curand, dc, sizeof(uint32_t) * 4 * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(de);
    cudaFree(dc);
    MQV_CK(e);
    return MQV_OK;
}

}  // extern "C"

// ---- batches -----------------------------------------------------------------------

namespace mqv {

// host mirror of the labelling Wolff's per-member seed (wolff_ccl.cuh)
struct CclSeedHost {
    int64_t rsite;
    int val, newq;
    float r[3];
};

struct Batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<Sim*> sims;
    int nrep = 0;
    bool f32 = false;
    std::vector<BatchRep> reps;  // host copy of the member table (kept alive for the upload)
    BatchRep* d_reps = nullptr;
    int64_t* d_prefix = nullptr;
    int32_t* d_block_rep = nullptr;
    int32_t* d_cbegin = nullptr;
    int32_t* d_ccount = nullptr;
    // members run by batch_resident (one CTA each, state in shared memory):
    // two classes by size (<= kResSmall sites: several CTAs per SM), each
    // listed largest first; resident[r] marks them
    std::vector<char> resident;
    int32_t* d_res_order = nullptr;
    int nres[2] = {0, 0};
    size_t res_smem[2] = {0, 0};  // dynamic shared memory of each class (its largest layout)
    // members held by thread-block clusters of c CTAs (c = 2 .. 8): ncl[c]
    // of them at d_res_order + cl_off[c]
    int ncl[9] = {};
    int cl_off[9] = {};
    int64_t* d_site_prefix = nullptr;
    int32_t* d_site_block_rep = nullptr;
    int32_t* d_meas_prefix = nullptr;
    int32_t* d_meas_rep = nullptr;
    void* d_ccl_seeds = nullptr;
    int wolff_mode = MQV_WOLFF_AUTO;
    // MQV_WOLFF_AUTO: ms per EMCS of breadth first [0] and labelling [1] when
    // last timed (-1: never), the one in use, EMCS since the other was tried
    double wolff_est[2] = {-1.0, -1.0};
    int wolff_best = 0;
    int64_t wolff_since_try = 0;
    cudaEvent_t ev[4] = {};
    std::vector<int> block_off, blocks;
    std::vector<int64_t> total;
    BatchCtr* d_ctr = nullptr;
    long long* d_acc = nullptr;
    double* d_obs = nullptr;
    int32_t* d_csize = nullptr;
    int cap_slots = 0;   // measurement slots in d_acc / d_obs (per member)
    int cap_cslots = 0;  // cluster-size slots in d_csize (per member)
    BatchLaunch L{};
    cudaGraphExec_t g_one[2] = {nullptr, nullptr}, g_many[2] = {nullptr, nullptr};  // [labelling clusters]
    int g_ncluster = -1, g_nmetro = -1, g_steps = 0;
    int graph_steps = 8;  // EMCS per graph launch
    uint64_t launches = 0;
    uint32_t temper_steps = 0;  // replica-exchange steps done (part of their draws' counters)
    // Members are independent, so the resident classes and the cluster sizes
    // run on side streams beside the graph members on `stream`: forked from
    // it by fork_ev, joined back by join_ev[i] before anything that reads
    // every member (exchanges, the chunk's reductions and copies).
    static constexpr int kSide = 9;  // 2 resident classes + cluster sizes 2 .. 8
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kSide] = {};
};

static void free_graphs(Batch* b)
{
    for (int w = 0; w < 2; ++w) {
        if (b->g_one[w]) cudaGraphExecDestroy(b->g_one[w]);
        if (b->g_many[w]) cudaGraphExecDestroy(b->g_many[w]);
        b->g_one[w] = b->g_many[w] = nullptr;
    }
    b->g_ncluster = b->g_nmetro = -1;
}

static void free_batch(Batch* b)
{
    if (!b) return;
    DeviceGuard g(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_graphs(b);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    for (int i = 0; i < Batch::kSide; ++i) {
        if (b->side[i]) cudaStreamSynchronize(b->side[i]);
        if (b->side[i]) cudaStreamDestroy(b->side[i]);
        if (b->join_ev[i]) cudaEventDestroy(b->join_ev[i]);
    }
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    for (Sim* s : b->sims) free_sim(s);
    for (void* p : {(void*)b->d_reps, (void*)b->d_prefix, (void*)b->d_block_rep, (void*)b->d_cbegin,
                    (void*)b->d_ccount, (void*)b->d_res_order, (void*)b->d_ctr,
                    (void*)b->d_acc, (void*)b->d_obs, (void*)b->d_csize, (void*)b->d_site_prefix,
                    (void*)b->d_site_block_rep, (void*)b->d_meas_prefix, (void*)b->d_meas_rep, b->d_ccl_seeds})
        if (p) cudaFree(p);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

static mqv_status batch_capacity(Batch* b, int slots, int cslots)
{
    if (slots > b->cap_slots) {
        if (b->d_acc) cudaFree(b->d_acc);
        if (b->d_obs) cudaFree(b->d_obs);
        b->d_acc = nullptr;
        b->d_obs = nullptr;
        b->cap_slots = 0;
        MQV_CK(cudaMalloc(&b->d_acc, sizeof(long long) * kAccStride * (size_t)slots * b->nrep));
        MQV_CK(cudaMalloc(&b->d_obs, sizeof(double) * 4 * (size_t)slots * b->nrep));
        b->cap_slots = slots;
    }
    if (cslots > b->cap_cslots) {
        if (b->d_csize) cudaFree(b->d_csize);
        b->d_csize = nullptr;
        b->cap_cslots = 0;
        MQV_CK(cudaMalloc(&b->d_csize, sizeof(int32_t) * (size_t)cslots * b->nrep));
        b->cap_cslots = cslots;
    }
    b->L.acc = b->d_acc;
    b->L.csize = b->d_csize;
    return MQV_OK;
}

// Capture `steps` EMCS of the batch into an executable graph.
static mqv_status batch_capture(Batch* b, int steps, int ncluster, int nmetro, cudaGraphExec_t* out)
{
    cudaGraph_t graph = nullptr;
    MQV_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < steps && e == cudaSuccess; ++k) e = batch_launch_emcs(b->L, b->stream, ncluster, nmetro);
    const cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
    MQV_CK(e);
    MQV_CK(e2);
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    MQV_CK(e);
    return MQV_OK;
}

static bool batch_kind_ok(int k)
{
    return k == MQV_MODEL_ISING || k == MQV_MODEL_ISING_EMBED || k == MQV_MODEL_POTTS || k == MQV_MODEL_BLUME_CAPEL ||
           k == MQV_MODEL_EA || k == MQV_MODEL_HEISENBERG || k == MQV_MODEL_PHI4 || k == MQV_MODEL_XXZ;
}

// calcMHratio's under/overflow guards (src/libmarqov/marqovscheduler.h:44-57)
static const double kTemperEnMin = std::log(std::numeric_limits<double>::min());
static const double kTemperEnMax = std::log(std::numeric_limits<double>::max());

// Replica exchange inside a run: after every `interval` EMCS the step's
// pairs (d_plan + 2 * npairs * step) attempt an exchange; d_perm tracks which
// member's state buffers each member holds, d_flags the outcomes.
struct TemperRun {
    int interval = 0;  // EMCS per step; 0 = no exchanges
    int npairs = 0;
    const int32_t* d_plan = nullptr;
    uint32_t step0 = 0;  // the batch's step counter when the run started
    uint64_t seed = 0;
    int32_t* d_perm = nullptr;
    int32_t* d_flags = nullptr;
};

// n_emcs EMCS of every member; observables / cluster means to the host, raw
// sums to the device samples buffer ([member][n_emcs][4]), each when given.
static mqv_status batch_run(Batch* b, int n_emcs, int ncluster, int nmetro, mqv_obs* obs, double* mean_cluster,
                            double* d_samples, const TemperRun* pt = nullptr)
{
    DeviceGuard guard_(b->device);
    if (n_emcs < 0 || ncluster < 0 || nmetro < 0) return fail(MQV_ERR_INVALID_ARG, "negative count");
    if (ncluster > 64 || nmetro > 64) return fail(MQV_ERR_INVALID_ARG, "at most 64 clusters and 64 sweeps per EMCS");
    for (Sim* s : b->sims) {
        if (!s->initialised) return fail(MQV_ERR_STATE, "state of a batch member not initialised");
        if (s->failed) return check_runnable(s);
        if (!b->f32) MQV_CK(ensure_cuts(s));
        if (ncluster > 0) {
            mqv_status st = check_wolff_supported(s);
            if (st) return st;
            st = ensure_wolff(s);
            if (st) return st;
        }
    }
    // member table at the start of the run
    b->reps.assign((size_t)b->nrep, BatchRep{});
    for (int i = 0; i < b->nrep; ++i) {
        const Sim* s = b->sims[(size_t)i];
        BatchRep& r = b->reps[(size_t)i];
        r.md = s->md;
        r.st = s->sten;
        r.csr = s->csr;
        r.lat_kind = s->lat_kind;
        r.order = s->d_order;
        if (!b->f32) r.w = wolff_int8_params(s->md);
        r.key = make_key(s->seed);
        r.replica = s->replica;
        r.sweep0 = (uint32_t)s->sweep;
        r.cluster0 = (uint32_t)s->cluster;
        r.s = s->state[s->cur];
        r.visited = s->d_visited;
        r.queue = s->d_queue;
        r.cuts = s->d_cuts;
        r.D = s->max_degree;
        r.resident = b->resident[(size_t)i] ? 1 : 0;
        r.tile = ccl_tile_kind(s->lat_kind, s->dim, s->len);
    }
    MQV_CK(cudaMemcpyAsync(b->d_reps, b->reps.data(), sizeof(BatchRep) * b->reps.size(), cudaMemcpyHostToDevice,
                           b->stream));
    const int CH = 256;  // EMCS per chunk of measurements
    const int slots = std::min(CH, std::max(n_emcs, 1));
    const long long* acc0 = b->d_acc;
    const int32_t* csize0 = b->d_csize;
    mqv_status st = batch_capacity(b, slots, slots * std::max(ncluster, 1));
    if (st) return st;
    if (b->d_acc != acc0 || b->d_csize != csize0) free_graphs(b);  // graphs hold the old pointers
    const int K = std::max(1, std::min(b->graph_steps, CH));
    // Cluster algorithm: fixed, or (MQV_WOLFF_AUTO) chosen by measurement.
    // Both give the same clusters, so switching never changes the chain; the
    // cost of breadth-first growth follows the clusters (it rises as a farm
    // orders), labelling costs the same every EMCS.  Each chunk is timed; the
    // algorithm not in use is tried on a few EMCS at the start of a chunk when
    // it has no estimate or its estimate is old (256 EMCS, scaled by how
    // much slower it was), and the faster estimate is used after that.
    const bool adapt = b->wolff_mode == MQV_WOLFF_AUTO && ncluster > 0;
    const int fixed = b->wolff_mode == MQV_WOLFF_LABEL ? 1 : 0;
    if (b->g_ncluster != ncluster || b->g_nmetro != nmetro || b->g_steps != K) {
        free_graphs(b);
        b->g_ncluster = ncluster;
        b->g_nmetro = nmetro;
        b->g_steps = K;
    }
    for (int w = 0; w < 2; ++w) {
        if (!adapt && w != fixed) continue;
        if (b->g_one[w] && (K == 1 || b->g_many[w])) continue;
        MQV_CK(cudaStreamSynchronize(b->stream));
        b->L.wolff_ccl = w;
        if (!b->g_one[w]) st = batch_capture(b, 1, ncluster, nmetro, &b->g_one[w]);
        if (!st && K > 1 && !b->g_many[w]) st = batch_capture(b, K, ncluster, nmetro, &b->g_many[w]);
        if (!st) {
            // upload now, so that the first timed launch is not the upload
            if (cudaGraphUpload(b->g_one[w], b->stream) != cudaSuccess ||
                (K > 1 && cudaGraphUpload(b->g_many[w], b->stream) != cudaSuccess))
                st = fail(MQV_ERR_CUDA, "graph upload failed");
        }
        if (st) {
            free_graphs(b);
            return st;
        }
    }
    if (adapt && !b->ev[0])
        for (auto& e : b->ev) MQV_CK(cudaEventCreate(&e));
    int done_run = 0;  // first EMCS of the chunk in progress
    uint64_t per_emcs[2];
    for (int w = 0; w < 2; ++w) {
        BatchLaunch l = b->L;
        l.wolff_ccl = w;
        per_emcs[w] = batch_launches_per_emcs(l, ncluster, nmetro);
    }
    // side streams of the resident classes and cluster sizes (created once)
    int nside_needed = (b->nres[0] ? 1 : 0) + (b->nres[1] ? 1 : 0);
    for (int c = 2; c <= 8; ++c) nside_needed += b->ncl[c] ? 1 : 0;
    if (nside_needed && !b->fork_ev) {
        MQV_CK(cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming));
        for (int i = 0; i < Batch::kSide; ++i) {
            MQV_CK(cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking));
            MQV_CK(cudaEventCreateWithFlags(&b->join_ev[i], cudaEventDisableTiming));
        }
    }
    // `count` EMCS of every member from chunk position k0: the resident
    // classes and each cluster size on their own side stream, the graph
    // members (algorithm w) on the batch stream, joined at the end
    auto launch_emcs = [&](int w, int count, int k0) -> mqv_status {
        int nside = 0;
        if (nside_needed) MQV_CK(cudaEventRecord(b->fork_ev, b->stream));
        // the next side stream, ordered after the fork
        auto side_stream = [&](cudaStream_t& st2) -> cudaError_t {
            st2 = b->side[nside];
            return cudaStreamWaitEvent(st2, b->fork_ev, 0);
        };
        auto side_done = [&](cudaStream_t st2) -> cudaError_t {
            const cudaError_t e = cudaEventRecord(b->join_ev[nside], st2);
            ++nside;
            return e;
        };
        for (int cls = 0; cls < 2; ++cls) {
            if (!b->nres[cls]) continue;
            cudaStream_t st2 = nullptr;
            MQV_CK(side_stream(st2));
            MQV_CK(batch_launch_resident(b->L, st2, b->d_res_order + (cls ? b->nres[0] : 0), b->nres[cls],
                                         b->res_smem[cls], (uint32_t)(done_run + k0), k0, count, ncluster, nmetro,
                                         b->device));
            MQV_CK(side_done(st2));
            b->launches++;
        }
        for (int c = 2; c <= 8; ++c) {
            if (!b->ncl[c]) continue;
            cudaStream_t st2 = nullptr;
            MQV_CK(side_stream(st2));
            MQV_CK(batch_launch_cluster(b->L, st2, b->d_res_order + b->cl_off[c], b->ncl[c], c,
                                        (uint32_t)(done_run + k0), k0, count, ncluster, nmetro));
            MQV_CK(side_done(st2));
            b->launches++;
        }
        int j = 0;
        if (K > 1)
            for (; j + K <= count; j += K) MQV_CK(cudaGraphLaunch(b->g_many[w], b->stream));
        for (; j < count; ++j) MQV_CK(cudaGraphLaunch(b->g_one[w], b->stream));
        b->launches += per_emcs[w] * (uint64_t)count;
        for (int i = 0; i < nside; ++i) MQV_CK(cudaStreamWaitEvent(b->stream, b->join_ev[i], 0));
        return MQV_OK;
    };
    // the exchange step that ends after EMCS `e` of the run, if any
    auto exchange_after = [&](int e) -> mqv_status {
        if (!pt || e % pt->interval != 0) return MQV_OK;
        const int t = e / pt->interval - 1;
        MQV_CK(batch_launch_temper(b->L, b->stream, pt->d_plan + (size_t)2 * pt->npairs * t, pt->npairs,
                                   pt->step0 + (uint32_t)t, pt->seed, kTemperEnMin, kTemperEnMax, pt->d_perm,
                                   pt->d_flags + (size_t)pt->npairs * t));
        b->launches++;
        return MQV_OK;
    };
    std::vector<int32_t> csz;
    int done = 0;
    while (done < n_emcs) {
        const int ch = std::min(n_emcs - done, CH);
        done_run = done;
        MQV_CK(cudaMemsetAsync(b->d_acc, 0, sizeof(long long) * kAccStride * (size_t)ch * b->nrep, b->stream));
        MQV_CK(batch_launch_chunk_start(b->L, b->stream, (uint32_t)done));
        b->launches++;
        const int w_main = adapt ? b->wolff_best : fixed, w_try = 1 - w_main;
        int x = 0;  // EMCS of this chunk that try the other algorithm
        if (adapt) {
            const double* est = b->wolff_est;
            const double r = est[w_try] > 0 && est[w_main] > 0 ? std::max(1.0, est[w_try] / est[w_main]) : 1.0;
            if (est[w_try] < 0 || (double)b->wolff_since_try >= 256.0 * r) x = std::min(4, ch / 2);
        }
        int k = 0;
        // `count` EMCS from chunk position k, an exchange step where one ends
        auto advance = [&](int w, int count) -> mqv_status {
            const int stop = k + count;
            while (k < stop) {
                int run = stop - k;
                if (pt) run = std::min(run, pt->interval - (done + k) % pt->interval);
                mqv_status s2 = launch_emcs(w, run, k);
                if (s2) return s2;
                k += run;
                s2 = exchange_after(done + k);
                if (s2) return s2;
            }
            return MQV_OK;
        };
        if (x) {
            MQV_CK(cudaEventRecord(b->ev[0], b->stream));
            st = advance(w_try, x);
            if (st) return st;
            MQV_CK(cudaEventRecord(b->ev[1], b->stream));
        }
        if (adapt) MQV_CK(cudaEventRecord(b->ev[2], b->stream));
        st = advance(w_main, ch - x);
        if (st) return st;
        if (adapt) MQV_CK(cudaEventRecord(b->ev[3], b->stream));
        if (d_samples) {
            MQV_CK(batch_launch_samples(b->L, b->stream, ch, done, n_emcs, d_samples));
            b->launches++;
        }
        if (obs) {
            MQV_CK(batch_launch_finalize(b->L, b->stream, ch, b->d_obs));
            b->launches++;
            MQV_CK(cudaMemcpyAsync(obs + (size_t)done * b->nrep, b->d_obs, sizeof(double) * 4 * (size_t)ch * b->nrep,
                                   cudaMemcpyDeviceToHost, b->stream));
        }
        if (mean_cluster && ncluster > 0) {
            csz.resize((size_t)ch * ncluster * b->nrep);
            MQV_CK(cudaMemcpyAsync(csz.data(), b->d_csize, sizeof(int32_t) * csz.size(), cudaMemcpyDeviceToHost,
                                   b->stream));
        }
        MQV_CK(cudaStreamSynchronize(b->stream));
        if (adapt) {
            float ms = 0;
            if (x) {
                MQV_CK(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
                b->wolff_est[w_try] = ms / x;
                b->wolff_since_try = 0;
            }
            if (ch > x) {
                MQV_CK(cudaEventElapsedTime(&ms, b->ev[2], b->ev[3]));
                b->wolff_est[w_main] = ms / (ch - x);
            }
            b->wolff_since_try += ch - x;
            if (b->wolff_est[0] > 0 && b->wolff_est[1] > 0) b->wolff_best = b->wolff_est[1] < b->wolff_est[0] ? 1 : 0;
        }
        if (mean_cluster) {
            for (int e = 0; e < ch; ++e)
                for (int r = 0; r < b->nrep; ++r) {
                    double a = 0;
                    for (int c = 0; c < ncluster; ++c) a += (double)csz[((size_t)e * ncluster + c) * b->nrep + r];
                    mean_cluster[(size_t)(done + e) * b->nrep + r] = ncluster > 0 ? a / ncluster : 0.0;
                }
        }
        done += ch;
    }
    MQV_CK(cudaStreamSynchronize(b->stream));
    for (Sim* s : b->sims) {
        s->sweep += (uint64_t)n_emcs * (uint64_t)nmetro;
        s->cluster += (uint64_t)n_emcs * (uint64_t)ncluster;
    }
    return MQV_OK;
}

// Partners of a replica exchange differ in beta only: the same model
// descriptor and the same lattice.
static bool temper_compatible(const Sim* a, const Sim* b)
{
    const mqv_model_desc &x = a->model, &y = b->model;
    if (x.kind != y.kind || x.q != y.q || x.proposal != y.proposal || x.J != y.J || x.h != y.h || x.h2 != y.h2 ||
        x.k != y.k || x.delta != y.delta || x.cap != y.cap)
        return false;
    if (a->lat_kind != b->lat_kind || a->n != b->n || a->termsel != b->termsel) return false;
    if (a->lat_kind == MQV_LATTICE_HYPERCUBIC)
        return a->dim == b->dim && a->len == b->len && a->lat_hash == b->lat_hash;  // hash: bonds (0 without)
    return a->lat_hash == b->lat_hash;
}

// Member r takes the state buffers member perm[r] held when the run started.
static void apply_state_permutation(Batch* b, const std::vector<int32_t>& perm)
{
    struct Bufs {
        void* s0;
        void* s1;
        int cur;
    };
    std::vector<Bufs> old;
    for (Sim* s : b->sims) old.push_back(Bufs{s->state[0], s->state[1], s->cur});
    for (int r = 0; r < b->nrep; ++r) {
        const Bufs& o = old[(size_t)perm[(size_t)r]];
        Sim* s = b->sims[(size_t)r];
        s->state[0] = o.s0;
        s->state[1] = o.s1;
        s->cur = o.cur;
    }
}

}  // namespace mqv

extern "C" {

MQV_API mqv_status mqv_batch_create(const mqv_sim_spec* specs, int32_t n, mqv_batch** out)
{
    if (!specs || !out) return fail(MQV_ERR_INVALID_ARG, "null argument");
    if (n < 1 || n > 65535) return fail(MQV_ERR_INVALID_ARG, "batch size must be in [1, 65535]");
    *out = nullptr;
    const int device = specs[0].params.device;
    for (int i = 0; i < n; ++i) {
        if (!batch_kind_ok(specs[i].model.kind))
            return fail(MQV_ERR_UNSUPPORTED_TERM, "unsupported model kind in batch member " + std::to_string(i));
        if (is_f32_kind(specs[i].model.kind) != is_f32_kind(specs[0].model.kind))
            return fail(MQV_ERR_UNSUPPORTED_TERM, "a batch holds int8 members or float members, not both");
        if (specs[i].params.device != device) return fail(MQV_ERR_INVALID_ARG, "all members of a batch share one device");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(MQV_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(MQV_ERR_INVALID_ARG, "device ordinal out of range");
    Batch* b = new (std::nothrow) Batch();
    if (!b) return fail(MQV_ERR_OUT_OF_MEMORY, "host allocation failed");
    b->device = device;
    auto bail = [&](mqv_status st) {
        free_batch(b);
        return st;
    };
    DeviceGuard g(device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("cudaStreamCreate failed");
        return bail(MQV_ERR_CUDA);
    }
    // members: ordinary handles on the batch's stream, one launch per colour
    // class (reference site order, no fused two-colour layout)
    b->nrep = n;
    b->f32 = is_f32_kind(specs[0].model.kind);
    b->sims.reserve((size_t)n);
    for (int i = 0; i < n; ++i) {
        mqv_run_params p = specs[i].params;
        p.flags |= MQV_FLAG_PER_COLOUR;
        mqv_sim* h = nullptr;
        mqv_status st = mqv_create(&specs[i].model, &specs[i].lattice, &p, &h);
        if (st) {
            const std::string msg = "batch member " + std::to_string(i) + ": " + g_err;
            return bail(fail(st, msg));
        }
        b->sims.push_back(reinterpret_cast<Sim*>(h));
        st = mqv_set_stream(h, b->stream);
        if (st) return bail(st);
    }
    // resident members: int8 stencil lattices that fit one CTA's shared
    // memory (or a thread-block cluster's) and whose spec asks for it
    b->resident.assign((size_t)n, 0);
    std::vector<int32_t> res_order[2], cl_order[9];
    bool cl_ok[9] = {};
    for (int c = 2; c <= 8; ++c) cl_ok[c] = cluster_launchable(c);
    for (int r = 0; r < n; ++r) {
        const Sim* s = b->sims[(size_t)r];
        // A resident member runs on one CTA (or one cluster) for a whole chunk
        // of EMCS, which leaves it at the speed of one SM (or a few): the
        // graph path, whose launches spread every member over all SMs, is the
        // default (the 256-replica Potts farm: 1.8 against 3.4 ms per EMCS);
        // members that ask for it (MQV_FLAG_RESIDENT) stay resident.
        if (!(specs[r].params.flags & MQV_FLAG_RESIDENT)) continue;
        if (resident_fits(s)) {
            b->resident[(size_t)r] = 1;
            res_order[s->n > kResSmall ? 1 : 0].push_back(r);
        } else if (!s->is_f32 && s->lat_kind == MQV_LATTICE_HYPERCUBIC) {
            const int c = cluster_ctas(s->n);
            if (c >= 2 && cl_ok[c]) {
                b->resident[(size_t)r] = 2;
                cl_order[c].push_back(r);
            }
        }
    }

    for (int k = 0; k < 2; ++k) {
        std::stable_sort(res_order[k].begin(), res_order[k].end(),
                         [&](int32_t x, int32_t y) { return b->sims[(size_t)x]->n > b->sims[(size_t)y]->n; });
        b->nres[k] = (int)res_order[k].size();
        b->res_smem[k] = 0;
        for (int32_t r : res_order[k]) b->res_smem[k] = std::max(b->res_smem[k], resident_smem_for(b->sims[(size_t)r]->sten));
    }
    std::vector<int32_t> res_all(res_order[0]);
    res_all.insert(res_all.end(), res_order[1].begin(), res_order[1].end());
    for (int c = 2; c <= 8; ++c) {
        b->cl_off[c] = (int)res_all.size();
        b->ncl[c] = (int)cl_order[c].size();
        res_all.insert(res_all.end(), cl_order[c].begin(), cl_order[c].end());
    }
    // per-colour work: colour c concatenates every graph member's colour-c
    // sites (resident members contribute none), each member's count padded
    // to whole blocks of kAccSites, so that a CTA's block lies in one member
    // (batch_metro)
    int ncol = 0;
    for (Sim* s : b->sims) ncol = std::max(ncol, (int)s->colour_ptr.size() - 1);
    std::vector<int64_t> prefix((size_t)ncol * (n + 1), 0);
    std::vector<int32_t> cbegin((size_t)n * ncol, 0), ccount((size_t)n * ncol, 0), brep;
    b->block_off.assign((size_t)ncol, 0);
    b->blocks.assign((size_t)ncol, 0);
    b->total.assign((size_t)ncol, 0);
    const int64_t per_cta = kAccSites;  // padded positions per CTA: one block
    for (int c = 0; c < ncol; ++c) {
        int64_t* pf = prefix.data() + (size_t)c * (n + 1);
        for (int r = 0; r < n; ++r) {
            const Sim* s = b->sims[(size_t)r];
            int64_t cnt = 0;
            if (c + 1 < (int)s->colour_ptr.size()) {
                cnt = s->colour_ptr[(size_t)c + 1] - s->colour_ptr[(size_t)c];
                cbegin[(size_t)r * ncol + c] = s->colour_ptr[(size_t)c];
            }
            if (b->resident[(size_t)r]) cnt = 0;
            ccount[(size_t)r * ncol + c] = (int32_t)cnt;
            pf[r + 1] = pf[r] + (cnt + kAccSites - 1) / kAccSites * kAccSites;
        }
        const int64_t tot = pf[n];
        const int64_t nb = (tot + per_cta - 1) / per_cta;
        if ((int64_t)brep.size() + nb >= (int64_t)1 << 31) return bail(fail(MQV_ERR_INVALID_ARG, "batch too large"));
        b->block_off[(size_t)c] = (int)brep.size();
        b->blocks[(size_t)c] = (int)nb;
        b->total[(size_t)c] = tot;
        for (int64_t k = 0, r = 0; k < nb; ++k) {
            while (k * per_cta >= pf[r + 1]) ++r;
            brep.push_back((int32_t)r);
        }
    }
    if (brep.empty()) brep.push_back(0);
    // site-level work of the labelling Wolff
    std::vector<int64_t> sprefix((size_t)n + 1, 0);
    for (int r = 0; r < n; ++r) sprefix[r + 1] = sprefix[r] + (b->resident[(size_t)r] ? 0 : b->sims[(size_t)r]->n);
    const int64_t sblocks = (sprefix[n] + kBatchMetroThreads - 1) / kBatchMetroThreads;
    if (sblocks >= (int64_t)1 << 31) return bail(fail(MQV_ERR_INVALID_ARG, "batch too large"));
    std::vector<int32_t> sbrep((size_t)std::max<int64_t>(sblocks, 1), 0);
    for (int64_t k = 0, r = 0; k < sblocks; ++k) {
        while (k * kBatchMetroThreads >= sprefix[r + 1]) ++r;
        sbrep[(size_t)k] = (int32_t)r;
    }
    auto dcopy = [&](void** dst, const void* src, size_t bytes) -> mqv_status {
        MQV_CK(cudaMalloc(dst, bytes));
        MQV_CK(upload_sync(b->stream, *dst, src, bytes));
        return MQV_OK;
    };
    // measurement CTAs: about 1024 sites each (four per thread: enough CTAs
    // to fill the SMs on farms of small members, few enough that the CTAs'
    // atomic adds and reductions stay a small part), at least one per member
    std::vector<int32_t> mprefix((size_t)n + 1, 0), mrep;
    for (int r = 0; r < n; ++r) {
        const int64_t parts =
            b->resident[(size_t)r] ? 0 : std::max<int64_t>(1, (b->sims[(size_t)r]->n + 1023) / 1024);
        if (mprefix[(size_t)r] + parts >= (int64_t)1 << 31) return bail(fail(MQV_ERR_INVALID_ARG, "batch too large"));
        mprefix[(size_t)r + 1] = mprefix[(size_t)r] + (int32_t)parts;
        for (int64_t k = 0; k < parts; ++k) mrep.push_back(r);
    }
    mqv_status st = dcopy((void**)&b->d_prefix, prefix.data(), sizeof(int64_t) * prefix.size());
    if (!st) st = dcopy((void**)&b->d_meas_prefix, mprefix.data(), sizeof(int32_t) * mprefix.size());
    if (mrep.empty()) mrep.push_back(0);
    if (res_all.empty()) res_all.push_back(0);
    if (!st) st = dcopy((void**)&b->d_meas_rep, mrep.data(), sizeof(int32_t) * mrep.size());
    if (!st) st = dcopy((void**)&b->d_res_order, res_all.data(), sizeof(int32_t) * res_all.size());
    if (!st) st = dcopy((void**)&b->d_block_rep, brep.data(), sizeof(int32_t) * brep.size());
    if (!st) st = dcopy((void**)&b->d_cbegin, cbegin.data(), sizeof(int32_t) * std::max<size_t>(cbegin.size(), 1));
    if (!st) st = dcopy((void**)&b->d_ccount, ccount.data(), sizeof(int32_t) * std::max<size_t>(ccount.size(), 1));
    if (!st) st = dcopy((void**)&b->d_site_prefix, sprefix.data(), sizeof(int64_t) * sprefix.size());
    if (!st) st = dcopy((void**)&b->d_site_block_rep, sbrep.data(), sizeof(int32_t) * sbrep.size());
    if (st) return bail(st);
    if (cudaMalloc(&b->d_ccl_seeds, sizeof(CclSeedHost) * (size_t)n) != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of the batch tables failed");
        return bail(MQV_ERR_OUT_OF_MEMORY);
    }
    if (cudaMalloc(&b->d_reps, sizeof(BatchRep) * (size_t)n) != cudaSuccess ||
        cudaMalloc(&b->d_ctr, sizeof(BatchCtr)) != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of the batch tables failed");
        return bail(MQV_ERR_OUT_OF_MEMORY);
    }
    b->L.reps = b->d_reps;
    b->L.nrep = n;
    b->L.f32 = b->f32 ? 1 : 0;
    b->L.ncol = ncol;
    b->L.prefix = b->d_prefix;
    b->L.block_rep = b->d_block_rep;
    b->L.cbegin = b->d_cbegin;
    b->L.ccount = b->d_ccount;
    b->L.block_off = b->block_off.data();
    b->L.blocks = b->blocks.data();
    b->L.total = b->total.data();
    b->L.meas_prefix = b->d_meas_prefix;
    b->L.meas_rep = b->d_meas_rep;
    b->L.meas_blocks = (int)mprefix[(size_t)n];
    b->L.site_prefix = b->d_site_prefix;
    b->L.site_block_rep = b->d_site_block_rep;
    b->L.total_sites = sprefix[n];
    b->L.site_blocks = (int)sblocks;
    b->L.ccl_seeds = b->d_ccl_seeds;
    b->L.wolff_ccl = 0;  // set per captured graph (mqv_batch_set_wolff, or timed: MQV_WOLFF_AUTO)
    b->L.ctr = b->d_ctr;
    *out = reinterpret_cast<mqv_batch*>(b);
    return MQV_OK;
}

MQV_API mqv_status mqv_batch_destroy(mqv_batch* h)
{
    free_batch(reinterpret_cast<Batch*>(h));
    return MQV_OK;
}

MQV_API mqv_status mqv_batch_member(mqv_batch* h, int32_t i, mqv_sim** sim)
{
    Batch* b = reinterpret_cast<Batch*>(h);
    if (!b || !sim) return fail(MQV_ERR_INVALID_ARG, "null argument");
    if (i < 0 || i >= b->nrep) return fail(MQV_ERR_INVALID_ARG, "member index out of range");
    *sim = reinterpret_cast<mqv_sim*>(b->sims[(size_t)i]);
    return MQV_OK;
}

MQV_API mqv_status mqv_batch_init_state(mqv_batch* h)
{
    Batch* b = reinterpret_cast<Batch*>(h);
    if (!b) return fail(MQV_ERR_INVALID_ARG, "null handle");
    for (Sim* s : b->sims) {
        const mqv_status st = mqv_init_state(reinterpret_cast<mqv_sim*>(s));
        if (st) return st;
    }
    return MQV_OK;
}

MQV_API mqv_status mqv_batch_set_graph_steps(mqv_batch* h, int32_t steps)
{
    Batch* b = reinterpret_cast<Batch*>(h);
    if (!b) return fail(MQV_ERR_INVALID_ARG, "null handle");
    if (steps < 1 || steps > 256) return fail(MQV_ERR_INVALID_ARG, "graph steps must be in [1, 256]");
    b->graph_steps = steps;
    return MQV_OK;
}

MQV_API mqv_status mqv_batch_set_wolff(mqv_batch* h, int32_t algorithm)
{
    Batch* b = reinterpret_cast<Batch*>(h);
    if (!b) return fail(MQV_ERR_INVALID_ARG, "null handle");
    if (algorithm != MQV_WOLFF_AUTO && algorithm != MQV_WOLFF_BFS && algorithm != MQV_WOLFF_LABEL)
        return fail(MQV_ERR_INVALID_ARG, "unknown cluster algorithm");
    b->wolff_mode = algorithm;
    if (algorithm == MQV_WOLFF_AUTO) {
        b->wolff_est[0] = b->wolff_est[1] = -1.0;
        b->wolff_best = 0;
        b->wolff_since_try = 0;
    }
    return MQV_OK;
}

MQV_API mqv_status mqv_batch_get_wolff(mqv_batch* h, int32_t* algorithm)
{
    Batch* b = reinterpret_cast<Batch*>(h);
    if (!b || !algorithm) return fail(MQV_ERR_INVALID_ARG, "null argument");
    const bool timed = b->wolff_est[0] > 0 && b->wolff_est[1] > 0;
    *algorithm = b->wolff_mode != MQV_WOLFF_AUTO ? b->wolff_mode
                 : !timed                       ? MQV_WOLFF_AUTO
                 : b->wolff_best == 1           ? MQV_WOLFF_LABEL
                                                : MQV_WOLFF_BFS;
    return MQV_OK;
}

MQV_API mqv_status mqv_batch_emcs(mqv_batch* h, int32_t n_emcs, int32_t ncluster, int32_t nmetro, mqv_obs* obs,
                                  double* mean_cluster)
{
    Batch* b = reinterpret_cast<Batch*>(h);
    if (!b) return fail(MQV_ERR_INVALID_ARG, "null handle");
    return batch_run(b, n_emcs, ncluster, nmetro, obs, mean_cluster, nullptr);
}

MQV_API mqv_status mqv_batch_emcs_samples(mqv_batch* h, int32_t n_emcs, int32_t ncluster, int32_t nmetro,
                                          double* d_samples)
{
    Batch* b = reinterpret_cast<Batch*>(h);
    if (!b) return fail(MQV_ERR_INVALID_ARG, "null handle");
    if (n_emcs > 0 && !d_samples) return fail(MQV_ERR_INVALID_ARG, "null sample buffer");
    return batch_run(b, n_emcs, ncluster, nmetro, nullptr, nullptr, d_samples);
}

MQV_API mqv_status mqv_batch_tempering(mqv_batch* h, int32_t n_steps, int32_t emcs_per_step, int32_t ncluster,
                                      int32_t nmetro, const int32_t* plan, int32_t pairs_per_step, uint64_t seed,
                                      mqv_obs* obs, int32_t* accepted)
{
    Batch* b = reinterpret_cast<Batch*>(h);
    if (!b || (!plan && n_steps > 0 && pairs_per_step > 0)) return fail(MQV_ERR_INVALID_ARG, "null argument");
    if (n_steps < 0 || emcs_per_step < 1 || pairs_per_step < 0)
        return fail(MQV_ERR_INVALID_ARG, "need n_steps >= 0, emcs_per_step >= 1, pairs_per_step >= 0");
    if ((int64_t)n_steps * emcs_per_step > INT32_MAX) return fail(MQV_ERR_INVALID_ARG, "too many EMCS");
    if (pairs_per_step > b->nrep) return fail(MQV_ERR_INVALID_ARG, "more pairs per step than members");
    DeviceGuard guard_(b->device);
    // the plan: member ids in range, pairs of a step disjoint, partners alike
    std::vector<int> seen((size_t)b->nrep, -1);
    for (int t = 0; t < n_steps; ++t)
        for (int k = 0; k < pairs_per_step; ++k) {
            const int32_t* pr = plan + ((size_t)t * pairs_per_step + k) * 2;
            const int a = pr[0], c = pr[1];
            if (a < 0 || a >= b->nrep || c < 0 || c >= b->nrep)
                return fail(MQV_ERR_INVALID_ARG, "plan step " + std::to_string(t) + ": member id out of range");
            if (a == c) continue;
            if (seen[(size_t)a] == t || seen[(size_t)c] == t)
                return fail(MQV_ERR_INVALID_ARG, "plan step " + std::to_string(t) + ": pairs share a member");
            seen[(size_t)a] = seen[(size_t)c] = t;
            if (!temper_compatible(b->sims[(size_t)a], b->sims[(size_t)c]))
                return fail(MQV_ERR_INVALID_ARG, "members " + std::to_string(a) + " and " + std::to_string(c) +
                                                     " differ in more than beta (model or lattice)");
        }
    const int n_emcs = n_steps * emcs_per_step;
    if (n_emcs == 0) return MQV_OK;
    const size_t nflags = (size_t)n_steps * pairs_per_step;
    int32_t *d_plan = nullptr, *d_perm = nullptr, *d_flags = nullptr;
    auto release = [&]() {
        for (void* p : {(void*)d_plan, (void*)d_perm, (void*)d_flags})
            if (p) cudaFree(p);
    };
    std::vector<int32_t> ident((size_t)b->nrep);
    for (int i = 0; i < b->nrep; ++i) ident[(size_t)i] = i;
    if (cudaMalloc(&d_plan, sizeof(int32_t) * std::max<size_t>(2 * nflags, 1)) != cudaSuccess ||
        cudaMalloc(&d_perm, sizeof(int32_t) * (size_t)b->nrep) != cudaSuccess ||
        cudaMalloc(&d_flags, sizeof(int32_t) * std::max<size_t>(nflags, 1)) != cudaSuccess) {
        cudaGetLastError();
        release();
        return fail(MQV_ERR_OUT_OF_MEMORY, "device allocation of the exchange plan failed");
    }
    cudaError_t ce = cudaSuccess;
    if (nflags) ce = upload_sync(b->stream, d_plan, plan, sizeof(int32_t) * 2 * nflags);
    if (ce == cudaSuccess) ce = upload_sync(b->stream, d_perm, ident.data(), sizeof(int32_t) * ident.size());
    if (ce != cudaSuccess) {
        release();
        return fail(MQV_ERR_CUDA, std::string("upload of the exchange plan failed: ") + cudaGetErrorString(ce));
    }
    TemperRun pt;
    pt.interval = emcs_per_step;
    pt.npairs = pairs_per_step;
    pt.d_plan = d_plan;
    pt.step0 = b->temper_steps;
    pt.seed = seed;
    pt.d_perm = d_perm;
    pt.d_flags = d_flags;
    mqv_status st = batch_run(b, n_emcs, ncluster, nmetro, obs, nullptr, nullptr, &pt);
    // the handles take the state buffers the exchanges left them (also after a failed run)
    std::vector<int32_t> perm((size_t)b->nrep);
    std::vector<int32_t> flags(nflags);
    ce = cudaStreamSynchronize(b->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpy(perm.data(), d_perm, sizeof(int32_t) * perm.size(), cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess && accepted && nflags)
        ce = cudaMemcpy(flags.data(), d_flags, sizeof(int32_t) * nflags, cudaMemcpyDeviceToHost);
    release();
    if (ce != cudaSuccess)
        return fail(MQV_ERR_CUDA, std::string("download of the exchange outcome failed: ") + cudaGetErrorString(ce));
    std::vector<char> hit((size_t)b->nrep, 0);
    for (int32_t q : perm) {
        if (q < 0 || q >= b->nrep || hit[(size_t)q]) return fail(MQV_ERR_CUDA, "exchange permutation corrupted");
        hit[(size_t)q] = 1;
    }
    apply_state_permutation(b, perm);
    if (st) return st;
    b->temper_steps += (uint32_t)n_steps;
    if (accepted && nflags) std::memcpy(accepted, flags.data(), sizeof(int32_t) * nflags);
    return MQV_OK;
}

MQV_API mqv_status mqv_batch_launch_count(mqv_batch* h, uint64_t* count)
{
    Batch* b = reinterpret_cast<Batch*>(h);
    if (!b || !count) return fail(MQV_ERR_INVALID_ARG, "null argument");
    *count = b->launches;
    return MQV_OK;
}

}  // extern "C"
