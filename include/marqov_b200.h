/*
 * marqov_b200 -- C ABI of the B200 Monte Carlo update engine.
 *
 * The engine runs MARQOV's elementary Monte Carlo step -- Wolff embedded
 * clusters followed by Metropolis sweeps -- on one GPU, with the state resident
 * in device memory.  Hosts that speak MARQOV's plugin API (Hamiltonian terms,
 * lattice neighbours, Metropolis / Wolff / Embedder specialisations) lower
 * their model and lattice into the plain descriptors below; every entry point
 * takes plain pointers and sizes and returns an int32 status.
 *
 * Reference interfaces replaced (file:line in the MARQOV source tree):
 *   mqv_create        MARQOV::makeCore            src/libmarqov/core.h:1223-1246
 *                     (Core constructor           src/libmarqov/core.h:469-530)
 *   mqv_init_state    Core::init / initstatespace src/libmarqov/core.h:829-834,
 *                                                 src/hamiltonian/Ising.h:99-107
 *   mqv_metropolis    the Metropolis sweeps of    src/libmarqov/emcs.h:91-106
 *                     Metropolis<H,L>::move       src/libmarqov/metropolis.h:88-126
 *   mqv_wolff         the cluster loop of         src/libmarqov/emcs.h:77-89
 *                     Wolff<H,L>::move            src/libmarqov/wolff.h:72-126
 *   mqv_emcs          EMCS<H,L>::move + measure   src/libmarqov/emcs.h:69-109,
 *                                                 src/libmarqov/core.h:1001-1028
 *   mqv_measure       Energy / Magnetization      src/hamiltonian/util/observables.h:47-65,331-352
 *   mqv_get_state /   the state space and its     src/libmarqov/core.h:249-342
 *   mqv_set_state     checkpoint dump             src/libmarqov/core.h:543-607
 *   mqv_last_error    exit(-1)/throw paths        src/libmarqov/metropolishelpers.h:297-302,
 *                                                 src/libmarqov/core.h:336-340
 *
 * Conventions: status 0 is success; no exception crosses the ABI; the library
 * owns device memory and the caller owns the host buffers it passes; a handle
 * is bound to one CUDA stream and is not thread safe, while distinct handles
 * may be used from distinct host threads (one MARQOV Core per thread).
 */
#ifndef MARQOV_B200_H
#define MARQOV_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MQV_API __attribute__((visibility("default")))
#else
#define MQV_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t mqv_status;

enum {
    MQV_OK = 0,
    MQV_ERR_INVALID_ARG = 1,      /* bad argument or size */
    MQV_ERR_UNSUPPORTED_TERM = 2, /* model / term shape the engine does not lower */
    MQV_ERR_BAD_DESCRIPTOR = 3,   /* inconsistent lattice or model descriptor */
    MQV_ERR_CUDA = 4,             /* CUDA runtime error (message in mqv_last_error) */
    MQV_ERR_TIMEOUT = 5,          /* a bounded device wait gave up; the handle refuses compute
                                     (MQV_ERR_STATE) until its state is set again.  Outside
                                     the injected test case treat it as fatal for the
                                     context: a bulk copy still in flight when the block
                                     left may land in reassigned shared memory, so destroy
                                     the device's handles and reset its context */
    MQV_ERR_CHECKSUM = 6,         /* checkpoint / state checksum mismatch */
    MQV_ERR_NO_DEVICE = 7,        /* no usable CUDA device */
    MQV_ERR_OUT_OF_MEMORY = 8,    /* device allocation failed */
    MQV_ERR_STATE = 9             /* call out of order (e.g. run before init) */
};

/* Model kinds: the reference Hamiltonians the engine lowers. */
enum {
    MQV_MODEL_ISING = 1,        /* Ising<int>: int8 +-1, flip proposal, Wolff<Ising<int>> (exact -expm1) */
    MQV_MODEL_ISING_EMBED = 2,  /* Ising<int8_t>: generic Wolff + default Embedder */
    MQV_MODEL_POTTS = 3,        /* Potts<Q>: int8 0..Q-1, flex delta term k */
    MQV_MODEL_BLUME_CAPEL = 4,  /* BlumeCapel / BlumeCapelBipartite: int8 -1/0/+1, Spin1 proposal,
                                   onsite terms h s^2 (D or DA) and h2 s^2 (DB) */
    MQV_MODEL_EA = 5,           /* EdwardsAndersonIsing: Ising with lattice bonds */
    MQV_MODEL_HEISENBERG = 6,   /* Heisenberg: float 3-vectors */
    MQV_MODEL_PHI4 = 7,         /* scalar phi^4: float, onsite h = mass/beta, h2 = lambda/beta */
    MQV_MODEL_XXZ = 8           /* XXZAntiferro / XXZAntiferroSingleAniso: float 3-vectors, interaction
                                   get(s) = (delta s_x, delta s_y, s_z) with coefficient J (the
                                   reference's J = +1), onsite terms h s_z (field H) and h2 s_z^2 (D) */
};

/* Metropolis proposal (Initializer<H>::newsv). */
enum {
    MQV_PROPOSAL_DEFAULT = 0,   /* the model's reference initializer */
    MQV_PROPOSAL_SMALL_CAP = 1  /* O(3): uniform in the cap cos(angle) >= cap around the old spin */
};

typedef struct mqv_model_desc {
    int32_t kind;      /* MQV_MODEL_* */
    int32_t q;         /* Potts states (2..64) */
    int32_t proposal;  /* MQV_PROPOSAL_* */
    int32_t reserved;
    double J;          /* interaction coefficient, reference sign: dE = J dot(s_new - s_old, sum_nbrs) */
    double h;          /* coefficient of onsite term 0 */
    double h2;         /* coefficient of onsite term 1 */
    double k;          /* flex (multisite) coefficient */
    double delta;      /* XXZ anisotropy */
    double cap;        /* proposal width: small-cap cos(half-angle), or phi^4 shift amplitude */
} mqv_model_desc;

/* Lattice kinds. */
enum {
    MQV_LATTICE_HYPERCUBIC = 1, /* FixedDimRegularHypercubic<d>: periodic, even len, stencil path */
    MQV_LATTICE_CSR = 2,        /* any lattice with nbrs(): CSR neighbours (+ optional bnds) */
    MQV_LATTICE_BIPARTITE = 3   /* SimpleBipartite (src/lattice/simple_bipartite.h): the hypercubic
                                   stencil with a termselector -- a site whose coordinate sum is even
                                   (sublattice A) takes onsite term 0 only, odd (B) term 1 only */
};

typedef struct mqv_lattice_desc {
    int32_t kind;              /* MQV_LATTICE_* */
    int32_t dim;               /* hypercubic dimension (1..4) */
    int32_t len;               /* hypercubic side length */
    int32_t n;                 /* CSR: number of sites */
    const int32_t* row_ptr;    /* CSR: n+1 offsets (host memory, copied) */
    const int32_t* col_idx;    /* CSR: neighbour ids in nbrs(0,i) order (host, copied) */
    const int8_t* bonds;       /* optional bond weights (bnds), symmetric: CSR, one per col_idx entry;
                                  hypercubic, 2 dim per site in the nbrs(0,i) order +x,-x,+y,-y,...
                                  (RegularRandomBond), kept on the stencil path */
    const int32_t* colours;    /* optional proper colouring; NULL = greedy colouring */
} mqv_lattice_desc;

/* Run flags. */
enum {
    MQV_FLAG_PER_COLOUR = 1,  /* always use one launch per colour class (no fused two-colour tiles) */
    MQV_FLAG_NO_RESIDENT = 2, /* never run an int8 stencil lattice on the resident path -- one CTA
                                 (<= 65536 sites) or one thread-block cluster (<= 262144 sites) that
                                 keeps the state in shared memory for a whole chunk of EMCS; launch
                                 per cluster, colour and measurement instead (same results) */
    MQV_FLAG_RESIDENT = 4     /* take the resident path wherever the lattice fits it.  Default (neither
                                 flag): a single handle is resident up to 16384 sites; batch members
                                 run on the batch's graph path */
};

typedef struct mqv_run_params {
    double beta;       /* inverse temperature */
    uint64_t seed;     /* Philox key */
    uint32_t replica;  /* replica id (24 bits), part of every counter */
    int32_t device;    /* CUDA device ordinal */
    uint32_t flags;    /* MQV_FLAG_* */
    uint32_t reserved;
} mqv_run_params;

/* Per-measurement observables (FP64): energy per site, |m|, m^2, m^4. */
typedef struct mqv_obs {
    double e, m, m2, m4;
} mqv_obs;

typedef struct mqv_sim mqv_sim;

MQV_API const char* mqv_version(void);
/* Number of CUDA devices visible to the engine (0 on a machine without GPUs). */
MQV_API mqv_status mqv_device_count(int32_t* count);
/* Copies the calling thread's last error message (NUL-terminated). */
MQV_API mqv_status mqv_last_error(char* buf, size_t len);

MQV_API mqv_status mqv_create(const mqv_model_desc* model, const mqv_lattice_desc* lattice,
                              const mqv_run_params* params, mqv_sim** out);
MQV_API mqv_status mqv_destroy(mqv_sim* sim);

/* Bind the handle to a caller stream (cudaStream_t passed as void*). */
MQV_API mqv_status mqv_set_stream(mqv_sim* sim, void* stream);
MQV_API mqv_status mqv_get_stream(mqv_sim* sim, void** stream);
MQV_API mqv_status mqv_set_beta(mqv_sim* sim, double beta);
MQV_API mqv_status mqv_set_model(mqv_sim* sim, const mqv_model_desc* model);

/* Random initial state from the INIT stream (reference initstatespace rules). */
MQV_API mqv_status mqv_init_state(mqv_sim* sim);
/* Host copy of the state in the reference layout: site-major, symd
 * components per site; int8 for integer models, float32 otherwise. */
MQV_API mqv_status mqv_get_state(mqv_sim* sim, void* host, size_t bytes);
MQV_API mqv_status mqv_set_state(mqv_sim* sim, const void* host, size_t bytes);
/* No counterpart in the reference.  mqv_get_state / mqv_set_state with a
 * checksum: *hash receives the FNV-1a 64-bit hash of the host bytes, and
 * mqv_set_state_checked refuses a buffer whose hash differs with
 * MQV_ERR_CHECKSUM (a corrupt or truncated stored state), leaving the
 * handle's state untouched.  The dump container stores the hash beside the
 * state (core.h:543-607 is the reference's restart-from-dump path). */
MQV_API mqv_status mqv_get_state_checked(mqv_sim* sim, void* host, size_t bytes, uint64_t* hash);
MQV_API mqv_status mqv_set_state_checked(mqv_sim* sim, const void* host, size_t bytes, uint64_t hash);
/* Device pointer of the current state (valid until the next engine call).
 * Layout: the reference site order, except (a) on the fused 2D Ising path,
 * whose rows hold the even-x sites, then the odd-x sites, with the 32 bytes
 * of each 32-site group transposed (site s of a group at byte 4 (s & 7) +
 * (s >> 3)), and (b) for 3-vector models (Heisenberg, XXZ), stored as one
 * float array per component (component c of site i at [c n + i]);
 * mqv_get_state / mqv_set_state convert. */
MQV_API mqv_status mqv_state_device_ptr(mqv_sim* sim, void** dev, size_t* bytes);
MQV_API mqv_status mqv_state_bytes(mqv_sim* sim, size_t* bytes);

/* Sweep / cluster counters: together with (seed, replica) they are the whole
 * random-number state, so checkpoint = state + counters. */
MQV_API mqv_status mqv_get_counters(mqv_sim* sim, uint64_t* sweep, uint64_t* cluster);
MQV_API mqv_status mqv_set_counters(mqv_sim* sim, uint64_t sweep, uint64_t cluster);

/* nsweeps colour-ordered Metropolis sweeps (asynchronous on the handle's stream). */
MQV_API mqv_status mqv_metropolis(mqv_sim* sim, int32_t nsweeps);
/* Cluster algorithms (same clusters either way, the seed's component of the
 * bonds activated on their keyed draws): growth by one CTA, breadth first
 * (a barrier per level of the cluster's depth), or labelling of the
 * activated-bond components in a fixed number of whole-lattice passes. */
enum { MQV_WOLFF_AUTO = 0, MQV_WOLFF_BFS = 1, MQV_WOLFF_LABEL = 2 };
/* No counterpart in the reference.  The cluster algorithm of a handle:
 * MQV_WOLFF_AUTO (default) labels int8 lattices of at least 2^18 sites and
 * grows the others breadth first; lattices on the resident path
 * (MQV_FLAG_NO_RESIDENT unset, int8 stencils of <= 262144 sites) label in
 * (distributed) shared memory. */
MQV_API mqv_status mqv_set_wolff(mqv_sim* sim, int32_t algorithm);
/* nclusters Wolff clusters; sizes (host, may be NULL) receives each size
 * (synchronises when sizes != NULL). */
MQV_API mqv_status mqv_wolff(mqv_sim* sim, int32_t nclusters, int32_t* sizes);
/* No counterpart in the reference.  mqv_wolff for int8 models (Ising,
 * embedded Ising, Potts) that allocates no device memory: the queue, the
 * visited bitmap and the size slots live in one static device array sized
 * for lattices of at most 1,048,576 sites (larger lattices are rejected with
 * MQV_ERR_INVALID_ARG).  For hosts that cannot have device memory allocated
 * while they run clusters (HBM budgeted up front for resident lattices, or
 * no cudaMalloc/cudaFree stalls allowed between their streams).  Same
 * clusters, sizes and counters as mqv_wolff.  The bitmap starts at zero
 * (module load) and every cluster leaves it zero.  The array is shared by
 * all handles on a device: calls whose kernels may overlap race on it, so
 * the caller orders them on the GPU (one stream, or an event or a
 * synchronisation between streams); host calls one after the other are not
 * enough when sizes is NULL, since the call then returns while its kernels
 * run.  The first call on a device looks up the array's address, keeps it
 * and may load the module, so it must come before any stream capture, and
 * the handle must not be used across a reset of its CUDA context. */
MQV_API mqv_status mqv_wolff_noalloc(mqv_sim* sim, int32_t nclusters, int32_t* sizes);
/* n_emcs elementary MC steps (ncluster clusters then nmetro sweeps each),
 * measuring after every step.  obs (host, may be NULL) receives n_emcs
 * records; mean_cluster (host, may be NULL) receives n_emcs mean sizes. */
MQV_API mqv_status mqv_emcs(mqv_sim* sim, int32_t n_emcs, int32_t ncluster, int32_t nmetro,
                            mqv_obs* obs, double* mean_cluster);
/* No counterpart in the reference.  mqv_emcs that keeps the raw lattice sums
 * of every EMCS on the device for gradient estimators: d_samples (DEVICE
 * pointer, n_emcs * 4 doubles) receives per EMCS the interaction sum
 * sum_i s_i sum_{j in nbrs(i)} s_j, sum_i s_i, sum_i s_i^2 and
 * sum_i (s_i^2 - 1)^2 (x components for vectors; 0 for the last sum of
 * integer models).  Asynchronous on the handle's stream. */
MQV_API mqv_status mqv_emcs_samples(mqv_sim* sim, int32_t n_emcs, int32_t ncluster, int32_t nmetro, double* d_samples);
/* No counterpart in the reference.  Fluctuation-dissipation gradients of
 * scalar phi^4 in the reference form (src/hamiltonian/Phi4.h:84-121),
 * S = -beta sum_<ij> phi_i phi_j + sum_i [mass phi_i^2 + lambda (phi_i^2 - 1)^2],
 * from the samples of nrep runs (d_samples: [nrep][nsamp][4] as written by
 * mqv_emcs_samples).  All arrays are DEVICE pointers: d_beta, d_lambda [nrep];
 * d_obs [nrep][3] = (<E>, <|m|>, U4); d_jac [nrep][3][2] = d obs / d(beta,
 * lambda); optional d_gout [nrep][3] and d_grads [nrep][2] = gout . jac.
 * stream: cudaStream_t (NULL = default stream). */
MQV_API mqv_status mqv_phi4_fdt(const double* d_samples, int32_t nrep, int32_t nsamp, int64_t nsites, double mass,
                                const double* d_beta, const double* d_lambda, double* d_obs, double* d_jac,
                                const double* d_gout, double* d_grads, void* stream);
/* Observables of the current state. */
MQV_API mqv_status mqv_measure(mqv_sim* sim, mqv_obs* out);
MQV_API mqv_status mqv_synchronize(mqv_sim* sim);
/* Human-readable description of the handle's kernel path (e.g. the autotuned
 * fused-sweep configuration), NUL-terminated. */
MQV_API mqv_status mqv_describe(mqv_sim* sim, char* buf, size_t len);
/* Number of engine kernel launches issued by this handle so far. */
MQV_API mqv_status mqv_launch_count(mqv_sim* sim, uint64_t* count);

/* ---- batches ------------------------------------------------------------
 * Many independent simulations on one GPU, advanced together: the farm of
 * MARQOV's scheduler (one Core per thread, src/libmarqov/marqovscheduler.h:
 * 64-494, createSimfromParameter / start at :75-144, 223-273) as one set of
 * batched kernels per EMCS, captured once in a CUDA graph and replayed.
 * Members: any model on hypercubic or CSR lattices of any sizes, each with
 * its own coefficients, beta, seed, replica id and bonds (disorder
 * realisations); one batch holds either int8 members (Ising, embedded Ising,
 * Potts, Blume-Capel, Edwards-Anderson) or float members (Heisenberg, XXZ,
 * phi^4).  A batched run produces the same states, cluster sizes and
 * observables as running each member handle with mqv_emcs. */
typedef struct mqv_sim_spec {
    mqv_model_desc model;
    mqv_lattice_desc lattice;
    mqv_run_params params; /* the same device for every member */
} mqv_sim_spec;

typedef struct mqv_batch mqv_batch;

MQV_API mqv_status mqv_batch_create(const mqv_sim_spec* specs, int32_t n, mqv_batch** out);
MQV_API mqv_status mqv_batch_destroy(mqv_batch* batch);
/* Member i as an ordinary handle (state, counters, measurement); owned by
 * the batch and bound to its stream. */
MQV_API mqv_status mqv_batch_member(mqv_batch* batch, int32_t i, mqv_sim** sim);
MQV_API mqv_status mqv_batch_init_state(mqv_batch* batch);
/* Cluster algorithms of a batch (MQV_WOLFF_*; same clusters either way):
 * growth by one CTA per member, breadth first; or labelling of the
 * activated-bond components of all members in a fixed number of
 * whole-lattice passes (cost independent of cluster depth; pays for
 * percolating clusters on large lattices).  The default, MQV_WOLFF_AUTO,
 * times every chunk of EMCS (up
 * to 256 between host synchronisations), tries the algorithm not in use on a
 * few EMCS at the start of a chunk when it has no estimate or an old one, and
 * uses the faster estimate: the chain is the same whichever runs. */
MQV_API mqv_status mqv_batch_set_wolff(mqv_batch* batch, int32_t algorithm);
/* The algorithm in use: MQV_WOLFF_BFS or MQV_WOLFF_LABEL, or MQV_WOLFF_AUTO
 * while the automatic choice has not been timed yet. */
MQV_API mqv_status mqv_batch_get_wolff(mqv_batch* batch, int32_t* algorithm);
/* EMCS per graph launch (1 .. 256; default 8). */
MQV_API mqv_status mqv_batch_set_graph_steps(mqv_batch* batch, int32_t steps);
/* n_emcs EMCS of every member (ncluster clusters, then nmetro sweeps, then a
 * measurement).  obs (host, may be NULL): n_emcs * n records, EMCS-major
 * (record e * n + i is member i after EMCS e); mean_cluster likewise. */
MQV_API mqv_status mqv_batch_emcs(mqv_batch* batch, int32_t n_emcs, int32_t ncluster, int32_t nmetro, mqv_obs* obs,
                                  double* mean_cluster);
/* No counterpart in the reference.  mqv_batch_emcs that keeps each member's
 * raw lattice sums on the device (as mqv_emcs_samples): d_samples is a
 * DEVICE pointer to [n][n_emcs][4] doubles. */
MQV_API mqv_status mqv_batch_emcs_samples(mqv_batch* batch, int32_t n_emcs, int32_t ncluster, int32_t nmetro,
                                          double* d_samples);
/* Replica exchange (parallel tempering) between batch members; replaces the
 * scheduler's PT loop, CXX11Scheduler::start / ptstep / calcprob /
 * exchange_statespace (src/libmarqov/marqovscheduler.h:44-57,223-273,374-470).
 * n_steps steps, each emcs_per_step EMCS of every member (one Core::gameloop)
 * followed by exchange attempts between the step's pairs:
 * plan[(t * pairs_per_step + k) * 2 + {0, 1}] are member ids; a pair (a, a)
 * is skipped (the reference's self swap), the other pairs of one step are
 * disjoint, and partners share model descriptor and lattice (they differ in
 * beta).  A pair exchanges its members' states with probability
 * min(1, exp(b_a E_a - b_a E_b + b_b E_b - b_b E_a)), E the total energy
 * after the step's last EMCS, the uniform drawn from the TEMPER stream keyed
 * by (seed, the batch's exchange-step counter, pair index).  Members keep
 * beta, seed and counters; member i's state is the one it holds after the
 * exchanges.  obs (optional): [n_steps * emcs_per_step][n]; accepted
 * (optional): [n_steps][pairs_per_step], 1 exchanged, 0 rejected, -1 self
 * pair.  No counterpart to the reference's plan generator: the caller passes
 * the pairs (the reference draws maxpt random pairs, marqovscheduler.h:203-210). */
MQV_API mqv_status mqv_batch_tempering(mqv_batch* batch, int32_t n_steps, int32_t emcs_per_step, int32_t ncluster,
                                      int32_t nmetro, const int32_t* plan, int32_t pairs_per_step, uint64_t seed,
                                      mqv_obs* obs, int32_t* accepted);
MQV_API mqv_status mqv_batch_launch_count(mqv_batch* batch, uint64_t* count);

/* Self test (host only, no device needed): the closed-form acceptance cut
 * the sweep kernels use, cut[i] = the smallest word >> 11 that
 * update_accepted<pref>(dE[i], beta[i], word) rejects (2^53: none). */
MQV_API mqv_status mqv_selftest_accept_cut(int32_t pref, int32_t n, const double* dE, const double* beta,
                                           uint64_t* cut);
/* Self test: Philox blocks for n counters (c0 = i, other words given) computed
 * on the device by the engine and by cuRAND's Philox4_32_10; out_engine and
 * out_curand receive 4n words each (host). */
MQV_API mqv_status mqv_selftest_philox(uint64_t seed, uint32_t c1, uint32_t c2, uint32_t c3,
                                       int32_t n, uint32_t* out_engine, uint32_t* out_curand);
/* Self test of the bounded device waits: the next fused 2D Ising sweep of
 * the handle (band kernel, L = 8192 or 16384) has CTA 0 withhold its staged
 * row `row` (2 .. 64) and waits at most wait_ns for a row, so that the wait
 * for the withheld row runs out.  The kernel then sets MQV_ERR_TIMEOUT,
 * lets the copies it issued land and returns; the call that reads the
 * device status reports MQV_ERR_TIMEOUT, and the handle refuses compute
 * (MQV_ERR_STATE) until its state is set again.  Nothing faults or hangs:
 * every other wait is bounded by the same limit. */
MQV_API mqv_status mqv_selftest_inject_timeout(mqv_sim* sim, int32_t row, uint64_t wait_ns);

#ifdef __cplusplus
}
#endif
#endif /* MARQOV_B200_H */
