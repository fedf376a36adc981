/*
 * tvbk.h -- C ABI of the B200 region-simulation kernels (libtvbk.so).
 *
 * The library runs TVB's region simulation loop -- delayed-history gather,
 * coupling pre/sum/post, model derivative, Euler/Heun (deterministic and
 * stochastic) step with additive noise, and the Raw / TemporalAverage / Bold
 * monitors -- for a batch of independent simulation instances in one launch.
 *
 * Every entry point takes plain pointers and sizes.  Device buffers are
 * allocated and owned by the caller; the library allocates nothing, except
 * where a function's comment says otherwise.  Functions return TVBK_OK (0) or
 * a negative status; tvbk_last_error() gives the message of the last failure
 * on the calling thread.  Launches are asynchronous on the caller's stream
 * (a cudaStream_t passed as void*; NULL is the legacy default stream).
 *
 * Which reference interface each entry point replaces (paths inside
 * the-virtual-brain/tvb-root):
 *   tvbk_idelays           tvb_library/tvb/datatypes/connectivity.py:275,308-326
 *                          (Connectivity.configure delays + set_idelays)
 *   tvbk_sparse_layout     tvb_library/tvb/simulator/history.py:221-244
 *                          (SparseHistory.__init__ non-zero arrays)
 *   tvbk_sim_run           tvb_library/tvb/simulator/simulator.py:322-366
 *                          (Simulator.__call__ step loop: history.py:197-204,251-256,
 *                          coupling.py:118-167, integrators.py:296-426, noise.py:195-232,
 *                          monitors.py:178-190,380-391,942-962)
 *   tvbk_gather_delayed    tvb_library/tvb/simulator/history.py:251-256
 *                          (SparseHistory.query_sparse, the delayed-state gather alone)
 *   tvbk_fc                tvb_framework/tvb/adapters/analyzers/cross_correlation_adapter.py:348-380
 *                          (numpy.corrcoef over the Bold time series, per instance)
 *   tvbk_project           tvb_library/tvb/simulator/monitors.py:602-614
 *                          (Projection.sample: gain.dot(state) of EEG / MEG / iEEG)
 *   tvbk_balloon           tvb_library/tvb/analyzers/fmri_balloon.py:198-364
 *                          (BalloonModel.evaluate: Balloon-Windkessel BOLD, float64)
 */
#ifndef TVBK_H
#define TVBK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TVBK_ABI_VERSION 3

/* status codes */
#define TVBK_OK 0
#define TVBK_ERR_INVALID (-1)     /* bad argument */
#define TVBK_ERR_UNSUPPORTED (-2) /* component combination not built */
#define TVBK_ERR_CUDA (-3)        /* CUDA runtime error (message has the CUDA error string) */
#define TVBK_ERR_TOO_LARGE (-4)   /* size beyond a documented limit */

/* per-instance status bits written by the simulation kernel */
#define TVBK_STATUS_NONFINITE 1   /* a state variable became NaN or Inf */
#define TVBK_STATUS_DEGREE 2      /* a row had more edges than launch.max_degree (coupling incomplete) */
#define TVBK_STATUS_UNSUPPORTED 4 /* the instance asks for something this kernel variant does not do
                                   * (AfferentCoupling on a variant other than the row kernel; a stimulus,
                                   * AfferentCoupling or projection stream with launch.extras = 0) */
#define TVBK_STATUS_TIMEOUT 8     /* a group barrier of a cooperative launch (launch.groups > 0) waited past its
                                   * limit (4 s), or another group's did: the launch stopped early and this
                                   * instance's state is incomplete */

/* components */
enum {
    TVBK_MODEL_G2D = 0,        /* Generic2dOscillator (models/oscillator.py:39-395) */
    TVBK_MODEL_JANSEN_RIT = 1, /* JansenRit (models/jansen_rit.py:38-289) */
    TVBK_MODEL_RWW = 2,        /* ReducedWongWang (models/wong_wang.py:36-181) */
    TVBK_MODEL_EPILEPTOR = 3,  /* Epileptor (models/epileptor.py:36-356) */
    TVBK_MODEL_SUM = 4         /* dx = x + c; the model of the reference's exact-propagation test */
};
enum {
    TVBK_CFUN_LINEAR = 0,        /* Linear: a*gx + b (coupling.py:170-200); Scaling is Linear with b = 0 */
    TVBK_CFUN_DIFFERENCE = 1,    /* Difference: a * sum w (x_j - x_i) (coupling.py:462-486) */
    TVBK_CFUN_SIGMOIDAL_JR = 2,  /* SigmoidalJansenRit (coupling.py:325-376) */
    TVBK_CFUN_SIGMOIDAL = 3,     /* Sigmoidal: cmin + (cmax-cmin) / (1 + exp(-a ((gx-midpoint)/sigma))),
                                  * cfun {cmin, cmax, midpoint, a, sigma} (coupling.py:270-322) */
    TVBK_CFUN_HYPERBOLIC_TANGENT = 4, /* pre a (1 + tanh((b x_j - midpoint)/sigma)), cfun {a, b, midpoint,
                                       * sigma} (coupling.py:227-267) */
    TVBK_CFUN_KURAMOTO = 5       /* pre sin(x_j - x_i), post a / ncvar * gx, cfun {a} (coupling.py:489-508) */
};
/* Couplings 3..5 run on the row kernel one step at a time (prefetch 0, lanes 1, no edge split, no cluster). */
enum {
    TVBK_SCHEME_EULER_DET = 0,   /* integrators.py:365-391 */
    TVBK_SCHEME_EULER_STOCH = 1, /* integrators.py:394-426 */
    TVBK_SCHEME_HEUN_DET = 2,    /* integrators.py:286-318 */
    TVBK_SCHEME_HEUN_STOCH = 3,  /* integrators.py:321-362 */
    TVBK_SCHEME_IDENTITY = 4,    /* integrators.py:483-507 */
    TVBK_SCHEME_RK4 = 5          /* RungeKutta4thOrderDeterministic, integrators.py:429-480 */
};
enum {
    TVBK_NOISE_NONE = 0,
    TVBK_NOISE_FED = 1,          /* caller-provided standard normals (e.g. the reference's own stream) */
    TVBK_NOISE_PHILOX = 2        /* counter-based Philox4x32-10 + Box-Muller, keyed by (seed, stream) */
};

/* Maximum sizes of this build. */
#define TVBK_MAX_REGIONS 1024    /* regions per instance (one thread per region) */
#define TVBK_MAX_VOI 8           /* observed variables per monitor set */
#define TVBK_MAX_PARAMS 20       /* model parameters */

/* One connectome edge as the gather reads it: off = (idelay * n - col) * ncvar,
 * so that the ring offset of the delayed value is (slot of step - 1) * n * ncvar
 * - off, plus ring_len * n * ncvar when that is negative. */
typedef struct tvbk_edge {
    int32_t off;
    float weight;
} tvbk_edge;

/*
 * One simulation instance.  All pointers are device pointers.  Arrays
 * indexed [..][n] are region-fastest.  The ring holds the coupling variables
 * of time t in slot t % ring_len, laid out [ring_len][n][ncvar]; ring_len is
 * at least horizon + 1 (see tvbk_ring_len).  Instances may share the
 * connectome arrays.  The kernel advances `step` itself, so a chunked run
 * re-launches the same descriptor array.
 */
typedef struct tvbk_inst {
    /* connectome: rows are target regions, edges in the reference's row-major non-zero order */
    const int32_t* row_ptr;      /* [n+1] */
    const tvbk_edge* edges;      /* [nnz] packed offsets and weights (tvbk_pack_edges) */
    const tvbk_edge* slots;      /* [n][slot_width] or NULL: the row kernel's gather slots of each row -- the
                                  * row's edges in an order where the 32 rows of a warp read distinct shared-
                                  * memory banks in every slot (needs ring_len * n a multiple of 32), padding
                                  * slots with weight 0; used when slot_width equals the kernel's register
                                  * slot count, else the packed edges are read */
    /* dynamic state */
    float* ring;                 /* [ring_len][n][ncvar] */
    float* pre_ring;             /* [ring_len][n] SigmoidalJansenRit with the row or cluster kernel and rings
                                  * read in place: the gather ring of pre-applied sigmoid values (scratch,
                                  * recomputed from `ring` at every launch); NULL otherwise */
    float* state;                /* [nsv][n] */
    /* parameters */
    const float* params;         /* [nparam][n] model parameters, one value per region */
    const float* noise_sigma;    /* [nintvar][n] sqrt(dt) * sqrt(2 nsig); NULL when deterministic */
    const float* noise_fed;      /* [*][nintvar][n] standard normals; step s reads row s - fed_base - 1 */
    /* region stimulus (patterns.py:146-186, simulator.py:290-306): step s adds
     * stim[s - stim_base - 1] * stim_weight[i] to the state variables in the
     * stim_vars bit mask, through dt * stimulus in the scheme (identity: + stimulus) */
    const float* stim;           /* [*] temporal pattern; NULL: no stimulus */
    const float* stim_weight;    /* [n] spatial pattern */
    /* monitors (NULL disables one) */
    float* raw;                  /* [*][nvoi][n]; step s writes row s - raw_base - 1 */
    float* sub;                  /* [*][nvoi][n] the state at every step s with s % sub_istep == 0 (SubSample,
                                  * and GlobalAverage / SpatialAverage reduce it): row s / sub_istep - sub_base - 1 */
    float* tavg;                 /* [*][nvoi][n]; sample s / tavg_istep - tavg_base - 1 */
    float* aff;                  /* [*][ncvar][n] AfferentCoupling (monitors.py:394-433): the coupling that step
                                  * s + 1 receives, taken after step s and averaged over aff_istep steps (1: every
                                  * step); sample s / aff_istep - aff_base - 1.  Row kernel only */
    float* aff_acc;              /* [ncvar][n] running sum of the current aff_istep period */
    float* proj;                 /* [*][nvoi][n] projection monitors (EEG / MEG / iEEG, monitors.py:436-831): the
                                  * mean of the observed variables over each proj_istep steps, sample
                                  * s / proj_istep - proj_base - 1; the host applies the sensor gain (a GEMM) */
    float* proj_acc;             /* [nvoi][n] running sum of the current proj_istep period */
    float* tavg_acc;             /* [nvoi][n] running sum of the current period */
    double* bold;                /* [*][nvoi][n]; sample s / bold_istep - bold_base - 1 */
    double* bold_acc;            /* [nvoi][n] running sum of the current 4 ms window */
    double* bold_stock;          /* [stock_len][nvoi][n] 4 ms averages, ring */
    const double* hrf;           /* [stock_len] reversed haemodynamic kernel */
    int64_t step;                /* last completed step (the reference's current_step) */
    int64_t step_end;            /* run until step == step_end */
    int64_t raw_base, fed_base, tavg_base, bold_base, sub_base, stim_base, aff_base, proj_base;
    int32_t n, nnz, horizon, ring_len;
    int32_t tavg_istep, bold_istep, bold_ii, stock_len, sub_istep;
    uint32_t stim_vars;          /* bit k: state variable k receives the stimulus (the model's stvar) */
    int32_t aff_istep, proj_istep;
    int32_t slot_width;
    float cfun[6];               /* coupling parameters, see tvbk_sim_run */
    uint32_t seed, stream;       /* Philox key */
    double bold_k1v0;            /* k_1 * V_0 of the FirstOrderVolterra kernel */
} tvbk_inst;

/* Launch description shared by all instances of one tvbk_sim_run call. */
typedef struct tvbk_launch {
    tvbk_inst* insts;            /* device array [n_inst]; the kernel advances each `step` */
    int32_t* status;             /* device array [n_inst], TVBK_STATUS_* bits are OR-ed in */
    int32_t n_inst;
    int32_t model, cfun, scheme, noise;
    int32_t nvoi;
    int32_t voi[TVBK_MAX_VOI];   /* indices into the model's observable expressions */
    int32_t max_n;               /* largest n over the instances (sets the block size) */
    int32_t max_ring_len;        /* largest ring_len; the ring is staged in shared memory if it fits */
    int32_t sync_every;          /* barrier interval K, 1 <= K <= min(d_min + 1, ring_len - horizon) */
    int32_t ring_in_smem;        /* 1: stage rings in shared memory (needs fit), 0: read them in place */
    int32_t max_degree;          /* largest row degree (non-zero weights of a target region) over the instances */
    int32_t edges_per_thread;    /* 0: one thread per row; 8, 12, 16 or 24: edge-parallel gather with that many
                                  * register slots per thread (rings in shared memory, Linear or
                                  * SigmoidalJansenRit only; ceil(nnz / block_threads) must not exceed it nor
                                  * the smallest non-zero row degree of any instance).  With cluster > 1: 0 (a
                                  * warp per row) or 8, 16, 32: edge runs -- each cluster CTA's edges, staged in
                                  * shared memory (cluster_edges), cut into runs of that many edges, one per
                                  * gather thread; it must not exceed the smallest non-zero row degree of a
                                  * CTA's rows and the runs must cover the CTA's edges (512 threads, less one
                                  * warp per 32 rows with prefetch); Difference is then summed as
                                  * sum w x_j - x_i sum w and may prefetch */
    int32_t block_threads;       /* CTA size for the edge-parallel gather (multiple of 32, >= max_n, <= 512) */
    int32_t prefetch;            /* 1: issue the gather of step s + 1 before the update of step s (row kernel,
                                  * Linear or SigmoidalJansenRit); needs every delay >= 1 and
                                  * 1 <= sync_every <= the smallest delay.  With rings in shared memory the
                                  * kernel then stages max_ring_len + TVBK_RING_GUARD slots per instance (the
                                  * guard slots mirror slots 0..TVBK_RING_GUARD-1).  2: the same overlap with separate
                                  * warps -- ceil(max_n / 32) gather warps sum the rows of step s + 1 while as
                                  * many update warps advance step s (rings in shared memory, row degrees
                                  * <= 64; one CTA barrier per step) */
    int32_t lanes;               /* 1, or 8 / ncvar: instance groups.  Consecutive groups of `lanes` instances
                                  * share connectome, ring length and step range; one thread advances one
                                  * (region, instance) pair and the group's rings are interleaved
                                  * [ring_len][n][ncvar][lanes] in the `ring` of the group's first instance,
                                  * read in place (regions * lanes <= 1024 threads; the edge list and two
                                  * staging buffers of max_degree * ncvar floats per thread must fit in
                                  * shared memory) */
    int32_t cluster;             /* 0 or 1: one CTA per instance; 2..16: a thread-block cluster of that many CTAs
                                  * per instance, each owning ceil(max_n / cluster) <= 480 rows, rings read in
                                  * place (lanes 1, row gather, rings not in shared memory).  With groups > 0,
                                  * 2..256 CTAs per instance without a hardware cluster (see groups) */
    int32_t cluster_edges;       /* cluster kernel: edges of one CTA's rows that it stages in shared memory; a CTA
                                  * with more edges reads them from global memory (0: always global) */
    int32_t ring_layout;         /* 0: rings [ring_len][n][ncvar] (time-major).  1: region-major rings for the
                                  * cluster kernel's blocked edge runs (cluster > 1, edges_per_thread > 0,
                                  * prefetch 1, Linear, Difference or SigmoidalJansenRit (whose ring of
                                  * pre-applied sigmoid values, one float per slot, is region-major too),
                                  * ncvar 1 or 2, sync_every a multiple of 4
                                  * with 4 <= sync_every <= the smallest delay - 3): region r's times sit in
                                  * [r][TVBK_RING_REGION_STRIDE(ring_len, ncvar)][ncvar], time t in slot
                                  * t % ring_len, and the slots past ring_len mirror slots 0, 1, ... (every write
                                  * of a mirrored slot also writes its mirror).  A block of block_steps steps'
                                  * couplings is gathered together, each edge reading its consecutive times with
                                  * 32-byte loads;
                                  * each instance's ring must be 32-byte aligned (else the instance is not
                                  * advanced and gets TVBK_STATUS_UNSUPPORTED) */
    int32_t block_steps;         /* ring_layout 1: steps per gather block, 4 (or 0) or 8.  8 reads each edge's
                                  * eight consecutive times at once (fewer scattered sector reads per step); it
                                  * needs sync_every a multiple of 8 with 8 <= sync_every <= the smallest
                                  * delay - 7, and launch.extras = 0 */
    int32_t groups;              /* 0: cluster > 1 launches one thread-block cluster per instance.  G > 0
                                  * (ring_layout 1 only): one cooperative launch of G x cluster CTAs, all
                                  * resident at once (at most the SMs' resident CTAs); each group of `cluster`
                                  * consecutive CTAs takes instances from a device-side queue in inst_order
                                  * order (index order when NULL) until the batch is done, its CTAs kept in
                                  * step by barriers through group_sync, each wait bounded (TVBK_STATUS_TIMEOUT).
                                  * The instances of a batch then need not fit the GPU's thread-block clusters
                                  * at once, and an instance may use more than 16 CTAs */
    uint32_t* group_sync;        /* groups > 0: device scratch of TVBK_GROUP_SYNC_WORDS(groups) words, 4-byte
                                  * aligned; tvbk_sim_run zeroes it on the launch stream before each launch */
    int32_t extras;              /* bit 0: some instance has a region stimulus; bit 1: some instance has an
                                  * AfferentCoupling monitor; bit 2: some instance has a projection stream.  0
                                  * lets the row kernel with rings in shared memory use a build without any of
                                  * them (an instance that has one then gets TVBK_STATUS_UNSUPPORTED) */
    const int32_t* inst_order;   /* device [n_inst] or NULL: CTA b advances insts[inst_order[b]] and ORs its status
                                  * bits into status[inst_order[b]] (row kernel: lanes 1, no edge split, prefetch 0
                                  * or 1; with cluster > 1, cluster b advances insts[inst_order[b]]; with groups > 0,
                                  * the groups take insts[inst_order[0]], insts[inst_order[1]], ... in turn).  Lets one
                                  * launch take any subset of a batch, e.g. a window of exactly one wave of resident
                                  * CTAs, or order it, e.g. the longest instances first */
    int32_t* occupancy;          /* host pointer or NULL: when set, tvbk_sim_run launches nothing and stores there
                                  * the CTAs per SM of the row kernel variant it would launch (same restrictions) */
    int64_t max_steps;           /* steps per launch (a chunk); instances stop at step_end */
    float dt;
} tvbk_launch;

/* Library information. */
int tvbk_abi_version(void);
const char* tvbk_last_error(void);

/* sizeof(tvbk_inst), sizeof(tvbk_launch), sizeof(tvbk_edge) for which = 0, 1, 2
 * (lets a binding check its struct mirrors); -1 otherwise. */
int64_t tvbk_sizeof(int32_t which);

/* Conduction delays in integration steps, exactly as the reference:
 * idelays = rint((tract_lengths / speed) / dt) in float64, round half to even;
 * *horizon = max(idelays) + 1 over all n_elems entries.  Host function. */
int tvbk_idelays(const double* tract_lengths, int64_t n_elems, double speed, double dt,
                 int32_t* idelays, int32_t* horizon);

/* Non-zero layout of an n x n weight matrix (row-major order of the non-zero
 * entries, as SparseHistory builds it).  Host function.  row_ptr has n+1
 * entries; col, idelay, weight have room for n*n entries; *nnz is set. */
int tvbk_sparse_layout(const double* weights, const int32_t* idelays, int32_t n,
                       int32_t* row_ptr, int32_t* col, int32_t* idelay, float* weight,
                       int32_t* nnz, int32_t* min_delay);

/* Pack CSR columns, delays and weights into gather edges for a ring with
 * n regions and ncvar coupling variables.  Host function. */
int tvbk_pack_edges(const int32_t* col, const int32_t* idelay, const float* weight, int32_t nnz,
                    int32_t n, int32_t ncvar, tvbk_edge* edges);

/* Slots past the end of a ring staged in shared memory with prefetch = 1:
 * they mirror slots 0..TVBK_RING_GUARD-1, so that the gathers of four steps
 * in a row take one ring address per edge (address + r slots, r <= 3). */
#define TVBK_RING_GUARD 3

/* Words of launch.group_sync for `groups` groups: the queue head, the abort
 * flag, then per group an arrival counter and the claimed queue index. */
#define TVBK_GROUP_SYNC_WORDS(groups) (2 + 2 * (groups))

/* Region-major rings (launch.ring_layout = 1): slots per region -- the
 * ring_len slots, then a guard of 10 (ncvar 2) or 14 (ncvar 1) slots mirroring
 * slots 0, 1, ... (a block's read loads up to three 32-byte chunks from the
 * 32-byte boundary at or below its first slot, which may lie just below
 * ring_len), rounded up so that every region starts on a 32-byte boundary.
 * The ring itself must be 32-byte aligned. */
#define TVBK_RING_REGION_GUARD(ncvar) ((ncvar) == 1 ? 14 : 10)
#define TVBK_RING_REGION_STRIDE(ring_len, ncvar) \
    ((((ring_len) + TVBK_RING_REGION_GUARD(ncvar)) + (8 / (ncvar)) - 1) / (8 / (ncvar)) * (8 / (ncvar)))

/* Smallest ring length (slots) usable with barrier interval sync_every. */
int32_t tvbk_ring_len(int32_t horizon, int32_t sync_every);

/* Shared memory bytes one instance needs to stage its ring; 0 if it cannot be staged. */
int64_t tvbk_ring_smem_bytes(int32_t n, int32_t ncvar, int32_t ring_len);

/* Number of coupling variables, state variables, integrated state variables
 * and observable expressions of a model. */
int tvbk_model_dims(int32_t model, int32_t* ncvar, int32_t* nsv, int32_t* nintvar, int32_t* nobs,
                    int32_t* nparam);

/* Run up to L->max_steps steps of every instance (one CTA per instance).
 * Coupling parameters in tvbk_inst.cfun: Linear {a, b}; Difference {a};
 * SigmoidalJansenRit {cmin, cmax, midpoint, r, a}.  SigmoidalJansenRit's
 * pre() depends on the source region only: the row kernel (lanes 1,
 * edges_per_thread 0) and the cluster kernel apply it once per region and
 * step and gather from a ring of those values, one float per (slot, region),
 * so their edges are packed with ncvar = 1 (tvbk_pack_edges) and, with rings
 * read in place, each instance needs a pre_ring; the edge-parallel and
 * instance-group kernels apply it per edge and use edges packed with
 * ncvar = 2. */
int tvbk_sim_run(const tvbk_launch* L, void* stream);

/* Delayed-state gather of one instance at step `step` (the values the
 * coupling of that step reads): out[e * ncvar + k] = ring value of variable k
 * of region col[e] at time step - 1 - idelay[e], for every edge e.  Used to
 * check the ring indexing bit-exactly against the reference; it reads the
 * ring in place (inst_host->ring) through inst_host->edges, the same address
 * arithmetic as the simulation kernel. */
int tvbk_gather_delayed(const tvbk_inst* inst_host, int32_t ncvar, int64_t step, float* out_dev,
                        void* stream);

/* Pearson correlation of each instance's series: x is [n_inst][T][n] float64
 * (instance-major), fc is [n_inst][n][n] float64.  Rows with zero variance
 * give NaN like numpy.corrcoef. */
int tvbk_fc(const double* x, int32_t n_inst, int32_t T, int32_t n, double* fc, void* stream);

/* Sensor signals of a projection monitor from the simulation's period-mean
 * stream (the launch's `proj` output), float64 on the device:
 *   y[t][v][s] = sum_r gain[s][r] * x[t][voi[v]][r]
 * x is [T][nvoi][n] float32 (the rows of several instances may be stacked
 * into T), voi [nvoi_m] int32 (device) picks the monitor's observed
 * variables, gain [S][n] float64 is the region lead field, y is
 * [T][nvoi_m][S] float64.  Each output is one fma chain over r in order, so
 * a row's value does not depend on the other rows of the launch. */
int tvbk_project(const float* x, int64_t T, int32_t nvoi, int32_t n, const int32_t* voi, int32_t nvoi_m,
                 const double* gain, int32_t S, double* y, void* stream);

/* Balloon-Windkessel BOLD of neural-activity series, float64
 * (tvb_library/tvb/analyzers/fmri_balloon.py:198-364, BalloonModel.evaluate with the
 * HeunDeterministic scheme).  x and bold are device arrays [T][nseries] (series fastest);
 * dt in seconds; params (host) = {tau_s, tau_f, tau_o, alpha, E0, V0, k1, k2, k3};
 * nonlinear = 1 for the non-linear BOLD equation, 0 for the linear one.  Every series
 * starts from s = 0, f = v = q = 1; bold[0] is the signal of that state. */
int tvbk_balloon(const double* x, int32_t T, int64_t nseries, double dt, const double* params, int32_t nonlinear,
                 double* bold, void* stream);

/* Bytes of device scratch that tvbk_sim_run_static keeps inside the library (per GPU). */
#define TVBK_STATIC_SCRATCH_BYTES (8 * 1024 * 1024)

/* No counterpart in the reference.  Runs one instance like tvbk_sim_run but
 * allocates nothing, for callers that cannot call cudaMalloc (an FFI or
 * plug-in host that only holds the input and output buffers it was given,
 * or code under a fixed memory budget).  The working memory that
 * tvbk_sim_run takes from the caller -- the ring the kernel advances, the
 * TemporalAverage, Bold, AfferentCoupling and projection-stream
 * accumulators, the Bold 4 ms stock, the descriptor and the status word --
 * lives in a static device array of TVBK_STATIC_SCRATCH_BYTES; larger
 * instances are rejected with TVBK_ERR_TOO_LARGE.  `inst` is a host struct:
 * inst->ring is the caller's initial ring (device, read only), inst->state
 * the caller's state buffer (read at the start, holds the final state at the
 * end), inst->tavg_acc, bold_acc, bold_stock, aff_acc and proj_acc are
 * ignored, every monitor starts from zero, and
 * all steps from inst->step to inst->step_end run in this call
 * (L->insts, L->status, L->n_inst, L->max_n, L->max_ring_len and
 * L->max_steps are ignored).  status_out, if not NULL, is a device int32
 * that receives the TVBK_STATUS_* bits.  The first call on a device looks up
 * the array's address with that device current; make it before any stream
 * capture.  That address does not survive a cudaDeviceReset of the device.
 * Calls share the array and keep the last call's contents: calls
 * that overlap on the GPU race, so serialise them. */
int tvbk_sim_run_static(const tvbk_launch* L, const tvbk_inst* inst, int32_t* status_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TVBK_H */
