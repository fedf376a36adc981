// C ABI of libtvbk.so: argument checks, host-side planning helpers
// (delays, non-zero layout, edge packing) and dispatch to the kernels.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "tvbk.h"
#include "tvbk_models.cuh"

namespace tvbk {
int launch_g2d(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_jr(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_rww(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_epileptor(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_sum(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int64_t fc_smem_bytes(int32_t T, int32_t n);
int fc_launch(const double* x, int32_t n_inst, int32_t T, int32_t n, double* fc, cudaStream_t stream);
}  // namespace tvbk

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* where) {
    return fail(TVBK_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

struct ModelDims {
    int ncvar, nsv, nint, nobs, nparam;
};

bool model_dims(int model, ModelDims* d) {
    using namespace tvbk;
    switch (model) {
        case TVBK_MODEL_G2D: *d = {G2D::NCV, G2D::NSV, G2D::NINT, G2D::NOBS, G2D::NP}; return true;
        case TVBK_MODEL_JANSEN_RIT:
            *d = {JansenRit::NCV, JansenRit::NSV, JansenRit::NINT, JansenRit::NOBS, JansenRit::NP};
            return true;
        case TVBK_MODEL_RWW: *d = {RWW::NCV, RWW::NSV, RWW::NINT, RWW::NOBS, RWW::NP}; return true;
        case TVBK_MODEL_EPILEPTOR:
            *d = {Epileptor::NCV, Epileptor::NSV, Epileptor::NINT, Epileptor::NOBS, Epileptor::NP};
            return true;
        case TVBK_MODEL_SUM:
            *d = {SumModel::NCV, SumModel::NSV, SumModel::NINT, SumModel::NOBS, SumModel::NP};
            return true;
        default: return false;
    }
}

constexpr int64_t kMaxSmemPerBlock = 227 * 1024;

// ------------------------------------------------------------------ kernels

__global__ void gather_kernel(const tvbk_edge* __restrict__ edges, const float* __restrict__ ring, int nnz,
                              int ncvar, int base_off, int ring_floats, float* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const int a = tvbk::gather_addr(base_off, edges[e].off, ring_floats);
    for (int k = 0; k < ncvar; ++k) out[(size_t)e * ncvar + k] = ring[a + k];
}

}  // namespace

namespace tvbk {
int set_error(int code, const char* msg) {
    g_last_error = msg;
    return code;
}
}  // namespace tvbk

// --------------------------------------------------------------------- ABI

extern "C" {

int tvbk_abi_version(void) { return TVBK_ABI_VERSION; }

int64_t tvbk_sizeof(int32_t which) {
    switch (which) {
        case 0: return (int64_t)sizeof(tvbk_inst);
        case 1: return (int64_t)sizeof(tvbk_launch);
        case 2: return (int64_t)sizeof(tvbk_edge);
        default: return -1;
    }
}

const char* tvbk_last_error(void) { return g_last_error.c_str(); }

int tvbk_idelays(const double* tract_lengths, int64_t n_elems, double speed, double dt, int32_t* idelays,
                 int32_t* horizon) {
    if (!tract_lengths || !idelays || !horizon || n_elems <= 0)
        return fail(TVBK_ERR_INVALID, "tvbk_idelays: null pointer or empty input");
    if (!(speed > 0.0) || !(dt > 0.0)) return fail(TVBK_ERR_INVALID, "tvbk_idelays: speed and dt must be > 0");
    int32_t mx = 0;
    for (int64_t k = 0; k < n_elems; ++k) {
        const double delay = tract_lengths[k] / speed;  // connectivity.py:275
        const double steps = std::rint(delay / dt);     // connectivity.py:321, round half to even
        if (!(steps >= 0.0) || steps > 2147483647.0)
            return fail(TVBK_ERR_INVALID, "tvbk_idelays: delay %g steps out of range at %lld", steps, (long long)k);
        idelays[k] = (int32_t)steps;
        mx = idelays[k] > mx ? idelays[k] : mx;
    }
    *horizon = mx + 1;  // connectivity.py:323
    return TVBK_OK;
}

int tvbk_sparse_layout(const double* weights, const int32_t* idelays, int32_t n, int32_t* row_ptr, int32_t* col,
                       int32_t* idelay, float* weight, int32_t* nnz, int32_t* min_delay) {
    if (!weights || !idelays || !row_ptr || !col || !idelay || !weight || !nnz || n <= 0)
        return fail(TVBK_ERR_INVALID, "tvbk_sparse_layout: null pointer or n <= 0");
    int32_t e = 0, dmin = 2147483647;
    for (int32_t i = 0; i < n; ++i) {
        row_ptr[i] = e;
        for (int32_t j = 0; j < n; ++j) {
            const double w = weights[(int64_t)i * n + j];
            if (w != 0.0) {  // history.py:224 (mask on the float64 weights)
                col[e] = j;
                idelay[e] = idelays[(int64_t)i * n + j];
                weight[e] = (float)w;  // stored float32, history.py:171,225
                dmin = idelay[e] < dmin ? idelay[e] : dmin;
                ++e;
            }
        }
    }
    row_ptr[n] = e;
    *nnz = e;
    if (min_delay) *min_delay = e > 0 ? dmin : 0;
    return TVBK_OK;
}

int tvbk_pack_edges(const int32_t* col, const int32_t* idelay, const float* weight, int32_t nnz, int32_t n,
                    int32_t ncvar, tvbk_edge* edges) {
    if ((nnz > 0 && (!col || !idelay || !weight || !edges)) || n <= 0 || ncvar <= 0)
        return fail(TVBK_ERR_INVALID, "tvbk_pack_edges: bad arguments");
    for (int32_t e = 0; e < nnz; ++e) {
        if (col[e] < 0 || col[e] >= n || idelay[e] < 0)
            return fail(TVBK_ERR_INVALID, "tvbk_pack_edges: edge %d out of range", e);
        const int64_t off = ((int64_t)idelay[e] * n - col[e]) * ncvar;
        if (off > 2147483647LL) return fail(TVBK_ERR_TOO_LARGE, "tvbk_pack_edges: ring offset overflows int32");
        edges[e].off = (int32_t)off;
        edges[e].weight = weight[e];
    }
    return TVBK_OK;
}

int32_t tvbk_ring_len(int32_t horizon, int32_t sync_every) {
    if (horizon < 1 || sync_every < 1) return -1;
    return horizon + sync_every;
}

int64_t tvbk_ring_smem_bytes(int32_t n, int32_t ncvar, int32_t ring_len) {
    const int64_t b = (int64_t)ring_len * n * ncvar * (int64_t)sizeof(float);
    return b <= kMaxSmemPerBlock ? b : 0;
}

int tvbk_model_dims(int32_t model, int32_t* ncvar, int32_t* nsv, int32_t* nintvar, int32_t* nobs,
                    int32_t* nparam) {
    ModelDims d;
    if (!model_dims(model, &d)) return fail(TVBK_ERR_INVALID, "tvbk_model_dims: unknown model %d", model);
    if (ncvar) *ncvar = d.ncvar;
    if (nsv) *nsv = d.nsv;
    if (nintvar) *nintvar = d.nint;
    if (nobs) *nobs = d.nobs;
    if (nparam) *nparam = d.nparam;
    return TVBK_OK;
}

int tvbk_sim_run(const tvbk_launch* L, void* stream) {
    if (!L) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: null launch");
    ModelDims d;
    if (!model_dims(L->model, &d)) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: unknown model %d", L->model);
    if (!L->insts || !L->status || L->n_inst <= 0)
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: need instances and a status array");
    if (L->n_inst > 2147483647 / 2) return fail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run: too many instances");
    if (L->max_n <= 0 || L->max_n > TVBK_MAX_REGIONS)
        return fail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run: %d regions, this build handles 1..%d", L->max_n,
                    TVBK_MAX_REGIONS);
    if (L->nvoi < 0 || L->nvoi > TVBK_MAX_VOI || L->nvoi > d.nobs)
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: nvoi %d out of 0..%d", L->nvoi,
                    d.nobs < TVBK_MAX_VOI ? d.nobs : TVBK_MAX_VOI);
    for (int v = 0; v < L->nvoi; ++v)
        if (L->voi[v] < 0 || L->voi[v] >= d.nobs)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: voi %d out of range", L->voi[v]);
    if (L->sync_every < 1) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: sync_every must be >= 1");
    if (L->max_degree < 0) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: max_degree < 0");
    if (L->prefetch < 0 || L->prefetch > 2) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: prefetch must be 0, 1 or 2");
    if (L->prefetch == 2 && (!L->ring_in_smem || L->lanes > 1 || L->edges_per_thread != 0 || L->cluster > 1 ||
                             L->cfun == TVBK_CFUN_DIFFERENCE || L->max_degree > 64 || L->model == TVBK_MODEL_SUM))
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: prefetch 2 (separate gather warps) needs rings in shared memory, "
                    "the row gather (lanes 1, no edge split, no cluster), Linear or SigmoidalJansenRit coupling and "
                    "row degrees <= 64");
    if (L->occupancy && (L->lanes > 1 || L->cluster > 1 || L->edges_per_thread != 0 || L->prefetch == 2))
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: occupancy applies to the row kernel (lanes 1, no "
                    "cluster, edges_per_thread 0, prefetch 0 or 1)");
    if (L->inst_order && (L->lanes > 1 || (L->cluster <= 1 && L->edges_per_thread != 0) || L->prefetch == 2))
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: inst_order applies to the row kernel (lanes 1, "
                    "edges_per_thread 0, prefetch 0 or 1) and to the cluster kernel");
    if (L->max_steps < 0) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: max_steps < 0");
    if (!(L->dt > 0.0f)) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: dt must be > 0");
    const bool stoch = L->scheme == TVBK_SCHEME_EULER_STOCH || L->scheme == TVBK_SCHEME_HEUN_STOCH;
    if (stoch && L->noise != TVBK_NOISE_FED && L->noise != TVBK_NOISE_PHILOX)
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: stochastic scheme needs fed or Philox noise");
    if (L->max_steps == 0) return TVBK_OK;
    if (L->cfun < 0 || L->cfun > TVBK_CFUN_KURAMOTO)
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: unknown coupling %d", L->cfun);
    if (L->cfun >= TVBK_CFUN_SIGMOIDAL && (L->prefetch != 0 || L->lanes > 1 || L->edges_per_thread != 0 ||
                                           L->cluster > 1))
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: Sigmoidal, HyperbolicTangent and Kuramoto run on the row kernel "
                    "one step at a time (prefetch 0, lanes 1, edges_per_thread 0, cluster 0)");
    if (L->ring_layout < 0 || L->ring_layout > 1 || (L->ring_layout == 1 && L->cluster <= 1))
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: ring_layout 1 (region-major) applies to clusters only");
    if (L->block_steps != 0 && L->block_steps != 4 && L->block_steps != 8)
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: block_steps %d is not 0, 4 or 8", L->block_steps);
    if (L->block_steps == 8 && (L->ring_layout != 1 || L->sync_every % 8 != 0 || L->extras != 0))
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: block_steps 8 needs ring_layout 1, sync_every a multiple of 8 "
                    "and extras 0");
    if (L->groups < 0 || (L->groups > 0 && (L->ring_layout != 1 || !L->group_sync)))
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: groups > 0 (cooperative launch) needs ring_layout 1 and "
                    "group_sync");
    if (L->groups > 0 && (reinterpret_cast<uintptr_t>(L->group_sync) & 3) != 0)
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: group_sync is not 4-byte aligned");
    if (L->cluster < 0 || L->cluster > (L->groups > 0 ? 256 : 16))
        return fail(TVBK_ERR_INVALID, "tvbk_sim_run: cluster %d out of 0..%d", L->cluster, L->groups > 0 ? 256 : 16);
    if (L->cluster > 1) {
        if (L->lanes > 1 || L->ring_in_smem)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: a cluster per instance reads its rings in place "
                        "(lanes 1, ring_in_smem 0)");
        const int E = L->edges_per_thread;
        if (E != 0 && E != 8 && E != 16 && E != 32)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: a cluster's edge runs have 8, 16 or 32 edges (or 0: a warp "
                        "per row)");
        if (L->ring_layout == 1) {
            if (E == 0 || L->prefetch != 1 || d.ncvar > 2 ||
                (L->cfun != TVBK_CFUN_LINEAR && L->cfun != TVBK_CFUN_DIFFERENCE &&
                 L->cfun != TVBK_CFUN_SIGMOIDAL_JR) ||
                L->sync_every < 4 || L->sync_every % 4 != 0 || L->max_n > 1024)
                return fail(TVBK_ERR_INVALID, "tvbk_sim_run: region-major rings need edge runs, prefetch 1, Linear, "
                            "Difference or SigmoidalJansenRit coupling, ncvar <= 2, sync_every a multiple of 4 and "
                            "at most 1024 regions");
        }
        if (E == 0 && L->prefetch && L->cfun == TVBK_CFUN_DIFFERENCE)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: a cluster with a warp per row cannot prefetch Difference "
                        "coupling (use edge runs)");
        if (L->model == TVBK_MODEL_SUM) return fail(TVBK_ERR_UNSUPPORTED, "tvbk_sim_run: clusters with the Sum model");
        const int64_t R = ((int64_t)L->max_n + L->cluster - 1) / L->cluster;
        if (R > 480)
            return fail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run: %lld rows per cluster CTA, at most 480 (use a larger cluster)",
                        (long long)R);
        if (L->cluster_edges < 0) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: cluster_edges < 0");
        const int64_t nacc = L->cfun == TVBK_CFUN_SIGMOIDAL_JR ? 1 : d.ncvar;
        // edge runs: row pointers, double-buffered partials of all 512 threads, the edges
        // blocked runs keep the partials of a block of steps
        const int64_t nbuf = L->ring_layout == 1 ? (L->block_steps == 8 ? 8 : 4) : 1;
        const int64_t b = E ? ((R + 1) * 4 + 15) / 16 * 16 + (2 * nbuf * 512 * 2 * nacc * 4 + 15) / 16 * 16 +
                                  ((int64_t)L->cluster_edges + E) * 8
                            : ((R + 1) * 4 + 15) / 16 * 16 + (2 * R * nacc * 4 + 15) / 16 * 16 +
                                  (int64_t)L->cluster_edges * 8;
        if (E && L->cluster_edges <= 0)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: edge runs need the CTAs' edges in shared memory "
                        "(cluster_edges > 0)");
        if (b > kMaxSmemPerBlock)
            return fail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run: cluster CTA needs %lld bytes of shared memory",
                        (long long)b);
    }
    size_t smem = 0;
    if (L->lanes > 1) {
        if (L->lanes * d.ncvar != 8)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: instance groups have 8 / ncvar = %d lanes", 8 / d.ncvar);
        if (L->n_inst % L->lanes != 0)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: %d instances are not groups of %d", L->n_inst, L->lanes);
        if (L->edges_per_thread != 0 || L->ring_in_smem)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: instance groups read their rings in place and use the "
                        "row gather");
        if (L->model == TVBK_MODEL_SUM) return fail(TVBK_ERR_UNSUPPORTED, "tvbk_sim_run: groups with the Sum model");
        const int64_t threads = ((int64_t)L->max_n * L->lanes + 31) / 32 * 32;
        const int64_t b = ((int64_t)L->max_n * L->max_degree * 8 + 15) / 16 * 16 +
                          (int64_t)2 * L->max_degree * d.ncvar * threads * 4;
        if (threads > 1024 || b > kMaxSmemPerBlock)
            return fail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run: a group of %d lanes x %d regions needs %lld threads and "
                        "%lld bytes of shared memory", L->lanes, L->max_n, (long long)threads, (long long)b);
    } else if (L->cluster <= 1 && L->edges_per_thread != 0) {
        const int E = L->edges_per_thread;
        if (E != 8 && E != 12 && E != 16 && E != 24)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: edges_per_thread must be 0, 8, 12, 16 or 24");
        if (L->cfun == TVBK_CFUN_DIFFERENCE)
            return fail(TVBK_ERR_UNSUPPORTED, "tvbk_sim_run: the edge-parallel gather needs Linear or "
                        "SigmoidalJansenRit coupling");
        if (!L->ring_in_smem) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: the edge-parallel gather needs rings "
                                          "in shared memory");
        if (L->block_threads < L->max_n || L->block_threads > 512 || L->block_threads % 32 != 0)
            return fail(TVBK_ERR_INVALID, "tvbk_sim_run: block_threads %d must be a multiple of 32 in [max_n, 512]",
                        L->block_threads);
        if (L->max_ring_len <= 0) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: max_ring_len <= 0");
        const int64_t ring = ((int64_t)L->max_ring_len * L->max_n * d.ncvar + 3) / 4 * 4;
        const int nacc = L->cfun == TVBK_CFUN_SIGMOIDAL_JR ? 1 : d.ncvar;
        const int64_t b = (ring + (int64_t)2 * L->block_threads * 2 * nacc) * (int64_t)sizeof(float);
        if (b > kMaxSmemPerBlock)
            return fail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run: ring and partials need %lld bytes of shared memory",
                        (long long)b);
        smem = (size_t)b;
    } else if (L->ring_in_smem) {
        if (L->max_ring_len <= 0) return fail(TVBK_ERR_INVALID, "tvbk_sim_run: max_ring_len <= 0");
        // the row kernel stages one pre-applied sigmoid value per (slot, region) for SigmoidalJansenRit
        const int64_t ncv_g = L->cfun == TVBK_CFUN_SIGMOIDAL_JR ? 1 : d.ncvar;
        // with prefetch 1 the row kernel keeps TVBK_RING_GUARD mirrored slots past the ring's end
        const bool guard = L->prefetch == 1 && L->lanes <= 1;
        const int64_t slots = (int64_t)L->max_ring_len + (guard ? TVBK_RING_GUARD : 0);
        int64_t b = slots * L->max_n * ncv_g * (int64_t)sizeof(float);
        // separate gather warps pass the sums through a double buffer after the ring
        if (L->prefetch == 2) b = (b + 15) / 16 * 16 + (int64_t)2 * L->max_n * d.ncvar * (int64_t)sizeof(float);
        if (b > kMaxSmemPerBlock || L->max_n > 256)
            return fail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run: ring of %lld bytes / %d regions cannot be staged in "
                        "shared memory", (long long)b, L->max_n);
        smem = (size_t)b;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (L->groups > 0) {
        // the queue head, the abort flag and every group's barrier counter start from zero
        const cudaError_t e = cudaMemsetAsync(L->group_sync, 0, sizeof(uint32_t) * TVBK_GROUP_SYNC_WORDS(L->groups), st);
        if (e != cudaSuccess) return cuda_fail(e, "tvbk_sim_run group_sync");
    }
    int rc;
    switch (L->model) {
        case TVBK_MODEL_G2D: rc = tvbk::launch_g2d(*L, st, smem); break;
        case TVBK_MODEL_JANSEN_RIT: rc = tvbk::launch_jr(*L, st, smem); break;
        case TVBK_MODEL_RWW: rc = tvbk::launch_rww(*L, st, smem); break;
        case TVBK_MODEL_EPILEPTOR: rc = tvbk::launch_epileptor(*L, st, smem); break;
        default: rc = tvbk::launch_sum(*L, st, smem); break;
    }
    if (rc == -1) return fail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run: instance too large for this kernel variant");
    if (rc == -4)
        return fail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run: %d groups x %d CTAs are more than the GPU holds at once",
                    L->groups, L->cluster);
    if (rc == -2)
        return fail(TVBK_ERR_UNSUPPORTED, "tvbk_sim_run: model %d / coupling %d / scheme %d not built", L->model,
                    L->cfun, L->scheme);
    if (rc != 0) return cuda_fail((cudaError_t)rc, "tvbk_sim_run launch");
    return TVBK_OK;
}

int tvbk_gather_delayed(const tvbk_inst* I, int32_t ncvar, int64_t step, float* out_dev, void* stream) {
    if (!I || !out_dev || !I->ring || !I->edges || ncvar < 1 || ncvar > 2)
        return fail(TVBK_ERR_INVALID, "tvbk_gather_delayed: bad arguments");
    if (I->nnz <= 0) return TVBK_OK;
    const int ring_floats = I->ring_len * I->n * ncvar;
    int64_t slot = (step - 1) % I->ring_len;
    if (slot < 0) slot += I->ring_len;
    const int base_off = (int)slot * I->n * ncvar;
    const int threads = 256, blocks = (I->nnz + threads - 1) / threads;
    gather_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(I->edges, I->ring, I->nnz, ncvar, base_off,
                                                                 ring_floats, out_dev);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TVBK_OK : cuda_fail(e, "tvbk_gather_delayed");
}

int tvbk_fc(const double* x, int32_t n_inst, int32_t T, int32_t n, double* fc, void* stream) {
    if (!x || !fc || n_inst <= 0 || T < 2 || n < 1) return fail(TVBK_ERR_INVALID, "tvbk_fc: bad arguments");
    if (tvbk::fc_smem_bytes(T, n) == 0)
        return fail(TVBK_ERR_TOO_LARGE, "tvbk_fc: series of %d x %d does not fit the shared-memory kernel", T, n);
    const int rc = tvbk::fc_launch(x, n_inst, T, n, fc, (cudaStream_t)stream);
    return rc == 0 ? TVBK_OK : cuda_fail((cudaError_t)rc, "tvbk_fc");
}

}  // extern "C"
