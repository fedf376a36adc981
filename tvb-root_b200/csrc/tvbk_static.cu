// tvbk_sim_run_static: one simulation instance with all of its working
// memory in a fixed array inside the library, for callers that cannot
// allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc at the point where they
// want to run a simulation: plug-in and FFI callers whose process owns no
// allocator of its own (the device memory belongs to another runtime that
// hands out only the input and output buffers), code paths that run under a
// fixed memory budget, and callers that must not allocate while other work
// is being recorded.  tvbk_sim_run needs caller-allocated scratch besides the
// inputs and outputs (the working copy of the delayed-history ring, the
// TemporalAverage, Bold, AfferentCoupling and projection-stream accumulators,
// the Bold 4 ms stock, the instance descriptor and its status word).  This
// variant keeps all of that in g_static_scratch below,
// TVBK_STATIC_SCRATCH_BYTES bytes per device, and allocates nothing: it calls
// no cudaMalloc, cudaFree or allocating library routine.  Every accumulator
// starts each call from zero; the caller's *_acc pointers are not read.
//
// The array exists on every GPU that loads the library and stays allocated
// until the process exits.  Its device address is looked up once per device
// (cudaGetSymbolAddress, with that device current) by the first call made on
// that device, so that first call should come before any stream capture.
// The looked-up address belongs to the device's context of that moment: after
// a cudaDeviceReset of the device (which this library never calls) it is
// stale, and the process must not call this entry point on that device again.
// All calls on a device share the one array and it keeps the contents of the
// last call: each call re-initialises what must start from zero or from the
// caller's inputs, and calls whose work overlaps on the GPU (concurrent
// streams, or several host threads on one device) race on it -- serialise
// them.
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>

#include "tvbk.h"
#include "tvbk_models.cuh"

namespace tvbk {
int launch_g2d(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_jr(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_rww(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_epileptor(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_sum(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int set_error(int code, const char* msg);
}  // namespace tvbk

namespace {

static __device__ __align__(256) unsigned char g_static_scratch[TVBK_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Failures are reported through tvbk_last_error() like every other entry point.
int sfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return tvbk::set_error(code, buf);
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Copies the caller's initial ring into the scratch ring, zeroes the
// accumulators and the status word, and writes the instance descriptor.
__global__ void static_setup(tvbk_inst d, tvbk_inst* desc, int32_t* status, const float* __restrict__ ring_src,
                             int64_t ring_floats, int64_t zero_bytes, unsigned char* zero_base) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = tid; k < ring_floats; k += stride) d.ring[k] = ring_src[k];
    for (int64_t k = tid; k < zero_bytes; k += stride) zero_base[k] = 0;
    if (tid == 0) {
        *desc = d;
        *status = 0;
    }
}

}  // namespace

extern "C" int tvbk_sim_run_static(const tvbk_launch* L, const tvbk_inst* inst, int32_t* status_out, void* stream) {
    if (!L || !inst) return sfail(TVBK_ERR_INVALID, "tvbk_sim_run_static: null launch or instance");
    int32_t ncvar, nsv, nint, nobs, nparam;
    if (tvbk_model_dims(L->model, &ncvar, &nsv, &nint, &nobs, &nparam) != TVBK_OK)
        return sfail(TVBK_ERR_INVALID, "tvbk_sim_run_static: unknown model %d", L->model);
    if (!inst->ring || !inst->state || !inst->row_ptr || !inst->params || inst->n <= 0 || inst->ring_len <= 0)
        return sfail(TVBK_ERR_INVALID, "tvbk_sim_run_static: instance needs ring, state, row_ptr, params, n, ring_len");
    if (inst->n > TVBK_MAX_REGIONS)
        return sfail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run_static: %d regions, at most %d", inst->n, TVBK_MAX_REGIONS);
    if (inst->ring_len < inst->horizon + L->sync_every)
        return sfail(TVBK_ERR_INVALID, "tvbk_sim_run_static: ring_len %d < horizon + sync_every", inst->ring_len);
    if (inst->step_end < inst->step) return sfail(TVBK_ERR_INVALID, "tvbk_sim_run_static: step_end < step");
    if (L->ring_layout != 0)
        return sfail(TVBK_ERR_UNSUPPORTED, "tvbk_sim_run_static: time-major rings only (ring_layout 0)");

    // scratch layout: descriptor | status | tavg_acc | bold_acc | bold_stock | aff_acc | proj_acc | ring | pre_ring
    const int64_t n = inst->n, nvoi = L->nvoi;
    const bool tavg = inst->tavg != nullptr, bold = inst->bold != nullptr;
    const bool aff = inst->aff != nullptr, proj = inst->proj != nullptr;
    if (bold && (!inst->hrf || inst->stock_len <= 0))
        return sfail(TVBK_ERR_INVALID, "tvbk_sim_run_static: Bold needs hrf and stock_len");
    size_t off = 0;
    const size_t o_desc = off;
    off = align256(off + sizeof(tvbk_inst));
    const size_t o_status = off;
    off = align256(off + sizeof(int32_t));
    const size_t o_zero = off;
    const size_t o_tacc = off;
    off = align256(off + (tavg ? nvoi * n * sizeof(float) : 0));
    const size_t o_bacc = off;
    off = align256(off + (bold ? nvoi * n * sizeof(double) : 0));
    const size_t o_stock = off;
    off = align256(off + (bold ? (size_t)inst->stock_len * nvoi * n * sizeof(double) : 0));
    // the AfferentCoupling and projection-stream period sums: both start every call from zero
    const size_t o_aff = off;
    off = align256(off + (aff ? (size_t)ncvar * n * sizeof(float) : 0));
    const size_t o_proj = off;
    off = align256(off + (proj ? (size_t)nvoi * n * sizeof(float) : 0));
    const size_t zero_bytes = off - o_zero;
    const size_t o_ring = off;
    const int64_t ring_floats = (int64_t)inst->ring_len * n * ncvar;
    off = align256(off + (size_t)ring_floats * sizeof(float));
    // SigmoidalJansenRit: the kernel's ring of pre-applied sigmoid values (filled by the kernel itself)
    const bool pre = L->cfun == TVBK_CFUN_SIGMOIDAL_JR;
    const size_t o_pre = off;
    off = align256(off + (pre ? (size_t)inst->ring_len * n * sizeof(float) : 0));
    if (off > (size_t)TVBK_STATIC_SCRATCH_BYTES)
        return sfail(TVBK_ERR_TOO_LARGE,
                     "tvbk_sim_run_static: needs %zu bytes of scratch (ring %lld floats%s), the library holds %d",
                     off, (long long)ring_floats, bold ? " + Bold stock" : "", (int)TVBK_STATIC_SCRATCH_BYTES);

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return sfail(TVBK_ERR_CUDA, "tvbk_sim_run_static: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return sfail(TVBK_ERR_TOO_LARGE, "tvbk_sim_run_static: device %d", dev);
    unsigned char* base;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_static_scratch);
            if (e != cudaSuccess || !p)
                return sfail(TVBK_ERR_CUDA, "tvbk_sim_run_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            g_scratch_addr[dev] = p;
        }
        base = static_cast<unsigned char*>(g_scratch_addr[dev]);
    }

    tvbk_inst d = *inst;
    d.ring = reinterpret_cast<float*>(base + o_ring);
    d.pre_ring = pre ? reinterpret_cast<float*>(base + o_pre) : nullptr;
    d.tavg_acc = tavg ? reinterpret_cast<float*>(base + o_tacc) : nullptr;
    d.bold_acc = bold ? reinterpret_cast<double*>(base + o_bacc) : nullptr;
    d.bold_stock = bold ? reinterpret_cast<double*>(base + o_stock) : nullptr;
    d.aff_acc = aff ? reinterpret_cast<float*>(base + o_aff) : nullptr;
    d.proj_acc = proj ? reinterpret_cast<float*>(base + o_proj) : nullptr;
    tvbk_inst* desc = reinterpret_cast<tvbk_inst*>(base + o_desc);
    int32_t* status = reinterpret_cast<int32_t*>(base + o_status);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t work = ring_floats > (int64_t)zero_bytes ? ring_floats : (int64_t)zero_bytes;
    int blocks = (int)((work + 255) / 256);
    blocks = blocks < 1 ? 1 : (blocks > 1024 ? 1024 : blocks);
    static_setup<<<blocks, 256, 0, st>>>(d, desc, status, inst->ring, ring_floats, (int64_t)zero_bytes,
                                         base + o_zero);
    e = cudaGetLastError();
    if (e != cudaSuccess) return sfail(TVBK_ERR_CUDA, "tvbk_sim_run_static setup: %s", cudaGetErrorString(e));

    tvbk_launch L2 = *L;
    L2.insts = desc;
    L2.status = status;
    L2.n_inst = 1;
    L2.lanes = 1;
    L2.max_n = inst->n;
    L2.max_ring_len = inst->ring_len;
    L2.max_steps = inst->step_end - inst->step;
    L2.inst_order = nullptr;  // one instance, the staged descriptor
    L2.occupancy = nullptr;   // always a launch
    const int rc = tvbk_sim_run(&L2, stream);
    if (rc != TVBK_OK) return rc;  // tvbk_sim_run has set the message
    if (status_out) {
        e = cudaMemcpyAsync(status_out, status, sizeof(int32_t), cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return sfail(TVBK_ERR_CUDA, "tvbk_sim_run_static status: %s", cudaGetErrorString(e));
    }
    return TVBK_OK;
}
