// reduce_static.cu — the global reductions without any device allocation.
//
// ssmd_reduce keeps its per-block partial sums in the caller's workspace
// buffer.  Some callers cannot provide one: a monitoring or post-processing
// plugin that is handed the simulation's LBMFields by the host application
// but owns no device memory of its own, or code running where cudaMalloc is
// off limits (it synchronises the whole device).  ssmd_reduce_static serves
// them: the same two reduction kernels, with the partial sums and the result
// in a fixed array that lives in this library's own device image.
//
// Limits and sharing rules:
//   * the array holds kStaticPartials = 512 partial sums of kRedVals doubles
//     plus one result row (41 KiB per GPU that loads the library, held until
//     the process exits).  The first pass launches at most 512 blocks that
//     stride over the cells, so 512 partials cover every lattice that
//     ssmd_validate accepts (nx*ny*nz <= 2^32 - 1); larger lattices are
//     refused by ssmd_validate before anything reaches the device.
//   * every call on a device uses the same array and leaves its contents
//     behind.  Pass 1 overwrites every partial that pass 2 reads and pass 2
//     overwrites the result row, so nothing has to start at zero.  Calls that
//     overlap on the GPU (different streams or threads at the same time) race
//     on the array and corrupt each other's results: serialise them.
//   * the call copies its result to the host and synchronises its stream, so
//     it cannot run inside a stream capture: a capturing stream is refused
//     with SSMD_ERR_INVALID_ARGUMENT, and it must not be called on the legacy
//     default stream while another stream of the device is being captured.
//   * the device address of the array is looked up with cudaGetSymbolAddress
//     on the first call in each CUDA context of a device (the device that is
//     current) and kept for later calls in the same context.  A device reset
//     or a released and re-created primary context gives a new context, in
//     which the next call looks the address up again.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "host.cuh"

using namespace ssmd;
using namespace ssmd::host;

namespace {

constexpr int kStaticPartials = 512;
constexpr int kMaxDevices = 64;
// ceil(cells / kRedThreads) blocks, clamped to kStaticPartials: pass 1 strides
// over the cells, so the clamp only lengthens each block's loop
static_assert(kStaticPartials <= kMaxRedBlocks, "pass 2 sums at most kMaxRedBlocks partial rows");

// [0, kRedVals * kStaticPartials): partials; last kRedVals doubles: result.
static __device__ __align__(256) double g_reduce_scratch[kRedVals * (kStaticPartials + 1)];

// Unique ID of the calling thread's current CUDA context (0 when none is
// current yet or the driver entry points are unavailable).
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(p);
    });
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

struct ScratchCache {
    unsigned long long ctx_id = 0; // context the address belongs to (0: none cached)
    double *ptr = nullptr;
};

std::mutex g_setup_mutex;
ScratchCache g_scratch[kMaxDevices];

// Device address of g_reduce_scratch in the current device's current context.
int scratch_address(double **out) {
    int dev = 0;
    if (int e = cuda_check(cudaGetDevice(&dev), "cudaGetDevice")) return e;
    if (dev < 0 || dev >= kMaxDevices)
        return fail(SSMD_ERR_UNSUPPORTED, "device index %d above %d", dev, kMaxDevices - 1);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    ScratchCache &c = g_scratch[dev];
    const unsigned long long id = current_context_id();
    if (id != 0 && c.ctx_id == id && c.ptr) {
        *out = c.ptr;
        return SSMD_OK;
    }
    // set-up for this device and context: the runtime makes the device's
    // primary context current here if nothing was current yet
    void *ptr = nullptr;
    if (int e = cuda_check(cudaGetSymbolAddress(&ptr, g_reduce_scratch),
                           "cudaGetSymbolAddress(reduction scratch)"))
        return e;
    c.ptr = static_cast<double *>(ptr);
    c.ctx_id = id != 0 ? id : current_context_id(); // 0 again: no cache, look up on every call
    *out = c.ptr;
    return SSMD_OK;
}

template <class T>
int reduce_static(const ssmd_params &p, const LBMFields &fl, uint64_t steps_done, double *out_host,
                  cudaStream_t st) {
    const Geometry G = make_geometry(p);
    const phase_t<T> *g = static_cast<const phase_t<T> *>((steps_done & 1ull) == 0ull ? fl.g : p.g_alt);
    const uint64_t want = (G.cells + kRedThreads - 1) / kRedThreads;
    const int nb = (int)(want < (uint64_t)kStaticPartials ? want : kStaticPartials);
    double *scratch = nullptr;
    if (int e = scratch_address(&scratch)) return e;
    double *partials = scratch;
    double *result = scratch + (size_t)kRedVals * kStaticPartials;
    reduce_pass1<phase_t<T>><<<nb, kRedThreads, 0, st>>>(G, make_fields(fl), g, partials);
    reduce_pass2<<<1, kRedThreads, 0, st>>>(partials, nb, result);
    if (int e = cuda_check(cudaGetLastError(), "static reduce launch")) return e;
    if (int e = cuda_check(cudaMemcpyAsync(out_host, result, sizeof(double) * kRedVals,
                                           cudaMemcpyDeviceToHost, st),
                           "static reduce copy"))
        return e;
    return cuda_check(cudaStreamSynchronize(st), "static reduce sync");
}

} // namespace

extern "C" int ssmd_reduce_static(const ssmd_params *p, const LBMFields *fields, uint64_t steps_done,
                                  ssmd_stats *out, ssmd_stream_t stream) {
    if (!out || !fields) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    if (int e = ssmd_validate(p)) return e;
    const void *need[] = {fields->rho, fields->ux, fields->uy, fields->uz, fields->phi, fields->g, p->g_alt};
    for (const void *q : need)
        if (!q) return fail(SSMD_ERR_INVALID_ARGUMENT, "a field, g or g_alt pointer is null");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (int e = cuda_check(cudaStreamIsCapturing(st, &cap), "cudaStreamIsCapturing")) return e;
    if (cap != cudaStreamCaptureStatusNone)
        return fail(SSMD_ERR_INVALID_ARGUMENT,
                    "ssmd_reduce_static synchronises its stream and cannot be captured: call it on a stream "
                    "that is not being captured");
    double v[kRedVals];
    int e;
    switch (p->storage) {
    case SSMD_STORAGE_F32: e = reduce_static<float>(*p, *fields, steps_done, v, st); break;
    case SSMD_STORAGE_F16: e = reduce_static<__half>(*p, *fields, steps_done, v, st); break;
    case SSMD_STORAGE_F16_G32: e = reduce_static<half_g32>(*p, *fields, steps_done, v, st); break;
    default: e = reduce_static<__nv_bfloat16>(*p, *fields, steps_done, v, st); break;
    }
    if (e) return e;
    out->phi_sum = v[0];
    out->phi_sum_next = v[1];
    out->mass = v[2];
    out->momentum[0] = v[3];
    out->momentum[1] = v[4];
    out->momentum[2] = v[5];
    out->kinetic = v[6];
    out->u_max = v[7];
    out->nonfinite = v[8];
    out->cells = v[9];
    if (v[8] > 0.0 || v[7] > (double)p->u_limit)
        return fail(SSMD_ERR_UNSTABLE, "unstable state: %g non-finite cells, max |u| = %g (limit %g)",
                    v[8], v[7], (double)p->u_limit);
    return SSMD_OK;
}
