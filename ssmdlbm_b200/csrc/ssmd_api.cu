// ssmd_api.cu — the C ABI declared in include/ssmd.h.
//
// Replaces the reference's host-side launch sequence (src/main.cu:105-186,
// src/cuda/CUDAGraph.cuh:34-57) with: one fused bulk kernel, then the
// boundary kernels of the active face kinds, all on the caller's stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/ssmd.h"
#include "host.cuh"

using namespace ssmd;

namespace ssmd {
namespace host {

thread_local std::string g_error;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

int cuda_check(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return SSMD_OK;
    return fail(SSMD_ERR_CUDA, "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
}

struct Profile {
    std::vector<cudaEvent_t> ev; // 2 per launch
    int used = 0;                // launches recorded
};
thread_local Profile g_prof;

void profile_next(cudaEvent_t *before, cudaEvent_t *after) {
    *before = *after = nullptr;
    Profile &P = g_prof;
    if (2 * (P.used + 1) > (int)P.ev.size()) return;
    *before = P.ev[2 * P.used];
    *after = P.ev[2 * P.used + 1];
    ++P.used;
}

void profile_free() {
    for (cudaEvent_t e : g_prof.ev) cudaEventDestroy(e);
    g_prof.ev.clear();
    g_prof.used = 0;
}

SSMD_DECLARE(19, float)
SSMD_DECLARE(19, __half)
SSMD_DECLARE(19, __nv_bfloat16)
SSMD_DECLARE(19, half_g32)
SSMD_DECLARE(27, float)
SSMD_DECLARE(27, __half)
SSMD_DECLARE(27, __nv_bfloat16)
SSMD_DECLARE(27, half_g32)

} // namespace host
} // namespace ssmd

using namespace ssmd::host;


namespace {

template <class T>
int launch_reduce(const ssmd_params &p, const LBMFields &fl, uint64_t steps_done, double *out_host,
                  cudaStream_t st) {
    const Geometry G = make_geometry(p);
    const phase_t<T> *g = static_cast<const phase_t<T> *>((steps_done & 1ull) == 0ull ? fl.g : p.g_alt);
    uint64_t nb64 = (G.cells + kRedThreads - 1) / kRedThreads;
    const int nb = (int)(nb64 < (uint64_t)kMaxRedBlocks ? nb64 : kMaxRedBlocks);
    char *ws = static_cast<char *>(p.workspace);
    double *partials = reinterpret_cast<double *>(ws + kPartialOff);
    double *out = reinterpret_cast<double *>(ws + kRedOutOff);
    reduce_pass1<phase_t<T>><<<nb, kRedThreads, 0, st>>>(G, make_fields(fl), g, partials);
    reduce_pass2<<<1, kRedThreads, 0, st>>>(partials, nb, out);
    if (int e = cuda_check(cudaGetLastError(), "reduce launch")) return e;
    if (int e = cuda_check(cudaMemcpyAsync(out_host, out, sizeof(double) * kRedVals,
                                           cudaMemcpyDeviceToHost, st),
                           "reduce copy"))
        return e;
    return cuda_check(cudaStreamSynchronize(st), "reduce sync");
}

template <class T, int NQ>
int launch_to_push(const ssmd_params &p, const void *src, void *dst, cudaStream_t st) {
    const Geometry G = make_geometry(p);
    const unsigned nb = (unsigned)((G.cells + 255) / 256);
    pull_to_push_kernel<T, NQ><<<nb, 256, 0, st>>>(G, static_cast<const T *>(src), static_cast<T *>(dst));
    return cuda_check(cudaGetLastError(), "pull_to_push launch");
}

bool finite_pos(float v) { return std::isfinite(v) && v > 0.0f; }

} // namespace

extern "C" {

int ssmd_abi_version(void) { return SSMD_ABI_VERSION; }

const char *ssmd_last_error(void) { return g_error.c_str(); }

size_t ssmd_scalar_bytes(const ssmd_params *p) {
    return p ? (size_t)p->nx * p->ny * p->nz * sizeof(float) : 0;
}
size_t ssmd_f_bytes(const ssmd_params *p) {
    return p ? (size_t)p->nx * p->ny * p->nz * (size_t)p->velocity_set * f_storage_size(p->storage) : 0;
}
size_t ssmd_g_bytes(const ssmd_params *p) {
    return p ? (size_t)p->nx * p->ny * p->nz * 7u * g_storage_size(p->storage) : 0;
}
size_t ssmd_workspace_bytes(const ssmd_params *p) {
    (void)p;
    return kWorkspaceBytes;
}

int ssmd_validate(const ssmd_params *p) {
    if (!p) return fail(SSMD_ERR_INVALID_ARGUMENT, "params is null");
    if (p->velocity_set != 19 && p->velocity_set != 27)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "velocity_set must be 19 or 27 (got %d)",
                    p->velocity_set);
    if (p->storage < SSMD_STORAGE_F32 || p->storage > SSMD_STORAGE_F16_G32)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "unknown storage %d", p->storage);
    if (p->bc_x != SSMD_BC_PERIODIC_COPY && p->bc_x != SSMD_BC_PERIODIC)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "bc_x must be PERIODIC_COPY or PERIODIC");
    if (p->bc_y < SSMD_BC_PERIODIC_COPY || p->bc_y > SSMD_BC_JET)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "bc_y must be PERIODIC_COPY, PERIODIC or JET");
    if (p->bc_z != SSMD_BC_JET && p->bc_z != SSMD_BC_PERIODIC)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "bc_z must be JET or PERIODIC");
    const uint32_t n[3] = {p->nx, p->ny, p->nz};
    const int bc[3] = {p->bc_x, p->bc_y, p->bc_z};
    for (int d = 0; d < 3; ++d) {
        const uint32_t need = bc[d] == SSMD_BC_PERIODIC ? 3u : 6u;
        if (n[d] < need || n[d] > 65535u)
            return fail(SSMD_ERR_INVALID_ARGUMENT, "axis %d: size %u outside [%u, 65535]", d, n[d],
                        need);
    }
    const uint64_t cells = (uint64_t)p->nx * p->ny * p->nz;
    if (cells > 0xFFFFFFFFull)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "nx*ny*nz = %llu exceeds 2^32 - 1 cells",
                    (unsigned long long)cells);
    if (!finite_pos(p->nu_water) || !finite_pos(p->nu_oil))
        return fail(SSMD_ERR_INVALID_ARGUMENT,
                    "viscosities must be finite and > 0 (tau > 1/2): nu_water=%g nu_oil=%g",
                    p->nu_water, p->nu_oil);
    if (!(p->omega_g > 0.0f && p->omega_g < 2.0f))
        return fail(SSMD_ERR_INVALID_ARGUMENT, "omega_g must be in (0, 2) (got %g)", p->omega_g);
    const float fl[] = {p->omco_water, p->omco_oil, p->omco_ref, p->sigma, p->gamma,
                        p->u_oil, p->oil_cx, p->oil_cy, p->oil_r2, p->u_water,
                        p->water_cx, p->water_cz, p->water_r2, p->noise_amp, p->u_limit};
    for (float v : fl)
        if (!std::isfinite(v)) return fail(SSMD_ERR_INVALID_ARGUMENT, "non-finite parameter");
    if (p->tile_z < 0) return fail(SSMD_ERR_INVALID_ARGUMENT, "tile_z must be >= 0");
    if (p->bulk_path < SSMD_PATH_AUTO || p->bulk_path > SSMD_PATH_SLAB)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "unknown bulk_path %d", p->bulk_path);
    return SSMD_OK;
}

int ssmd_params_reference(ssmd_params *p, uint32_t nx, uint32_t ny, uint32_t nz,
                          int32_t velocity_set, float u_water, float u_oil, int32_t diam_water,
                          int32_t diam_oil, int32_t radius_water, int32_t radius_oil,
                          double reynolds_water, double reynolds_oil, double weber,
                          float interface_width) {
    if (!p) return fail(SSMD_ERR_INVALID_ARGUMENT, "params is null");
    *p = ssmd_params{};
    p->nx = nx;
    p->ny = ny;
    p->nz = nz;
    p->velocity_set = velocity_set;
    p->storage = SSMD_STORAGE_F32;
    p->bc_x = SSMD_BC_PERIODIC_COPY;
    p->bc_y = SSMD_BC_JET;
    p->bc_z = SSMD_BC_JET;
    // globalFunctions.cuh:234-242 (FP64 product and quotient, then FP32)
    p->nu_water = (float)(((double)u_water * (double)diam_water) / reynolds_water);
    p->nu_oil = (float)(((double)u_oil * (double)diam_oil) / reynolds_oil);
    // :244-247, :269-282
    const float om_w = (float)(1.0 / (0.5 + 3.0 * (double)p->nu_water));
    const float om_o = (float)(1.0 / (0.5 + 3.0 * (double)p->nu_oil));
    p->omco_water = 1.0f - om_w;
    p->omco_oil = 1.0f - om_o;
    p->omco_ref = p->omco_water;
    // constants.cuh:93 (FP32 constexpr)
    p->sigma = (u_oil * u_oil * (float)diam_oil) / (float)weber;
    // constants.cuh:97-100 with tau_g = 1 and the D3Q7 cs2 = 1/4
    const float cs2 = (float)(1.0 / 4.0);
    const float diff_int = cs2 * (1.0f - 0.5f);
    const float kappa = 4.0f * diff_int / interface_width;
    p->gamma = kappa / cs2;
    p->omega_g = 1.0f;
    // globalFunctions.cuh:70-103
    const int rw = radius_water >= 0 ? radius_water : diam_water / 2;
    const int ro = radius_oil >= 0 ? radius_oil : diam_oil / 2;
    p->water_r2 = (float)(rw * rw);
    p->oil_r2 = (float)(ro * ro);
    const float center_x = (float)(nx - 1) * 0.5f;
    const float center_y = (float)(ny - 1) * 0.5f;
    const float center_z = (float)(nz - 1) * 0.5f;
    p->oil_cx = center_x;
    p->oil_cy = 0.5f * center_y;
    p->water_cx = center_x;
    p->water_cz = 0.7f * center_z;
    p->u_oil = u_oil;
    p->u_water = u_water;
    p->noise_amp = 0.0f;
    p->u_limit = 0.3f;
    p->seed = 0;
    return SSMD_OK;
}

int ssmd_init(const ssmd_params *p, LBMFields *fields, ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (int e = check_fields(*p, fields)) return e;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const Geometry G = make_geometry(*p);
    const unsigned nb = (unsigned)((G.cells + 255) / 256);
    init_macros_kernel<<<nb, 256, 0, st>>>(G, make_physics(*p), make_fields(*fields), fields->fsx,
                                           fields->fsy, fields->fsz);
    if (int e = cuda_check(cudaGetLastError(), "init_macros launch")) return e;
    return ssmd_init_from_macros(p, fields, stream);
}

int ssmd_init_from_macros(const ssmd_params *p, LBMFields *fields, ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (int e = check_fields(*p, fields)) return e;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int e = SSMD_OK;
    switch (p->velocity_set * 4 + p->storage) {
    case 19 * 4 + SSMD_STORAGE_F32: e = launch_init_pops<19, float>(*p, *fields, st); break;
    case 19 * 4 + SSMD_STORAGE_F16: e = launch_init_pops<19, __half>(*p, *fields, st); break;
    case 19 * 4 + SSMD_STORAGE_BF16: e = launch_init_pops<19, __nv_bfloat16>(*p, *fields, st); break;
    case 27 * 4 + SSMD_STORAGE_F32: e = launch_init_pops<27, float>(*p, *fields, st); break;
    case 27 * 4 + SSMD_STORAGE_F16: e = launch_init_pops<27, __half>(*p, *fields, st); break;
    case 27 * 4 + SSMD_STORAGE_BF16: e = launch_init_pops<27, __nv_bfloat16>(*p, *fields, st); break;
    case 19 * 4 + SSMD_STORAGE_F16_G32: e = launch_init_pops<19, half_g32>(*p, *fields, st); break;
    case 27 * 4 + SSMD_STORAGE_F16_G32: e = launch_init_pops<27, half_g32>(*p, *fields, st); break;
    default: return fail(SSMD_ERR_UNSUPPORTED, "unsupported velocity set / storage");
    }
    if (e) return e;
    set_status_kernel<<<1, 1, 0, st>>>(status_of(*p), ~0ull);
    return cuda_check(cudaGetLastError(), "status reset");
}

int ssmd_step(LBMFields *fields, const ssmd_params *p, uint64_t step, uint32_t flags,
              ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (int e = check_fields(*p, fields)) return e;
    if (flags & ~(SSMD_STEP_STORE_MACROS | SSMD_STEP_AVERAGE))
        return fail(SSMD_ERR_INVALID_ARGUMENT, "unknown step flags 0x%x", flags);
    if ((flags & SSMD_STEP_AVERAGE) && !p->derived)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "SSMD_STEP_AVERAGE needs params.derived");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    switch (p->velocity_set * 4 + p->storage) {
    case 19 * 4 + SSMD_STORAGE_F32: return launch_step<19, float>(*p, *fields, step, flags, st);
    case 19 * 4 + SSMD_STORAGE_F16: return launch_step<19, __half>(*p, *fields, step, flags, st);
    case 19 * 4 + SSMD_STORAGE_BF16:
        return launch_step<19, __nv_bfloat16>(*p, *fields, step, flags, st);
    case 27 * 4 + SSMD_STORAGE_F32: return launch_step<27, float>(*p, *fields, step, flags, st);
    case 27 * 4 + SSMD_STORAGE_F16: return launch_step<27, __half>(*p, *fields, step, flags, st);
    case 27 * 4 + SSMD_STORAGE_BF16:
        return launch_step<27, __nv_bfloat16>(*p, *fields, step, flags, st);
    case 19 * 4 + SSMD_STORAGE_F16_G32: return launch_step<19, half_g32>(*p, *fields, step, flags, st);
    case 27 * 4 + SSMD_STORAGE_F16_G32: return launch_step<27, half_g32>(*p, *fields, step, flags, st);
    default: return fail(SSMD_ERR_UNSUPPORTED, "unsupported velocity set / storage");
    }
}

int ssmd_capture_graph(const ssmd_params *p, LBMFields *fields, uint64_t first_step, int32_t steps,
                       uint32_t flags, ssmd_stream_t stream, ssmd_graph_exec_t *out) {
    if (!out) return fail(SSMD_ERR_INVALID_ARGUMENT, "out is null");
    if (steps <= 0 || (steps & 1))
        return fail(SSMD_ERR_INVALID_ARGUMENT, "steps must be a positive even number (got %d)",
                    steps);
    if (int e = ssmd_validate(p)) return e;
    if (int e = check_fields(*p, fields)) return e;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int e = cuda_check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal),
                           "begin capture"))
        return e;
    int err = SSMD_OK;
    for (int32_t i = 0; i < steps && !err; ++i) err = ssmd_step(fields, p, first_step + i, flags, stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (err) {
        if (graph) cudaGraphDestroy(graph);
        return err;
    }
    if (int e = cuda_check(ce, "end capture")) return e;
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (int e = cuda_check(ie, "graph instantiate")) return e;
    *out = reinterpret_cast<ssmd_graph_exec_t>(exec);
    return SSMD_OK;
}

int ssmd_graph_launch(ssmd_graph_exec_t exec, ssmd_stream_t stream) {
    if (!exec) return fail(SSMD_ERR_INVALID_ARGUMENT, "graph exec is null");
    return cuda_check(cudaGraphLaunch(reinterpret_cast<cudaGraphExec_t>(exec),
                                      reinterpret_cast<cudaStream_t>(stream)),
                      "graph launch");
}

int ssmd_graph_destroy(ssmd_graph_exec_t exec) {
    if (!exec) return SSMD_OK;
    return cuda_check(cudaGraphExecDestroy(reinterpret_cast<cudaGraphExec_t>(exec)), "graph destroy");
}

int ssmd_reduce(const ssmd_params *p, const LBMFields *fields, uint64_t steps_done, ssmd_stats *out,
                ssmd_stream_t stream) {
    if (!out) return fail(SSMD_ERR_INVALID_ARGUMENT, "out is null");
    if (int e = ssmd_validate(p)) return e;
    if (int e = check_fields(*p, fields)) return e;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    double v[kRedVals];
    int e;
    switch (p->storage) {
    case SSMD_STORAGE_F32: e = launch_reduce<float>(*p, *fields, steps_done, v, st); break;
    case SSMD_STORAGE_F16: e = launch_reduce<__half>(*p, *fields, steps_done, v, st); break;
    case SSMD_STORAGE_F16_G32: e = launch_reduce<half_g32>(*p, *fields, steps_done, v, st); break;
    default: e = launch_reduce<__nv_bfloat16>(*p, *fields, steps_done, v, st); break;
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

int ssmd_populations_to_push(const ssmd_params *p, const LBMFields *fields, uint64_t steps_done,
                             int32_t which, void *out, ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (int e = check_fields(*p, fields)) return e;
    if (!out) return fail(SSMD_ERR_INVALID_ARGUMENT, "out is null");
    if (which != 0 && which != 1) return fail(SSMD_ERR_INVALID_ARGUMENT, "which must be 0 or 1");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const bool even = (steps_done & 1ull) == 0ull;
    const void *src = which == 0 ? (even ? fields->f : p->f_alt) : (even ? fields->g : p->g_alt);
    if (which == 1) {
        if (g_storage_size(p->storage) == 4) return launch_to_push<float, 7>(*p, src, out, st);
        return launch_to_push<unsigned short, 7>(*p, src, out, st);
    }
    const bool f32 = p->storage == SSMD_STORAGE_F32;
    if (p->velocity_set == 19)
        return f32 ? launch_to_push<float, 19>(*p, src, out, st)
                   : launch_to_push<unsigned short, 19>(*p, src, out, st);
    return f32 ? launch_to_push<float, 27>(*p, src, out, st)
               : launch_to_push<unsigned short, 27>(*p, src, out, st);
}

int ssmd_profile_enable(int32_t max_launches) {
    if (max_launches <= 0 || max_launches > (1 << 20))
        return fail(SSMD_ERR_INVALID_ARGUMENT, "max_launches must be in [1, 2^20]");
    profile_free();
    g_prof.ev.resize(2 * (size_t)max_launches, nullptr);
    for (auto &e : g_prof.ev)
        if (int r = cuda_check(cudaEventCreate(&e), "event create")) {
            e = nullptr;
            profile_free();
            return r;
        }
    return SSMD_OK;
}

int ssmd_profile_read(float *ms, int32_t max, int32_t *count) {
    if (!count) return fail(SSMD_ERR_INVALID_ARGUMENT, "count is null");
    const int n = g_prof.used < max ? g_prof.used : max;
    for (int i = 0; i < n; ++i) {
        if (int r = cuda_check(cudaEventSynchronize(g_prof.ev[2 * i + 1]), "event sync")) return r;
        float t = 0.f;
        if (int r = cuda_check(cudaEventElapsedTime(&t, g_prof.ev[2 * i], g_prof.ev[2 * i + 1]),
                               "event elapsed"))
            return r;
        if (ms) ms[i] = t;
    }
    *count = n;
    return SSMD_OK;
}

int ssmd_profile_disable(void) {
    profile_free();
    return SSMD_OK;
}

int ssmd_check_status(const ssmd_params *p, uint32_t *status_out, ssmd_stream_t stream) {
    if (!p || !status_out || !p->workspace)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    DeviceStatus *s = status_of(*p);
    unsigned int flags = 0;
    if (int e = cuda_check(cudaMemcpyAsync(&flags, &s->flags, sizeof flags, cudaMemcpyDeviceToHost, st),
                           "status copy"))
        return e;
    if (int e = cuda_check(cudaMemsetAsync(&s->flags, 0, sizeof flags, st), "status clear")) return e;
    if (int e = cuda_check(cudaStreamSynchronize(st), "status sync")) return e;
    *status_out = flags;
    return SSMD_OK;
}

} // extern "C"
