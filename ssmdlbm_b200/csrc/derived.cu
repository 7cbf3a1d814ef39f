// derived.cu — derived fields: running means and vorticity.
//
// Reference: src/derivedFields/operators/timeAverage.cuh:37-82 (means of phi
// and u), reynoldsMoments.cuh:37-96 (means of u_i u_j), vorticityFields.cuh:
// 37-96 (curl u by central differences on interior cells, zero on the
// outermost layer, and its magnitude).  The reference launches these once
// per step after the boundaries (src/main.cu:175) with t = STEP + 1; here t
// is a device counter of updates since ssmd_init, so a captured graph
// replays correctly.  The same running-mean update also runs inside the
// fused step (SSMD_STEP_AVERAGE).
#include <cuda_runtime.h>

#include "host.cuh"

using namespace ssmd;
using namespace ssmd::host;

namespace {

__global__ void vorticity_kernel(Geometry G, Fields F, float *wx_out, float *wy_out, float *wz_out, float *wm_out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= G.cells) return;
    const uint32_t c = (uint32_t)i;
    const uint32_t x = c % G.nx, y = (c / G.nx) % G.ny, z = c / G.nxy;
    float wx = 0.f, wy = 0.f, wz = 0.f;
    if (x > 0 && x < G.nx - 1 && y > 0 && y < G.ny - 1 && z > 0 && z < G.nz - 1) {
        const uint32_t xp = c + 1, xm = c - 1, yp = c + G.nx, ym = c - G.nx, zp = c + G.nxy, zm = c - G.nxy;
        // each difference and product rounded on its own, as written
        const float duz_dy = __fmul_rn(0.5f, __fsub_rn(F.uz[yp], F.uz[ym]));
        const float duy_dz = __fmul_rn(0.5f, __fsub_rn(F.uy[zp], F.uy[zm]));
        const float dux_dz = __fmul_rn(0.5f, __fsub_rn(F.ux[zp], F.ux[zm]));
        const float duz_dx = __fmul_rn(0.5f, __fsub_rn(F.uz[xp], F.uz[xm]));
        const float duy_dx = __fmul_rn(0.5f, __fsub_rn(F.uy[xp], F.uy[xm]));
        const float dux_dy = __fmul_rn(0.5f, __fsub_rn(F.ux[yp], F.ux[ym]));
        wx = __fsub_rn(duz_dy, duy_dz);
        wy = __fsub_rn(dux_dz, duz_dx);
        wz = __fsub_rn(duy_dx, dux_dy);
    }
    if (wx_out) wx_out[c] = wx;
    if (wy_out) wy_out[c] = wy;
    if (wz_out) wz_out[c] = wz;
    if (wm_out) wm_out[c] = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(wx, wx), __fmul_rn(wy, wy)), __fmul_rn(wz, wz)));
}

} // namespace

extern "C" int ssmd_derived_update(const ssmd_params *p, const LBMFields *fields, uint32_t what,
                                   ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (!fields || !p->derived) return fail(SSMD_ERR_INVALID_ARGUMENT, "null fields or params.derived");
    if (what & ~(SSMD_DERIVED_AVERAGES | SSMD_DERIVED_VORTICITY))
        return fail(SSMD_ERR_INVALID_ARGUMENT, "unknown bits in what (0x%x)", what);
    if (!fields->ux || !fields->uy || !fields->uz || !fields->phi)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null macroscopic field");
    if (!p->workspace) return fail(SSMD_ERR_INVALID_ARGUMENT, "workspace is null");
    const Geometry G = make_geometry(*p);
    const Fields F = make_fields(*fields);
    const ssmd_derived &d = *p->derived;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const unsigned nb = (unsigned)((G.cells + 255) / 256);
    if (what & SSMD_DERIVED_AVERAGES) {
        averages_kernel<<<nb, 256, 0, st>>>(G, F, make_averages(*p), status_of(*p), 0);
        advance_avg_kernel<<<1, 1, 0, st>>>(status_of(*p));
    }
    if ((what & SSMD_DERIVED_VORTICITY) && (d.vort_x || d.vort_y || d.vort_z || d.vort_mag))
        vorticity_kernel<<<nb, 256, 0, st>>>(G, F, d.vort_x, d.vort_y, d.vort_z, d.vort_mag);
    return cuda_check(cudaGetLastError(), "derived-field launch");
}
