// closure.cu — features, training targets and application of the learned closure.
//
// The closure runs the plain method on a 2x coarser lattice and corrects it
// per cell: an eddy viscosity nu_t added to nu(phi), and a factor on the
// surface tension.  Training data come from the solver's own fine runs:
// ssmd_closure_filter box-filters a fine lattice onto the coarse one (the
// resolved fields, the subgrid stress and the fine interface area density),
// ssmd_closure_targets turns them into the two targets, and
// ssmd_closure_features computes the network inputs from any lattice's
// macroscopic fields, so filtered fine data and a live coarse run are
// described by the same numbers.  Derivatives are central differences;
// exact-periodic axes wrap, the others clamp at the faces.
#include <cuda_runtime.h>

#include "closure.cuh"
#include "host.cuh"

using namespace ssmd;
using namespace ssmd::host;
using namespace ssmd::closure;

namespace {

__global__ void features_kernel(Grid g, const float *rho, const float *ux, const float *uy, const float *uz,
                                const float *phi, float nu_w, float nu_dow, float *feat) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t cells = (int64_t)g.nx * g.ny * g.nz;
    if (i >= cells) return;
    float f[SSMD_MLP_IN];
    closure::cell_features(g, rho, ux, uy, uz, phi, nu_w, nu_dow, i, f);
#pragma unroll
    for (int k = 0; k < SSMD_MLP_IN; ++k) feat[i * SSMD_MLP_IN + k] = f[k];
}

// One thread per coarse cell: means over the 2 x 2 x 2 fine block.
__global__ void filter_kernel(Grid fg, Grid cg, const float *rho, const float *ux, const float *uy, const float *uz,
                              const float *phi, float *coarse, float *tau, float *area) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t cells = (int64_t)cg.nx * cg.ny * cg.nz;
    if (i >= cells) return;
    const int X = (int)(i % cg.nx), Y = (int)((i / cg.nx) % cg.ny), Z = (int)(i / ((int64_t)cg.nx * cg.ny));
    double m[5] = {0, 0, 0, 0, 0}, uu[6] = {0, 0, 0, 0, 0, 0}, a = 0.0;
    for (int k = 0; k < 2; ++k)
        for (int j = 0; j < 2; ++j)
            for (int l = 0; l < 2; ++l) {
                const int x = 2 * X + l, y = 2 * Y + j, z = 2 * Z + k;
                const int64_t c = idx(fg, x, y, z);
                const float u0 = ux[c], u1 = uy[c], u2 = uz[c];
                m[0] += rho[c];
                m[1] += u0;
                m[2] += u1;
                m[3] += u2;
                m[4] += phi[c];
                uu[0] += (double)u0 * u0;
                uu[1] += (double)u1 * u1;
                uu[2] += (double)u2 * u2;
                uu[3] += (double)u0 * u1;
                uu[4] += (double)u0 * u2;
                uu[5] += (double)u1 * u2;
                float gx, gy, gz;
                grad3(fg, phi, x, y, z, gx, gy, gz);
                a += sqrt((double)gx * gx + (double)gy * gy + (double)gz * gz);
            }
    for (int q = 0; q < 5; ++q) m[q] *= 0.125;
    for (int q = 0; q < 6; ++q) uu[q] *= 0.125;
    for (int q = 0; q < 5; ++q) coarse[q * cells + i] = (float)m[q];
    tau[0 * cells + i] = (float)(uu[0] - m[1] * m[1]);
    tau[1 * cells + i] = (float)(uu[1] - m[2] * m[2]);
    tau[2 * cells + i] = (float)(uu[2] - m[3] * m[3]);
    tau[3 * cells + i] = (float)(uu[3] - m[1] * m[2]);
    tau[4 * cells + i] = (float)(uu[4] - m[1] * m[3]);
    tau[5 * cells + i] = (float)(uu[5] - m[2] * m[3]);
    area[i] = (float)(0.125 * a);
}

__global__ void targets_kernel(Grid g, const float *cf, const float *tau, const float *area, float nut_max,
                               float *targets, float *weights) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t cells = (int64_t)g.nx * g.ny * g.nz;
    if (i >= cells) return;
    const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / ((int64_t)g.nx * g.ny));
    const float *ux = cf + 1 * cells, *uy = cf + 2 * cells, *uz = cf + 3 * cells, *phi = cf + 4 * cells;
    float d[3][3];
    strain(g, ux, uy, uz, x, y, z, d);
    const float t[3][3] = {{tau[0 * cells + i], tau[3 * cells + i], tau[4 * cells + i]},
                           {tau[3 * cells + i], tau[1 * cells + i], tau[5 * cells + i]},
                           {tau[4 * cells + i], tau[5 * cells + i], tau[2 * cells + i]}};
    const float tr = (t[0][0] + t[1][1] + t[2][2]) * (1.0f / 3.0f);
    float num = 0.f, den = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const float s = 0.5f * (d[a][b] + d[b][a]);
            num += (t[a][b] - (a == b ? tr : 0.f)) * s;
            den += s * s;
        }
    // signed: negative values (backscatter) are kept, the coarse run bounds them
    const float nut = fminf(fmaxf(-num / (2.0f * den + 1e-12f), -nut_max), nut_max);
    float gx, gy, gz;
    grad3(g, phi, x, y, z, gx, gy, gz);
    const float gm = sqrtf(gx * gx + gy * gy + gz * gz);
    float cs = 1.0f;
    if (gm >= 1e-2f) cs = fminf(fmaxf(2.0f * area[i] / gm, 0.25f), 4.0f);
    const float ph = phi[i];
    targets[2 * i + 0] = nut;
    targets[2 * i + 1] = cs;
    weights[2 * i + 0] = 1.0f;
    weights[2 * i + 1] = 4.0f * ph * (1.0f - ph) + 0.01f;
}

// nu_t is bounded below by -nu(phi)/2 (feature 11), so the total viscosity
// stays at least half the molecular one and the relaxation rate below 2.
__global__ void apply_kernel(int64_t cells, const float *out, const float *feat, float nut_max, float *nut,
                             float *cs) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const float lo = fmaxf(-0.5f * feat[i * SSMD_MLP_IN + 11], -nut_max);
    nut[i] = fminf(fmaxf(out[2 * i + 0], lo), nut_max);
    cs[i] = fminf(fmaxf(out[2 * i + 1], 0.25f), 4.0f);
}

unsigned blocks_for(int64_t n) { return (unsigned)((n + 255) / 256); }

} // namespace

extern "C" int ssmd_closure_features(const ssmd_params *p, const LBMFields *fields, float *features,
                                     ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (!fields || !fields->rho || !fields->ux || !fields->uy || !fields->uz || !fields->phi || !features)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    const Grid g = grid_of(*p);
    const int64_t cells = (int64_t)g.nx * g.ny * g.nz;
    features_kernel<<<blocks_for(cells), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        g, fields->rho, fields->ux, fields->uy, fields->uz, fields->phi, p->nu_water, p->nu_oil - p->nu_water,
        features);
    return cuda_check(cudaGetLastError(), "features launch");
}

extern "C" int ssmd_closure_filter(const ssmd_params *fine, const LBMFields *fine_fields, float *coarse, float *tau,
                                   float *area, ssmd_stream_t stream) {
    if (int e = ssmd_validate(fine)) return e;
    if (!fine_fields || !fine_fields->rho || !fine_fields->ux || !fine_fields->uy || !fine_fields->uz ||
        !fine_fields->phi || !coarse || !tau || !area)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    if ((fine->nx | fine->ny | fine->nz) & 1u)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "filtering needs even lattice sizes (%u x %u x %u)", fine->nx,
                    fine->ny, fine->nz);
    const Grid fg = grid_of(*fine);
    Grid cg = fg;
    cg.nx /= 2;
    cg.ny /= 2;
    cg.nz /= 2;
    const int64_t cells = (int64_t)cg.nx * cg.ny * cg.nz;
    filter_kernel<<<blocks_for(cells), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        fg, cg, fine_fields->rho, fine_fields->ux, fine_fields->uy, fine_fields->uz, fine_fields->phi, coarse, tau,
        area);
    return cuda_check(cudaGetLastError(), "filter launch");
}

extern "C" int ssmd_closure_targets(const ssmd_params *coarse, const float *coarse_fields, const float *tau,
                                    const float *area, float nut_max, float *targets, float *weights,
                                    ssmd_stream_t stream) {
    if (int e = ssmd_validate(coarse)) return e;
    if (!coarse_fields || !tau || !area || !targets || !weights)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    const Grid g = grid_of(*coarse);
    const int64_t cells = (int64_t)g.nx * g.ny * g.nz;
    targets_kernel<<<blocks_for(cells), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        g, coarse_fields, tau, area, nut_max, targets, weights);
    return cuda_check(cudaGetLastError(), "targets launch");
}

extern "C" int ssmd_closure_apply(const ssmd_params *coarse, const float *net, const float *features, float *out,
                                  float *nut, float *sigma_scale, float nut_max, ssmd_stream_t stream) {
    if (int e = ssmd_validate(coarse)) return e;
    if (!net || !features || !out || !nut || !sigma_scale) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    const int64_t cells = (int64_t)coarse->nx * coarse->ny * coarse->nz;
    if (int e = ssmd_mlp_forward(net, features, cells, out, stream)) return e;
    apply_kernel<<<blocks_for(cells), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(cells, out, features,
                                                                                        nut_max, nut, sigma_scale);
    return cuda_check(cudaGetLastError(), "closure apply launch");
}
