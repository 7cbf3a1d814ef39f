// closure.cuh — per-cell features of the learned closure, shared by the
// features kernel (closure.cu) and the fused closure refresh (mlp.cu), so both
// give the network the same numbers.  Derivatives are central differences;
// exact-periodic axes wrap, the others clamp at the faces.
#pragma once

#include <cstdint>

#include "../../include/ssmd.h"

namespace ssmd {
namespace closure {

struct Grid {
    int nx, ny, nz;
    bool px, py, pz;
};

inline Grid grid_of(const ssmd_params &p) {
    return Grid{(int)p.nx, (int)p.ny, (int)p.nz, p.bc_x == SSMD_BC_PERIODIC, p.bc_y == SSMD_BC_PERIODIC,
                p.bc_z == SSMD_BC_PERIODIC};
}

__device__ __forceinline__ int nbr(int c, int d, int n, bool per) {
    int v = c + d;
    if (per) v = v < 0 ? v + n : (v >= n ? v - n : v);
    else v = v < 0 ? 0 : (v >= n ? n - 1 : v);
    return v;
}

__device__ __forceinline__ int64_t idx(const Grid &g, int x, int y, int z) {
    return (int64_t)x + (int64_t)g.nx * ((int64_t)y + (int64_t)g.ny * z);
}

// Central-difference gradient of a scalar array at (x, y, z).
__device__ __forceinline__ void grad3(const Grid &g, const float *a, int x, int y, int z, float &gx, float &gy,
                                      float &gz) {
    gx = 0.5f * (a[idx(g, nbr(x, 1, g.nx, g.px), y, z)] - a[idx(g, nbr(x, -1, g.nx, g.px), y, z)]);
    gy = 0.5f * (a[idx(g, x, nbr(y, 1, g.ny, g.py), z)] - a[idx(g, x, nbr(y, -1, g.ny, g.py), z)]);
    gz = 0.5f * (a[idx(g, x, y, nbr(z, 1, g.nz, g.pz))] - a[idx(g, x, y, nbr(z, -1, g.nz, g.pz))]);
}

// Velocity gradient d[i][j] = d u_i / d x_j and the strain rate S = (d + d^T)/2.
__device__ __forceinline__ void strain(const Grid &g, const float *ux, const float *uy, const float *uz, int x,
                                       int y, int z, float (&d)[3][3]) {
    grad3(g, ux, x, y, z, d[0][0], d[0][1], d[0][2]);
    grad3(g, uy, x, y, z, d[1][0], d[1][1], d[1][2]);
    grad3(g, uz, x, y, z, d[2][0], d[2][1], d[2][2]);
}

// The six face neighbours of a cell, as 32-bit cell indices (a lattice has
// fewer than 2^32 cells): the same cells nbr() and idx() give, found with one
// 32-bit division chain per cell instead of 64-bit arithmetic per load.
struct Faces {
    uint32_t xp, xm, yp, ym, zp, zm;
};

__device__ __forceinline__ Faces faces(const Grid &g, uint32_t c) {
    const uint32_t nx = (uint32_t)g.nx, nxy = nx * (uint32_t)g.ny;
    const uint32_t z = c / nxy, rxy = c - z * nxy, y = rxy / nx, x = rxy - y * nx;
    // step d along an axis of n cells at coordinate v, stride s: wrap or clamp like nbr()
    auto up = [](uint32_t v, uint32_t n, uint32_t s, bool per) { return v + 1 < n ? s : (per ? s - n * s : 0u); };
    auto dn = [](uint32_t v, uint32_t n, uint32_t s, bool per) { return v > 0 ? 0u - s : (per ? n * s - s : 0u); };
    Faces f;
    f.xp = c + up(x, nx, 1u, g.px);
    f.xm = c + dn(x, nx, 1u, g.px);
    f.yp = c + up(y, (uint32_t)g.ny, nx, g.py);
    f.ym = c + dn(y, (uint32_t)g.ny, nx, g.py);
    f.zp = c + up(z, (uint32_t)g.nz, nxy, g.pz);
    f.zm = c + dn(z, (uint32_t)g.nz, nxy, g.pz);
    return f;
}

// The SSMD_MLP_IN features of cell i.
__device__ __forceinline__ void cell_features(const Grid &g, const float *rho, const float *ux, const float *uy,
                                              const float *uz, const float *phi, float nu_w, float nu_dow, int64_t i,
                                              float (&f)[SSMD_MLP_IN]) {
    const Faces n6 = faces(g, (uint32_t)i);
    const float ph = phi[i];
    auto diff = [&](const float *a, uint32_t p, uint32_t m) { return 0.5f * (a[p] - a[m]); };
    const float gx = diff(phi, n6.xp, n6.xm), gy = diff(phi, n6.yp, n6.ym), gz = diff(phi, n6.zp, n6.zm);
    const float gmag = sqrtf(gx * gx + gy * gy + gz * gz);
    const float lap = phi[n6.xp] + phi[n6.xm] + phi[n6.yp] + phi[n6.ym] + phi[n6.zp] + phi[n6.zm] - 6.0f * ph;
    float d[3][3];
    const float *u3[3] = {ux, uy, uz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        d[a][0] = diff(u3[a], n6.xp, n6.xm);
        d[a][1] = diff(u3[a], n6.yp, n6.ym);
        d[a][2] = diff(u3[a], n6.zp, n6.zm);
    }
    float ss = 0.f, nsn = 0.f;
    const float inv = 1.0f / (gmag + 1e-9f);
    const float n[3] = {gx * inv, gy * inv, gz * inv};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const float s = 0.5f * (d[a][b] + d[b][a]);
            ss += s * s;
            nsn += n[a] * s * n[b];
        }
    const float wx = d[2][1] - d[1][2], wy = d[0][2] - d[2][0], wz = d[1][0] - d[0][1];
    const float u0 = ux[i], u1 = uy[i], u2 = uz[i];
    f[0] = ph;
    f[1] = 4.0f * ph * (1.0f - ph);
    f[2] = gmag;
    f[3] = lap;
    f[4] = sqrtf(2.0f * ss);
    f[5] = sqrtf(wx * wx + wy * wy + wz * wz);
    f[6] = nsn;
    f[7] = sqrtf(u0 * u0 + u1 * u1 + u2 * u2);
    f[8] = u2;
    f[9] = rho[i] - 1.0f;
    f[10] = d[0][0] + d[1][1] + d[2][2];
    f[11] = fmaf(ph, nu_dow, nu_w);
}

} // namespace closure
} // namespace ssmd
