// init.cuh — initial state and layout conversion kernels.
#pragma once

#include "common.cuh"
#include "noise.h"
#include "surface.cuh"

namespace ssmd {

// rho = 1, u = 0, phi = 0, Pi = 0, then the water disc (phi = 0,
// uy = u_water) and the oil disc (phi = 1, uz = u_oil), in the reference's
// order setWaterJet, setOilJet, setInitialDensity (initialConditions.cu:33-97).
static __global__ void init_macros_kernel(Geometry G, Physics P, Fields F, float *fsx, float *fsy,
                                   float *fsz) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= G.cells) return;
    const uint32_t c = (uint32_t)i;
    const uint32_t x = c % G.nx, y = (c / G.nx) % G.ny, z = c / G.nxy;
    float phi = 0.f, ux = 0.f, uy = 0.f, uz = 0.f;
    if (G.bcy == BC_JET && y == 0) {
        const float dx = float(x) - P.water_cx, dz = float(z) - P.water_cz;
        if (dx * dx + dz * dz <= P.water_r2) {
            phi = 0.f;
            uy = P.u_water;
        }
    }
    if (G.bcz == BC_JET && z == 0) {
        const float dx = float(x) - P.oil_cx, dy = float(y) - P.oil_cy;
        if (dx * dx + dy * dy <= P.oil_r2) {
            phi = 1.f;
            uz = P.noise_amp != 0.0f ? inlet_speed(P, 0, c) : P.u_oil;
        }
    }
    F.rho[c] = 1.0f;
    F.phi[c] = phi;
    F.ux[c] = ux;
    F.uy[c] = uy;
    F.uz[c] = uz;
    F.pxx[c] = F.pyy[c] = F.pzz[c] = 0.f;
    F.pxy[c] = F.pxz[c] = F.pyz[c] = 0.f;
    if (fsx) fsx[c] = 0.f;
    if (fsy) fsy[c] = 0.f;
    if (fsz) fsz[c] = 0.f;
}

// f = f_eq(rho, u) and g = g_eq(phi, u) of the cell each slot streams into
// (setDistros, initialConditions.cu:99-140, in pull layout), written into both
// buffers so that slots no kernel ever rewrites agree between them.
template <int Q, class TF, class TG>
__global__ void init_populations_kernel(Geometry G, Fields F, TF *fa, TF *fb, TG *ga, TG *gb) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= G.cells) return;
    const uint32_t c = (uint32_t)i;
    const int x = c % G.nx, y = (c / G.nx) % G.ny, z = c / G.nxy;
    const bool px = G.bcx == BC_PERIODIC, py = G.bcy == BC_PERIODIC, pz = G.bcz == BC_PERIODIC;
    unroll<0, Q>([&](auto q) {
        int tx = axis_nb(x + cx27(q), G.nx, px), ty = axis_nb(y + cy27(q), G.ny, py),
            tz = axis_nb(z + cz27(q), G.nz, pz);
        const uint32_t t = (tx < 0 || ty < 0 || tz < 0) ? c : cell_index(G, tx, ty, tz);
        const float v = feq_dir<Q, q>(F.rho[t], F.ux[t], F.uy[t], F.uz[t]);
        Store<TF>::st(fa + slot(G, q, c), v);
        Store<TF>::st(fb + slot(G, q, c), v);
    });
    unroll<0, 7>([&](auto q) {
        int tx = axis_nb(x + cx27(q), G.nx, px), ty = axis_nb(y + cy27(q), G.ny, py),
            tz = axis_nb(z + cz27(q), G.nz, pz);
        const uint32_t t = (tx < 0 || ty < 0 || tz < 0) ? c : cell_index(G, tx, ty, tz);
        const float w = q == 0 ? kW7_0 : kW7_1;
        const float cu = float(cx27(q)) * F.ux[t] + float(cy27(q)) * F.uy[t] + float(cz27(q)) * F.uz[t];
        const float v = w * F.phi[t] * (1.0f + 4.0f * cu);
        Store<TG>::st(ga + slot(G, q, c), v);
        Store<TG>::st(gb + slot(G, q, c), v);
    });
}

// Pull layout -> the reference's push (post-stream) layout:
// push[q][t] = pull[q][t - c_q]; zero where t - c_q leaves the lattice.
template <class T, int NQ>
__global__ void pull_to_push_kernel(Geometry G, const T *pull, T *push) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= G.cells) return;
    const uint32_t c = (uint32_t)i;
    const int x = c % G.nx, y = (c / G.nx) % G.ny, z = c / G.nxy;
    const bool px = G.bcx == BC_PERIODIC, py = G.bcy == BC_PERIODIC, pz = G.bcz == BC_PERIODIC;
    unroll<0, NQ>([&](auto q) {
        const int sx = axis_nb(x - cx27(q), G.nx, px), sy = axis_nb(y - cy27(q), G.ny, py),
                  sz = axis_nb(z - cz27(q), G.nz, pz);
        T v = T(0.0f);
        if (sx >= 0 && sy >= 0 && sz >= 0) v = pull[slot(G, q, cell_index(G, sx, sy, sz))];
        push[slot(G, q, c)] = v;
    });
}

} // namespace ssmd
