// surface.cuh — boundary kernels, one per reference boundary launch.
//
// The reference applies, after its four bulk kernels and in this order
// (src/main.cu:165-169): water inflow at y = 0, oil inflow at z = 0, outflow
// at y = ny-1, outflow at z = nz-1, copy-periodic x.  Each writes
// post-stream population slots whose source cell is a ghost cell; in pull
// layout those slots live in the ghost cell itself, so every kernel here
// writes ghost-cell slots of the destination buffer only.  The kernels keep
// the reference's order because later ones read what earlier ones wrote
// (outflow z reads u on the y = ny-1 face, copy-periodic x copies slots and
// phi written by the outflows, copy-periodic y reads the x ghosts).
#pragma once

#include "common.cuh"
#include "noise.h"

namespace ssmd {

// Shifted equilibrium of direction q (D3Q19.cuh:133-140, D3Q27.cuh:147-154).
template <int Q, int q>
__device__ __forceinline__ float feq_dir(float rho, float ux, float uy, float uz) {
    constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
    constexpr float w = VS<Q>::w(q);
    const float uu = 1.5f * (ux * ux + uy * uy + uz * uz);
    const float cu = 3.0f * (float(cx) * ux + float(cy) * uy + float(cz) * uz);
    float b = 1.0f - uu + cu + 0.5f * cu * cu;
    if constexpr (Q == 27) b += cu * cu * cu * float(1.0 / 6.0) - uu * cu;
    return w * rho * b - w;
}

// Hermite non-equilibrium of direction q (D3Q19.cuh:142-161, D3Q27.cuh:156-185).
template <int Q, int q>
__device__ __forceinline__ float fneq_dir(float pxx, float pyy, float pzz, float pxy, float pxz,
                                          float pyz, float ux, float uy, float uz) {
    constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
    constexpr float w = VS<Q>::w(q);
    float h = (float(cx * cx) - kCs2) * pxx + (float(cy * cy) - kCs2) * pyy +
              (float(cz * cz) - kCs2) * pzz +
              2.0f * (float(cx * cy) * pxy + float(cx * cz) * pxz + float(cy * cz) * pyz);
    if constexpr (Q == 27) {
        h += 3.0f * ((float(cx * cx * cy) - kCs2 * float(cy)) * (pxx * uy + 2.0f * ux * pxy) +
                     (float(cx * cx * cz) - kCs2 * float(cz)) * (pxx * uz + 2.0f * ux * pxz) +
                     (float(cx * cy * cy) - kCs2 * float(cx)) * (pyy * ux + 2.0f * uy * pxy) +
                     (float(cy * cy * cz) - kCs2 * float(cz)) * (pyy * uz + 2.0f * uy * pyz) +
                     (float(cx * cz * cz) - kCs2 * float(cx)) * (pzz * ux + 2.0f * uz * pxz) +
                     (float(cy * cz * cz) - kCs2 * float(cy)) * (pzz * uy + 2.0f * uz * pyz)) +
             6.0f * float(cx * cy * cz) * (ux * pyz + uy * pxz + uz * pxy);
    }
    return (w * 4.5f) * h;
}

__device__ __forceinline__ bool in_range(int v, int lo, int hi) { return v >= lo && v <= hi; }

// Oil inlet speed u_oil (1 + a N(seed, step, cell)), rounded step by step
// (no contraction) so that host code evaluating the same expression in FP32
// gets the same bits.
__device__ __forceinline__ float inlet_speed(const Physics &P, unsigned long long step, uint32_t cell) {
    const float n = float(ssmd_noise::gaussian(P.seed, step, cell, 0u));
    return __fmul_rn(P.u_oil, __fadd_rn(1.0f, __fmul_rn(P.noise_amp, n)));
}

// Regularized inflow / outflow write of direction q into the ghost cell `home`:
// f = f_eq(rho_b, u_b) + omco f_neq(Pi(fn), u(fn)) at fluid node fn.
template <int Q, int q, class TF, class TG>
__device__ __forceinline__ void regularized_slot(const StepArgs<TF, TG> &a, uint32_t home,
                                                 uint32_t fn, float rho, float ux, float uy,
                                                 float uz, float omco) {
    const Fields &F = a.fld;
    const float feq = feq_dir<Q, q>(rho, ux, uy, uz);
    const float fneq = fneq_dir<Q, q>(F.pxx[fn], F.pyy[fn], F.pzz[fn], F.pxy[fn], F.pxz[fn],
                                      F.pyz[fn], F.ux[fn], F.uy[fn], F.uz[fn]);
    Store<TF>::st(a.f_dst + slot(a.geo, q, home), feq + omco * fneq);
}

// Water inflow disc on y = 0 (BoundaryConditions.cuh:36-99).  Thread (x, z).
template <int Q, class TF, class TG>
__device__ __forceinline__ void bc_water_inflow_at(const StepArgs<TF, TG> &a, const int x, const int z) {
    const Geometry &G = a.geo;
    const Physics &P = a.phys;
    if (x >= (int)G.nx || z >= (int)G.nz) return;
    const float dx = float(x) - P.water_cx, dz = float(z) - P.water_cz;
    if (dx * dx + dz * dz > P.water_r2) return;
    const uint32_t b = cell_index(G, x, 0, z);
    const float uw = P.u_water;
    a.fld.rho[b] = 1.0f;
    a.fld.phi[b] = 0.0f;
    a.fld.ux[b] = 0.0f;
    a.fld.uy[b] = uw;
    a.fld.uz[b] = 0.0f;
    unroll<0, Q>([&](auto q) {
        if constexpr (cy27(q) == 1) {
            const int xx = axis_nb(x + cx27(q), G.nx, G.bcx == BC_PERIODIC);
            const int zz = axis_nb(z + cz27(q), G.nz, G.bcz == BC_PERIODIC);
            if (xx < 0 || zz < 0) return; // outside the lattice (the reference reads out of bounds)
            regularized_slot<Q, q>(a, b, cell_index(G, xx, 1, zz), 1.0f, 0.0f, uw, 0.0f,
                                   P.omco_water);
        }
    });
    Store<TG>::st(a.g_dst + slot(G, 3, b), 0.0f); // w_3 * phi (1 + 4 u_y) with phi = 0
}

// Oil inflow disc on z = 0 (BoundaryConditions.cuh:101-168).  Thread (x, y).
template <int Q, class TF, class TG>
__device__ __forceinline__ void bc_oil_inflow_at(const StepArgs<TF, TG> &a, const int x, const int y) {
    const Geometry &G = a.geo;
    const Physics &P = a.phys;
    if (x >= (int)G.nx || y >= (int)G.ny) return;
    const float dx = float(x) - P.oil_cx, dy = float(y) - P.oil_cy;
    if (dx * dx + dy * dy > P.oil_r2) return;
    const uint32_t b = cell_index(G, x, y, 0);
    float uin = P.u_oil;
    if (P.noise_amp != 0.0f) {
        uin = inlet_speed(P, a.status->step, b);
    }
    a.fld.rho[b] = 1.0f;
    a.fld.phi[b] = 1.0f;
    a.fld.ux[b] = 0.0f;
    a.fld.uy[b] = 0.0f;
    a.fld.uz[b] = uin;
    unroll<0, Q>([&](auto q) {
        if constexpr (cz27(q) == 1) {
            const int xx = axis_nb(x + cx27(q), G.nx, G.bcx == BC_PERIODIC);
            const int yy = axis_nb(y + cy27(q), G.ny, G.bcy == BC_PERIODIC);
            if (xx < 0 || yy < 0 || !in_range(xx, G.x_lo, G.x_hi) || !in_range(yy, G.y_lo, G.y_hi))
                return;
            regularized_slot<Q, q>(a, b, cell_index(G, xx, yy, 1), 1.0f, 0.0f, 0.0f, uin,
                                   P.omco_oil);
        }
    });
    Store<TG>::st(a.g_dst + slot(G, 5, b), kW7_1 * 1.0f * (1.0f + 4.0f * uin));
}

// Outflow on y = ny-1 (BoundaryConditions.cuh:170-233).  Thread (x, z).
template <int Q, class TF, class TG>
__device__ __forceinline__ void bc_outflow_y_at(const StepArgs<TF, TG> &a, const int x, const int z) {
    const Geometry &G = a.geo;
    if (!in_range(x, G.x_lo, G.x_hi) || !in_range(z, G.z_lo, G.z_hi)) return;
    const uint32_t b = cell_index(G, x, G.ny - 1, z);
    const uint32_t i1 = cell_index(G, x, G.ny - 2, z);
    Fields F = a.fld;
    const float rho = F.rho[i1], phi = F.phi[i1], ux = F.ux[i1], uy = F.uy[i1], uz = F.uz[i1];
    F.rho[b] = rho;
    F.phi[b] = phi;
    F.ux[b] = ux;
    F.uy[b] = uy;
    F.uz[b] = uz;
    unroll<0, Q>([&](auto q) {
        if constexpr (cy27(q) == -1) {
            const int xx = axis_nb(x + cx27(q), G.nx, G.bcx == BC_PERIODIC);
            const int zz = axis_nb(z + cz27(q), G.nz, G.bcz == BC_PERIODIC);
            if (xx < 0 || zz < 0 || !in_range(xx, G.x_lo, G.x_hi) || !in_range(zz, G.z_lo, G.z_hi))
                return;
            regularized_slot<Q, q>(a, b, cell_index(G, xx, G.ny - 2, zz), rho, ux, uy, uz,
                                   a.phys.omco_ref);
        }
    });
    Store<TG>::st(a.g_dst + slot(G, 4, b), kW7_1 * phi * (1.0f - 4.0f * uy));
}

// Outflow on z = nz-1 (BoundaryConditions.cuh:235-293).  Thread (x, y).
template <int Q, class TF, class TG>
__device__ __forceinline__ void bc_outflow_z_at(const StepArgs<TF, TG> &a, const int x, const int y) {
    const Geometry &G = a.geo;
    if (!in_range(x, G.x_lo, G.x_hi) || !in_range(y, G.y_lo, G.y_hi)) return;
    const uint32_t b = cell_index(G, x, y, G.nz - 1);
    const uint32_t i1 = cell_index(G, x, y, G.nz - 2);
    Fields F = a.fld;
    const float rho = F.rho[i1], phi = F.phi[i1], ux = F.ux[i1], uy = F.uy[i1], uz = F.uz[i1];
    F.rho[b] = rho;
    F.phi[b] = phi;
    F.ux[b] = ux;
    F.uy[b] = uy;
    F.uz[b] = uz;
    unroll<0, Q>([&](auto q) {
        if constexpr (cz27(q) == -1) {
            // no fluid-range check here, as in the reference (ghost nodes allowed)
            const int xx = axis_nb(x + cx27(q), G.nx, G.bcx == BC_PERIODIC);
            const int yy = axis_nb(y + cy27(q), G.ny, G.bcy == BC_PERIODIC);
            if (xx < 0 || yy < 0) return;
            regularized_slot<Q, q>(a, b, cell_index(G, xx, yy, G.nz - 2), rho, ux, uy, uz,
                                   a.phys.omco_ref);
        }
    });
    Store<TG>::st(a.g_dst + slot(G, 6, b), kW7_1 * phi * (1.0f - 4.0f * uz));
}

// Copy-periodic x (BoundaryConditions.cuh:295-349).  Thread (y, z), all y, z.
// Push slot (1, y, z) <- (nx-2, y, z) for c_x > 0 is pull slot
// (0, y-c_y, z-c_z) <- (nx-3, y-c_y, z-c_z); c_x < 0 likewise with
// (nx-1, .) <- (2, .).  Slots whose pull home leaves the lattice are never
// read by a fluid cell and are skipped.
template <int Q, class TF, class TG>
__device__ __forceinline__ void bc_copy_x_at(const StepArgs<TF, TG> &a, const int y, const int z) {
    const Geometry &G = a.geo;
    if (y >= (int)G.ny || z >= (int)G.nz) return;
    const int nx = G.nx;
    const bool py = G.bcy == BC_PERIODIC, pz = G.bcz == BC_PERIODIC;
    unroll<0, Q>([&](auto q) {
        constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
        if constexpr (cx != 0) {
            const int hy = axis_nb(y - cy, G.ny, py), hz = axis_nb(z - cz, G.nz, pz);
            if (hy < 0 || hz < 0) return;
            const int to = cx > 0 ? 0 : nx - 1;
            const int from = cx > 0 ? nx - 3 : 2;
            TF *f = a.f_dst;
            f[slot(G, q, cell_index(G, to, hy, hz))] = f[slot(G, q, cell_index(G, from, hy, hz))];
        }
    });
    TG *g = a.g_dst;
    g[slot(G, 1, cell_index(G, 0, y, z))] = g[slot(G, 1, cell_index(G, nx - 3, y, z))];
    g[slot(G, 2, cell_index(G, nx - 1, y, z))] = g[slot(G, 2, cell_index(G, 2, y, z))];
    const uint32_t gL = cell_index(G, 0, y, z), gR = cell_index(G, nx - 1, y, z);
    const uint32_t bL = cell_index(G, 1, y, z), bR = cell_index(G, nx - 2, y, z);
    Fields F = a.fld;
    F.phi[gL] = F.phi[bR];
    F.phi[gR] = F.phi[bL];
    F.ux[gL] = F.ux[bR];
    F.ux[gR] = F.ux[bL];
    F.uy[gL] = F.uy[bR];
    F.uy[gR] = F.uy[bL];
    F.uz[gL] = F.uz[bR];
    F.uz[gR] = F.uz[bL];
}

// Copy-periodic y: the same rule as copy-periodic x applied to y (the
// reference only has the x version; this completes the x,y-periodic jet box).
// Thread (x, z), all x, z.
template <int Q, class TF, class TG>
__device__ __forceinline__ void bc_copy_y_at(const StepArgs<TF, TG> &a, const int x, const int z) {
    const Geometry &G = a.geo;
    if (x >= (int)G.nx || z >= (int)G.nz) return;
    const int ny = G.ny;
    const bool px = G.bcx == BC_PERIODIC, pz = G.bcz == BC_PERIODIC;
    unroll<0, Q>([&](auto q) {
        constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
        if constexpr (cy != 0) {
            const int hx = axis_nb(x - cx, G.nx, px), hz = axis_nb(z - cz, G.nz, pz);
            if (hx < 0 || hz < 0) return;
            const int to = cy > 0 ? 0 : ny - 1;
            const int from = cy > 0 ? ny - 3 : 2;
            TF *f = a.f_dst;
            f[slot(G, q, cell_index(G, hx, to, hz))] = f[slot(G, q, cell_index(G, hx, from, hz))];
        }
    });
    TG *g = a.g_dst;
    g[slot(G, 3, cell_index(G, x, 0, z))] = g[slot(G, 3, cell_index(G, x, ny - 3, z))];
    g[slot(G, 4, cell_index(G, x, ny - 1, z))] = g[slot(G, 4, cell_index(G, x, 2, z))];
    const uint32_t gL = cell_index(G, x, 0, z), gR = cell_index(G, x, ny - 1, z);
    const uint32_t bL = cell_index(G, x, 1, z), bR = cell_index(G, x, ny - 2, z);
    Fields F = a.fld;
    F.phi[gL] = F.phi[bR];
    F.phi[gR] = F.phi[bL];
    F.ux[gL] = F.ux[bR];
    F.ux[gR] = F.ux[bL];
    F.uy[gL] = F.uy[bR];
    F.uy[gR] = F.uy[bL];
    F.uz[gL] = F.uz[bR];
    F.uz[gR] = F.uz[bL];
}


// ---- kernels: one thread per face cell (i0, i1) ------------------------------
template <int Q, class TF, class TG>
__global__ void bc_water_inflow(const StepArgs<TF, TG> a) {
    bc_water_inflow_at<Q>(a, (int)(threadIdx.x + blockIdx.x * blockDim.x), (int)(threadIdx.y + blockIdx.y * blockDim.y));
}
template <int Q, class TF, class TG>
__global__ void bc_oil_inflow(const StepArgs<TF, TG> a) {
    bc_oil_inflow_at<Q>(a, (int)(threadIdx.x + blockIdx.x * blockDim.x), (int)(threadIdx.y + blockIdx.y * blockDim.y));
}
template <int Q, class TF, class TG>
__global__ void bc_outflow_y(const StepArgs<TF, TG> a) {
    bc_outflow_y_at<Q>(a, (int)(threadIdx.x + blockIdx.x * blockDim.x), (int)(threadIdx.y + blockIdx.y * blockDim.y));
}
template <int Q, class TF, class TG>
__global__ void bc_outflow_z(const StepArgs<TF, TG> a) {
    bc_outflow_z_at<Q>(a, (int)(threadIdx.x + blockIdx.x * blockDim.x), (int)(threadIdx.y + blockIdx.y * blockDim.y));
}
// Oil inflow (blockIdx.z 0) and outflow z (blockIdx.z 1) in one launch, for a
// lattice whose only jet faces are the z pair: inflow writes plane 0 and reads
// plane 1, outflow writes plane nz-1 and reads plane nz-2, so with nz >= 3
// neither reads what the other writes and their order does not matter.
template <int Q, class TF, class TG>
__global__ void bc_jet_z(const StepArgs<TF, TG> a) {
    const int i0 = (int)(threadIdx.x + blockIdx.x * blockDim.x), i1 = (int)(threadIdx.y + blockIdx.y * blockDim.y);
    if (blockIdx.z == 0) bc_oil_inflow_at<Q>(a, i0, i1);
    else bc_outflow_z_at<Q>(a, i0, i1);
}
template <int Q, class TF, class TG>
__global__ void bc_copy_x(const StepArgs<TF, TG> a) {
    bc_copy_x_at<Q>(a, (int)(threadIdx.x + blockIdx.x * blockDim.x), (int)(threadIdx.y + blockIdx.y * blockDim.y));
}
template <int Q, class TF, class TG>
__global__ void bc_copy_y(const StepArgs<TF, TG> a) {
    bc_copy_y_at<Q>(a, (int)(threadIdx.x + blockIdx.x * blockDim.x), (int)(threadIdx.y + blockIdx.y * blockDim.y));
}

} // namespace ssmd
