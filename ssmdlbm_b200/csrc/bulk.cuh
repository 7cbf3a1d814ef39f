// bulk.cuh — the fused per-step kernel for every fluid cell.
//
// One launch performs what the reference does in four
// (src/cuda/CUDAGraph.cuh:44-49):
//   computePhase   phi^n = sum_q g^n                (src/phaseField.cuh:31-52)
//   computeForces  n, |grad phi|, kappa, F_s         (src/phaseField.cuh:54-294)
//   computeMoments rho, u, Pi_neq                    (src/lbm.cu:33-128)
//   streamCollide  regularized collision + phase update (src/lbm.cu:130-270)
//
// Layout: populations are in pull layout (slot q of cell s is read by s + c_q),
// two buffers; this kernel reads src and writes only fluid-cell slots of dst.
// The boundary kernels write only ghost-cell slots of dst, so the two never
// overlap, and every slot the reference leaves untouched stays constant in
// both buffers.
//
// Work item: a 32 x 8 column of cells marching over `zchunk` z planes.  phi is
// rebuilt from g on the fly (never re-read from DRAM) into a 5-plane ring with
// a 2-cell halo; interface normals and |grad phi| live in a 3-plane ring with a
// 1-cell halo; the populations of the cell are gathered straight from DRAM
// (pull) and written back to the cell's own slots (aligned, coalesced).
#pragma once

#include "common.cuh"

namespace ssmd {

#ifndef SSMD_BULK_MIN_BLOCKS
#define SSMD_BULK_MIN_BLOCKS 3 // resident work items per SM the register budget targets
#endif

constexpr int kTX = 32, kTY = 8, kThreads = kTX * kTY;
constexpr int kHX = kTX + 4, kHY = kTY + 4; // phi ring (halo 2)
constexpr int kNX = kTX + 2, kNY = kTY + 2; // normal ring (halo 1)

struct BulkSmem {
    float phiR[5][kHY][kHX]; // phi as the reference's streamCollide sees it (ghost values kept)
    float phiZ[5][kHY][kHX]; // phi as computeForces sees it (ghost / outside read as 0)
    float nrm[3][4][kNY][kNX]; // n_x, n_y, n_z, |grad phi| on the zeroed field
};

// Ring slot of plane p; planes never go below -2, so the unsigned form is exact.
__device__ __forceinline__ int ring5(int p) { return (int)((unsigned)(p + 10) % 5u); }
__device__ __forceinline__ int ring3(int p) { return (int)((unsigned)(p + 9) % 3u); }

template <int Q, class TF, class TG>
struct Bulk {
    using A = StepArgs<TF, TG>;

    // phi^n at fluid cell (x, y, z) with linear index c, from the post-stream
    // phase populations (pull layout: direction q is read at c - c_q).
    static __device__ __forceinline__ float phi_from_g(const A &a, int x, int y, int z, uint32_t c) {
        const Geometry &G = a.geo;
        const int64_t N = (int64_t)G.cells, sy = G.nx, sz = G.nxy;
        // Offsets of the source cells (pull: direction q is read at c - c_q); a
        // fluid cell only wraps on an exact-periodic axis, handled by a per-lane
        // correction instead of a branch so that a warp never runs two paths.
        const int64_t wxm = (x == 0) ? (int64_t)G.nx : 0;                 // c - 1 wraps to +nx-1
        const int64_t wxp = (x == (int)G.nx - 1) ? -(int64_t)G.nx : 0;
        const int64_t wym = (y == 0) ? (int64_t)G.nxy : 0;
        const int64_t wyp = (y == (int)G.ny - 1) ? -(int64_t)G.nxy : 0;
        const int64_t wzm = (z == 0) ? N : 0;
        const int64_t wzp = (z == (int)G.nz - 1) ? -N : 0;
        const TG *pg = a.g_src + c;
        float s = Store<TG>::ld(pg);
        s += Store<TG>::ld(pg + (1 * N - 1 + wxm));
        s += Store<TG>::ld(pg + (2 * N + 1 + wxp));
        s += Store<TG>::ld(pg + (3 * N - sy + wym));
        s += Store<TG>::ld(pg + (4 * N + sy + wyp));
        s += Store<TG>::ld(pg + (5 * N - sz + wzm));
        s += Store<TG>::ld(pg + (6 * N + sz + wzp));
        return s;
    }

    static __device__ __forceinline__ bool fluid(const Geometry &G, int x, int y, int z) {
        return x >= G.x_lo && x <= G.x_hi && y >= G.y_lo && y <= G.y_hi && z >= G.z_lo &&
               z <= G.z_hi;
    }

    // Halo coordinate along one axis: one conditional wrap suffices unless the
    // host flagged an axis shorter than the tile halo (halo_mod).
    static __device__ __forceinline__ int halo_axis(const A &a, int c, int n, bool periodic) {
        if (a.halo_mod) return axis_halo(c, n, periodic);
        return axis_nb(c, n, periodic);
    }

    // Fill ring slot of plane pz with phi over the tile + 2-cell halo.
    static __device__ void fill_phi(const A &a, BulkSmem &S, int x0, int y0, int pz, int tid) {
        const Geometry &G = a.geo;
        const int gz = halo_axis(a, pz, G.nz, G.bcz == BC_PERIODIC);
        const int s = ring5(pz);
        const bool zfluid = gz >= G.z_lo && gz <= G.z_hi;
        for (int i = tid; i < kHX * kHY; i += kThreads) {
            const int hx = i % kHX, hy = i / kHX;
            const int gx = halo_axis(a, x0 - 2 + hx, G.nx, G.bcx == BC_PERIODIC);
            const int gy = halo_axis(a, y0 - 2 + hy, G.ny, G.bcy == BC_PERIODIC);
            float raw = 0.f, zer = 0.f;
            if (gx >= 0 && gy >= 0 && gz >= 0) {
                const uint32_t c = cell_index(G, gx, gy, gz);
                if (zfluid && gx >= G.x_lo && gx <= G.x_hi && gy >= G.y_lo && gy <= G.y_hi) {
                    raw = phi_from_g(a, gx, gy, gz, c);
                    zer = raw;
                } else {
                    raw = a.fld.phi[c];
                }
            }
            S.phiR[s][hy][hx] = raw;
            S.phiZ[s][hy][hx] = zer;
        }
    }

    // Isotropic gradient 3 sum_q w_q c_q phi(x + c_q) with the hydrodynamic
    // set's weights (phaseField.cuh:158-218); (hx, hy) is the centre in ring
    // coordinates, p0 the centre plane.
    template <class Ring>
    static __device__ __forceinline__ void grad(const Ring &R, int hx, int hy, int sm, int s0, int sp,
                                                float &gx, float &gy, float &gz) {
        auto at = [&](int dx, int dy, int dz) -> float {
            const int sl = dz < 0 ? sm : (dz > 0 ? sp : s0);
            return R[sl][hy + dy][hx + dx];
        };
        float sx = 0.f, sy = 0.f, sz = 0.f;
        unroll<0, (Q - 1) / 2>([&](auto k) {
            constexpr int q = 2 * k + 1;
            constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
            constexpr float w = (q <= 6) ? VS<Q>::w1 : (q <= 18 ? VS<Q>::w2 : VS<Q>::w3);
            const float d = w * (at(cx, cy, cz) - at(-cx, -cy, -cz));
            if constexpr (cx != 0) sx += cx > 0 ? d : -d;
            if constexpr (cy != 0) sy += cy > 0 ? d : -d;
            if constexpr (cz != 0) sz += cz > 0 ? d : -d;
        });
        gx = 3.0f * sx;
        gy = 3.0f * sy;
        gz = 3.0f * sz;
    }

    // Normals and |grad phi| of plane pz over the tile + 1-cell halo.
    static __device__ void fill_nrm(BulkSmem &S, int pz, int tid) {
        const int s = ring3(pz);
        for (int i = tid; i < kNX * kNY; i += kThreads) {
            const int nxh = i % kNX, nyh = i / kNX;
            float gx, gy, gz;
            grad(S.phiZ, nxh + 1, nyh + 1, ring5(pz - 1), ring5(pz), ring5(pz + 1), gx, gy, gz);
            const float ind = sqrtf(gx * gx + gy * gy + gz * gz);
            const float inv = 1.0f / (ind + 1e-9f);
            S.nrm[s][0][nyh][nxh] = gx * inv;
            S.nrm[s][1][nyh][nxh] = gy * inv;
            S.nrm[s][2][nyh][nxh] = gz * inv;
            S.nrm[s][3][nyh][nxh] = ind;
        }
    }

    // Update of one fluid cell (x, y, z); (tx, ty) its position in the tile.
    static __device__ __forceinline__ void cell(const A &a, const BulkSmem &S, int x, int y, int z,
                                                int tx, int ty) {
        const Geometry &G = a.geo;
        const Physics &P = a.phys;
        const bool px = G.bcx == BC_PERIODIC, py = G.bcy == BC_PERIODIC, pz = G.bcz == BC_PERIODIC;
        const uint32_t c0 = cell_index(G, x, y, z);

        // ---- surface tension from the zeroed-ghost field (phaseField.cuh:246-293)
        const int hx = tx + 2, hy = ty + 2; // phi ring centre
        const int nxh = tx + 1, nyh = ty + 1; // normal ring centre
        const int sm = ring3(z - 1), s0 = ring3(z), sp = ring3(z + 1);
        auto nat = [&](int comp, int dx, int dy, int dz) -> float {
            const int sl = dz < 0 ? sm : (dz > 0 ? sp : s0);
            return S.nrm[sl][comp][nyh + dy][nxh + dx];
        };
        float div = 0.f;
        unroll<0, (Q - 1) / 2>([&](auto k) {
            constexpr int q = 2 * k + 1;
            constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
            constexpr float w = (q <= 6) ? VS<Q>::w1 : (q <= 18 ? VS<Q>::w2 : VS<Q>::w3);
            float d = 0.f;
            if constexpr (cx != 0) d += float(cx) * (nat(0, cx, cy, cz) - nat(0, -cx, -cy, -cz));
            if constexpr (cy != 0) d += float(cy) * (nat(1, cx, cy, cz) - nat(1, -cx, -cy, -cz));
            if constexpr (cz != 0) d += float(cz) * (nat(2, cx, cy, cz) - nat(2, -cx, -cy, -cz));
            div += w * d;
        });
        const float curvature = 3.0f * div;
        const float stc = -P.sigma * curvature * nat(3, 0, 0, 0);
        const float fx = stc * nat(0, 0, 0, 0);
        const float fy = stc * nat(1, 0, 0, 0);
        const float fz = stc * nat(2, 0, 0, 0);

        // ---- normals of the phase update from phi with ghost values (lbm.cu:157-224).
        // Away from ghost layers the raw and zeroed fields agree on the 3x3x3
        // neighbourhood, so the ring's normal is the same number.
        const bool near_ghost = (!px && (x <= G.x_lo || x >= G.x_hi)) ||
                                (!py && (y <= G.y_lo || y >= G.y_hi)) ||
                                (!pz && (z <= G.z_lo || z >= G.z_hi));
        float nx = nat(0, 0, 0, 0), ny = nat(1, 0, 0, 0), nz = nat(2, 0, 0, 0);
        if (near_ghost) {
            float gx, gy, gz;
            grad(S.phiR, hx, hy, ring5(z - 1), ring5(z), ring5(z + 1), gx, gy, gz);
            const float ind = sqrtf(gx * gx + gy * gy + gz * gz);
            const float inv = 1.0f / (ind + 1e-9f);
            nx = gx * inv;
            ny = gy * inv;
            nz = gz * inv;
        }
        const float phi = S.phiR[ring5(z)][hy][hx];

        // ---- gather f^n (after the stencil work, so that the Q values are live
        // only across the moments and the collision).  The source of direction q
        // is c0 - (cx + cy nx + cz nx ny), one warp-uniform offset per q, plus a
        // per-lane correction where an exact-periodic axis wraps (no branch, so
        // the warp holding the wrapping lane does not run two gathers).
        const int64_t N = (int64_t)G.cells, sy = G.nx, sz = G.nxy;
        const int64_t wxm = (px && x == 0) ? (int64_t)G.nx : 0; // source x-1 -> x-1+nx
        const int64_t wxp = (px && x == (int)G.nx - 1) ? -(int64_t)G.nx : 0;
        const int64_t wym = (py && y == 0) ? (int64_t)G.nxy : 0;
        const int64_t wyp = (py && y == (int)G.ny - 1) ? -(int64_t)G.nxy : 0;
        const int64_t wzm = (pz && z == 0) ? N : 0;
        const int64_t wzp = (pz && z == (int)G.nz - 1) ? -N : 0;
        auto src_off = [&](auto q) -> int64_t {
            constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
            int64_t o = (int64_t)q * N - (cx + cy * sy + cz * sz);
            if constexpr (cx > 0) o += wxm;
            if constexpr (cx < 0) o += wxp;
            if constexpr (cy > 0) o += wym;
            if constexpr (cy < 0) o += wyp;
            if constexpr (cz > 0) o += wzm;
            if constexpr (cz < 0) o += wzp;
            return o;
        };
        float f[Q];
        const TF *pf = a.f_src + c0;
        unroll<0, Q>([&](auto q) { f[q] = Store<TF>::ld(pf + src_off(q)); });
        float gin[7];
        const bool bgk = a.phys.omega_g != 1.0f;
        if (bgk) {
            const TG *pg = a.g_src + c0;
            unroll<0, 7>([&](auto q) { gin[q] = Store<TG>::ld(pg + src_off(q)); });
        }

        // ---- hydrodynamics
        const Moments m = moments<Q>(f, fx, fy, fz);
        const float nu = fmaf(phi, P.nu_oil_minus_water, P.nu_water);
        const float omega = 1.0f / (0.5f + 3.0f * nu);
        float fo[Q];
        collide<Q>(m, 1.0f - omega, fx, fy, fz, fo);
        TF *pfd = a.f_dst + c0;
        unroll<0, Q>([&](auto q) { Store<TF>::st(pfd + (int64_t)q * N, fo[q]); });

        // ---- conservative Allen-Cahn update, D3Q7 (lbm.cu:256-269; D3Q7.cuh:124-148)
        const float sharp = P.gamma * phi * (1.0f - phi);
        float go[7];
        go[0] = kW7_0 * phi;
        const float ax = 4.0f * phi * m.ux + sharp * nx;
        const float ay = 4.0f * phi * m.uy + sharp * ny;
        const float az = 4.0f * phi * m.uz + sharp * nz;
        go[1] = kW7_1 * (phi + ax);
        go[2] = kW7_1 * (phi - ax);
        go[3] = kW7_1 * (phi + ay);
        go[4] = kW7_1 * (phi - ay);
        go[5] = kW7_1 * (phi + az);
        go[6] = kW7_1 * (phi - az);
        if (bgk) {
            // BGK with the anti-diffusion flux inside the equilibrium; omega_g = 1
            // reduces to the reference's g = g_eq + h.
            unroll<0, 7>([&](auto q) { go[q] = gin[q] + P.omega_g * (go[q] - gin[q]); });
        }
        TG *pgd = a.g_dst + c0;
        unroll<0, 7>([&](auto q) { Store<TG>::st(pgd + (int64_t)q * N, go[q]); });

        // ---- macroscopic fields needed by the boundaries (or all, on save steps)
        const bool bplane = (G.bcx == BC_COPY && (x == 1 || x == (int)G.nx - 2)) ||
                            (G.bcy != BC_PERIODIC && (y == 1 || y == (int)G.ny - 2)) ||
                            (G.bcz != BC_PERIODIC && (z == 1 || z == (int)G.nz - 2));
        if (bplane || (a.flags & 1u)) {
            a.fld.rho[c0] = m.rho;
            a.fld.ux[c0] = m.ux;
            a.fld.uy[c0] = m.uy;
            a.fld.uz[c0] = m.uz;
            a.fld.phi[c0] = phi;
            a.fld.pxx[c0] = m.pxx;
            a.fld.pyy[c0] = m.pyy;
            a.fld.pzz[c0] = m.pzz;
            a.fld.pxy[c0] = m.pxy;
            a.fld.pxz[c0] = m.pxz;
            a.fld.pyz[c0] = m.pyz;
        }
        if (!isfinite(m.rho)) atomicOr(&a.status->flags, 1u);
    }
};

template <int Q, class TF, class TG>
__global__ void __launch_bounds__(kThreads, SSMD_BULK_MIN_BLOCKS) bulk_kernel(const StepArgs<TF, TG> a) {
    using B = Bulk<Q, TF, TG>;
    __shared__ BulkSmem S;
    const Geometry &G = a.geo;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kTX * ty;
    if (blockIdx.x == 0 && tid == 0) a.status->step += 1ull; // step in progress

    int w = blockIdx.x;
    const int bx = w % a.tiles_x;
    w /= a.tiles_x;
    const int by = w % a.tiles_y;
    const int bz = w / a.tiles_y;
    const int x0 = bx * kTX, y0 = by * kTY;
    const int zs = G.z_lo + bz * a.zchunk;
    const int ze = min(zs + a.zchunk, G.z_hi + 1);
    const int x = x0 + tx, y = y0 + ty;
    const bool active = x >= G.x_lo && x <= G.x_hi && y >= G.y_lo && y <= G.y_hi;

    for (int p = zs - 2; p <= zs + 2; ++p) B::fill_phi(a, S, x0, y0, p, tid);
    __syncthreads();
    B::fill_nrm(S, zs - 1, tid);
    B::fill_nrm(S, zs, tid);
    for (int z = zs; z < ze; ++z) {
        B::fill_nrm(S, z + 1, tid);
        __syncthreads();
        if (active) B::cell(a, S, x, y, z, tx, ty);
        if (z + 1 < ze) B::fill_phi(a, S, x0, y0, z + 3, tid);
        __syncthreads();
    }
}

} // namespace ssmd
