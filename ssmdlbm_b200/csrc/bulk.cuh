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
// rebuilt from g on the fly (never re-read from DRAM) into a 6-plane ring with
// a 2-cell halo; interface normals and |grad phi| live in a 3-plane ring with a
// 1-cell halo, both filled ahead of the plane being updated so that one barrier
// per plane suffices; the curvature stencil is split into per-plane partial sums
// that each thread carries along its own column in registers; the
// populations of the cell are gathered straight from DRAM (pull) and written
// back to the cell's own slots (aligned, coalesced).
#pragma once

#include <type_traits>

#include "common.cuh"
#include "tma.cuh"

namespace ssmd {

// Resident work items per SM the register budget targets: 4 (64 registers),
// with the long-lived gradient and curvature carries in shared memory.
template <int Q>
constexpr int kBulkMinBlocks = 4;

constexpr int kTX = 32, kTY = 8, kThreads = kTX * kTY;
constexpr int kHX = kTX + 4, kHY = kTY + 4; // phi ring (halo 2)
constexpr int kNX = kTX + 2, kNY = kTY + 2; // normal ring (halo 1)

// Shared-memory boxes of g for the phi halo, filled by TMA: per stage, one box
// per D3Q7 direction q, kHY rows x WX columns starting at
// (x0 - XH, y0 - 2 - c_qy, plane - c_qz), so that the value direction q
// contributes to halo cell (hx, hy) sits at row hy, column hx + XH - 2 - c_qx.
template <class TG>
struct GBox {
    static constexpr int XH = 16 / (int)sizeof(TG); // halo columns: 16-byte aligned box start
    static constexpr int WX = kTX + 2 * XH;
    static constexpr int BOX = WX * kHY;                       // elements per box
    static constexpr uint32_t BOX_BYTES = BOX * sizeof(TG);     // multiple of 128
    static constexpr uint32_t STAGE_BYTES = 7 * BOX_BYTES;
    static constexpr size_t SMEM = 2 * (size_t)STAGE_BYTES + 64; // two stages + barriers + flag
};

// Shared-memory slabs of the populations of one z plane, filled by TMA (the
// slab path): per direction q one box of kTY rows x WX columns starting at
// (x0 - XH or x0, y0 - c_qy, z - c_qz), so the value cell (tx, ty) pulls from
// direction q sits at row ty, column tx - c_qx + (c_qx < 0 ? 0 : XH).
template <class T>
struct Slab {
    static constexpr int XH = 16 / (int)sizeof(T); // 16-byte aligned left start
    static constexpr int WX = kTX + XH;
    static constexpr int ELEMS = WX * kTY;
    static constexpr uint32_t BYTES = ELEMS * sizeof(T); // multiple of 128
    template <int cx>
    static constexpr int col0() { return cx < 0 ? 1 : XH - cx; } // column of tx = 0
    template <int Q>
    static constexpr size_t smem() { return 2 * (size_t)(Q + 7) * BYTES + 64; }
};

// Threads 0 .. kPhiBorder - 1 each fill one element of the phi ring's
// 2-cell border on every plane (the others fill only their own column).
constexpr int kPhiBorder = kHX * kHY - kThreads; // 176
constexpr uint32_t kNoCell = 0xFFFFFFFFu;
static_assert(kHX * kHY <= 1024, "a ring position fits the 10 bits BulkSmem::bpack gives it");

struct BulkSmem {
    float phiZ[6][kHY][kHX]; // phi as computeForces sees it (ghost / outside read as 0)
    float nrm[3][4][kNY][kNX]; // n_x, n_y, n_z, |grad phi| on the zeroed field
    float carry[11][kThreads]; // gradient and curvature carries, one column per thread
    // the border element of thread tid, the same on every plane of a work
    // item: its in-plane cell index (kNoCell where the element is a ghost or
    // outside cell in x or y) and, packed, its position in a ring plane
    // (hy * kHX + hx, bits 0-9) and which of its x-1, x+1, y-1, y+1
    // neighbours wrap an exact-periodic axis (bits 10-13); 1 KB, so that four
    // blocks (of the batched kernel too) stay within the 164 KB shared-memory
    // carve-out and leave the L1 cache its 92 KB
    uint32_t bcell[kPhiBorder];
    uint16_t bpack[kPhiBorder];
};

// Ring slot of plane p; planes never go below -2, so the unsigned form is exact.
__device__ __forceinline__ int ringP(int p) { return (int)((unsigned)(p + 12) % 6u); } // phi: 6 planes
__device__ __forceinline__ int ringN(int p) { return (int)((unsigned)(p + 3) % 3u); }  // normals: 3 planes

template <int Q, class TF, class TG>
struct Bulk {
    using A = StepArgs<TF, TG>;

    // phi^n at fluid cell (x, y, z) with linear index c, from the post-stream
    // phase populations (pull layout: direction q is read at c - c_q).
    static __device__ __forceinline__ float phi_from_g(const A &a, int x, int y, int z, uint32_t c) {
        float g[7];
        gather_g(a, x, y, z, c, g);
        return (((((g[0] + g[1]) + g[2]) + g[3]) + g[4]) + g[5]) + g[6];
    }

    // The 7 post-stream phase populations of fluid cell (x, y, z), index c.
    static __device__ __forceinline__ void gather_g(const A &a, int x, int y, int z, uint32_t c, float (&g)[7]) {
        const Geometry &G = a.geo;
        // 32-bit source cell indices (pull: direction q is read at c - c_q); a
        // fluid cell only wraps on an exact-periodic axis, selected per lane
        // (no branch, so a warp never runs two paths).  Population q of cell i
        // is then one wide multiply-add away from the warp-uniform base g + q N.
        // The loads keep their lines in L2 (evict-last): the neighbouring
        // tiles' ring borders and this cell's own update read them again.
        const uint32_t xm = c + (x == 0 ? G.nx - 1 : (uint32_t)-1);
        const uint32_t xp = c + (x == (int)G.nx - 1 ? (uint32_t)(1 - (int)G.nx) : 1u);
        const uint32_t ym = c + (y == 0 ? G.nxy - G.nx : (uint32_t)-(int)G.nx);
        const uint32_t yp = c + (y == (int)G.ny - 1 ? (uint32_t)-(int)(G.nxy - G.nx) : G.nx);
        const uint32_t zm = c + (z == 0 ? (uint32_t)(G.cells - G.nxy) : (uint32_t)-(int)G.nxy);
        const uint32_t zp = c + (z == (int)G.nz - 1 ? (uint32_t)-(int64_t)(G.cells - G.nxy) : G.nxy);
        g[0] = Store<TG>::ld_keep(a.gq_src[0] + c);
        g[1] = Store<TG>::ld_keep(a.gq_src[1] + xm);
        g[2] = Store<TG>::ld_keep(a.gq_src[2] + xp);
        g[3] = Store<TG>::ld_keep(a.gq_src[3] + ym);
        g[4] = Store<TG>::ld_keep(a.gq_src[4] + yp);
        g[5] = Store<TG>::ld_keep(a.gq_src[5] + zm);
        g[6] = Store<TG>::ld_keep(a.gq_src[6] + zp);
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

    // The phi ring of a plane (36 x 12 cells: the tile and a 2-cell border)
    // is filled one element per thread for the thread's own column and one
    // more for tid < kPhiBorder, which covers the border: rows 0-1 and 10-11,
    // then columns 0, 1, 34, 35 of rows 2-9.
    static __device__ __forceinline__ void phi_border_pos(int tid, int &hx, int &hy) {
        if (tid < 2 * kHX) {
            hy = tid / kHX;
            hx = tid - hy * kHX;
        } else if (tid < 4 * kHX) {
            const int k = tid - 2 * kHX, r = k / kHX;
            hy = kHY - 2 + r;
            hx = k - r * kHX;
        } else {
            const int k = tid - 4 * kHX, c = k & 3;
            hy = 2 + (k >> 2);
            hx = c < 2 ? c : kHX - 4 + c;
        }
    }

    // Thread tid's border element, once per work item (BulkSmem::bcell, bpack).
    static __device__ void border_setup(const A &a, BulkSmem &S, int x0, int y0, int tid) {
        const Geometry &G = a.geo;
        int hx, hy;
        phi_border_pos(tid, hx, hy);
        const int bx = halo_axis(a, x0 - 2 + hx, G.nx, G.bcx == BC_PERIODIC);
        const int by = halo_axis(a, y0 - 2 + hy, G.ny, G.bcy == BC_PERIODIC);
        const bool fl = bx >= G.x_lo && bx <= G.x_hi && by >= G.y_lo && by <= G.y_hi;
        S.bcell[tid] = fl ? (uint32_t)bx + G.nx * (uint32_t)by : kNoCell;
        S.bpack[tid] = (uint16_t)((hy * kHX + hx) | (bx == 0 ? 1 << 10 : 0) | (bx == (int)G.nx - 1 ? 1 << 11 : 0) |
                                  (by == 0 ? 1 << 12 : 0) | (by == (int)G.ny - 1 ? 1 << 13 : 0));
    }

    // The 7 phase populations of fluid cell c (lattice index) whose in-plane
    // neighbours wrap as `wrap` says (bits 10-13 of BulkSmem::bpack), on plane
    // gz: the gathers of phi_from_g.
    static __device__ __forceinline__ void border_gather(const A &a, uint32_t c, uint32_t wrap, int gz,
                                                         float (&g)[7]) {
        const Geometry &G = a.geo;
        const uint32_t xm = c + ((wrap & (1u << 10)) ? G.nx - 1 : (uint32_t)-1);
        const uint32_t xp = c + ((wrap & (1u << 11)) ? (uint32_t)(1 - (int)G.nx) : 1u);
        const uint32_t ym = c + ((wrap & (1u << 12)) ? G.nxy - G.nx : (uint32_t)-(int)G.nx);
        const uint32_t yp = c + ((wrap & (1u << 13)) ? (uint32_t)-(int)(G.nxy - G.nx) : G.nx);
        const uint32_t zm = c + (gz == 0 ? (uint32_t)(G.cells - G.nxy) : (uint32_t)-(int)G.nxy);
        const uint32_t zp = c + (gz == (int)G.nz - 1 ? (uint32_t)-(int64_t)(G.cells - G.nxy) : G.nxy);
        g[0] = Store<TG>::ld_keep(a.gq_src[0] + c);
        g[1] = Store<TG>::ld_keep(a.gq_src[1] + xm);
        g[2] = Store<TG>::ld_keep(a.gq_src[2] + xp);
        g[3] = Store<TG>::ld_keep(a.gq_src[3] + ym);
        g[4] = Store<TG>::ld_keep(a.gq_src[4] + yp);
        g[5] = Store<TG>::ld_keep(a.gq_src[5] + zm);
        g[6] = Store<TG>::ld_keep(a.gq_src[6] + zp);
    }
    static __device__ __forceinline__ float sum7(const float (&g)[7]) {
        return (((((g[0] + g[1]) + g[2]) + g[3]) + g[4]) + g[5]) + g[6];
    }

    // Fill ring slot of plane pz with phi over the tile + 2-cell halo: fluid
    // cells from g, ghost and outside cells 0 (the field computeForces sees,
    // phaseField.cuh:118-142).  Both of a thread's elements gather before
    // either sum, so their load latencies overlap.
    static __device__ void fill_phi(const A &a, BulkSmem &S, int x0, int y0, int pz, int tid) {
        const Geometry &G = a.geo;
        const bool px = G.bcx == BC_PERIODIC, py = G.bcy == BC_PERIODIC;
        const int gz = halo_axis(a, pz, G.nz, G.bcz == BC_PERIODIC);
        const int s = ringP(pz);
        const bool zfluid = gz >= G.z_lo && gz <= G.z_hi; // (gz = -1 outside a non-periodic axis)
        auto fluid_xy = [&](int gx, int gy) { return gx >= G.x_lo && gx <= G.x_hi && gy >= G.y_lo && gy <= G.y_hi; };
        const int tx = tid % kTX, ty = tid / kTX;
        const int ox = halo_axis(a, x0 + tx, G.nx, px), oy = halo_axis(a, y0 + ty, G.ny, py);
        const bool fo = zfluid && fluid_xy(ox, oy);
        const bool border = tid < kPhiBorder;
        int hx = 0, hy = 0, bx = 0, by = 0;
        if (border) {
            phi_border_pos(tid, hx, hy);
            bx = halo_axis(a, x0 - 2 + hx, G.nx, px);
            by = halo_axis(a, y0 - 2 + hy, G.ny, py);
        }
        const bool fb = border && zfluid && fluid_xy(bx, by);
        float go[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, gb[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (fo) gather_g(a, ox, oy, gz, cell_index(G, ox, oy, gz), go);
        if (fb) gather_g(a, bx, by, gz, cell_index(G, bx, by, gz), gb);
        S.phiZ[s][ty + 2][tx + 2] = (((((go[0] + go[1]) + go[2]) + go[3]) + go[4]) + go[5]) + go[6];
        if (border) S.phiZ[s][hy][hx] = (((((gb[0] + gb[1]) + gb[2]) + gb[3]) + gb[4]) + gb[5]) + gb[6];
    }

    static __device__ __forceinline__ float tofloat(float v) { return v; }
    static __device__ __forceinline__ float tofloat(__half v) { return __half2float(v); }
    static __device__ __forceinline__ float tofloat(half_g32 v) { return __half2float(v.h); }
    static __device__ __forceinline__ float tofloat(__nv_bfloat16 v) { return __bfloat162float(v); }

    // Same as fill_phi, with the g values of fluid cells taken from the TMA
    // boxes of this plane; cells whose 7-point stencil wraps an exact-periodic
    // axis (outside the boxes) fall back to the gather.
    static __device__ void fill_phi_box(const A &a, BulkSmem &S, const TG *B, int x0, int y0, int pz,
                                        int tid) {
        using GB = GBox<TG>;
        const Geometry &G = a.geo;
        const bool px = G.bcx == BC_PERIODIC, py = G.bcy == BC_PERIODIC;
        const int gz = halo_axis(a, pz, G.nz, G.bcz == BC_PERIODIC);
        const int s = ringP(pz);
        const bool zfluid = gz >= G.z_lo && gz <= G.z_hi;
        for (int i = tid; i < kHX * kHY; i += kThreads) {
            const int hx = i % kHX, hy = i / kHX;
            const int rx = x0 - 2 + hx, ry = y0 - 2 + hy;
            const int gx = halo_axis(a, rx, G.nx, px);
            const int gy = halo_axis(a, ry, G.ny, py);
            float v = 0.f;
            if (zfluid && gx >= G.x_lo && gx <= G.x_hi && gy >= G.y_lo && gy <= G.y_hi) {
                const bool edge = (px && (rx < 1 || rx > (int)G.nx - 2)) || (py && (ry < 1 || ry > (int)G.ny - 2));
                if (edge) {
                    v = phi_from_g(a, gx, gy, gz, cell_index(G, gx, gy, gz));
                } else {
                    const int col = hy * GB::WX + hx + GB::XH - 2;
                    v = tofloat(B[0 * GB::BOX + col]);
                    v += tofloat(B[1 * GB::BOX + col - 1]);
                    v += tofloat(B[2 * GB::BOX + col + 1]);
                    v += tofloat(B[3 * GB::BOX + col]);
                    v += tofloat(B[4 * GB::BOX + col]);
                    v += tofloat(B[5 * GB::BOX + col]);
                    v += tofloat(B[6 * GB::BOX + col]);
                }
            }
            S.phiZ[s][hy][hx] = v;
        }
    }

    // Thread 0: TMA loads of the 7 g boxes phi of plane pz needs.
    static __device__ void issue_boxes(const A &a, const CUtensorMap *map, TG *B, uint64_t *bar, int x0,
                                       int y0, int pz) {
        using GB = GBox<TG>;
        const Geometry &G = a.geo;
        const bool pzp = G.bcz == BC_PERIODIC;
        fence_proxy_async();
        mbar_arrive_expect_tx(bar, GB::STAGE_BYTES);
        unroll<0, 7>([&](auto q) {
            constexpr int cy = cy27(q), cz = cz27(q);
            const int zq = pzp ? axis_halo(pz - cz, G.nz, true) : pz - cz;
            tma_load_4d(B + q * GB::BOX, map, x0 - GB::XH, y0 - 2 - cy, zq, q, bar);
        });
    }

    // One work item on the gather path: the 32 x 8 column at (x0, y0) over
    // planes [zs, ze).  One barrier per plane: iteration z updates plane z
    // and fills the normals of plane z + 2 and phi of plane z + 4, which
    // later iterations read; the ring slots they overwrite (z - 1, z - 2)
    // were last read before the previous barrier, so the gathers of the
    // cell update and the stencil arithmetic of the fills interleave freely.
    // Ends with a block-wide barrier.  BORDER_PRE: the phi ring's border
    // element from its sources found once per work item (border_setup);
    // otherwise found on every plane, which the batched kernel keeps (its
    // extra live state spills more with the precompute: 18 872 against
    // 19 590 MLUPS on the 48-lattice sweep, measured back to back).  Both
    // give the same bits.
    template <bool BORDER_PRE = true>
    static __device__ void run_gather(const A &a, BulkSmem &S, int x0, int y0, int zs, int ze, int tx, int ty,
                                      int tid) {
        const Geometry &G = a.geo;
        const int x = x0 + tx, y = y0 + ty;
        const bool active = x >= G.x_lo && x <= G.x_hi && y >= G.y_lo && y <= G.y_hi;
        for (int p = zs - 2; p <= zs + 3; ++p) fill_phi(a, S, x0, y0, p, tid);
        if (BORDER_PRE && tid < kPhiBorder) border_setup(a, S, x0, y0, tid); // read back by this thread only
        __syncthreads();
        GradCarry gc(S, tid);
        gc.start(S.phiZ[ringP(zs - 2)], S.phiZ[ringP(zs - 1)], tx + 2, ty + 2);
        for (int p = zs - 1; p <= zs + 1; ++p) fill_nrm_carry(S, p, tid, gc);
        __syncthreads();
        Curv cv(S, tid);
        cv.start(S, zs, tx, ty);
        __syncthreads();
        for (int z = zs; z < ze; ++z) {
            // the plane terms after the population gathers are issued (D3Q19:
            // before them, measured faster on B200 for FP32 and 16-bit storage)
            constexpr bool kEarly = Q == 19;
            if (active) cell_lazy<kEarly>(a, S, x, y, z, tx, ty, [&] { return cv.advance(S, z, tx, ty); });
            else cv.advance(S, z, tx, ty);
            {
                // fill_phi(z + 4) split around the normals of plane z + 2: the own
                // column's 7 gathers are in flight while the normals are computed,
                // then its sum and the border element (ghost / outside: 0)
                const bool more = z + 4 <= ze + 1;
                const int gz = halo_axis(a, z + 4, G.nz, G.bcz == BC_PERIODIC);
                const bool zf = gz >= G.z_lo && gz <= G.z_hi;
                const int ox = halo_axis(a, x, G.nx, G.bcx == BC_PERIODIC);
                const int oy = halo_axis(a, y, G.ny, G.bcy == BC_PERIODIC);
                float go[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (more && zf && ox >= G.x_lo && ox <= G.x_hi && oy >= G.y_lo && oy <= G.y_hi)
                    gather_g(a, ox, oy, gz, cell_index(G, ox, oy, gz), go);
                if (z + 2 <= ze) fill_nrm_carry(S, z + 2, tid, gc);
                if (more) {
                    const int sp = ringP(z + 4);
                    S.phiZ[sp][ty + 2][tx + 2] = sum7(go);
                    if (BORDER_PRE && tid < kPhiBorder) {
                        // the border element: its cell and wraps from border_setup
                        const uint32_t c = S.bcell[tid], pk = S.bpack[tid];
                        float v = 0.f;
                        if (zf && c != kNoCell) {
                            float gb[7];
                            border_gather(a, c + (uint32_t)gz * G.nxy, pk, gz, gb);
                            v = sum7(gb);
                        }
                        (&S.phiZ[sp][0][0])[pk & 0x3FFu] = v;
                    } else if (!BORDER_PRE && tid < kPhiBorder) {
                        int hx, hy;
                        phi_border_pos(tid, hx, hy);
                        const int bx = halo_axis(a, x0 - 2 + hx, G.nx, G.bcx == BC_PERIODIC);
                        const int by = halo_axis(a, y0 - 2 + hy, G.ny, G.bcy == BC_PERIODIC);
                        float v = 0.f;
                        if (zf && bx >= G.x_lo && bx <= G.x_hi && by >= G.y_lo && by <= G.y_hi)
                            v = phi_from_g(a, bx, by, gz, cell_index(G, bx, by, gz));
                        S.phiZ[sp][hy][hx] = v;
                    }
                }
            }
            __syncthreads();
        }
    }

    // Thread 0: TMA loads of the population slabs of plane z (f, and g when the
    // phase field relaxes with omega_g != 1).
    static __device__ void issue_slabs(const A &a, const CUtensorMap *fmap, const CUtensorMap *gmap, TF *Fs,
                                       TG *Gs, uint64_t *bar, int x0, int y0, int z) {
        const Geometry &G = a.geo;
        const bool pzp = G.bcz == BC_PERIODIC;
        const bool bgk = a.phys.omega_g != 1.0f;
        fence_proxy_async();
        mbar_arrive_expect_tx(bar, (uint32_t)(Q + (bgk ? 7 : 0)) * Slab<TF>::BYTES);
        unroll<0, Q>([&](auto q) {
            constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
            const int zq = pzp ? axis_halo(z - cz, G.nz, true) : z - cz;
            tma_load_4d(Fs + q * Slab<TF>::ELEMS, fmap, cx < 0 ? x0 : x0 - Slab<TF>::XH, y0 - cy, zq, q, bar);
        });
        if (bgk)
            unroll<0, 7>([&](auto q) {
                constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
                const int zq = pzp ? axis_halo(z - cz, G.nz, true) : z - cz;
                tma_load_4d(Gs + q * Slab<TG>::ELEMS, gmap, cx < 0 ? x0 : x0 - Slab<TG>::XH, y0 - cy, zq, q, bar);
            });
    }

    // Isotropic gradient 3 sum_q w_q c_q phi(x + c_q) with the hydrodynamic
    // set's weights (phaseField.cuh:158-218); (hx, hy) is the centre in ring
    // coordinates, p0 the centre plane.
    template <class Ring>
    static __device__ __forceinline__ void grad(const Ring &R, int hx, int hy, int sm, int s0, int sp,
                                                float &gx, float &gy, float &gz) {
        grad_at(
            [&](int dx, int dy, int dz) -> float {
                const int sl = dz < 0 ? sm : (dz > 0 ? sp : s0);
                return R[sl][hy + dy][hx + dx];
            },
            gx, gy, gz);
    }

    // The same gradient of the field phi(dx, dy, dz) around the centre.
    template <class At>
    static __device__ __forceinline__ void grad_at(At &&at, float &gx, float &gy, float &gz) {
        float sx = 0.f, sy = 0.f, sz = 0.f;
        unroll<0, (Q - 1) / 2>([&](auto k) {
            constexpr int q = 2 * k + 1;
            constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
            constexpr float w = (q <= 6) ? VS<Q>::w1 : (q <= 18 ? VS<Q>::w2 : VS<Q>::w3);
            // explicit fused forms: every instantiation rounds alike
            const float d = at(cx, cy, cz) - at(-cx, -cy, -cz);
            if constexpr (cx != 0) sx = fmaf(cx > 0 ? w : -w, d, sx);
            if constexpr (cy != 0) sy = fmaf(cy > 0 ? w : -w, d, sy);
            if constexpr (cz != 0) sz = fmaf(cz > 0 ? w : -w, d, sz);
        });
        gx = 3.0f * sx;
        gy = 3.0f * sy;
        gz = 3.0f * sz;
    }

    // The normal ring (34 x 10) is filled like the phi ring: the thread's own
    // column, and for tid < kNrmBorder one element of the 1-cell border (rows 0
    // and 9, then columns 0 and 33 of rows 1-8).
    static constexpr int kNrmBorder = kNX * kNY - kThreads; // 84
    static __device__ __forceinline__ void nrm_border_pos(int tid, int &nxh, int &nyh) {
        if (tid < kNX) {
            nxh = tid;
            nyh = 0;
        } else if (tid < 2 * kNX) {
            nxh = tid - kNX;
            nyh = kNY - 1;
        } else {
            const int k = tid - 2 * kNX;
            nyh = 1 + (k >> 1);
            nxh = (k & 1) ? kNX - 1 : 0;
        }
    }


    // Normal, |grad phi| of one ring element from its gradient.
    static __device__ __forceinline__ void store_nrm(BulkSmem &S, int s, int nxh, int nyh, float gx, float gy,
                                                     float gz) {
        const float ind = sqrt_sfu(fmaf(gx, gx, fmaf(gy, gy, gz * gz)));
        const float inv = rcp_sfu(ind + 1e-9f); // 1 / (ind + 1e-9)
        S.nrm[s][0][nyh][nxh] = gx * inv;
        S.nrm[s][1][nyh][nxh] = gy * inv;
        S.nrm[s][2][nyh][nxh] = gz * inv;
        S.nrm[s][3][nyh][nxh] = ind;
    }

    static __device__ __forceinline__ void nrm_elem(BulkSmem &S, int s, int sm, int s0, int sp, int nxh, int nyh) {
        float gx, gy, gz;
        grad(S.phiZ, nxh + 1, nyh + 1, sm, s0, sp, gx, gy, gz);
        store_nrm(S, s, nxh, nyh, gx, gy, gz);
    }

    // Gradient of phi along the thread's own column from in-plane partial sums
    // carried from plane to plane.  With the stencil weights of the velocity
    // set the isotropic gradient 3 sum_q w_q c_q phi(x + c_q)
    // (phaseField.cuh:158-218) splits by planes:
    //   D3Q27, w = b(c_x) b(c_y) b(c_z) / 216 with b(0) = 4, b(+-1) = 1:
    //     g_x(p) = 3/216 [Gx(p-1) + 4 Gx(p) + Gx(p+1)],  Gx = D_x S_y phi
    //     g_y(p) = 3/216 [Gy(p-1) + 4 Gy(p) + Gy(p+1)],  Gy = D_y S_x phi
    //     g_z(p) = 3/216 [Sxy(p+1) - Sxy(p-1)],          Sxy = S_x S_y phi
    //   D3Q19, w = 2/36 on the faces and 1/36 on the edges:
    //     g_x(p) = 3/36 [Cx(p) + Ax(p-1) + Ax(p+1)],  Ax = D_x phi,
    //              Cx = 2 Ax + D_x phi(y + 1) + D_x phi(y - 1)  (same for y)
    //     g_z(p) = 3/36 [T(p+1) - T(p-1)],  T = 2 phi + the 4 in-plane neighbours
    // where S is the 1-4-1 sum and D the central difference along one axis.
    // Each plane's 3 x 3 neighbourhood is read once (9 loads, not 18 / 26).
    // The carried sums: plane p - 1: Gx, Gy, Sxy (D3Q27) / Ax, Ay, T (D3Q19);
    // plane p: the same, and Cx, Cy (D3Q19).  They live in the thread's column
    // of BulkSmem::carry (rows 0-7), which frees the registers of the
    // 4-blocks-per-SM budget.
    struct GradCarry {
        float *col; // &BulkSmem::carry[0][tid]
        __device__ __forceinline__ GradCarry(BulkSmem &S, int tid) : col(&S.carry[0][tid]) {}
        __device__ __forceinline__ float &v(int k) { return col[k * kThreads]; }
        __device__ __forceinline__ float &px() { return v(0); }
        __device__ __forceinline__ float &py() { return v(1); }
        __device__ __forceinline__ float &pz() { return v(2); }
        __device__ __forceinline__ float &cx() { return v(3); }
        __device__ __forceinline__ float &cy() { return v(4); }
        __device__ __forceinline__ float &cz() { return v(5); }
        __device__ __forceinline__ float &ccx() { return v(6); }
        __device__ __forceinline__ float &ccy() { return v(7); }

        // partials of ring plane P at ring position (hx, hy)
        static __device__ __forceinline__ void partials(const float (&P)[kHY][kHX], int hx, int hy, float &a,
                                                        float &b, float &c, float &d, float &e) {
            auto f = [&](int i, int j) { return P[hy + j][hx + i]; };
            if constexpr (Q == 27) {
                const float sym = fmaf(4.0f, f(-1, 0), f(-1, -1) + f(-1, 1));
                const float sy0 = fmaf(4.0f, f(0, 0), f(0, -1) + f(0, 1));
                const float syp = fmaf(4.0f, f(1, 0), f(1, -1) + f(1, 1));
                const float sxm = fmaf(4.0f, f(0, -1), f(-1, -1) + f(1, -1));
                const float sxp = fmaf(4.0f, f(0, 1), f(-1, 1) + f(1, 1));
                a = syp - sym;
                b = sxp - sxm;
                c = fmaf(4.0f, sy0, sym + syp);
                d = e = 0.0f;
            } else {
                a = f(1, 0) - f(-1, 0);
                b = f(0, 1) - f(0, -1);
                c = fmaf(2.0f, f(0, 0), (f(1, 0) + f(-1, 0)) + (f(0, 1) + f(0, -1)));
                d = fmaf(2.0f, a, (f(1, 1) - f(-1, 1)) + (f(1, -1) - f(-1, -1)));
                e = fmaf(2.0f, b, (f(1, 1) - f(1, -1)) + (f(-1, 1) - f(-1, -1)));
            }
        }
        // planes p - 1 and p enter (ring planes Pm, P0)
        __device__ __forceinline__ void start(const float (&Pm)[kHY][kHX], const float (&P0)[kHY][kHX], int hx,
                                              int hy) {
            float a, b, c, d, e;
            partials(Pm, hx, hy, a, b, c, d, e);
            px() = a;
            py() = b;
            pz() = c;
            partials(P0, hx, hy, a, b, c, d, e);
            cx() = a;
            cy() = b;
            cz() = c;
            ccx() = d;
            ccy() = e;
        }
        // plane p + 1 enters: gradient at plane p
        __device__ __forceinline__ void advance(const float (&Pp)[kHY][kHX], int hx, int hy, float &gx, float &gy,
                                                float &gz) {
            float a, b, c, d, e;
            partials(Pp, hx, hy, a, b, c, d, e);
            if constexpr (Q == 27) {
                constexpr float k = float(3.0 / 216.0);
                gx = k * fmaf(4.0f, cx(), px() + a);
                gy = k * fmaf(4.0f, cy(), py() + b);
                gz = k * (c - pz());
            } else {
                constexpr float k = float(3.0 / 36.0);
                gx = k * (ccx() + (px() + a));
                gy = k * (ccy() + (py() + b));
                gz = k * (c - pz());
            }
            px() = cx();
            py() = cy();
            pz() = cz();
            cx() = a;
            cy() = b;
            cz() = c;
            ccx() = d;
            ccy() = e;
        }
    };

    // Normals and |grad phi| of plane pz over the tile + 1-cell halo: the
    // thread's own column from its carried partial sums (planes pz - 1 and pz
    // in gc; plane pz + 1 must be in the phi ring), the border element (tid <
    // kNrmBorder) from the full stencil.
    static __device__ void fill_nrm_carry(BulkSmem &S, int pz, int tid, GradCarry &gc) {
        const int s = ringN(pz);
        const int tx = tid % kTX, ty = tid / kTX;
        float gx, gy, gz;
        gc.advance(S.phiZ[ringP(pz + 1)], tx + 2, ty + 2, gx, gy, gz);
        store_nrm(S, s, tx + 1, ty + 1, gx, gy, gz);
        if (tid < kNrmBorder) {
            const int sm = ringP(pz - 1), s0 = ringP(pz), sp = ringP(pz + 1);
            int nxh, nyh;
            nrm_border_pos(tid, nxh, nyh);
            nrm_elem(S, s, sm, s0, sp, nxh, nyh);
        }
    }

    // Curvature by planes.  The divergence 3 sum_q w_q c_q . n(x + c_q)
    // (phaseField.cuh:246-275) groups by c_qz: the plane of the cell itself
    // contributes C, each neighbouring plane z +- 1 contributes S +- Z, where
    // (dx, dy) runs over the 3 x 3 in-plane pattern of the velocity set:
    //   C = w1 A + w2 B,  S = w2 A + w3 B,  Z = w1 nz + w2 (4 edge nz) + w3 (4 corner nz)
    //   A = nx(+1, 0) - nx(-1, 0) + ny(0, +1) - ny(0, -1)
    //   B = sum over the 4 corners (dx, dy) of dx nx + dy ny
    // (w3 = 0 for D3Q19).  Every thread evaluates them once per plane for its
    // own column and keeps those of the previous planes in its column of
    // shared memory (Curv), so the cell update combines three carried sums
    // instead of reading the full 3 x 3 x 3 stencil of normals.
    static __device__ __forceinline__ void plane_terms(const BulkSmem &S, int pz, int tx, int ty, float &C,
                                                       float &Sv, float &Zv) {
        const int s = ringN(pz);
        const int cx = tx + 1, cy = ty + 1;
        auto nx = [&](int dx, int dy) { return S.nrm[s][0][cy + dy][cx + dx]; };
        auto ny = [&](int dx, int dy) { return S.nrm[s][1][cy + dy][cx + dx]; };
        auto nz = [&](int dx, int dy) { return S.nrm[s][2][cy + dy][cx + dx]; };
        const float A = (nx(1, 0) - nx(-1, 0)) + (ny(0, 1) - ny(0, -1));
        const float B = ((nx(1, 1) - nx(-1, 1)) + (nx(1, -1) - nx(-1, -1))) +
                        ((ny(1, 1) - ny(1, -1)) + (ny(-1, 1) - ny(-1, -1)));
        const float E = (nz(1, 0) + nz(-1, 0)) + (nz(0, 1) + nz(0, -1));
        C = fmaf(VS<Q>::w1, A, VS<Q>::w2 * B);
        if constexpr (Q == 27) {
            const float K = (nz(1, 1) + nz(-1, 1)) + (nz(1, -1) + nz(-1, -1));
            Sv = fmaf(VS<Q>::w2, A, VS<Q>::w3 * B);
            Zv = fmaf(VS<Q>::w1, nz(0, 0), fmaf(VS<Q>::w2, E, VS<Q>::w3 * K));
        } else {
            Sv = VS<Q>::w2 * A;
            Zv = fmaf(VS<Q>::w1, nz(0, 0), VS<Q>::w2 * E);
        }
    }

    // Per-thread curvature state along the column: C of the current plane and
    // S - Z of the current and previous planes, in rows 8-10 of the thread's
    // column of BulkSmem::carry.
    struct Curv {
        float *col;
        __device__ __forceinline__ Curv(BulkSmem &S, int tid) : col(&S.carry[8][tid]) {}
        __device__ __forceinline__ float &prev_d() { return col[0]; }
        __device__ __forceinline__ float &cur_c() { return col[kThreads]; }
        __device__ __forceinline__ float &cur_d() { return col[2 * kThreads]; }
        // planes zs - 1 and zs must be in the normal ring; ends before any
        // thread may overwrite plane zs - 1 (the caller's next barrier)
        __device__ __forceinline__ void start(const BulkSmem &S, int zs, int tx, int ty) {
            float c, sv, zv;
            plane_terms(S, zs - 1, tx, ty, c, sv, zv);
            prev_d() = sv - zv;
            plane_terms(S, zs, tx, ty, c, sv, zv);
            cur_c() = c;
            cur_d() = sv - zv;
        }
        // plane z + 1 just entered the ring: returns the divergence at plane z
        __device__ __forceinline__ float advance(const BulkSmem &S, int z, int tx, int ty) {
            float c, sv, zv;
            plane_terms(S, z + 1, tx, ty, c, sv, zv);
            const float div = cur_c() + (sv + zv) + prev_d();
            prev_d() = cur_d();
            cur_c() = c;
            cur_d() = sv - zv;
            return div;
        }
    };

    // Update of one fluid cell (x, y, z); (tx, ty) its position in the tile.
    // fs / gs: this plane's population slabs (slab path) or null (gather path).
    static __device__ __forceinline__ void cell(const A &a, const BulkSmem &S, int x, int y, int z,
                                                int tx, int ty, float div, const TF *fs = nullptr,
                                                const TG *gs = nullptr) {
        cell_lazy(a, S, x, y, z, tx, ty, [div] { return div; }, fs, gs);
    }

    // cell() with the normal divergence produced by divfn() after the
    // population gathers are issued, so that their latency covers the plane
    // terms (the gather loop passes Curv::advance); EARLY evaluates it and the
    // surface tension before the gathers instead.
    template <bool EARLY = false, class DivFn>
    static __device__ __forceinline__ void cell_lazy(const A &a, const BulkSmem &S, int x, int y, int z, int tx,
                                                     int ty, DivFn &&divfn, const TF *fs = nullptr,
                                                     const TG *gs = nullptr) {
        const Geometry &G = a.geo;
        const Physics &P = a.phys;
        const bool px = G.bcx == BC_PERIODIC, py = G.bcy == BC_PERIODIC, pz = G.bcz == BC_PERIODIC;
        const uint32_t c0 = cell_index(G, x, y, z);

        // (the surface tension from the zeroed-ghost field, phaseField.cuh:246-293,
        // follows the gathers below: its divergence comes from the plane terms)
        const int hx = tx + 2, hy = ty + 2; // phi ring centre
        const int nxh = tx + 1, nyh = ty + 1; // normal ring centre
        const int s0 = ringN(z);
        auto nat = [&](int comp) -> float { return S.nrm[s0][comp][nyh][nxh]; };
        // surface tension: -sigma kappa |grad phi| n, kappa = 3 div
        auto tension = [&](float &fx, float &fy, float &fz) {
            const float curvature = 3.0f * divfn();
            const float sigma = a.clo_cs ? P.sigma * a.clo_cs[c0] : P.sigma;
            const float stc = -sigma * curvature * nat(3);
            fx = stc * nat(0);
            fy = stc * nat(1);
            fz = stc * nat(2);
        };
        float fx, fy, fz;
        if constexpr (EARLY) tension(fx, fy, fz);

        // ---- normals of the phase update from phi with ghost values (lbm.cu:157-224).
        // Away from ghost layers the raw and zeroed fields agree on the 3x3x3
        // neighbourhood, so the ring's normal is the same number.
        const bool near_ghost = (!px && (x <= G.x_lo || x >= G.x_hi)) ||
                                (!py && (y <= G.y_lo || y >= G.y_hi)) ||
                                (!pz && (z <= G.z_lo || z >= G.z_hi));
        float nx = nat(0), ny = nat(1), nz = nat(2);
        if (near_ghost) {
            // phi with ghost values: the ring's for fluid cells, the phi array
            // (written by the boundaries, constant during this kernel) for ghost
            // cells, 0 outside the lattice
            auto raw = [&](int dx, int dy, int dz) -> float {
                const int gx = axis_nb(x + dx, (int)G.nx, px), gy = axis_nb(y + dy, (int)G.ny, py);
                const int gz = axis_nb(z + dz, (int)G.nz, pz);
                if (gx < 0 || gy < 0 || gz < 0) return 0.f;
                if (fluid(G, gx, gy, gz)) return S.phiZ[ringP(z + dz)][hy + dy][hx + dx];
                return a.fld.phi[cell_index(G, gx, gy, gz)];
            };
            float gx, gy, gz;
            grad_at(raw, gx, gy, gz);
            const float ind = sqrtf(fmaf(gx, gx, fmaf(gy, gy, gz * gz)));
            const float inv = __frcp_rn(ind + 1e-9f);
            nx = gx * inv;
            ny = gy * inv;
            nz = gz * inv;
        }
        const float phi = S.phiZ[ringP(z)][hy][hx];

        // ---- gather f^n (after the stencil work, so that the Q values are live
        // only across the moments and the collision).  The source of direction q
        // is c0 - (cx + cy nx + cz nx ny), one warp-uniform offset per q, plus a
        // per-lane correction where an exact-periodic axis wraps (no branch, so
        // the warp holding the wrapping lane does not run two gathers).
        // Source cell of direction q: c0 + DX[cx] + DY[cy] + DZ[cz] in 32 bits,
        // the per-lane deltas already wrapped on exact-periodic axes.
        const uint64_t N = G.cells;
        const uint32_t dxm = (px && x == 0) ? G.nx - 1 : (uint32_t)-1;            // c_x = +1 reads x - 1
        const uint32_t dxp = (px && x == (int)G.nx - 1) ? (uint32_t)(1 - (int)G.nx) : 1u;
        const uint32_t dym = (py && y == 0) ? G.nxy - G.nx : (uint32_t)-(int)G.nx;
        const uint32_t dyp = (py && y == (int)G.ny - 1) ? (uint32_t)-(int)(G.nxy - G.nx) : G.nx;
        const uint32_t dzm = (pz && z == 0) ? (uint32_t)(N - G.nxy) : (uint32_t)-(int)G.nxy;
        const uint32_t dzp = (pz && z == (int)G.nz - 1) ? (uint32_t)-(int64_t)(N - G.nxy) : G.nxy;
        auto src = [&](auto q) -> uint32_t {
            constexpr int cx = cx27(q), cy = cy27(q), cz = cz27(q);
            uint32_t i = c0;
            if constexpr (cx > 0) i += dxm;
            if constexpr (cx < 0) i += dxp;
            if constexpr (cy > 0) i += dym;
            if constexpr (cy < 0) i += dyp;
            if constexpr (cz > 0) i += dzm;
            if constexpr (cz < 0) i += dzp;
            return i;
        };
        float f[Q];
        float gin[7];
        const bool bgk = a.phys.omega_g != 1.0f;
        if (fs == nullptr) {
            unroll<0, Q>([&](auto q) { f[q] = Store<TF>::ld(a.fq_src[q] + src(q)); });
            if (bgk) unroll<0, 7>([&](auto q) { gin[q] = Store<TG>::ld(a.gq_src[q] + src(q)); });
        } else {
            // slab path: immediate shared-memory offsets; lanes whose source wraps an
            // exact-periodic x or y axis (outside the slab) reload those directions
            unroll<0, Q>([&](auto q) {
                constexpr int cx = cx27(q);
                f[q] = tofloat(fs[q * Slab<TF>::ELEMS + ty * Slab<TF>::WX + tx + Slab<TF>::template col0<cx>()]);
            });
            if (bgk)
                unroll<0, 7>([&](auto q) {
                    constexpr int cx = cx27(q);
                    gin[q] = tofloat(gs[q * Slab<TG>::ELEMS + ty * Slab<TG>::WX + tx + Slab<TG>::template col0<cx>()]);
                });
            const bool wx0 = px && x == 0, wx1 = px && x == (int)G.nx - 1;
            const bool wy0 = py && y == 0, wy1 = py && y == (int)G.ny - 1;
            if (wx0 || wx1 || wy0 || wy1) {
                unroll<0, Q>([&](auto q) {
                    constexpr int cx = cx27(q), cy = cy27(q);
                    const bool w = (cx > 0 && wx0) || (cx < 0 && wx1) || (cy > 0 && wy0) || (cy < 0 && wy1);
                    if (w) f[q] = Store<TF>::ld(a.fq_src[q] + src(q));
                });
                if (bgk)
                    unroll<0, 7>([&](auto q) {
                        constexpr int cx = cx27(q), cy = cy27(q);
                        const bool w = (cx > 0 && wx0) || (cx < 0 && wx1) || (cy > 0 && wy0) || (cy < 0 && wy1);
                        if (w) gin[q] = Store<TG>::ld(a.gq_src[q] + src(q));
                    });
            }
        }

        if constexpr (!EARLY) tension(fx, fy, fz);

        // ---- hydrodynamics
        const Moments m = moments<Q>(f, fx, fy, fz);
        float nu = fmaf(phi, P.nu_oil_minus_water, P.nu_water);
        if (a.clo_nut) nu += a.clo_nut[c0];
        const float omega = rcp_sfu(fmaf(3.0f, nu, 0.5f)); // 1 / (0.5 + 3 nu)
        float fo[Q];
        collide<Q>(m, 1.0f - omega, fx, fy, fz, fo);
        unroll<0, Q>([&](auto q) { Store<TF>::st(a.fq_dst[q] + c0, fo[q]); });

        // ---- conservative Allen-Cahn update, D3Q7 (lbm.cu:256-269; D3Q7.cuh:124-148)
        const float sharp = P.gamma * phi * (1.0f - phi);
        float go[7];
        go[0] = kW7_0 * phi;
        const float phi4 = 4.0f * phi;
        const float ax = fmaf(phi4, m.ux, sharp * nx);
        const float ay = fmaf(phi4, m.uy, sharp * ny);
        const float az = fmaf(phi4, m.uz, sharp * nz);
        go[1] = kW7_1 * (phi + ax);
        go[2] = kW7_1 * (phi - ax);
        go[3] = kW7_1 * (phi + ay);
        go[4] = kW7_1 * (phi - ay);
        go[5] = kW7_1 * (phi + az);
        go[6] = kW7_1 * (phi - az);
        if (bgk) {
            // BGK with the anti-diffusion flux inside the equilibrium; omega_g = 1
            // reduces to the reference's g = g_eq + h.
            unroll<0, 7>([&](auto q) { go[q] = fmaf(P.omega_g, go[q] - gin[q], gin[q]); });
        }
        unroll<0, 7>([&](auto q) { Store<TG>::st(a.gq_dst[q] + c0, go[q]); });

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
        if (a.flags & SSMD_STEP_AVERAGE)
            accumulate_averages(a.avg, c0, (float)(a.status->avg_t + 1u), phi, m.ux, m.uy, m.uz);
        if (!isfinite(m.rho)) atomicOr(&a.status->flags, 1u);
    }
};

// Waits for TMA stages are bounded: after kTmaWaitNs without completion the
// block records status bit 1, waits (bounded again) for its own copies in
// flight and returns.
constexpr uint64_t kTmaWaitNs = 2000000000ull;

// PATH: 1 = per-cell gathers, 2 = TMA boxes for the phi halo, 3 = TMA slabs
// for the populations (phi halo by gathers).
template <int Q, class TF, class TG, int PATH>
__global__ void __launch_bounds__(kThreads, PATH == 3 ? 2 : kBulkMinBlocks<Q>)
    bulk_kernel(const StepArgs<TF, TG> a, const __grid_constant__ CUtensorMap gmap,
                const __grid_constant__ CUtensorMap fmap) {
    using B = Bulk<Q, TF, TG>;
    using GB = GBox<TG>;
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

    if constexpr (PATH == 3) {
        extern __shared__ __align__(128) unsigned char dyn3[];
        using SL = Slab<TF>;
        static_assert(sizeof(TF) == sizeof(TG), "a slab stage holds f and g slabs of one element size");
        constexpr size_t STAGE = (size_t)(Q + 7) * SL::BYTES;
        auto fstage = [&](int k) { return reinterpret_cast<TF *>(dyn3 + (k & 1) * STAGE); };
        auto gstage = [&](int k) { return reinterpret_cast<TG *>(dyn3 + (k & 1) * STAGE + (size_t)Q * SL::BYTES); };
        uint64_t *bars = reinterpret_cast<uint64_t *>(dyn3 + 2 * STAGE);
        volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 2);
        int issued = 0, consumed = 0; // thread 0 only
        if (tid == 0) {
            mbar_init(&bars[0], 1);
            mbar_init(&bars[1], 1);
            *abort_flag = 0;
            fence_barrier_init();
        }
        __syncthreads();
        auto issue = [&](int z) {
            if (tid == 0 && z < ze) {
                const int k = z - zs;
                B::issue_slabs(a, &fmap, &gmap, fstage(k), gstage(k), &bars[k & 1], x0, y0, z);
                ++issued;
            }
        };
        issue(zs);
        for (int p = zs - 2; p <= zs + 2; ++p) B::fill_phi(a, S, x0, y0, p, tid);
        __syncthreads();
        typename B::GradCarry gc(S, tid);
        gc.start(S.phiZ[ringP(zs - 2)], S.phiZ[ringP(zs - 1)], tx + 2, ty + 2);
        B::fill_nrm_carry(S, zs - 1, tid, gc);
        B::fill_nrm_carry(S, zs, tid, gc);
        __syncthreads();
        typename B::Curv cv(S, tid);
        cv.start(S, zs, tx, ty);
        __syncthreads();
        bool ok = true;
        for (int z = zs; z < ze; ++z) {
            const int k = z - zs;
            issue(z + 1);
            B::fill_nrm_carry(S, z + 1, tid, gc);
            if (tid == 0) {
                if (!mbar_wait_bounded(&bars[k & 1], (uint32_t)(k >> 1) & 1u, kTmaWaitNs)) *abort_flag = 1;
                else ++consumed;
            }
            __syncthreads();
            if (*abort_flag) {
                ok = false;
                break;
            }
            mbar_wait_bounded(&bars[k & 1], (uint32_t)(k >> 1) & 1u, kTmaWaitNs); // complete: visibility
            const float div = cv.advance(S, z, tx, ty);
            if (active) B::cell(a, S, x, y, z, tx, ty, div, fstage(k), gstage(k));
            if (z + 1 < ze) B::fill_phi(a, S, x0, y0, z + 3, tid);
            __syncthreads();
        }
        if (!ok && tid == 0) {
            atomicOr(&a.status->flags, 2u);
            for (int k = consumed; k < issued; ++k)
                mbar_wait_bounded(&bars[k & 1], (uint32_t)(k >> 1) & 1u, kTmaWaitNs);
        }
    } else if constexpr (PATH == 1) {
        B::run_gather(a, S, x0, y0, zs, ze, tx, ty, tid);
    } else {
        extern __shared__ __align__(128) unsigned char dyn[];
        TG *const stage0 = reinterpret_cast<TG *>(dyn);
        TG *const stage1 = reinterpret_cast<TG *>(dyn + GB::STAGE_BYTES);
        uint64_t *bars = reinterpret_cast<uint64_t *>(dyn + 2 * (size_t)GB::STAGE_BYTES);
        volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 2);
        const int p_first = zs - 2;
        const int p_last = max(zs + 2, ze + 1);
        int issued = 0, consumed = 0; // thread 0 only
        if (tid == 0) {
            mbar_init(&bars[0], 1);
            mbar_init(&bars[1], 1);
            *abort_flag = 0;
            fence_barrier_init();
        }
        __syncthreads();
        auto issue = [&](int p) {
            if (tid == 0 && p <= p_last) {
                const int k = p - p_first;
                B::issue_boxes(a, &gmap, (k & 1) ? stage1 : stage0, &bars[k & 1], x0, y0, p);
                ++issued;
            }
        };
        // thread 0 polls (bounded), then everybody learns the outcome after a barrier
        auto poll = [&](int p) {
            if (tid == 0) {
                const int k = p - p_first;
                if (!mbar_wait_bounded(&bars[k & 1], (uint32_t)(k >> 1) & 1u, kTmaWaitNs)) *abort_flag = 1;
                else ++consumed;
            }
        };
        auto confirm = [&](int p) {
            const int k = p - p_first;
            mbar_wait_bounded(&bars[k & 1], (uint32_t)(k >> 1) & 1u, kTmaWaitNs); // already complete
            return (k & 1) ? stage1 : stage0;
        };
        bool ok = true;
        issue(p_first);
        issue(p_first + 1);
        for (int p = zs - 2; p <= zs + 2 && ok; ++p) {
            poll(p);
            __syncthreads();
            if (*abort_flag) {
                ok = false;
                break;
            }
            B::fill_phi_box(a, S, confirm(p), x0, y0, p, tid);
            __syncthreads();
            issue(p + 2);
        }
        if (ok) {
            typename B::GradCarry gc(S, tid);
            gc.start(S.phiZ[ringP(zs - 2)], S.phiZ[ringP(zs - 1)], tx + 2, ty + 2);
            B::fill_nrm_carry(S, zs - 1, tid, gc);
            B::fill_nrm_carry(S, zs, tid, gc);
            __syncthreads();
            typename B::Curv cv(S, tid);
            cv.start(S, zs, tx, ty);
            __syncthreads();
            for (int z = zs; z < ze; ++z) {
                B::fill_nrm_carry(S, z + 1, tid, gc);
                const bool more = z + 1 < ze;
                if (more) poll(z + 3);
                __syncthreads();
                if (*abort_flag) {
                    ok = false;
                    break;
                }
                const float div = cv.advance(S, z, tx, ty);
                if (active) B::cell(a, S, x, y, z, tx, ty, div);
                if (more) B::fill_phi_box(a, S, confirm(z + 3), x0, y0, z + 3, tid);
                __syncthreads();
                if (more) issue(z + 5);
            }
        }
        if (!ok && tid == 0) {
            atomicOr(&a.status->flags, 2u);
            // wait (bounded) for this block's copies still in flight before leaving
            for (int k = consumed; k < issued; ++k)
                mbar_wait_bounded(&bars[k & 1], (uint32_t)(k >> 1) & 1u, kTmaWaitNs);
        }
    }
}

} // namespace ssmd
