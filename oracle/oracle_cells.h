// oracle_cells.h — the oracle's per-cell arithmetic.  TEST INFRASTRUCTURE.
//
// One restatement of the reference's time step, cell by cell, shared by the
// two instances of the oracle:
//   * ssmd_oracle.cpp  — CPU loops (OpenMP over z), R = float or double;
//   * ssmd_oracle_gpu.cu — the same functions as FP64 CUDA kernels, one
//     thread per cell, for lattices too large for the host cores.
// Both are compiled without FMA contraction (g++ -ffp-contract=off, nvcc
// --fmad=false) and use only correctly rounded +, -, *, / and sqrt, so the
// two instances give the same bits.
//
// Layout and order follow the reference: push (post-stream, in place)
// populations [q][cell] with f stored shifted by -w_q, cell index
// x + nx (y + ny z), and the step
//   computePhase    src/phaseField.cuh:31-52
//   computeForces   src/phaseField.cuh:54-294   (ghost/outside phi read as 0)
//   computeMoments  src/lbm.cu:33-128
//   streamCollide   src/lbm.cu:130-270          (ghost phi values kept)
//   boundaries      src/BoundaryConditions.cuh:36-349 in the order of
//                   src/main.cu:165-169, plus a copy-periodic y mirroring
//                   periodicX for the x,y-periodic jet box
//   initial state   src/initialConditions.cu:33-140
//   velocity sets   src/velocitySet/D3Q19.cuh:65-177, D3Q27.cuh:70-201,
//                   D3Q7.cuh:60-148
// Run-time extensions beyond the reference (exact periodic axes, phase-field
// BGK rate omega_g != 1, seeded inlet noise) follow the formulas the CUDA
// path documents.  Every per-cell function writes only its own cell's slots
// (or, for the push writes, the slots no other cell of the same pass writes),
// so each pass is data-parallel.
#pragma once

#include <math.h>
#include <stdint.h>

#include "../include/ssmd.h"
#include "../ssmdlbm_b200/csrc/noise.h"

#if defined(__CUDACC__)
#define ORC_HD __host__ __device__ __forceinline__
#else
#define ORC_HD inline
#endif

namespace ssmd_oracle {

// D3Q27 velocity order (D3Q19 = the first 19), D3Q19.cuh:82-131,
// D3Q27.cuh:91-140; each component + 1 packed in 2 bits per direction so
// that host and device read the same table without memory.
constexpr int kCX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
constexpr int kCY[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
constexpr int kCZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
constexpr uint64_t pack(const int (&c)[27]) {
    uint64_t v = 0;
    for (int q = 0; q < 27; ++q) v |= (uint64_t)(c[q] + 1) << (2 * q);
    return v;
}
constexpr uint64_t kPX = pack(kCX), kPY = pack(kCY), kPZ = pack(kCZ);
ORC_HD int CX(int q) { return (int)((kPX >> (2 * q)) & 3u) - 1; }
ORC_HD int CY(int q) { return (int)((kPY >> (2 * q)) & 3u) - 1; }
ORC_HD int CZ(int q) { return (int)((kPZ >> (2 * q)) & 3u) - 1; }

enum { BC_COPY = 0, BC_PERIODIC = 1, BC_JET = 2 };

ORC_HD double osqrt(double a) { return sqrt(a); }
ORC_HD float osqrt(float a) { return sqrtf(a); }
ORC_HD float ofma(float a, float b, float c) { return fmaf(a, b, c); }

template <class R>
struct Lattice {
    ssmd_params p;
    int Q;
    int nx, ny, nz;
    int64_t N;
    int lo[3], hi[3];
    bool per[3];
    R w[27];  // hydrodynamic weights
    R sw[27]; // gradient-stencil weights (w_1, w_2, w_3 per shell)
    R as2, cs2, oos;
    // fields (N each), populations (Q N, 7 N), BGK copy of g (7 N, or null),
    // normals and |grad phi| of computeForces (N each)
    R *rho, *ux, *uy, *uz, *pxx, *pyy, *pzz, *pxy, *pxz, *pyz, *phi, *fsx, *fsy, *fsz;
    R *f, *g, *gold, *nX, *nY, *nZ, *nI;
    uint64_t step; // index of the step being taken (inlet noise)

    // geometry and weights from the parameters (pointers set by the owner)
    void setup(const ssmd_params &pp) {
        p = pp;
        Q = p.velocity_set;
        nx = (int)p.nx;
        ny = (int)p.ny;
        nz = (int)p.nz;
        N = (int64_t)nx * ny * nz;
        const int bc[3] = {p.bc_x, p.bc_y, p.bc_z};
        const int n[3] = {nx, ny, nz};
        for (int d = 0; d < 3; ++d) {
            per[d] = bc[d] == BC_PERIODIC;
            lo[d] = per[d] ? 0 : 1;
            hi[d] = per[d] ? n[d] - 1 : n[d] - 2;
        }
        // D3Q19.cuh:50-80, D3Q27.cuh:50-89 (weights computed in FP64 then cast)
        for (int q = 0; q < 27; ++q) {
            if (Q == 19) {
                w[q] = q == 0 ? R(1.0 / 3.0) : (q <= 6 ? R(1.0 / 18.0) : R(1.0 / 36.0));
            } else {
                w[q] = q == 0 ? R(8.0 / 27.0)
                              : (q <= 6 ? R(2.0 / 27.0) : (q <= 18 ? R(1.0 / 54.0) : R(1.0 / 216.0)));
            }
            sw[q] = w[q];
        }
        as2 = R(3);
        cs2 = R(1.0 / 3.0);
        oos = R(1.0 / 6.0);
        step = 0;
    }

    ORC_HD int64_t idx(int x, int y, int z) const { return x + (int64_t)nx * (y + (int64_t)ny * z); }
    // coordinate along axis d, wrapped on exact-periodic axes, -1 outside
    ORC_HD int nb(int d, int c) const {
        const int n = d == 0 ? nx : (d == 1 ? ny : nz);
        if (per[d]) return c < 0 ? c + n : (c >= n ? c - n : c);
        return (c < 0 || c >= n) ? -1 : c;
    }
    ORC_HD bool fluid(int x, int y, int z) const {
        return x >= lo[0] && x <= hi[0] && y >= lo[1] && y <= hi[1] && z >= lo[2] && z <= hi[2];
    }
    ORC_HD size_t slot(int q, int64_t i) const { return (size_t)q * (size_t)N + (size_t)i; }

    // ------------------------------------------------ velocity-set formulas
    // f_eq (D3Q19.cuh:133-140, D3Q27.cuh:147-154), shifted by -w
    ORC_HD R f_eq(int q, R r, R uu, R cu) const {
        if (Q == 19) return w[q] * r * (R(1) - uu + cu + R(0.5) * cu * cu) - w[q];
        return w[q] * r * (R(1) - uu + cu + R(0.5) * cu * cu + oos * cu * cu * cu - uu * cu) - w[q];
    }
    // f_neq (D3Q19.cuh:142-161, D3Q27.cuh:156-185)
    ORC_HD R f_neq(int q, R Pxx, R Pyy, R Pzz, R Pxy, R Pxz, R Pyz, R Ux, R Uy, R Uz) const {
        const R cx = R(CX(q)), cy = R(CY(q)), cz = R(CZ(q));
        R h = (cx * cx - cs2) * Pxx + (cy * cy - cs2) * Pyy + (cz * cz - cs2) * Pzz +
              R(2) * (cx * cy * Pxy + cx * cz * Pxz + cy * cz * Pyz);
        if (Q == 27) {
            h += (cx * cx * cx - cx) * (as2 * Ux * Pxx) + (cy * cy * cy - cy) * (as2 * Uy * Pyy) +
                 (cz * cz * cz - cz) * (as2 * Uz * Pzz) +
                 as2 * ((cx * cx * cy - cs2 * cy) * (Pxx * Uy + R(2) * Ux * Pxy) +
                        (cx * cx * cz - cs2 * cz) * (Pxx * Uz + R(2) * Ux * Pxz) +
                        (cx * cy * cy - cs2 * cx) * (Pyy * Ux + R(2) * Uy * Pxy) +
                        (cy * cy * cz - cs2 * cz) * (Pyy * Uz + R(2) * Uy * Pyz) +
                        (cx * cz * cz - cs2 * cx) * (Pzz * Ux + R(2) * Uz * Pxz) +
                        (cy * cz * cz - cs2 * cy) * (Pzz * Uy + R(2) * Uz * Pyz)) +
                 R(6) * cx * cy * cz * (Ux * Pyz + Uy * Pxz + Uz * Pxy);
        }
        return (w[q] * R(4.5)) * h;
    }
    // Guo force (D3Q19.cuh:163-177, D3Q27.cuh:187-201)
    ORC_HD R force(int q, R cu, R Ux, R Uy, R Uz, R Fx, R Fy, R Fz) const {
        const R cx = R(CX(q)), cy = R(CY(q)), cz = R(CZ(q));
        return w[q] * ((as2 * (cx - Ux) + as2 * cu * cx) * Fx + (as2 * (cy - Uy) + as2 * cu * cy) * Fy +
                       (as2 * (cz - Uz) + as2 * cu * cz) * Fz);
    }
    // D3Q7 g_eq and anti-diffusion (D3Q7.cuh:124-148)
    ORC_HD static R w7(int q) { return q == 0 ? R(1.0 / 4.0) : R(1.0 / 8.0); }
    ORC_HD R g_eq(int q, R ph, R Ux, R Uy, R Uz) const {
        return w7(q) * ph * (R(1) + R(4) * (R(CX(q)) * Ux + R(CY(q)) * Uy + R(CZ(q)) * Uz));
    }
    ORC_HD R anti_diffusion(int q, R sharp, R Nx, R Ny, R Nz) const {
        return w7(q) * sharp * (R(CX(q)) * Nx + R(CY(q)) * Ny + R(CZ(q)) * Nz);
    }
    // isotropic gradient 3 sum_q w_q c_q a(x + c_q) of field a, with
    // out-of-lattice neighbours read as `outside` (phaseField.cuh:158-218 and
    // lbm.cu:157-217 written as a loop over the stencil)
    template <class Get>
    ORC_HD void gradient(int x, int y, int z, Get get, R &gx, R &gy, R &gz) const {
        R sx = 0, sy = 0, sz = 0;
        for (int q = 1; q < Q; ++q) {
            const R v = get(x + CX(q), y + CY(q), z + CZ(q));
            sx += sw[q] * R(CX(q)) * v;
            sy += sw[q] * R(CY(q)) * v;
            sz += sw[q] * R(CZ(q)) * v;
        }
        gx = as2 * sx;
        gy = as2 * sy;
        gz = as2 * sz;
    }

    ORC_HD float inlet_speed(uint64_t s, uint32_t cell) const {
        if (p.noise_amp == 0.0f) return p.u_oil;
        return p.u_oil * (1.0f + p.noise_amp * float(ssmd_noise::gaussian(p.seed, s, cell, 0u)));
    }

    // ------------------------------------------------------- initial state
    // setWaterJet / setOilJet / setInitialDensity (initialConditions.cu:33-97),
    // in three passes: every cell cleared, then the nozzle discs, then rho = 1
    ORC_HD void init_clear(int64_t i) {
        rho[i] = ux[i] = uy[i] = uz[i] = phi[i] = R(0);
        pxx[i] = pyy[i] = pzz[i] = pxy[i] = pxz[i] = pyz[i] = R(0);
        fsx[i] = fsy[i] = fsz[i] = R(0);
    }
    ORC_HD void init_water_disc(int x, int z) { // face y = 0
        const float dx = float(x) - p.water_cx, dz = float(z) - p.water_cz;
        if (dx * dx + dz * dz > p.water_r2) return;
        phi[idx(x, 0, z)] = R(0);
        uy[idx(x, 0, z)] = R(p.u_water);
    }
    ORC_HD void init_oil_disc(int x, int y) { // face z = 0
        const float dx = float(x) - p.oil_cx, dy = float(y) - p.oil_cy;
        if (dx * dx + dy * dy > p.oil_r2) return;
        phi[idx(x, y, 0)] = R(1);
        uz[idx(x, y, 0)] = R(inlet_speed(0, (uint32_t)idx(x, y, 0)));
    }
    ORC_HD void init_density(int64_t i) { rho[i] = R(1); }

    // setDistros (initialConditions.cu:99-140): f = f_eq, g = g_eq at own cell
    ORC_HD void set_distros_cell(int x, int y, int z) {
        const int64_t i = idx(x, y, z);
        const R Ux = ux[i], Uy = uy[i], Uz = uz[i];
        const R uu = R(1.5) * (Ux * Ux + Uy * Uy + Uz * Uz);
        for (int q = 0; q < Q; ++q) {
            const R cu = as2 * (R(CX(q)) * Ux + R(CY(q)) * Uy + R(CZ(q)) * Uz);
            f[slot(q, i)] = f_eq(q, rho[i], uu, cu);
        }
        for (int q = 0; q < 7; ++q) g[slot(q, i)] = g_eq(q, phi[i], Ux, Uy, Uz);
    }

    // ------------------------------------------------------------ one step
    ORC_HD void phase_cell(int x, int y, int z) { // phaseField.cuh:31-52
        if (!fluid(x, y, z)) return;
        const int64_t i = idx(x, y, z);
        R s = 0;
        for (int q = 0; q < 7; ++q) s += g[slot(q, i)];
        phi[i] = s;
    }

    // computeForces, first half (phaseField.cuh:107-227): normals and
    // |grad phi| on every lattice cell from phi with ghost cells and outside
    // cells read as zero; a normal read outside the lattice only happens for
    // ghost cells, which get F = 0
    ORC_HD void normal_cell(int x, int y, int z) {
        auto phiz = [&](int xx, int yy, int zz) -> R {
            xx = nb(0, xx);
            yy = nb(1, yy);
            zz = nb(2, zz);
            if (xx < 0 || yy < 0 || zz < 0) return R(0);
            if (!fluid(xx, yy, zz)) return R(0);
            return phi[idx(xx, yy, zz)];
        };
        R gx, gy, gz;
        gradient(x, y, z, phiz, gx, gy, gz);
        const R ind = osqrt(gx * gx + gy * gy + gz * gz);
        const R inv = R(1) / (ind + R(1e-9));
        const int64_t i = idx(x, y, z);
        nX[i] = gx * inv;
        nY[i] = gy * inv;
        nZ[i] = gz * inv;
        nI[i] = ind;
    }

    // computeForces, second half (phaseField.cuh:238-293)
    ORC_HD void force_cell(int x, int y, int z) {
        const int64_t i = idx(x, y, z);
        if (!fluid(x, y, z)) { // :238-244
            fsx[i] = fsy[i] = fsz[i] = R(0);
            return;
        }
        R scx = 0, scy = 0, scz = 0; // :250-284
        for (int q = 1; q < Q; ++q) {
            const int64_t j = idx(nb(0, x + CX(q)), nb(1, y + CY(q)), nb(2, z + CZ(q)));
            scx += sw[q] * R(CX(q)) * nX[j];
            scy += sw[q] * R(CY(q)) * nY[j];
            scz += sw[q] * R(CZ(q)) * nZ[j];
        }
        const R curvature = as2 * (scx + scy + scz);
        const R stCurv = -R(p.sigma) * curvature * nI[i];
        fsx[i] = stCurv * nX[i];
        fsy[i] = stCurv * nY[i];
        fsz[i] = stCurv * nZ[i];
    }

    ORC_HD void moments_cell(int x, int y, int z) { // lbm.cu:33-128
        if (!fluid(x, y, z)) return;
        const int64_t i = idx(x, y, z);
        R pop[27];
        R r = 0;
        for (int q = 0; q < Q; ++q) {
            pop[q] = f[slot(q, i)];
            r += pop[q];
        }
        r += R(1);
        rho[i] = r;
        const R Fx = fsx[i], Fy = fsy[i], Fz = fsz[i];
        const R invRho = R(1) / r;
        R jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < Q; ++q) {
            jx += R(CX(q)) * pop[q];
            jy += R(CY(q)) * pop[q];
            jz += R(CZ(q)) * pop[q];
        }
        R Ux = invRho * jx, Uy = invRho * jy, Uz = invRho * jz;
        Ux += Fx * R(0.5) * invRho;
        Uy += Fy * R(0.5) * invRho;
        Uz += Fz * R(0.5) * invRho;
        ux[i] = Ux;
        uy[i] = Uy;
        uz[i] = Uz;
        R Pxx = 0, Pyy = 0, Pzz = 0, Pxy = 0, Pxz = 0, Pyz = 0;
        const R uu = R(1.5) * (Ux * Ux + Uy * Uy + Uz * Uz);
        for (int q = 0; q < Q; ++q) {
            const R cx = R(CX(q)), cy = R(CY(q)), cz = R(CZ(q));
            const R cu = as2 * (cx * Ux + cy * Uy + cz * Uz);
            const R fneq = pop[q] - f_eq(q, r, uu, cu) + R(0.5) * force(q, cu, Ux, Uy, Uz, Fx, Fy, Fz);
            Pxx += fneq * cx * cx;
            Pyy += fneq * cy * cy;
            Pzz += fneq * cz * cz;
            Pxy += fneq * cx * cy;
            Pxz += fneq * cx * cz;
            Pyz += fneq * cy * cz;
        }
        const R trace = Pxx + Pyy + Pzz;
        pxx[i] = Pxx - cs2 * trace;
        pyy[i] = Pyy - cs2 * trace;
        pzz[i] = Pzz - cs2 * trace;
        pxy[i] = Pxy;
        pxz[i] = Pxz;
        pyz[i] = Pyz;
    }

    // lbm.cu:130-270; with omega_g != 1, gold holds this step's post-stream g
    ORC_HD void collide_cell(int x, int y, int z) {
        if (!fluid(x, y, z)) return;
        const bool bgk = p.omega_g != 1.0f;
        const R visc_w = R(p.nu_water), visc_o = R(p.nu_oil);
        const R dvisc = R(p.nu_oil - p.nu_water);
        const R gam = R(p.gamma), omg = R(p.omega_g);
        auto phir = [&](int xx, int yy, int zz) -> R { // raw phi incl. ghost values
            return phi[idx(nb(0, xx), nb(1, yy), nb(2, zz))];
        };
        const int64_t i = idx(x, y, z);
        const R r = rho[i], Ux = ux[i], Uy = uy[i], Uz = uz[i];
        const R Fx = fsx[i], Fy = fsy[i], Fz = fsz[i];
        R gx, gy, gz;
        gradient(x, y, z, phir, gx, gy, gz);
        const R ind = osqrt(gx * gx + gy * gy + gz * gz);
        const R invInd = R(1) / (ind + R(1e-9));
        const R Nx = gx * invInd, Ny = gy * invInd, Nz = gz * invInd;
        const R ph = phi[i];
        R nu;
        if constexpr (sizeof(R) == 4) nu = ofma(ph, dvisc, visc_w);
        else nu = ph * (visc_o - visc_w) + visc_w;
        const R omega = R(1) / (R(0.5) + as2 * nu);
        const R omco = R(1) - omega;
        const R uu = R(1.5) * (Ux * Ux + Uy * Uy + Uz * Uz);
        for (int q = 0; q < Q; ++q) {
            const R cu = as2 * (R(CX(q)) * Ux + R(CY(q)) * Uy + R(CZ(q)) * Uz);
            const R feq = f_eq(q, r, uu, cu);
            const R frc = force(q, cu, Ux, Uy, Uz, Fx, Fy, Fz);
            const R fneq = f_neq(q, pxx[i], pyy[i], pzz[i], pxy[i], pxz[i], pyz[i], Ux, Uy, Uz);
            const int64_t j = idx(nb(0, x + CX(q)), nb(1, y + CY(q)), nb(2, z + CZ(q)));
            f[slot(q, j)] = feq + omco * fneq + R(0.5) * frc;
        }
        const R sharp = gam * ph * (R(1) - ph);
        for (int q = 0; q < 7; ++q) {
            R gn = g_eq(q, ph, Ux, Uy, Uz) + anti_diffusion(q, sharp, Nx, Ny, Nz);
            if (bgk) {
                const R gi = gold[slot(q, i)];
                gn = gi + omg * (gn - gi);
            }
            const int64_t j = idx(nb(0, x + CX(q)), nb(1, y + CY(q)), nb(2, z + CZ(q)));
            g[slot(q, j)] = gn;
        }
    }

    // regularized inflow/outflow value (BoundaryConditions.cuh:87-94 etc.)
    ORC_HD R reg(int q, R r, R Ux, R Uy, R Uz, int64_t fn, R omco) const {
        const R uu = R(1.5) * (Ux * Ux + Uy * Uy + Uz * Uz);
        const R cu = as2 * (R(CX(q)) * Ux + R(CY(q)) * Uy + R(CZ(q)) * Uz);
        return f_eq(q, r, uu, cu) +
               omco * f_neq(q, pxx[fn], pyy[fn], pzz[fn], pxy[fn], pxz[fn], pyz[fn], ux[fn], uy[fn], uz[fn]);
    }

    ORC_HD void water_inflow_cell(int x, int z) { // BoundaryConditions.cuh:36-99
        const float dx = float(x) - p.water_cx, dz = float(z) - p.water_cz;
        if (dx * dx + dz * dz > p.water_r2) return;
        const int64_t b = idx(x, 0, z), b1 = idx(x, 1, z);
        const R uw = R(p.u_water);
        rho[b] = R(1);
        phi[b] = R(0);
        ux[b] = R(0);
        uy[b] = uw;
        uz[b] = R(0);
        for (int q = 0; q < Q; ++q) {
            if (CY(q) != 1) continue;
            const int xx = nb(0, x + CX(q)), zz = nb(2, z + CZ(q));
            if (xx < 0 || zz < 0) continue;
            const int64_t fn = idx(xx, 1, zz);
            f[slot(q, fn)] = reg(q, R(1), R(0), uw, R(0), fn, R(p.omco_water));
        }
        g[slot(3, b1)] = w7(3) * R(0) * (R(1) + R(4) * uw);
    }

    ORC_HD void oil_inflow_cell(int x, int y) { // BoundaryConditions.cuh:101-168
        const float dx = float(x) - p.oil_cx, dy = float(y) - p.oil_cy;
        if (dx * dx + dy * dy > p.oil_r2) return;
        const int64_t b = idx(x, y, 0), b1 = idx(x, y, 1);
        const R uin = R(inlet_speed(step, (uint32_t)b));
        rho[b] = R(1);
        phi[b] = R(1);
        ux[b] = R(0);
        uy[b] = R(0);
        uz[b] = uin;
        for (int q = 0; q < Q; ++q) {
            if (CZ(q) != 1) continue;
            const int xx = nb(0, x + CX(q)), yy = nb(1, y + CY(q));
            if (xx < 0 || yy < 0 || xx < lo[0] || xx > hi[0] || yy < lo[1] || yy > hi[1]) continue;
            const int64_t fn = idx(xx, yy, 1);
            f[slot(q, fn)] = reg(q, R(1), R(0), R(0), uin, fn, R(p.omco_oil));
        }
        g[slot(5, b1)] = w7(5) * R(1) * (R(1) + R(4) * uin);
    }

    ORC_HD void outflow_y_cell(int x, int z) { // BoundaryConditions.cuh:170-233 (fluid x, z)
        const int64_t b = idx(x, ny - 1, z), i1 = idx(x, ny - 2, z);
        rho[b] = rho[i1];
        phi[b] = phi[i1];
        ux[b] = ux[i1];
        uy[b] = uy[i1];
        uz[b] = uz[i1];
        const R r = rho[b], ph = phi[b], Ux = ux[b], Uy = uy[b], Uz = uz[b];
        for (int q = 0; q < Q; ++q) {
            if (CY(q) != -1) continue;
            const int xx = nb(0, x + CX(q)), zz = nb(2, z + CZ(q));
            if (xx < 0 || zz < 0 || xx < lo[0] || xx > hi[0] || zz < lo[2] || zz > hi[2]) continue;
            const int64_t fn = idx(xx, ny - 2, zz);
            f[slot(q, fn)] = reg(q, r, Ux, Uy, Uz, fn, R(p.omco_ref));
        }
        g[slot(4, i1)] = w7(4) * ph * (R(1) - R(4) * Uy);
    }

    ORC_HD void outflow_z_cell(int x, int y) { // BoundaryConditions.cuh:235-293 (fluid x, y)
        const int64_t b = idx(x, y, nz - 1), i1 = idx(x, y, nz - 2);
        rho[b] = rho[i1];
        phi[b] = phi[i1];
        ux[b] = ux[i1];
        uy[b] = uy[i1];
        uz[b] = uz[i1];
        const R r = rho[b], ph = phi[b], Ux = ux[b], Uy = uy[b], Uz = uz[b];
        for (int q = 0; q < Q; ++q) {
            if (CZ(q) != -1) continue;
            const int xx = nb(0, x + CX(q)), yy = nb(1, y + CY(q));
            if (xx < 0 || yy < 0) continue;
            const int64_t fn = idx(xx, yy, nz - 2);
            f[slot(q, fn)] = reg(q, r, Ux, Uy, Uz, fn, R(p.omco_ref));
        }
        g[slot(6, i1)] = w7(6) * ph * (R(1) - R(4) * Uz);
    }

    ORC_HD void copy_x_cell(int y, int z) { // BoundaryConditions.cuh:295-349
        const int64_t bL = idx(1, y, z), bR = idx(nx - 2, y, z);
        for (int q = 0; q < Q; ++q) {
            if (CX(q) > 0) f[slot(q, bL)] = f[slot(q, bR)];
            if (CX(q) < 0) f[slot(q, bR)] = f[slot(q, bL)];
        }
        g[slot(1, bL)] = g[slot(1, bR)];
        g[slot(2, bR)] = g[slot(2, bL)];
        const int64_t gL = idx(0, y, z), gR = idx(nx - 1, y, z);
        phi[gL] = phi[bR];
        phi[gR] = phi[bL];
        ux[gL] = ux[bR];
        ux[gR] = ux[bL];
        uy[gL] = uy[bR];
        uy[gR] = uy[bL];
        uz[gL] = uz[bR];
        uz[gR] = uz[bL];
    }

    ORC_HD void copy_y_cell(int x, int z) { // periodicX's rule applied to y
        const int64_t bL = idx(x, 1, z), bR = idx(x, ny - 2, z);
        for (int q = 0; q < Q; ++q) {
            if (CY(q) > 0) f[slot(q, bL)] = f[slot(q, bR)];
            if (CY(q) < 0) f[slot(q, bR)] = f[slot(q, bL)];
        }
        g[slot(3, bL)] = g[slot(3, bR)];
        g[slot(4, bR)] = g[slot(4, bL)];
        const int64_t gL = idx(x, 0, z), gR = idx(x, ny - 1, z);
        phi[gL] = phi[bR];
        phi[gR] = phi[bL];
        ux[gL] = ux[bR];
        ux[gR] = ux[bL];
        uy[gL] = uy[bR];
        uy[gR] = uy[bL];
        uz[gL] = uz[bR];
        uz[gR] = uz[bL];
    }
};

} // namespace ssmd_oracle
