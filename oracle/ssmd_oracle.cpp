// ssmd_oracle.cpp — CPU oracle for the ssmd_b200 hot path.  TEST INFRASTRUCTURE.
//
// This file is the checker, never the product: only the tests, the smoke
// check and the CPU-baseline leg of bench.py load it.  It restates, loop by
// loop and in the reference's own push (post-stream, in-place) layout, the
// reference ssmdLBM kernels of one time step:
//
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
//
// Templated on the real type: R = float mirrors the reference's FP32
// arithmetic (compile with -ffp-contract=off), R = double is the FP64
// transcription.  Run-time extensions beyond the reference (exact periodic
// axes, phase-field BGK rate omega_g != 1, seeded inlet noise) follow the
// same formulas the CUDA path documents.  Loops are OpenMP-parallel over z.
//
// Parity pin: tests compare this file against outputs of the reference's own
// CUDA kernels (oracle/_ref harness runs) committed under tests/golden/.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../include/ssmd.h"
#include "../ssmdlbm_b200/csrc/noise.h"

namespace {

constexpr int CX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
constexpr int CY[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
constexpr int CZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};

enum { BC_COPY = 0, BC_PERIODIC = 1, BC_JET = 2 };

template <class R>
struct Oracle {
    ssmd_params p;
    int Q;
    int nx, ny, nz;
    int64_t N;
    int lo[3], hi[3];
    bool per[3];
    R w[27];      // hydrodynamic weights
    R sw[27];     // gradient-stencil weights (w_1, w_2, w_3 per shell)
    R as2, cs2, oos;
    std::vector<R> rho, ux, uy, uz, pxx, pyy, pzz, pxy, pxz, pyz, phi, fsx, fsy, fsz;
    std::vector<R> f, g, gold;
    uint64_t step = 0; // index of the next step

    explicit Oracle(const ssmd_params &pp) : p(pp) {
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
        for (auto *v : {&rho, &ux, &uy, &uz, &pxx, &pyy, &pzz, &pxy, &pxz, &pyz, &phi, &fsx, &fsy, &fsz})
            v->assign(N, R(0));
        f.assign((size_t)Q * N, R(0));
        g.assign((size_t)7 * N, R(0));
    }

    int64_t idx(int x, int y, int z) const { return x + (int64_t)nx * (y + (int64_t)ny * z); }
    // coordinate along axis d, wrapped on exact-periodic axes, -1 outside
    int nb(int d, int c) const {
        const int n = d == 0 ? nx : (d == 1 ? ny : nz);
        if (per[d]) return c < 0 ? c + n : (c >= n ? c - n : c);
        return (c < 0 || c >= n) ? -1 : c;
    }
    bool fluid(int x, int y, int z) const {
        return x >= lo[0] && x <= hi[0] && y >= lo[1] && y <= hi[1] && z >= lo[2] && z <= hi[2];
    }

    // ------------------------------------------------ velocity-set formulas
    // f_eq (D3Q19.cuh:133-140, D3Q27.cuh:147-154), shifted by -w
    R f_eq(int q, R r, R uu, R cu) const {
        if (Q == 19) return w[q] * r * (R(1) - uu + cu + R(0.5) * cu * cu) - w[q];
        return w[q] * r * (R(1) - uu + cu + R(0.5) * cu * cu + oos * cu * cu * cu - uu * cu) - w[q];
    }
    // f_neq (D3Q19.cuh:142-161, D3Q27.cuh:156-185)
    R f_neq(int q, R Pxx, R Pyy, R Pzz, R Pxy, R Pxz, R Pyz, R Ux, R Uy, R Uz) const {
        const R cx = R(CX[q]), cy = R(CY[q]), cz = R(CZ[q]);
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
    R force(int q, R cu, R Ux, R Uy, R Uz, R Fx, R Fy, R Fz) const {
        const R cx = R(CX[q]), cy = R(CY[q]), cz = R(CZ[q]);
        return w[q] * ((as2 * (cx - Ux) + as2 * cu * cx) * Fx + (as2 * (cy - Uy) + as2 * cu * cy) * Fy +
                       (as2 * (cz - Uz) + as2 * cu * cz) * Fz);
    }
    // D3Q7 g_eq and anti-diffusion (D3Q7.cuh:124-148)
    static R w7(int q) { return q == 0 ? R(1.0 / 4.0) : R(1.0 / 8.0); }
    R g_eq(int q, R ph, R Ux, R Uy, R Uz) const {
        return w7(q) * ph * (R(1) + R(4) * (R(CX[q]) * Ux + R(CY[q]) * Uy + R(CZ[q]) * Uz));
    }
    R anti_diffusion(int q, R sharp, R Nx, R Ny, R Nz) const {
        return w7(q) * sharp * (R(CX[q]) * Nx + R(CY[q]) * Ny + R(CZ[q]) * Nz);
    }

    // isotropic gradient 3 sum_q w_q c_q a(x + c_q) of field a, with
    // out-of-lattice neighbours read as `outside` (phaseField.cuh:158-218 and
    // lbm.cu:157-217 written as a loop over the stencil)
    template <class Get>
    void gradient(int x, int y, int z, Get get, R &gx, R &gy, R &gz) const {
        R sx = 0, sy = 0, sz = 0;
        for (int q = 1; q < Q; ++q) {
            const R v = get(x + CX[q], y + CY[q], z + CZ[q]);
            sx += sw[q] * R(CX[q]) * v;
            sy += sw[q] * R(CY[q]) * v;
            sz += sw[q] * R(CZ[q]) * v;
        }
        gx = as2 * sx;
        gy = as2 * sy;
        gz = as2 * sz;
    }

    // ------------------------------------------------------- initial state
    // setWaterJet / setOilJet / setInitialDensity (initialConditions.cu:33-97)
    void init_jets() {
        for (int64_t i = 0; i < N; ++i) {
            rho[i] = ux[i] = uy[i] = uz[i] = phi[i] = R(0);
            pxx[i] = pyy[i] = pzz[i] = pxy[i] = pxz[i] = pyz[i] = R(0);
            fsx[i] = fsy[i] = fsz[i] = R(0);
        }
        if (p.bc_y == BC_JET) {
            for (int z = 0; z < nz; ++z)
                for (int x = 0; x < nx; ++x) {
                    const float dx = float(x) - p.water_cx, dz = float(z) - p.water_cz;
                    if (dx * dx + dz * dz > p.water_r2) continue;
                    phi[idx(x, 0, z)] = R(0);
                    uy[idx(x, 0, z)] = R(p.u_water);
                }
        }
        if (p.bc_z == BC_JET) {
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    const float dx = float(x) - p.oil_cx, dy = float(y) - p.oil_cy;
                    if (dx * dx + dy * dy > p.oil_r2) continue;
                    phi[idx(x, y, 0)] = R(1);
                    uz[idx(x, y, 0)] = R(inlet_speed(0, (uint32_t)idx(x, y, 0)));
                }
        }
        for (int64_t i = 0; i < N; ++i) rho[i] = R(1);
        set_distros();
    }

    float inlet_speed(uint64_t s, uint32_t cell) const {
        if (p.noise_amp == 0.0f) return p.u_oil;
        return p.u_oil * (1.0f + p.noise_amp * float(ssmd_noise::gaussian(p.seed, s, cell, 0u)));
    }

    // setDistros (initialConditions.cu:99-140): f = f_eq, g = g_eq at own cell
    void set_distros() {
#pragma omp parallel for
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    const int64_t i = idx(x, y, z);
                    const R Ux = ux[i], Uy = uy[i], Uz = uz[i];
                    const R uu = R(1.5) * (Ux * Ux + Uy * Uy + Uz * Uz);
                    for (int q = 0; q < Q; ++q) {
                        const R cu = as2 * (R(CX[q]) * Ux + R(CY[q]) * Uy + R(CZ[q]) * Uz);
                        f[(size_t)q * N + i] = f_eq(q, rho[i], uu, cu);
                    }
                    for (int q = 0; q < 7; ++q) g[(size_t)q * N + i] = g_eq(q, phi[i], Ux, Uy, Uz);
                }
        step = 0;
    }

    // ------------------------------------------------------------ one step
    void compute_phase() { // phaseField.cuh:31-52
#pragma omp parallel for
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    if (!fluid(x, y, z)) continue;
                    const int64_t i = idx(x, y, z);
                    R s = 0;
                    for (int q = 0; q < 7; ++q) s += g[(size_t)q * N + i];
                    phi[i] = s;
                }
    }

    void compute_forces() { // phaseField.cuh:54-294
        // phi with ghost cells and outside cells read as zero (:107-143)
        auto phiz = [&](int x, int y, int z) -> R {
            x = nb(0, x);
            y = nb(1, y);
            z = nb(2, z);
            if (x < 0 || y < 0 || z < 0) return R(0);
            if (!fluid(x, y, z)) return R(0);
            return phi[idx(x, y, z)];
        };
        // normals and |grad phi| on every lattice cell (:147-227); a normal
        // read outside the lattice only happens for ghost cells, which get F = 0
        std::vector<R> nX(N), nY(N), nZ(N), nI(N);
#pragma omp parallel for
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    R gx, gy, gz;
                    gradient(x, y, z, phiz, gx, gy, gz);
                    const R ind = std::sqrt(gx * gx + gy * gy + gz * gz);
                    const R inv = R(1) / (ind + R(1e-9));
                    const int64_t i = idx(x, y, z);
                    nX[i] = gx * inv;
                    nY[i] = gy * inv;
                    nZ[i] = gz * inv;
                    nI[i] = ind;
                }
#pragma omp parallel for
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    const int64_t i = idx(x, y, z);
                    if (!fluid(x, y, z)) { // :238-244
                        fsx[i] = fsy[i] = fsz[i] = R(0);
                        continue;
                    }
                    R scx = 0, scy = 0, scz = 0; // :250-284
                    for (int q = 1; q < Q; ++q) {
                        const int64_t j = idx(nb(0, x + CX[q]), nb(1, y + CY[q]), nb(2, z + CZ[q]));
                        scx += sw[q] * R(CX[q]) * nX[j];
                        scy += sw[q] * R(CY[q]) * nY[j];
                        scz += sw[q] * R(CZ[q]) * nZ[j];
                    }
                    const R curvature = as2 * (scx + scy + scz);
                    const R stCurv = -R(p.sigma) * curvature * nI[i];
                    fsx[i] = stCurv * nX[i];
                    fsy[i] = stCurv * nY[i];
                    fsz[i] = stCurv * nZ[i];
                }
    }

    void compute_moments() { // lbm.cu:33-128
#pragma omp parallel for
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    if (!fluid(x, y, z)) continue;
                    const int64_t i = idx(x, y, z);
                    R pop[27];
                    R r = 0;
                    for (int q = 0; q < Q; ++q) {
                        pop[q] = f[(size_t)q * N + i];
                        r += pop[q];
                    }
                    r += R(1);
                    rho[i] = r;
                    const R Fx = fsx[i], Fy = fsy[i], Fz = fsz[i];
                    const R invRho = R(1) / r;
                    R jx = 0, jy = 0, jz = 0;
                    for (int q = 0; q < Q; ++q) {
                        jx += R(CX[q]) * pop[q];
                        jy += R(CY[q]) * pop[q];
                        jz += R(CZ[q]) * pop[q];
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
                        const R cx = R(CX[q]), cy = R(CY[q]), cz = R(CZ[q]);
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
    }

    void stream_collide() { // lbm.cu:130-270
        const bool bgk = p.omega_g != 1.0f;
        if (bgk) gold = g; // post-stream g of this step (BGK extension only)
        const R visc_w = R(p.nu_water), visc_o = R(p.nu_oil);
        const R dvisc = R(p.nu_oil - p.nu_water);
        const R gam = R(p.gamma), omg = R(p.omega_g);
        auto phir = [&](int x, int y, int z) -> R { // raw phi incl. ghost values
            return phi[idx(nb(0, x), nb(1, y), nb(2, z))];
        };
#pragma omp parallel for
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    if (!fluid(x, y, z)) continue;
                    const int64_t i = idx(x, y, z);
                    const R r = rho[i], Ux = ux[i], Uy = uy[i], Uz = uz[i];
                    const R Fx = fsx[i], Fy = fsy[i], Fz = fsz[i];
                    R gx, gy, gz;
                    gradient(x, y, z, phir, gx, gy, gz);
                    const R ind = std::sqrt(gx * gx + gy * gy + gz * gz);
                    const R invInd = R(1) / (ind + R(1e-9));
                    const R Nx = gx * invInd, Ny = gy * invInd, Nz = gz * invInd;
                    const R ph = phi[i];
                    R nu;
                    if constexpr (sizeof(R) == 4) nu = std::fma(ph, dvisc, visc_w);
                    else nu = ph * (visc_o - visc_w) + visc_w;
                    const R omega = R(1) / (R(0.5) + as2 * nu);
                    const R omco = R(1) - omega;
                    const R uu = R(1.5) * (Ux * Ux + Uy * Uy + Uz * Uz);
                    for (int q = 0; q < Q; ++q) {
                        const R cu = as2 * (R(CX[q]) * Ux + R(CY[q]) * Uy + R(CZ[q]) * Uz);
                        const R feq = f_eq(q, r, uu, cu);
                        const R frc = force(q, cu, Ux, Uy, Uz, Fx, Fy, Fz);
                        const R fneq = f_neq(q, pxx[i], pyy[i], pzz[i], pxy[i], pxz[i], pyz[i], Ux, Uy, Uz);
                        const int64_t j = idx(nb(0, x + CX[q]), nb(1, y + CY[q]), nb(2, z + CZ[q]));
                        f[(size_t)q * N + j] = feq + omco * fneq + R(0.5) * frc;
                    }
                    const R sharp = gam * ph * (R(1) - ph);
                    for (int q = 0; q < 7; ++q) {
                        R gn = g_eq(q, ph, Ux, Uy, Uz) + anti_diffusion(q, sharp, Nx, Ny, Nz);
                        if (bgk) {
                            const R gi = gold[(size_t)q * N + i];
                            gn = gi + omg * (gn - gi);
                        }
                        const int64_t j = idx(nb(0, x + CX[q]), nb(1, y + CY[q]), nb(2, z + CZ[q]));
                        g[(size_t)q * N + j] = gn;
                    }
                }
    }

    // regularized inflow/outflow value (BoundaryConditions.cuh:87-94 etc.)
    R reg(int q, R r, R Ux, R Uy, R Uz, int64_t fn, R omco) const {
        const R uu = R(1.5) * (Ux * Ux + Uy * Uy + Uz * Uz);
        const R cu = as2 * (R(CX[q]) * Ux + R(CY[q]) * Uy + R(CZ[q]) * Uz);
        return f_eq(q, r, uu, cu) +
               omco * f_neq(q, pxx[fn], pyy[fn], pzz[fn], pxy[fn], pxz[fn], pyz[fn], ux[fn], uy[fn], uz[fn]);
    }

    void water_inflow() { // BoundaryConditions.cuh:36-99
        for (int z = 0; z < nz; ++z)
            for (int x = 0; x < nx; ++x) {
                const float dx = float(x) - p.water_cx, dz = float(z) - p.water_cz;
                if (dx * dx + dz * dz > p.water_r2) continue;
                const int64_t b = idx(x, 0, z), b1 = idx(x, 1, z);
                const R uw = R(p.u_water);
                rho[b] = R(1);
                phi[b] = R(0);
                ux[b] = R(0);
                uy[b] = uw;
                uz[b] = R(0);
                for (int q = 0; q < Q; ++q) {
                    if (CY[q] != 1) continue;
                    const int xx = nb(0, x + CX[q]), zz = nb(2, z + CZ[q]);
                    if (xx < 0 || zz < 0) continue;
                    const int64_t fn = idx(xx, 1, zz);
                    f[(size_t)q * N + fn] = reg(q, R(1), R(0), uw, R(0), fn, R(p.omco_water));
                }
                g[(size_t)3 * N + b1] = w7(3) * R(0) * (R(1) + R(4) * uw);
            }
    }

    void oil_inflow() { // BoundaryConditions.cuh:101-168
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const float dx = float(x) - p.oil_cx, dy = float(y) - p.oil_cy;
                if (dx * dx + dy * dy > p.oil_r2) continue;
                const int64_t b = idx(x, y, 0), b1 = idx(x, y, 1);
                const R uin = R(inlet_speed(step, (uint32_t)b));
                rho[b] = R(1);
                phi[b] = R(1);
                ux[b] = R(0);
                uy[b] = R(0);
                uz[b] = uin;
                for (int q = 0; q < Q; ++q) {
                    if (CZ[q] != 1) continue;
                    const int xx = nb(0, x + CX[q]), yy = nb(1, y + CY[q]);
                    if (xx < 0 || yy < 0 || xx < lo[0] || xx > hi[0] || yy < lo[1] || yy > hi[1]) continue;
                    const int64_t fn = idx(xx, yy, 1);
                    f[(size_t)q * N + fn] = reg(q, R(1), R(0), R(0), uin, fn, R(p.omco_oil));
                }
                g[(size_t)5 * N + b1] = w7(5) * R(1) * (R(1) + R(4) * uin);
            }
    }

    void outflow_y() { // BoundaryConditions.cuh:170-233
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int x = lo[0]; x <= hi[0]; ++x) {
                const int64_t b = idx(x, ny - 1, z), i1 = idx(x, ny - 2, z);
                rho[b] = rho[i1];
                phi[b] = phi[i1];
                ux[b] = ux[i1];
                uy[b] = uy[i1];
                uz[b] = uz[i1];
                const R r = rho[b], ph = phi[b], Ux = ux[b], Uy = uy[b], Uz = uz[b];
                for (int q = 0; q < Q; ++q) {
                    if (CY[q] != -1) continue;
                    const int xx = nb(0, x + CX[q]), zz = nb(2, z + CZ[q]);
                    if (xx < 0 || zz < 0 || xx < lo[0] || xx > hi[0] || zz < lo[2] || zz > hi[2]) continue;
                    const int64_t fn = idx(xx, ny - 2, zz);
                    f[(size_t)q * N + fn] = reg(q, r, Ux, Uy, Uz, fn, R(p.omco_ref));
                }
                g[(size_t)4 * N + i1] = w7(4) * ph * (R(1) - R(4) * Uy);
            }
    }

    void outflow_z() { // BoundaryConditions.cuh:235-293
        for (int y = lo[1]; y <= hi[1]; ++y)
            for (int x = lo[0]; x <= hi[0]; ++x) {
                const int64_t b = idx(x, y, nz - 1), i1 = idx(x, y, nz - 2);
                rho[b] = rho[i1];
                phi[b] = phi[i1];
                ux[b] = ux[i1];
                uy[b] = uy[i1];
                uz[b] = uz[i1];
                const R r = rho[b], ph = phi[b], Ux = ux[b], Uy = uy[b], Uz = uz[b];
                for (int q = 0; q < Q; ++q) {
                    if (CZ[q] != -1) continue;
                    const int xx = nb(0, x + CX[q]), yy = nb(1, y + CY[q]);
                    if (xx < 0 || yy < 0) continue;
                    const int64_t fn = idx(xx, yy, nz - 2);
                    f[(size_t)q * N + fn] = reg(q, r, Ux, Uy, Uz, fn, R(p.omco_ref));
                }
                g[(size_t)6 * N + i1] = w7(6) * ph * (R(1) - R(4) * Uz);
            }
    }

    void copy_x() { // BoundaryConditions.cuh:295-349
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y) {
                const int64_t bL = idx(1, y, z), bR = idx(nx - 2, y, z);
                for (int q = 0; q < Q; ++q) {
                    if (CX[q] > 0) f[(size_t)q * N + bL] = f[(size_t)q * N + bR];
                    if (CX[q] < 0) f[(size_t)q * N + bR] = f[(size_t)q * N + bL];
                }
                g[(size_t)1 * N + bL] = g[(size_t)1 * N + bR];
                g[(size_t)2 * N + bR] = g[(size_t)2 * N + bL];
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
    }

    void copy_y() { // periodicX's rule applied to y
        for (int z = 0; z < nz; ++z)
            for (int x = 0; x < nx; ++x) {
                const int64_t bL = idx(x, 1, z), bR = idx(x, ny - 2, z);
                for (int q = 0; q < Q; ++q) {
                    if (CY[q] > 0) f[(size_t)q * N + bL] = f[(size_t)q * N + bR];
                    if (CY[q] < 0) f[(size_t)q * N + bR] = f[(size_t)q * N + bL];
                }
                g[(size_t)3 * N + bL] = g[(size_t)3 * N + bR];
                g[(size_t)4 * N + bR] = g[(size_t)4 * N + bL];
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
    }

    // main.cu:159-169 with the graph of CUDAGraph.cuh:44-49
    void one_step() {
        compute_phase();
        compute_forces();
        compute_moments();
        stream_collide();
        if (p.bc_y == BC_JET) water_inflow();
        if (p.bc_z == BC_JET) oil_inflow();
        if (p.bc_y == BC_JET) outflow_y();
        if (p.bc_z == BC_JET) outflow_z();
        if (p.bc_x == BC_COPY) copy_x();
        if (p.bc_y == BC_COPY) copy_y();
        ++step;
    }
};

struct Handle {
    int precision;
    void *o;
};

template <class R>
Oracle<R> &O(Handle *h) {
    return *static_cast<Oracle<R> *>(h->o);
}

template <class R, class T>
int get_field(Oracle<R> &o, int id, T *out) {
    const std::vector<R> *v = nullptr;
    switch (id) {
    case 0: v = &o.rho; break;
    case 1: v = &o.ux; break;
    case 2: v = &o.uy; break;
    case 3: v = &o.uz; break;
    case 4: v = &o.phi; break;
    case 5: v = &o.pxx; break;
    case 6: v = &o.pyy; break;
    case 7: v = &o.pzz; break;
    case 8: v = &o.pxy; break;
    case 9: v = &o.pxz; break;
    case 10: v = &o.pyz; break;
    case 11: v = &o.fsx; break;
    case 12: v = &o.fsy; break;
    case 13: v = &o.fsz; break;
    case 20: v = &o.f; break;
    case 21: v = &o.g; break;
    default: return 1;
    }
    for (size_t i = 0; i < v->size(); ++i) out[i] = (T)(*v)[i];
    return 0;
}

template <class R>
int set_field(Oracle<R> &o, int id, const float *in) {
    std::vector<R> *v = nullptr;
    switch (id) {
    case 0: v = &o.rho; break;
    case 1: v = &o.ux; break;
    case 2: v = &o.uy; break;
    case 3: v = &o.uz; break;
    case 4: v = &o.phi; break;
    case 20: v = &o.f; break;
    case 21: v = &o.g; break;
    default: return 1;
    }
    for (size_t i = 0; i < v->size(); ++i) (*v)[i] = (R)in[i];
    return 0;
}

} // namespace

extern "C" {

void *oracle_new(const ssmd_params *p, int precision) {
    if (!p || (precision != 32 && precision != 64)) return nullptr;
    auto *h = new Handle{precision, nullptr};
    if (precision == 32) h->o = new Oracle<float>(*p);
    else h->o = new Oracle<double>(*p);
    return h;
}

void oracle_free(void *hv) {
    auto *h = static_cast<Handle *>(hv);
    if (!h) return;
    if (h->precision == 32) delete &O<float>(h);
    else delete &O<double>(h);
    delete h;
}

int oracle_init_jets(void *hv) {
    auto *h = static_cast<Handle *>(hv);
    if (h->precision == 32) O<float>(h).init_jets();
    else O<double>(h).init_jets();
    return 0;
}

// rho, ux, uy, uz, phi (N floats each) then setDistros
int oracle_init_macros(void *hv, const float *r, const float *x, const float *y, const float *z,
                       const float *ph) {
    auto *h = static_cast<Handle *>(hv);
    auto doit = [&](auto &o) {
        set_field(o, 0, r);
        set_field(o, 1, x);
        set_field(o, 2, y);
        set_field(o, 3, z);
        set_field(o, 4, ph);
        o.set_distros();
    };
    if (h->precision == 32) doit(O<float>(h));
    else doit(O<double>(h));
    return 0;
}

int oracle_step(void *hv, int n) {
    auto *h = static_cast<Handle *>(hv);
    for (int i = 0; i < n; ++i) {
        if (h->precision == 32) O<float>(h).one_step();
        else O<double>(h).one_step();
    }
    return 0;
}

int oracle_get(void *hv, int id, double *out) {
    auto *h = static_cast<Handle *>(hv);
    return h->precision == 32 ? get_field(O<float>(h), id, out) : get_field(O<double>(h), id, out);
}

int oracle_set(void *hv, int id, const float *in) {
    auto *h = static_cast<Handle *>(hv);
    return h->precision == 32 ? set_field(O<float>(h), id, in) : set_field(O<double>(h), id, in);
}

// Centreline mean of u_z and phi over the cells nearest the oil-nozzle axis
// (the definition of ssmd_centreline), FP64, nz values each.
int oracle_centreline(void *hv, double *uz_out, double *phi_out) {
    auto *h = static_cast<Handle *>(hv);
    auto run = [&](auto &o) {
        const int x0 = (int)std::floor(o.p.oil_cx), x1 = (int)std::ceil(o.p.oil_cx);
        const int y0 = (int)std::floor(o.p.oil_cy), y1 = (int)std::ceil(o.p.oil_cy);
        for (int z = 0; z < o.nz; ++z) {
            double su = 0, sp = 0;
            int n = 0;
            for (int y = y0; y <= y1; ++y)
                for (int x = x0; x <= x1; ++x) {
                    if (x < 0 || y < 0 || x >= o.nx || y >= o.ny) continue;
                    su += (double)(float)o.uz[o.idx(x, y, z)];
                    sp += (double)(float)o.phi[o.idx(x, y, z)];
                    ++n;
                }
            uz_out[z] = n ? su / n : 0.0;
            phi_out[z] = n ? sp / n : 0.0;
        }
    };
    if (h->precision == 32) run(O<float>(h));
    else run(O<double>(h));
    return 0;
}

// Connected components of fluid cells with phi > thr (6-neighbour, exact
// periodic axes wrap), by breadth-first search in index order, so the first
// cell reached is the component's smallest index.  Per component: root, cell
// count, FP64 sum of phi (as float, the precision the device reads) and
// whether it reaches the first fluid plane.  Sorted by root.
int oracle_droplets(void *hv, float thr, uint32_t *root, uint32_t *cells, double *vol, uint32_t *touch, int max,
                    int *n_out) {
    auto *h = static_cast<Handle *>(hv);
    auto run = [&](auto &o) {
        const int64_t N = o.N;
        std::vector<float> phi(N);
        for (int64_t i = 0; i < N; ++i) phi[i] = (float)o.phi[i];
        auto fg = [&](int x, int y, int z) { return o.fluid(x, y, z) && phi[o.idx(x, y, z)] > thr; };
        std::vector<uint8_t> seen(N, 0);
        std::vector<int64_t> queue;
        int n = 0;
        for (int z = 0; z < o.nz; ++z)
            for (int y = 0; y < o.ny; ++y)
                for (int x = 0; x < o.nx; ++x) {
                    const int64_t i = o.idx(x, y, z);
                    if (seen[i] || !fg(x, y, z)) continue;
                    uint32_t cnt = 0;
                    double v = 0;
                    uint32_t t = 0;
                    queue.assign(1, i);
                    seen[i] = 1;
                    for (size_t k = 0; k < queue.size(); ++k) {
                        const int64_t c = queue[k];
                        const int cx = (int)(c % o.nx), cy = (int)((c / o.nx) % o.ny), cz = (int)(c / ((int64_t)o.nx * o.ny));
                        ++cnt;
                        v += (double)phi[c];
                        if (cz == o.lo[2]) t = 1;
                        const int d[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
                        for (auto &e : d) {
                            const int qx = o.nb(0, cx + e[0]), qy = o.nb(1, cy + e[1]), qz = o.nb(2, cz + e[2]);
                            if (qx < 0 || qy < 0 || qz < 0 || !fg(qx, qy, qz)) continue;
                            const int64_t j = o.idx(qx, qy, qz);
                            if (!seen[j]) {
                                seen[j] = 1;
                                queue.push_back(j);
                            }
                        }
                    }
                    if (n < max) {
                        root[n] = (uint32_t)i;
                        cells[n] = cnt;
                        vol[n] = v;
                        touch[n] = t;
                    }
                    ++n;
                }
        *n_out = n;
    };
    if (h->precision == 32) run(O<float>(h));
    else run(O<double>(h));
    return 0;
}

double oracle_noise(uint64_t seed, uint64_t step, uint32_t cell, uint32_t stream) {
    return ssmd_noise::gaussian(seed, step, cell, stream);
}

} // extern "C"
