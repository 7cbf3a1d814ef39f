// ssmd_oracle.cpp — CPU oracle for the ssmd_b200 hot path.  TEST INFRASTRUCTURE.
//
// This file is the checker, never the product: only the tests, the smoke
// check and the CPU-baseline leg of bench.py load it.  It runs the
// reference's time step, restated cell by cell in oracle_cells.h (which cites
// the reference lines each function follows), over the whole lattice with
// OpenMP over z.  Templated on the real type: R = float mirrors the
// reference's FP32 arithmetic (compile with -ffp-contract=off), R = double is
// the FP64 transcription.  ssmd_oracle_gpu.cu runs the same functions as FP64
// CUDA kernels.
//
// Parity pin: tests compare this file against outputs of the reference's own
// CUDA kernels (oracle/_ref harness runs) committed under tests/golden/.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle_cells.h"

namespace {

using ssmd_oracle::Lattice;
using ssmd_oracle::BC_COPY;
using ssmd_oracle::BC_JET;

template <class R>
struct Oracle {
    Lattice<R> L;
    std::vector<R> rho, ux, uy, uz, pxx, pyy, pzz, pxy, pxz, pyz, phi, fsx, fsy, fsz;
    std::vector<R> f, g, gold, nX, nY, nZ, nI;
    const ssmd_params &p;
    int &nx, &ny, &nz;
    const int64_t &N;
    uint64_t step = 0; // index of the next step

    explicit Oracle(const ssmd_params &pp) : p(L.p), nx(L.nx), ny(L.ny), nz(L.nz), N(L.N) {
        L.setup(pp);
        for (auto *v : {&rho, &ux, &uy, &uz, &pxx, &pyy, &pzz, &pxy, &pxz, &pyz, &phi, &fsx, &fsy, &fsz,
                        &nX, &nY, &nZ, &nI})
            v->assign(N, R(0));
        f.assign((size_t)L.Q * N, R(0));
        g.assign((size_t)7 * N, R(0));
        if (p.omega_g != 1.0f) gold.assign((size_t)7 * N, R(0));
        R **ptrs[] = {&L.rho, &L.ux, &L.uy, &L.uz, &L.pxx, &L.pyy, &L.pzz, &L.pxy, &L.pxz, &L.pyz,
                      &L.phi, &L.fsx, &L.fsy, &L.fsz, &L.nX, &L.nY, &L.nZ, &L.nI};
        std::vector<R> *vecs[] = {&rho, &ux, &uy, &uz, &pxx, &pyy, &pzz, &pxy, &pxz, &pyz,
                                  &phi, &fsx, &fsy, &fsz, &nX, &nY, &nZ, &nI};
        for (size_t k = 0; k < sizeof(vecs) / sizeof(vecs[0]); ++k) *ptrs[k] = vecs[k]->data();
        L.f = f.data();
        L.g = g.data();
        L.gold = gold.empty() ? nullptr : gold.data();
    }

    int64_t idx(int x, int y, int z) const { return L.idx(x, y, z); }
    int nb(int d, int c) const { return L.nb(d, c); }
    bool fluid(int x, int y, int z) const { return L.fluid(x, y, z); }

    template <class Fn>
    void cells(Fn fn) {
#pragma omp parallel for
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) fn(x, y, z);
    }

    void init_jets() {
        for (int64_t i = 0; i < N; ++i) L.init_clear(i);
        if (p.bc_y == BC_JET)
            for (int z = 0; z < nz; ++z)
                for (int x = 0; x < nx; ++x) L.init_water_disc(x, z);
        if (p.bc_z == BC_JET)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) L.init_oil_disc(x, y);
        for (int64_t i = 0; i < N; ++i) L.init_density(i);
        set_distros();
    }

    void set_distros() {
        cells([&](int x, int y, int z) { L.set_distros_cell(x, y, z); });
        step = 0;
    }

    // main.cu:159-169 with the graph of CUDAGraph.cuh:44-49
    void one_step() {
        L.step = step;
        cells([&](int x, int y, int z) { L.phase_cell(x, y, z); });
        cells([&](int x, int y, int z) { L.normal_cell(x, y, z); });
        cells([&](int x, int y, int z) { L.force_cell(x, y, z); });
        cells([&](int x, int y, int z) { L.moments_cell(x, y, z); });
        if (p.omega_g != 1.0f) std::copy(g.begin(), g.end(), gold.begin()); // post-stream g (BGK only)
        cells([&](int x, int y, int z) { L.collide_cell(x, y, z); });
        if (p.bc_y == BC_JET)
            for (int z = 0; z < nz; ++z)
                for (int x = 0; x < nx; ++x) L.water_inflow_cell(x, z);
        if (p.bc_z == BC_JET)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) L.oil_inflow_cell(x, y);
        if (p.bc_y == BC_JET)
            for (int z = L.lo[2]; z <= L.hi[2]; ++z)
                for (int x = L.lo[0]; x <= L.hi[0]; ++x) L.outflow_y_cell(x, z);
        if (p.bc_z == BC_JET)
            for (int y = L.lo[1]; y <= L.hi[1]; ++y)
                for (int x = L.lo[0]; x <= L.hi[0]; ++x) L.outflow_z_cell(x, y);
        if (p.bc_x == BC_COPY)
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y) L.copy_x_cell(y, z);
        if (p.bc_y == BC_COPY)
            for (int z = 0; z < nz; ++z)
                for (int x = 0; x < nx; ++x) L.copy_y_cell(x, z);
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

template <class R, class F>
void centreline_of(const Lattice<R> &o, const F *uz, const F *phi, double *uz_out, double *phi_out) {
    const int x0 = (int)std::floor(o.p.oil_cx), x1 = (int)std::ceil(o.p.oil_cx);
    const int y0 = (int)std::floor(o.p.oil_cy), y1 = (int)std::ceil(o.p.oil_cy);
    for (int z = 0; z < o.nz; ++z) {
        double su = 0, sp = 0;
        int n = 0;
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x) {
                if (x < 0 || y < 0 || x >= o.nx || y >= o.ny) continue;
                su += (double)(float)uz[o.idx(x, y, z)];
                sp += (double)(float)phi[o.idx(x, y, z)];
                ++n;
            }
        uz_out[z] = n ? su / n : 0.0;
        phi_out[z] = n ? sp / n : 0.0;
    }
}

template <class R, class F>
void droplets_of(const Lattice<R> &o, const F *phi_in, float thr, uint32_t *root, uint32_t *cells, double *vol,
                 uint32_t *touch, int max, int *n_out) {
    const int64_t N = o.N;
    std::vector<float> phi(N);
    for (int64_t i = 0; i < N; ++i) phi[i] = (float)phi_in[i];
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
    if (h->precision == 32) centreline_of(O<float>(h).L, O<float>(h).uz.data(), O<float>(h).phi.data(), uz_out, phi_out);
    else centreline_of(O<double>(h).L, O<double>(h).uz.data(), O<double>(h).phi.data(), uz_out, phi_out);
    return 0;
}

// The same from host arrays (N doubles each, [z][y][x]) of a lattice with
// parameters p: the statistics of the FP64 GPU instance, read back.
int oracle_centreline_arrays(const ssmd_params *p, const double *uz, const double *phi, double *uz_out,
                             double *phi_out) {
    Lattice<double> L{};
    L.setup(*p);
    centreline_of(L, uz, phi, uz_out, phi_out);
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
    if (h->precision == 32) droplets_of(O<float>(h).L, O<float>(h).phi.data(), thr, root, cells, vol, touch, max, n_out);
    else droplets_of(O<double>(h).L, O<double>(h).phi.data(), thr, root, cells, vol, touch, max, n_out);
    return 0;
}

int oracle_droplets_arrays(const ssmd_params *p, const double *phi, float thr, uint32_t *root, uint32_t *cells,
                           double *vol, uint32_t *touch, int max, int *n_out) {
    Lattice<double> L{};
    L.setup(*p);
    droplets_of(L, phi, thr, root, cells, vol, touch, max, n_out);
    return 0;
}

double oracle_noise(uint64_t seed, uint64_t step, uint32_t cell, uint32_t stream) {
    return ssmd_noise::gaussian(seed, step, cell, stream);
}

} // extern "C"
