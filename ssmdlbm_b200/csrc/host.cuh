// host.cuh — host-side helpers shared by the API and the per-lattice kernel TUs.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <queue>
#include <string>
#include <vector>

#include "../../include/ssmd.h"
#include "bulk.cuh"
#include "tma.cuh"
#include "init.cuh"
#include "reduce.cuh"
#include "surface.cuh"

namespace ssmd {
namespace host {

int fail(int code, const char *fmt, ...);
int cuda_check(cudaError_t e, const char *what);

// Bulk-kernel timing events of the calling thread (ssmd_profile_*); returns the
// event pair for the next launch, or nulls when profiling is off or full.
void profile_next(cudaEvent_t *before, cudaEvent_t *after);

constexpr size_t kStatusOff = 0;
constexpr size_t kRedOutOff = 256;
constexpr size_t kPartialOff = 512;
constexpr int kMaxRedBlocks = 1024;
constexpr size_t kWorkspaceBytes = kPartialOff + sizeof(double) * kRedVals * kMaxRedBlocks;

// element sizes of the hydrodynamic (f) and phase (g) populations
inline size_t f_storage_size(int s) { return s == SSMD_STORAGE_F32 ? 4 : 2; }
inline size_t g_storage_size(int s) { return (s == SSMD_STORAGE_F32 || s == SSMD_STORAGE_F16_G32) ? 4 : 2; }

inline Geometry make_geometry(const ssmd_params &p) {
    Geometry G{};
    G.nx = p.nx;
    G.ny = p.ny;
    G.nz = p.nz;
    G.nxy = p.nx * p.ny;
    G.cells = (uint64_t)p.nx * p.ny * p.nz;
    G.bcx = p.bc_x;
    G.bcy = p.bc_y;
    G.bcz = p.bc_z;
    auto lohi = [](int bc, uint32_t n, int &lo, int &hi) {
        lo = bc == SSMD_BC_PERIODIC ? 0 : 1;
        hi = bc == SSMD_BC_PERIODIC ? (int)n - 1 : (int)n - 2;
    };
    lohi(p.bc_x, p.nx, G.x_lo, G.x_hi);
    lohi(p.bc_y, p.ny, G.y_lo, G.y_hi);
    lohi(p.bc_z, p.nz, G.z_lo, G.z_hi);
    return G;
}

inline Physics make_physics(const ssmd_params &p) {
    Physics P{};
    P.nu_water = p.nu_water;
    P.nu_oil_minus_water = p.nu_oil - p.nu_water; // FP32, as the reference's constexpr difference
    P.omco_water = p.omco_water;
    P.omco_oil = p.omco_oil;
    P.omco_ref = p.omco_ref;
    P.sigma = p.sigma;
    P.gamma = p.gamma;
    P.omega_g = p.omega_g;
    P.u_oil = p.u_oil;
    P.oil_cx = p.oil_cx;
    P.oil_cy = p.oil_cy;
    P.oil_r2 = p.oil_r2;
    P.u_water = p.u_water;
    P.water_cx = p.water_cx;
    P.water_cz = p.water_cz;
    P.water_r2 = p.water_r2;
    P.noise_amp = p.noise_amp;
    P.seed = p.seed;
    return P;
}

inline Fields make_fields(const LBMFields &f) {
    Fields F{};
    F.rho = f.rho;
    F.ux = f.ux;
    F.uy = f.uy;
    F.uz = f.uz;
    F.pxx = f.pxx;
    F.pyy = f.pyy;
    F.pzz = f.pzz;
    F.pxy = f.pxy;
    F.pxz = f.pxz;
    F.pyz = f.pyz;
    F.phi = f.phi;
    return F;
}

inline DeviceStatus *status_of(const ssmd_params &p) {
    return reinterpret_cast<DeviceStatus *>(static_cast<char *>(p.workspace) + kStatusOff);
}

inline int check_fields(const ssmd_params &p, const LBMFields *f) {
    if (!f) return fail(SSMD_ERR_INVALID_ARGUMENT, "fields is null");
    const void *need[] = {f->rho, f->ux, f->uy, f->uz, f->pxx, f->pyy, f->pzz, f->pxy, f->pxz,
                          f->pyz, f->phi, f->f, f->g, p.f_alt, p.g_alt, p.workspace};
    const char *names[] = {"rho", "ux", "uy", "uz", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz",
                           "phi", "f", "g", "f_alt", "g_alt", "workspace"};
    for (int i = 0; i < 16; ++i)
        if (!need[i]) return fail(SSMD_ERR_INVALID_ARGUMENT, "device pointer %s is null", names[i]);
    if (p.workspace_bytes < kWorkspaceBytes)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "workspace_bytes %zu < required %zu",
                    p.workspace_bytes, kWorkspaceBytes);
    return SSMD_OK;
}

static __global__ void set_status_kernel(DeviceStatus *s, unsigned long long step) {
    s->flags = 0u;
    s->step = step;
    s->work_next = 0u;
    s->avg_t = 0u;
}

inline Averages make_averages(const ssmd_params &p) {
    Averages A{};
    if (const ssmd_derived *d = p.derived) {
        A.phi = d->avg_phi;
        A.ux = d->avg_ux;
        A.uy = d->avg_uy;
        A.uz = d->avg_uz;
        A.uxux = d->avg_uxux;
        A.uyuy = d->avg_uyuy;
        A.uzuz = d->avg_uzuz;
        A.uxuy = d->avg_uxuy;
        A.uxuz = d->avg_uxuz;
        A.uyuz = d->avg_uyuz;
    }
    return A;
}

// Running means at cells the bulk kernel does not update (ghost layers), from
// the macroscopic fields the boundary kernels wrote; t = avg_t + 1.
static __global__ void averages_kernel(Geometry G, Fields F, Averages A, const DeviceStatus *status,
                                       int ghost_only) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= G.cells) return;
    if (ghost_only) {
        const uint32_t c = (uint32_t)i;
        const int x = c % G.nx, y = (c / G.nx) % G.ny, z = c / G.nxy;
        if (x >= G.x_lo && x <= G.x_hi && y >= G.y_lo && y <= G.y_hi && z >= G.z_lo && z <= G.z_hi) return;
    }
    const float t = (float)(status->avg_t + 1u);
    accumulate_averages(A, i, t, F.phi[i], F.ux[i], F.uy[i], F.uz[i]);
}

static __global__ void advance_avg_kernel(DeviceStatus *status) { status->avg_t += 1u; }

// Dynamic shared memory of a bulk instantiation (TMA boxes or slabs).
template <int Q, class T, int PATH>
constexpr size_t bulk_dyn_smem() {
    return PATH == 2 ? GBox<phase_t<T>>::SMEM : (PATH == 3 ? Slab<T>::template smem<Q>() : 0);
}

// Resident bulk work items per SM for this instantiation (queried once per
// device and kernel, after raising its dynamic shared-memory limit) and the
// SM count.
template <int Q, class T, int PATH>
inline void bulk_slots(int &per_sm, int &sms) {
    static thread_local int cached_dev = -1, cached_per_sm = 0, cached_sms = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != cached_dev) {
        int n = 0, m = 0;
        const size_t dyn = bulk_dyn_smem<Q, T, PATH>();
        if (dyn > 0)
            cudaFuncSetAttribute(bulk_kernel<Q, T, phase_t<T>, PATH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dyn);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bulk_kernel<Q, T, phase_t<T>, PATH>, kThreads, dyn) !=
            cudaSuccess)
            n = 1;
        if (cudaDeviceGetAttribute(&m, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) m = 148;
        cached_dev = dev;
        cached_per_sm = n > 0 ? n : 1;
        cached_sms = m > 0 ? m : 1;
    }
    per_sm = cached_per_sm;
    sms = cached_sms;
}

// Makespan of a z chunk under the hardware's greedy block scheduling, in
// plane-updates: the work items in launch order (columns fastest, then
// chunks), each holding a resident slot for its planes plus kProloguePlanes
// (the ring prologue), the next item starting on the first slot to free.  On
// B200 this model tracks the measured kernel time across chunk sizes
// (correlation 0.98 on the 128 x 128 x 512 jet, chunks of 12-32 planes, and
// it ranks 56 planes, one wave of 4 items per SM, first among 28-64 there,
// as measured).
constexpr double kProloguePlanes = 4.0;
constexpr int kMaxAutoChunk = 64;

inline double chunk_makespan(long cols, int nzf, int zc, int slots) {
    std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
    for (int i = 0; i < slots; ++i) free_at.push(0.0);
    double end = 0.0;
    for (int z0 = 0; z0 < nzf; z0 += zc) {
        const double len = std::min(zc, nzf - z0) + kProloguePlanes;
        for (long c = 0; c < cols; ++c) {
            const double t = free_at.top() + len;
            free_at.pop();
            free_at.push(t);
            end = std::max(end, t);
        }
    }
    return end;
}

// Bulk tiling: 32 x 8 columns.  Unless the caller fixes tile_z, the z chunk
// (8..64 planes, the range the model was checked on) minimises
// chunk_makespan; the choice is cached per lattice shape and slot count (the
// search costs a few ms on the largest lattices).
inline void tiling(const ssmd_params &p, const Geometry &G, int slots, int &tiles_x, int &tiles_y,
                   int &zchunk, int &nchunks) {
    tiles_x = (int)((G.nx + kTX - 1) / kTX);
    tiles_y = (int)((G.ny + kTY - 1) / kTY);
    const int nzf = G.z_hi - G.z_lo + 1;
    const long cols = (long)tiles_x * tiles_y;
    if (p.tile_z > 0) {
        zchunk = p.tile_z;
    } else {
        thread_local long c_cols = -1;
        thread_local int c_nzf = -1, c_slots = -1, c_best = 16;
        if (cols != c_cols || nzf != c_nzf || slots != c_slots) {
            double best = 1e300;
            int arg = std::min(16, nzf);
            for (int zc = std::min(8, nzf); zc <= std::min(nzf, kMaxAutoChunk); ++zc) {
                const double t = chunk_makespan(cols, nzf, zc, slots);
                if (t <= best * (1.0 + 1e-9)) { // ties: the longer chunk (fewer prologues)
                    best = std::min(best, t);
                    arg = zc;
                }
            }
            c_cols = cols;
            c_nzf = nzf;
            c_slots = slots;
            c_best = arg;
        }
        zchunk = c_best;
    }
    if (zchunk > nzf) zchunk = nzf;
    nchunks = (nzf + zchunk - 1) / zchunk;
}

template <class TF, class TG>
inline void set_closure(StepArgs<TF, TG> &a, const ssmd_params &p) {
    a.clo_nut = p.closure ? p.closure->nut : nullptr;
    a.clo_cs = (p.closure && p.closure->nut) ? p.closure->sigma_scale : nullptr;
    a.avg = make_averages(p);
}

template <int Q, class T>
int launch_step(const ssmd_params &p, const LBMFields &fl, uint64_t step, uint32_t flags,
                cudaStream_t st) {
    using TG = phase_t<T>;
    StepArgs<T, TG> a{};
    a.geo = make_geometry(p);
    a.phys = make_physics(p);
    a.fld = make_fields(fl);
    const bool even = (step & 1ull) == 0ull;
    a.f_src = static_cast<const T *>(even ? fl.f : p.f_alt);
    a.f_dst = static_cast<T *>(even ? p.f_alt : fl.f);
    a.g_src = static_cast<const TG *>(even ? fl.g : p.g_alt);
    a.g_dst = static_cast<TG *>(even ? p.g_alt : fl.g);
    set_bases(a, Q);
    a.status = status_of(p);
    set_closure(a, p);
    a.flags = flags;
    // Kernel path: per-cell gathers (default), TMA boxes for the phi halo, or
    // TMA slabs for the populations; the TMA paths need a 16-byte aligned x pitch.
    CUtensorMap gmap{}, fmap{};
    int path = p.bulk_path == SSMD_PATH_AUTO ? SSMD_PATH_GATHER : p.bulk_path;
    if (path == SSMD_PATH_TMA &&
        !encode_populations<TG>(&gmap, a.g_src, a.geo.nx, a.geo.ny, a.geo.nz, 7, GBox<TG>::WX, kHY))
        return fail(SSMD_ERR_UNSUPPORTED, "TMA path needs nx * element size to be a multiple of 16 bytes");
    // the slab path stages f and g slabs of one element size
    constexpr bool kSlabs = sizeof(T) == sizeof(TG);
    if (path == SSMD_PATH_SLAB && !kSlabs)
        return fail(SSMD_ERR_UNSUPPORTED, "slab path needs f and g of one element size");
    if (path == SSMD_PATH_SLAB &&
        !(encode_populations<TG>(&gmap, a.g_src, a.geo.nx, a.geo.ny, a.geo.nz, 7, Slab<TG>::WX, kTY) &&
          encode_populations<T>(&fmap, a.f_src, a.geo.nx, a.geo.ny, a.geo.nz, Q, Slab<T>::WX, kTY)))
        return fail(SSMD_ERR_UNSUPPORTED, "slab path needs nx * element size to be a multiple of 16 bytes");
    int per_sm = 1, sms = 1;
    if (path == SSMD_PATH_TMA) bulk_slots<Q, T, 2>(per_sm, sms);
    else if (path == SSMD_PATH_SLAB) {
        if constexpr (kSlabs) bulk_slots<Q, T, 3>(per_sm, sms);
    } else bulk_slots<Q, T, 1>(per_sm, sms);
    tiling(p, a.geo, per_sm * sms, a.tiles_x, a.tiles_y, a.zchunk, a.nzchunks);
    a.halo_mod = (a.geo.bcx == BC_PERIODIC && a.geo.nx < (uint32_t)(kTX + 4)) ||
                 (a.geo.bcy == BC_PERIODIC && a.geo.ny < (uint32_t)(kTY + 4)) ||
                 (a.geo.bcz == BC_PERIODIC && a.geo.nz < 6u);

    const dim3 blk(kTX, kTY);
    const unsigned nblk = (unsigned)(a.tiles_x * a.tiles_y * a.nzchunks);
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    profile_next(&ev0, &ev1);
    if (ev0) cudaEventRecord(ev0, st);
    if (path == SSMD_PATH_TMA)
        bulk_kernel<Q, T, TG, 2><<<nblk, blk, bulk_dyn_smem<Q, T, 2>(), st>>>(a, gmap, fmap);
    else if (path == SSMD_PATH_SLAB) {
        if constexpr (kSlabs) bulk_kernel<Q, T, TG, 3><<<nblk, blk, bulk_dyn_smem<Q, T, 3>(), st>>>(a, gmap, fmap);
    } else
        bulk_kernel<Q, T, TG, 1><<<nblk, blk, 0, st>>>(a, gmap, fmap);
    if (ev1) cudaEventRecord(ev1, st);
    if (int e = cuda_check(cudaGetLastError(), "bulk_kernel launch")) return e;

    const Geometry &G = a.geo;
    const dim3 b2(32, 4);
    auto grid2 = [&](uint32_t n0, uint32_t n1) {
        return dim3((n0 + b2.x - 1) / b2.x, (n1 + b2.y - 1) / b2.y);
    };
    if (G.bcz == BC_JET && G.bcy != BC_JET && G.nz >= 3) {
        // the two z faces are independent: one launch (reference order otherwise)
        dim3 g = grid2(G.nx, G.ny);
        g.z = 2;
        bc_jet_z<Q, T, TG><<<g, b2, 0, st>>>(a);
    } else {
        if (G.bcy == BC_JET) bc_water_inflow<Q, T, TG><<<grid2(G.nx, G.nz), b2, 0, st>>>(a);
        if (G.bcz == BC_JET) bc_oil_inflow<Q, T, TG><<<grid2(G.nx, G.ny), b2, 0, st>>>(a);
        if (G.bcy == BC_JET) bc_outflow_y<Q, T, TG><<<grid2(G.nx, G.nz), b2, 0, st>>>(a);
        if (G.bcz == BC_JET) bc_outflow_z<Q, T, TG><<<grid2(G.nx, G.ny), b2, 0, st>>>(a);
    }
    if (G.bcx == BC_COPY) bc_copy_x<Q, T, TG><<<grid2(G.ny, G.nz), b2, 0, st>>>(a);
    if (G.bcy == BC_COPY) bc_copy_y<Q, T, TG><<<grid2(G.nx, G.nz), b2, 0, st>>>(a);
    if (flags & SSMD_STEP_AVERAGE) {
        // the bulk kernel updated the fluid cells; the ghost layers follow, then t advances
        const unsigned nb = (unsigned)((G.cells + 255) / 256);
        averages_kernel<<<nb, 256, 0, st>>>(G, a.fld, a.avg, a.status, 1);
        advance_avg_kernel<<<1, 1, 0, st>>>(a.status);
    }
    return cuda_check(cudaGetLastError(), "boundary kernel launch");
}

template <int Q, class T>
int launch_init_pops(const ssmd_params &p, const LBMFields &fl, cudaStream_t st) {
    const Geometry G = make_geometry(p);
    const unsigned nb = (unsigned)((G.cells + 255) / 256);
    using TG = phase_t<T>;
    init_populations_kernel<Q, T, TG><<<nb, 256, 0, st>>>(G, make_fields(fl), static_cast<T *>(fl.f),
                                                           static_cast<T *>(p.f_alt),
                                                           static_cast<TG *>(fl.g),
                                                           static_cast<TG *>(p.g_alt));
    return cuda_check(cudaGetLastError(), "init_populations launch");
}


#define SSMD_INSTANTIATE(Q, T)                                                                     \
    template int launch_step<Q, T>(const ssmd_params &, const LBMFields &, uint64_t, uint32_t,      \
                                   cudaStream_t);                                                   \
    template int launch_init_pops<Q, T>(const ssmd_params &, const LBMFields &, cudaStream_t);

#define SSMD_DECLARE(Q, T)                                                                         \
    extern template int launch_step<Q, T>(const ssmd_params &, const LBMFields &, uint64_t,        \
                                          uint32_t, cudaStream_t);                                  \
    extern template int launch_init_pops<Q, T>(const ssmd_params &, const LBMFields &, cudaStream_t);

} // namespace host
} // namespace ssmd
