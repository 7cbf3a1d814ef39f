// common.cuh — storage types, kernel arguments and lattice indexing.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>

#include "../../include/ssmd.h"
#include "lattice.cuh"

namespace ssmd {

// ------------------------------------------------------------- storage
// Populations are kept "shifted" (f - w_q, reference src/cuda/utils.cuh:67-99);
// the reduced types only change the element type, arithmetic stays FP32.
// L2 policy for loads whose lines are read again within a few planes: the
// phase populations gathered into the phi ring are gathered again by the
// neighbouring tiles' ring borders and by the cell update four planes later,
// while the hydrodynamic stream passing through L2 in between is touched
// once.  Marking the ring's loads evict-last keeps more of those lines (on
// the 128 x 128 x 512 jet: D3Q27 FP32 0.483 -> 0.474 ms, D3Q19 FP32 0.397 ->
// 0.391 ms).  (createpolicy / ld.global.nc.L2::cache_hint, sm_80 and later.)
__device__ __forceinline__ uint64_t l2_keep_policy() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

template <class T>
struct Store;

template <>
struct Store<float> {
    static __device__ __forceinline__ float ld(const float *p) { return __ldg(p); }
    static __device__ __forceinline__ float ldc(const float *p) { return *p; } // coherent (same-kernel writers)
    static __device__ __forceinline__ float ld_keep(const float *p) { // read-only, L2 evict-last
        float v;
        asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(l2_keep_policy()));
        return v;
    }
    static __device__ __forceinline__ void st(float *p, float v) { *p = v; }
};
template <>
struct Store<__half> {
    static __device__ __forceinline__ float ld(const __half *p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ float ldc(const __half *p) { return __half2float(*p); }
    static __device__ __forceinline__ float ld_keep(const __half *p) {
        unsigned short v;
        asm("ld.global.nc.L2::cache_hint.b16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(l2_keep_policy()));
        return __half2float(__ushort_as_half(v));
    }
    static __device__ __forceinline__ void st(__half *p, float v) { *p = __float2half_rn(v); }
};
template <>
struct Store<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16 *p) {
        return __bfloat162float(__ldg(p));
    }
    static __device__ __forceinline__ float ldc(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
    static __device__ __forceinline__ float ld_keep(const __nv_bfloat16 *p) {
        unsigned short v;
        asm("ld.global.nc.L2::cache_hint.b16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(l2_keep_policy()));
        return __bfloat162float(__ushort_as_bfloat16(v));
    }
    static __device__ __forceinline__ void st(__nv_bfloat16 *p, float v) { *p = __float2bfloat16_rn(v); }
};

// Element type of the hydrodynamic populations under SSMD_STORAGE_F16_G32: an
// IEEE half like __half, as its own type so that its lattice keeps the phase
// populations in float (the reference's ENABLE_FP16=1 layout).
struct __align__(2) half_g32 {
    __half h;
};
template <>
struct Store<half_g32> {
    static __device__ __forceinline__ float ld(const half_g32 *p) { return __half2float(__ldg(&p->h)); }
    static __device__ __forceinline__ float ldc(const half_g32 *p) { return __half2float(p->h); }
    static __device__ __forceinline__ float ld_keep(const half_g32 *p) { return Store<__half>::ld_keep(&p->h); }
    static __device__ __forceinline__ void st(half_g32 *p, float v) { p->h = __float2half_rn(v); }
};

// Phase-population (g) storage for a storage type: the same type, except that
// BF16 runs keep g in IEEE half.  g carries phi in [0, 1], which needs mantissa
// bits rather than exponent range; with BF16's 8 bits the small anti-diffusion
// increments round away and the phi mass drifts (0.6 % after 1000 steps of a
// 64 x 64 x 128 jet, against 0.04 % with half).  Both are 2 bytes, so buffer
// sizes and layouts do not change.
template <class T>
struct PhaseStore {
    using type = T;
};
template <>
struct PhaseStore<__nv_bfloat16> {
    using type = __half;
};
template <>
struct PhaseStore<half_g32> {
    using type = float;
};
template <class T>
using phase_t = typename PhaseStore<T>::type;

// ------------------------------------------------------------- arguments
enum : int { BC_COPY = 0, BC_PERIODIC = 1, BC_JET = 2 };

struct DeviceStatus {
    unsigned int flags;      // bit 0: non-finite density seen in the bulk
    unsigned int pad0;
    unsigned long long step; // index of the step in progress (inlet noise)
    unsigned int work_next;  // persistent-kernel work counter
    unsigned int avg_t;      // running-mean updates done (derived fields)
    unsigned int pad1[10];
};

// Running means of the derived fields (null members are skipped).
struct Averages {
    float *phi, *ux, *uy, *uz;
    float *uxux, *uyuy, *uzuz, *uxuy, *uxuz, *uyuz;
};

// avg <- avg + (v - avg) / t, every operation rounded on its own (no FMA),
// the form of the reference's update (timeAverage.cuh:58-61).
__device__ __forceinline__ float avg_update(float avg, float v, float t) {
    return __fadd_rn(avg, __fdiv_rn(__fsub_rn(v, avg), t));
}

__device__ __forceinline__ void accumulate_averages(const Averages &A, uint64_t c, float t, float phi, float ux,
                                                    float uy, float uz) {
    if (A.phi) A.phi[c] = avg_update(A.phi[c], phi, t);
    if (A.ux) A.ux[c] = avg_update(A.ux[c], ux, t);
    if (A.uy) A.uy[c] = avg_update(A.uy[c], uy, t);
    if (A.uz) A.uz[c] = avg_update(A.uz[c], uz, t);
    if (A.uxux) A.uxux[c] = avg_update(A.uxux[c], __fmul_rn(ux, ux), t);
    if (A.uyuy) A.uyuy[c] = avg_update(A.uyuy[c], __fmul_rn(uy, uy), t);
    if (A.uzuz) A.uzuz[c] = avg_update(A.uzuz[c], __fmul_rn(uz, uz), t);
    if (A.uxuy) A.uxuy[c] = avg_update(A.uxuy[c], __fmul_rn(ux, uy), t);
    if (A.uxuz) A.uxuz[c] = avg_update(A.uxuz[c], __fmul_rn(ux, uz), t);
    if (A.uyuz) A.uyuz[c] = avg_update(A.uyuz[c], __fmul_rn(uy, uz), t);
}

struct Geometry {
    uint32_t nx, ny, nz;
    uint32_t nxy;   // nx * ny
    uint64_t cells; // nx * ny * nz
    int bcx, bcy, bcz;
    // fluid (colliding) index range per axis: [lo, hi]
    int x_lo, x_hi, y_lo, y_hi, z_lo, z_hi;
};

struct Physics {
    float nu_water, nu_oil_minus_water;
    float omco_water, omco_oil, omco_ref;
    float sigma, gamma, omega_g;
    float u_oil, oil_cx, oil_cy, oil_r2;
    float u_water, water_cx, water_cz, water_r2;
    float noise_amp;
    unsigned long long seed;
};

struct Fields {
    float *rho, *ux, *uy, *uz;
    float *pxx, *pyy, *pzz, *pxy, *pxz, *pyz;
    float *phi;
};

template <class TF, class TG>
struct StepArgs {
    Geometry geo;
    Physics phys;
    Fields fld;
    const TF *__restrict__ f_src;
    TF *__restrict__ f_dst;
    const TG *__restrict__ g_src;
    TG *__restrict__ g_dst;
    // per-direction bases f_src + q N, ... (set_bases): the bulk kernel reads
    // them from the parameter space, so every population access is a 32-bit
    // cell index scaled onto a base the kernel does not compute
    const TF *fq_src[27];
    TF *fq_dst[27];
    const TG *gq_src[7];
    TG *gq_dst[7];
    DeviceStatus *status;
    Averages avg;         // derived running means (SSMD_STEP_AVERAGE)
    const float *clo_nut; // learned closure: eddy viscosity per cell (null: off)
    const float *clo_cs;  // learned closure: surface-tension factor per cell
    uint32_t flags;       // SSMD_STEP_*
    int tiles_x, tiles_y; // bulk tiling
    int zchunk, nzchunks;
    int halo_mod;         // 1: a tile halo may wrap a periodic axis more than once
};

template <class TF, class TG>
inline void set_bases(StepArgs<TF, TG> &a, int Q) {
    for (int q = 0; q < 27; ++q) {
        a.fq_src[q] = q < Q ? a.f_src + (uint64_t)q * a.geo.cells : nullptr;
        a.fq_dst[q] = q < Q ? a.f_dst + (uint64_t)q * a.geo.cells : nullptr;
    }
    for (int q = 0; q < 7; ++q) {
        a.gq_src[q] = a.g_src + (uint64_t)q * a.geo.cells;
        a.gq_dst[q] = a.g_dst + (uint64_t)q * a.geo.cells;
    }
}

// ------------------------------------------------------------- indexing
__host__ __device__ __forceinline__ uint32_t cell_index(const Geometry &g, uint32_t x, uint32_t y,
                                                        uint32_t z) {
    return x + g.nx * y + g.nxy * z;
}

__host__ __device__ __forceinline__ uint64_t slot(const Geometry &g, int q, uint32_t idx) {
    return (uint64_t)q * g.cells + idx;
}

// Neighbour coordinate along one axis, with wrap when the axis is periodic.
// Returns -1 when the coordinate leaves a non-periodic lattice.
__host__ __device__ __forceinline__ int axis_nb(int c, int n, bool periodic) {
    if (periodic) {
        if (c < 0) return c + n;
        if (c >= n) return c - n;
        return c;
    }
    return (c < 0 || c >= n) ? -1 : c;
}

// Same for halo coordinates that may lie several lattice lengths away
// (tile halos on small periodic axes): full modulo.
__host__ __device__ __forceinline__ int axis_halo(int c, int n, bool periodic) {
    if (periodic) {
        int m = c % n;
        return m < 0 ? m + n : m;
    }
    return (c < 0 || c >= n) ? -1 : c;
}

} // namespace ssmd
