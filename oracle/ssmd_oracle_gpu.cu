// ssmd_oracle_gpu.cu — the oracle as CUDA kernels.  TEST INFRASTRUCTURE.
//
// The per-cell functions of oracle_cells.h (the oracle's restatement of the
// reference's step), launched one thread per cell (one per face cell for the
// boundaries) in the order the CPU oracle runs them, in FP64 (R = double) or
// FP32 (R = float, the reference's arithmetic).  Compiled with --fmad=false:
// no contraction, and +, -, *, / and sqrt correctly rounded, as in the CPU
// build (g++ -ffp-contract=off), so both instances produce the same bits;
// tests check that on the 64 x 64 x 128 jet.  It exists for lattices whose
// oracle runs take hours on the host cores (the 128 x 128 x 512 jet over
// 5000 steps, lattices beyond 2^32 population slots).  Only tests and
// fixture scripts load it; it owns its device memory.
//
// C API (oracle/oracle.py wraps it): oracle_gpu_new / _free / _init_jets /
// _init_macros / _step / _get / _last_error.  Field ids as in
// ssmd_oracle.cpp (0-13 scalar fields, 20 f, 21 g); _get returns doubles.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "oracle_cells.h"

namespace {

using ssmd_oracle::BC_COPY;
using ssmd_oracle::BC_JET;

thread_local std::string g_err;

int cuda_ok(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return 0;
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return 1;
}

constexpr int kThreads = 256;

unsigned blocks_for(int64_t n) {
    const int64_t b = (n + kThreads - 1) / kThreads;
    return (unsigned)(b < 65535 * 64 ? b : 65535 * 64);
}

// grid-stride loops over cells (x fastest) and over face cells
template <int PASS, class R>
__global__ void cell_pass(ssmd_oracle::Lattice<R> L) {
    const int64_t N = L.N;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % L.nx);
        const int64_t r = i / L.nx;
        const int y = (int)(r % L.ny);
        const int z = (int)(r / L.ny);
        if constexpr (PASS == 0) L.init_clear(i);
        if constexpr (PASS == 1) L.init_density(i);
        if constexpr (PASS == 2) L.set_distros_cell(x, y, z);
        if constexpr (PASS == 3) L.phase_cell(x, y, z);
        if constexpr (PASS == 4) L.normal_cell(x, y, z);
        if constexpr (PASS == 5) L.force_cell(x, y, z);
        if constexpr (PASS == 6) L.moments_cell(x, y, z);
        if constexpr (PASS == 7) L.collide_cell(x, y, z);
    }
}

// face passes over (a, b) in [a0, a1] x [b0, b1]
template <int FACE, class R>
__global__ void face_pass(ssmd_oracle::Lattice<R> L, int a0, int a1, int b0, int b1) {
    const int64_t na = a1 - a0 + 1, nb = b1 - b0 + 1, n = na * nb;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int a = a0 + (int)(k % na), b = b0 + (int)(k / na);
        if constexpr (FACE == 0) L.init_water_disc(a, b);   // (x, z)
        if constexpr (FACE == 1) L.init_oil_disc(a, b);     // (x, y)
        if constexpr (FACE == 2) L.water_inflow_cell(a, b); // (x, z)
        if constexpr (FACE == 3) L.oil_inflow_cell(a, b);   // (x, y)
        if constexpr (FACE == 4) L.outflow_y_cell(a, b);    // (x, z)
        if constexpr (FACE == 5) L.outflow_z_cell(a, b);    // (x, y)
        if constexpr (FACE == 6) L.copy_x_cell(a, b);       // (y, z)
        if constexpr (FACE == 7) L.copy_y_cell(a, b);       // (x, z)
    }
}

template <class R>
__global__ void widen(const float *in, R *out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (R)in[i];
}

template <class R>
__global__ void to_double(const R *in, double *out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

struct GpuOracleBase {
    virtual ~GpuOracleBase() = default;
    virtual int setup(const ssmd_params &p) = 0;
    virtual int init_jets() = 0;
    virtual int init_macros(const float *const host[5]) = 0;
    virtual void one_step() = 0;
    virtual int get(int id, double *out) = 0;
};

template <class R>
struct GpuOracle final : GpuOracleBase {
    using Lat = ssmd_oracle::Lattice<R>;
    Lat L{};
    std::vector<R *> owned;
    uint64_t step = 0; // index of the next step

    ~GpuOracle() override {
        for (R *p : owned) cudaFree(p);
    }

    int alloc(R **p, size_t n) {
        if (cuda_ok(cudaMalloc(p, n * sizeof(R)), "cudaMalloc")) return 1;
        owned.push_back(*p);
        return cuda_ok(cudaMemset(*p, 0, n * sizeof(R)), "cudaMemset");
    }

    int setup(const ssmd_params &p) override {
        L.setup(p);
        const size_t N = (size_t)L.N;
        R **fields[] = {&L.rho, &L.ux, &L.uy, &L.uz, &L.pxx, &L.pyy, &L.pzz, &L.pxy, &L.pxz, &L.pyz,
                             &L.phi, &L.fsx, &L.fsy, &L.fsz, &L.nX, &L.nY, &L.nZ, &L.nI};
        for (R **f : fields)
            if (alloc(f, N)) return 1;
        if (alloc(&L.f, (size_t)L.Q * N) || alloc(&L.g, 7 * N)) return 1;
        L.gold = nullptr;
        if (p.omega_g != 1.0f && alloc(&L.gold, 7 * N)) return 1;
        return 0;
    }

    template <int PASS>
    void cells() {
        cell_pass<PASS, R><<<blocks_for(L.N), kThreads>>>(L);
    }
    template <int FACE>
    void face(int a0, int a1, int b0, int b1) {
        if (a1 < a0 || b1 < b0) return;
        face_pass<FACE, R><<<blocks_for((int64_t)(a1 - a0 + 1) * (b1 - b0 + 1)), kThreads>>>(L, a0, a1, b0, b1);
    }

    int init_jets() override {
        cells<0>();
        if (L.p.bc_y == BC_JET) face<0>(0, L.nx - 1, 0, L.nz - 1);
        if (L.p.bc_z == BC_JET) face<1>(0, L.nx - 1, 0, L.ny - 1);
        cells<1>();
        cells<2>();
        step = 0;
        return cuda_ok(cudaDeviceSynchronize(), "init_jets");
    }

    int init_macros(const float *const host[5]) override {
        const size_t N = (size_t)L.N;
        float *tmp = nullptr;
        if (cuda_ok(cudaMalloc(&tmp, N * sizeof(float)), "cudaMalloc")) return 1;
        R *dst[5] = {L.rho, L.ux, L.uy, L.uz, L.phi};
        int e = 0;
        for (int k = 0; k < 5 && !e; ++k) {
            e = cuda_ok(cudaMemcpy(tmp, host[k], N * sizeof(float), cudaMemcpyHostToDevice), "upload");
            if (!e) widen<R><<<blocks_for(L.N), kThreads>>>(tmp, dst[k], L.N);
        }
        cudaFree(tmp);
        if (e) return e;
        cells<2>();
        step = 0;
        return cuda_ok(cudaDeviceSynchronize(), "init_macros");
    }

    // main.cu:159-169 with the graph of CUDAGraph.cuh:44-49
    void one_step() override {
        L.step = step;
        cells<3>();
        cells<4>();
        cells<5>();
        cells<6>();
        if (L.gold) cudaMemcpyAsync(L.gold, L.g, 7 * (size_t)L.N * sizeof(R), cudaMemcpyDeviceToDevice);
        cells<7>();
        if (L.p.bc_y == BC_JET) face<2>(0, L.nx - 1, 0, L.nz - 1);
        if (L.p.bc_z == BC_JET) face<3>(0, L.nx - 1, 0, L.ny - 1);
        if (L.p.bc_y == BC_JET) face<4>(L.lo[0], L.hi[0], L.lo[2], L.hi[2]);
        if (L.p.bc_z == BC_JET) face<5>(L.lo[0], L.hi[0], L.lo[1], L.hi[1]);
        if (L.p.bc_x == BC_COPY) face<6>(0, L.ny - 1, 0, L.nz - 1);
        if (L.p.bc_y == BC_COPY) face<7>(0, L.nx - 1, 0, L.nz - 1);
        ++step;
    }

    const R *field(int id, size_t &n) const {
        const size_t N = (size_t)L.N;
        n = N;
        switch (id) {
        case 0: return L.rho;
        case 1: return L.ux;
        case 2: return L.uy;
        case 3: return L.uz;
        case 4: return L.phi;
        case 5: return L.pxx;
        case 6: return L.pyy;
        case 7: return L.pzz;
        case 8: return L.pxy;
        case 9: return L.pxz;
        case 10: return L.pyz;
        case 11: return L.fsx;
        case 12: return L.fsy;
        case 13: return L.fsz;
        case 20: n = (size_t)L.Q * N; return L.f;
        case 21: n = 7 * N; return L.g;
        default: return nullptr;
        }
    }

    // field `id` to host doubles (through a device staging buffer for FP32)
    int get(int id, double *out) override {
        size_t n = 0;
        const R *src = field(id, n);
        if (!src) {
            g_err = "unknown field id";
            return 1;
        }
        if constexpr (sizeof(R) == sizeof(double))
            return cuda_ok(cudaMemcpy(out, src, n * sizeof(double), cudaMemcpyDeviceToHost), "download");
        const size_t chunk = (size_t)1 << 26;
        double *tmp = nullptr;
        if (cuda_ok(cudaMalloc(&tmp, chunk * sizeof(double)), "cudaMalloc")) return 1;
        int e = 0;
        for (size_t i = 0; i < n && !e; i += chunk) {
            const size_t m = n - i < chunk ? n - i : chunk;
            to_double<R><<<blocks_for((int64_t)m), kThreads>>>(src + i, tmp, (int64_t)m);
            e = cuda_ok(cudaMemcpy(out + i, tmp, m * sizeof(double), cudaMemcpyDeviceToHost), "download");
        }
        cudaFree(tmp);
        return e;
    }
};

} // namespace

extern "C" {

// precision: 64 (FP64 transcription) or 32 (the reference's FP32 arithmetic)
void *oracle_gpu_new(const ssmd_params *p, int precision) {
    if (!p || (precision != 32 && precision != 64)) return nullptr;
    GpuOracleBase *o = precision == 64 ? static_cast<GpuOracleBase *>(new GpuOracle<double>())
                                       : static_cast<GpuOracleBase *>(new GpuOracle<float>());
    if (o->setup(*p)) {
        delete o;
        return nullptr;
    }
    return o;
}

void oracle_gpu_free(void *h) { delete static_cast<GpuOracleBase *>(h); }

int oracle_gpu_init_jets(void *h) { return static_cast<GpuOracleBase *>(h)->init_jets(); }

int oracle_gpu_init_macros(void *h, const float *r, const float *x, const float *y, const float *z, const float *ph) {
    const float *const host[5] = {r, x, y, z, ph};
    return static_cast<GpuOracleBase *>(h)->init_macros(host);
}

int oracle_gpu_step(void *h, int n) {
    auto *o = static_cast<GpuOracleBase *>(h);
    for (int i = 0; i < n; ++i) o->one_step();
    return cuda_ok(cudaDeviceSynchronize(), "oracle_gpu_step");
}

// Copies field `id` as doubles to host memory `out`.
int oracle_gpu_get(void *h, int id, double *out) { return static_cast<GpuOracleBase *>(h)->get(id, out); }

const char *oracle_gpu_last_error(void) { return g_err.c_str(); }

} // extern "C"
