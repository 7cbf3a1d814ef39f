// stats.cu — jet statistics on the device: centreline profile and droplets.
//
// The reference writes raw phi / rho fields only (src/main.cu:121-145) and
// leaves statistics to offline post-processing; its optional running means
// (src/derivedFields/operators/timeAverage.cuh:37-82) are the closest
// counterpart.  These kernels read the macroscopic arrays, so they need a
// step with SSMD_STEP_STORE_MACROS (or the initial state) first.
//
//   centreline: for every z, the mean of u_z and of phi over the (one, two
//     or four) cells nearest the oil nozzle axis (x, y) = (oil_cx, oil_cy), FP64.
//   droplets: connected components of {fluid cells with phi > threshold}
//     under 6-neighbour connectivity (exact-periodic axes wrap), labelled with
//     a lock-free union-find: every label points at a smaller or equal index,
//     unions hook the larger root under the smaller one with atomicMin
//     (the GPU union-find of Playne and Hawick, IEEE TPDS 2018), then every
//     label is compressed to its root (the smallest index of the component).
//     Per component: cell count, FP64 sum of phi (the "volume"), and whether
//     it touches the first fluid plane above the oil inlet.
#include <cuda_runtime.h>

#include "host.cuh"

using namespace ssmd;
using namespace ssmd::host;

namespace {

constexpr uint32_t kBG = 0xFFFFFFFFu;

struct DropScratch {
    uint32_t *label;
    uint32_t *count;
    double *volume;
    uint32_t *touch;
    uint32_t *n_out;
    ssmd_droplet *list;
    int max_list;
};

__device__ __forceinline__ bool fluid_cell(const Geometry &G, int x, int y, int z) {
    return x >= G.x_lo && x <= G.x_hi && y >= G.y_lo && y <= G.y_hi && z >= G.z_lo && z <= G.z_hi;
}

__global__ void centreline_kernel(Geometry G, Fields F, float cx, float cy, double *uz_out, double *phi_out) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= (int)G.nz) return;
    const int x0 = (int)floorf(cx), x1 = (int)ceilf(cx);
    const int y0 = (int)floorf(cy), y1 = (int)ceilf(cy);
    double su = 0.0, sp = 0.0;
    int n = 0;
    for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x) {
            if (x < 0 || y < 0 || x >= (int)G.nx || y >= (int)G.ny) continue;
            const uint32_t c = cell_index(G, x, y, z);
            su += (double)F.uz[c];
            sp += (double)F.phi[c];
            ++n;
        }
    uz_out[z] = n ? su / n : 0.0;
    phi_out[z] = n ? sp / n : 0.0;
}

__global__ void ccl_init(Geometry G, const float *phi, float thr, DropScratch S) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= G.cells) return;
    const uint32_t c = (uint32_t)i;
    const int x = c % G.nx, y = (c / G.nx) % G.ny, z = c / G.nxy;
    S.label[c] = (fluid_cell(G, x, y, z) && phi[c] > thr) ? c : kBG;
    S.count[c] = 0u;
    S.volume[c] = 0.0;
    S.touch[c] = 0u;
}

__device__ __forceinline__ uint32_t find_root(const uint32_t *L, uint32_t a) {
    uint32_t p = ((volatile const uint32_t *)L)[a];
    while (p != a) {
        a = p;
        p = ((volatile const uint32_t *)L)[a];
    }
    return a;
}

__device__ __forceinline__ void unite(uint32_t *L, uint32_t a, uint32_t b) {
    // bounded: each retry strictly lowers the label at one of the two roots
    for (int guard = 0; guard < (1 << 20); ++guard) {
        a = find_root(L, a);
        b = find_root(L, b);
        if (a == b) return;
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicMin(&L[b], a);
        if (old == b) return;
        b = old;
    }
}

__global__ void ccl_union(Geometry G, DropScratch S) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= G.cells) return;
    const uint32_t c = (uint32_t)i;
    if (S.label[c] == kBG) return;
    const int x = c % G.nx, y = (c / G.nx) % G.ny, z = c / G.nxy;
    const int nb[3][3] = {{x + 1, y, z}, {x, y + 1, z}, {x, y, z + 1}};
    const bool per[3] = {G.bcx == BC_PERIODIC, G.bcy == BC_PERIODIC, G.bcz == BC_PERIODIC};
    const int n[3] = {(int)G.nx, (int)G.ny, (int)G.nz};
    for (int d = 0; d < 3; ++d) {
        int q[3] = {nb[d][0], nb[d][1], nb[d][2]};
        if (q[d] >= n[d]) {
            if (!per[d]) continue;
            q[d] -= n[d];
        }
        if (!fluid_cell(G, q[0], q[1], q[2])) continue;
        const uint32_t j = cell_index(G, q[0], q[1], q[2]);
        if (S.label[j] == kBG) continue;
        unite(S.label, c, j);
    }
}

__global__ void ccl_compress_accumulate(Geometry G, const float *phi, DropScratch S) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= G.cells) return;
    const uint32_t c = (uint32_t)i;
    if (S.label[c] == kBG) return;
    const uint32_t r = find_root(S.label, c);
    atomicAdd(&S.count[r], 1u);
    atomicAdd(&S.volume[r], (double)phi[c]);
    if ((int)(c / G.nxy) == G.z_lo) S.touch[r] = 1u;
}

__global__ void ccl_collect(Geometry G, DropScratch S) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= G.cells) return;
    const uint32_t c = (uint32_t)i;
    const uint32_t n = S.count[c];
    if (n == 0u) return;
    const uint32_t slot_i = atomicAdd(S.n_out, 1u);
    if ((int)slot_i >= S.max_list) return;
    ssmd_droplet d;
    d.root = c;
    d.cells = n;
    d.volume = S.volume[c];
    d.touches_inlet = S.touch[c];
    d.reserved = 0u;
    S.list[slot_i] = d;
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// Phase-field populations that cross the boundary of the fluid region in the
// step just taken.  In the pull layout fluid cell x gathers direction q from
// slot q of x - c_q, so phi enters from ghost slots (q, x - c_q) and leaves
// through the fluid slots (q, x) whose x + c_q is a ghost cell.  FP64 sums;
// with the collision conserving phi per cell this closes the budget
// sum phi^{n+1} = sum phi^n + inflow - outflow.
template <class TG>
__global__ void phase_flux_kernel(Geometry G, const TG *g, double *acc) {
    __shared__ double s_in[256], s_out[256];
    double in = 0.0, out = 0.0;
    const bool per[3] = {G.bcx == BC_PERIODIC, G.bcy == BC_PERIODIC, G.bcz == BC_PERIODIC};
    const int n[3] = {(int)G.nx, (int)G.ny, (int)G.nz};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < G.cells;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = (uint32_t)i;
        const int p[3] = {(int)(c % G.nx), (int)((c / G.nx) % G.ny), (int)(c / G.nxy)};
        if (!fluid_cell(G, p[0], p[1], p[2])) continue;
        for (int q = 1; q < 7; ++q) {
            const int axis = (q - 1) >> 1, sgn = (q & 1) ? 1 : -1; // 1:+x 2:-x 3:+y 4:-y 5:+z 6:-z
            int a[3] = {p[0], p[1], p[2]}, b[3] = {p[0], p[1], p[2]};
            a[axis] = axis_nb(p[axis] - sgn, n[axis], per[axis]); // source of direction q
            b[axis] = axis_nb(p[axis] + sgn, n[axis], per[axis]); // where this cell's q goes
            if (!fluid_cell(G, a[0], a[1], a[2])) in += (double)Store<TG>::ld(g + slot(G, q, cell_index(G, a[0], a[1], a[2])));
            if (!fluid_cell(G, b[0], b[1], b[2])) out += (double)Store<TG>::ld(g + slot(G, q, c));
        }
    }
    s_in[threadIdx.x] = in;
    s_out[threadIdx.x] = out;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            s_in[threadIdx.x] += s_in[threadIdx.x + w];
            s_out[threadIdx.x] += s_out[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(&acc[0], s_in[0]);
        atomicAdd(&acc[1], s_out[0]);
    }
}

} // namespace

extern "C" int ssmd_centreline(const ssmd_params *p, const LBMFields *fields, double *uz_out, double *phi_out,
                               ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (!fields || !fields->uz || !fields->phi || !uz_out || !phi_out)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    const Geometry G = make_geometry(*p);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    centreline_kernel<<<(G.nz + 127) / 128, 128, 0, st>>>(G, make_fields(*fields), p->oil_cx, p->oil_cy, uz_out,
                                                         phi_out);
    return cuda_check(cudaGetLastError(), "centreline launch");
}

extern "C" size_t ssmd_droplets_scratch_bytes(const ssmd_params *p, int32_t max_droplets) {
    if (!p || max_droplets < 0) return 0;
    const size_t n = (size_t)p->nx * p->ny * p->nz;
    return round256(n * 4) * 3 + round256(n * 8) + 256 + round256((size_t)max_droplets * sizeof(ssmd_droplet));
}

extern "C" int ssmd_droplets(const ssmd_params *p, const LBMFields *fields, float threshold, void *scratch,
                             size_t scratch_bytes, ssmd_droplet *out, int32_t max_droplets, int32_t *n_out,
                             ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (!fields || !fields->phi || !scratch || !out || !n_out || max_droplets <= 0)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    if (scratch_bytes < ssmd_droplets_scratch_bytes(p, max_droplets))
        return fail(SSMD_ERR_INVALID_ARGUMENT, "scratch_bytes %zu < required %zu", scratch_bytes,
                    ssmd_droplets_scratch_bytes(p, max_droplets));
    const Geometry G = make_geometry(*p);
    const size_t n = G.cells;
    char *s = static_cast<char *>(scratch);
    DropScratch S{};
    S.label = reinterpret_cast<uint32_t *>(s);
    s += round256(n * 4);
    S.count = reinterpret_cast<uint32_t *>(s);
    s += round256(n * 4);
    S.touch = reinterpret_cast<uint32_t *>(s);
    s += round256(n * 4);
    S.volume = reinterpret_cast<double *>(s);
    s += round256(n * 8);
    S.n_out = reinterpret_cast<uint32_t *>(s);
    s += 256;
    S.list = reinterpret_cast<ssmd_droplet *>(s);
    S.max_list = max_droplets;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (int e = cuda_check(cudaMemsetAsync(S.n_out, 0, sizeof(uint32_t), st), "droplet counter")) return e;
    ccl_init<<<nb, 256, 0, st>>>(G, fields->phi, threshold, S);
    ccl_union<<<nb, 256, 0, st>>>(G, S);
    ccl_compress_accumulate<<<nb, 256, 0, st>>>(G, fields->phi, S);
    ccl_collect<<<nb, 256, 0, st>>>(G, S);
    if (int e = cuda_check(cudaGetLastError(), "droplet kernels")) return e;
    uint32_t found = 0;
    if (int e = cuda_check(cudaMemcpyAsync(&found, S.n_out, sizeof found, cudaMemcpyDeviceToHost, st), "count"))
        return e;
    if (int e = cuda_check(cudaStreamSynchronize(st), "droplet sync")) return e;
    const int32_t k = (int32_t)(found < (uint32_t)max_droplets ? found : (uint32_t)max_droplets);
    if (k > 0) {
        if (int e = cuda_check(cudaMemcpyAsync(out, S.list, sizeof(ssmd_droplet) * k, cudaMemcpyDeviceToHost, st),
                               "droplet list"))
            return e;
        if (int e = cuda_check(cudaStreamSynchronize(st), "droplet sync")) return e;
    }
    *n_out = (int32_t)found;
    return found > (uint32_t)max_droplets
               ? fail(SSMD_ERR_INVALID_ARGUMENT, "%u droplets found, only %d returned", found, max_droplets)
               : SSMD_OK;
}

extern "C" int ssmd_phase_flux(const ssmd_params *p, const LBMFields *fields, uint64_t steps_done, double *inflow,
                               double *outflow, ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (int e = check_fields(*p, fields)) return e;
    if (!inflow || !outflow) return fail(SSMD_ERR_INVALID_ARGUMENT, "null output");
    const Geometry G = make_geometry(*p);
    const void *g = (steps_done & 1ull) == 0ull ? fields->g : p->g_alt;
    double *acc = reinterpret_cast<double *>(static_cast<char *>(p->workspace) + kPartialOff);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int e = cuda_check(cudaMemsetAsync(acc, 0, 2 * sizeof(double), st), "flux clear")) return e;
    uint64_t nb64 = (G.cells + 255) / 256;
    const unsigned nb = (unsigned)(nb64 < 4096 ? nb64 : 4096);
    switch (p->storage) {
    case SSMD_STORAGE_F32: phase_flux_kernel<float><<<nb, 256, 0, st>>>(G, static_cast<const float *>(g), acc); break;
    case SSMD_STORAGE_F16: phase_flux_kernel<__half><<<nb, 256, 0, st>>>(G, static_cast<const __half *>(g), acc); break;
    case SSMD_STORAGE_F16_G32: // g as float
        phase_flux_kernel<float><<<nb, 256, 0, st>>>(G, static_cast<const float *>(g), acc);
        break;
    default: { // BF16 runs keep g in half
        using TG = phase_t<__nv_bfloat16>;
        phase_flux_kernel<TG><<<nb, 256, 0, st>>>(G, static_cast<const TG *>(g), acc);
        break;
    }
    }
    if (int e = cuda_check(cudaGetLastError(), "flux launch")) return e;
    double h[2] = {0.0, 0.0};
    if (int e = cuda_check(cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, st), "flux copy")) return e;
    if (int e = cuda_check(cudaStreamSynchronize(st), "flux sync")) return e;
    *inflow = h[0];
    *outflow = h[1];
    return SSMD_OK;
}
