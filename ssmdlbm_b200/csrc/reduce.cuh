// reduce.cuh — FP64 global reductions over the fluid cells.
//
// Deterministic two-pass sum: pass 1 leaves one partial per block in a
// scratch array, pass 2 folds the partials in a fixed order, so the result
// does not depend on block scheduling.
#pragma once

#include "common.cuh"

namespace ssmd {

constexpr int kRedThreads = 256;
constexpr int kRedVals = 10; // phi, phi_next, mass, mx, my, mz, kinetic, umax, nonfinite, cells

__device__ __forceinline__ void block_reduce(double (&v)[kRedVals], double *sm) {
    // sm: kRedVals * kRedThreads doubles; entry 7 is a max, the rest sums
    const int t = threadIdx.x;
#pragma unroll
    for (int k = 0; k < kRedVals; ++k) sm[k * kRedThreads + t] = v[k];
    __syncthreads();
    for (int s = kRedThreads / 2; s > 0; s >>= 1) {
        if (t < s) {
#pragma unroll
            for (int k = 0; k < kRedVals; ++k) {
                const double o = sm[k * kRedThreads + t + s];
                double &d = sm[k * kRedThreads + t];
                d = (k == 7) ? fmax(d, o) : d + o;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < kRedVals; ++k) v[k] = sm[k * kRedThreads];
}

template <class TG>
__global__ void __launch_bounds__(kRedThreads) reduce_pass1(Geometry G, Fields F, const TG *g,
                                                            double *partials) {
    __shared__ double sm[kRedVals * kRedThreads];
    double v[kRedVals] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const bool px = G.bcx == BC_PERIODIC, py = G.bcy == BC_PERIODIC, pz = G.bcz == BC_PERIODIC;
    for (uint64_t i = blockIdx.x * (uint64_t)kRedThreads + threadIdx.x; i < G.cells;
         i += (uint64_t)gridDim.x * kRedThreads) {
        const uint32_t c = (uint32_t)i;
        const int x = c % G.nx, y = (c / G.nx) % G.ny, z = c / G.nxy;
        if (x < G.x_lo || x > G.x_hi || y < G.y_lo || y > G.y_hi || z < G.z_lo || z > G.z_hi)
            continue;
        const double rho = F.rho[c], ux = F.ux[c], uy = F.uy[c], uz = F.uz[c], phi = F.phi[c];
        double pn = Store<TG>::ld(g + slot(G, 0, c));
        pn += Store<TG>::ld(g + slot(G, 1, cell_index(G, axis_nb(x - 1, G.nx, px), y, z)));
        pn += Store<TG>::ld(g + slot(G, 2, cell_index(G, axis_nb(x + 1, G.nx, px), y, z)));
        pn += Store<TG>::ld(g + slot(G, 3, cell_index(G, x, axis_nb(y - 1, G.ny, py), z)));
        pn += Store<TG>::ld(g + slot(G, 4, cell_index(G, x, axis_nb(y + 1, G.ny, py), z)));
        pn += Store<TG>::ld(g + slot(G, 5, cell_index(G, x, y, axis_nb(z - 1, G.nz, pz))));
        pn += Store<TG>::ld(g + slot(G, 6, cell_index(G, x, y, axis_nb(z + 1, G.nz, pz))));
        const double u2 = ux * ux + uy * uy + uz * uz;
        const bool bad = !(isfinite(rho) && isfinite(u2) && isfinite(phi) && isfinite(pn));
        v[0] += phi;
        v[1] += pn;
        v[2] += rho;
        v[3] += rho * ux;
        v[4] += rho * uy;
        v[5] += rho * uz;
        v[6] += 0.5 * rho * u2;
        v[7] = fmax(v[7], bad ? 0.0 : sqrt(u2));
        v[8] += bad ? 1.0 : 0.0;
        v[9] += 1.0;
    }
    block_reduce(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < kRedVals; ++k) partials[(uint64_t)k * gridDim.x + blockIdx.x] = v[k];
    }
}

static __global__ void __launch_bounds__(kRedThreads) reduce_pass2(const double *partials, int nparts,
                                                            double *out) {
    __shared__ double sm[kRedVals * kRedThreads];
    double v[kRedVals] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < nparts; i += kRedThreads) {
#pragma unroll
        for (int k = 0; k < kRedVals; ++k) {
            const double p = partials[(uint64_t)k * nparts + i];
            v[k] = (k == 7) ? fmax(v[k], p) : v[k] + p;
        }
    }
    block_reduce(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < kRedVals; ++k) out[k] = v[k];
    }
}

} // namespace ssmd
