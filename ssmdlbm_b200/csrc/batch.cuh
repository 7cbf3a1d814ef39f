// batch.cuh — many independent lattices in one persistent launch.
//
// A parameter sweep (many jets of different sizes and parameters) is run as
// one launch of the bulk kernel per step: a device table holds, per
// instance, its step arguments for both buffer parities and the first index
// of its work items; resident blocks pull work items (instance, 32 x 8
// column, z chunk) from an atomic counter, so uneven lattices balance across
// the SMs.  Boundaries run as one launch per boundary kind, blockIdx.z
// selecting the instance.  The last block to leave the work loop clears the
// work counter (a second counter of finished blocks tells it that it is the
// last), so every launch finds it at zero: graphs replay without memset
// nodes and batched steps mix freely with single-lattice steps.
#pragma once

#include "bulk.cuh"
#include "surface.cuh"

namespace ssmd {

struct BatchHeader {
    uint32_t count;       // instances
    uint32_t total_items; // work items per step, all instances
    uint32_t counter;     // next work item of the running launch
    uint32_t finished;    // blocks of the running launch that left the work loop
    uint32_t pad[60];
};

template <class T>
struct BatchInst {
    StepArgs<T, phase_t<T>> args[2]; // parity 0: A -> B, parity 1: B -> A
    uint32_t item_begin;
    uint32_t items;
    uint32_t pad[2];
};

template <int Q, class T>
__global__ void __launch_bounds__(kThreads, kBulkMinBlocks<Q>)
    bulk_batch_kernel(BatchHeader *hdr, const BatchInst<T> *inst, int parity, uint32_t flags) {
    using B = Bulk<Q, T, phase_t<T>>;
    __shared__ BulkSmem S;
    __shared__ StepArgs<T, phase_t<T>> sa;
    __shared__ uint32_t s_item, s_inst;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kTX * ty;
    const uint32_t count = hdr->count, total = hdr->total_items;
    if (blockIdx.x == 0) {
        for (uint32_t i = tid; i < count; i += kThreads) inst[i].args[parity].status->step += 1ull;
    }
    while (true) {
        if (tid == 0) {
            const uint32_t item = atomicAdd(&hdr->counter, 1u);
            s_item = item;
            uint32_t lo = 0, hi = count; // last instance with item_begin <= item
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) / 2;
                if (inst[mid].item_begin <= item) lo = mid;
                else hi = mid;
            }
            s_inst = lo;
        }
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= total) {
            // this block takes no further item; the last block out resets both counters
            if (tid == 0) {
                __threadfence();
                if (atomicAdd(&hdr->finished, 1u) == gridDim.x - 1) {
                    atomicExch(&hdr->counter, 0u);
                    atomicExch(&hdr->finished, 0u);
                }
            }
            break;
        }
        {   // this instance's arguments into shared memory
            const uint32_t *src = reinterpret_cast<const uint32_t *>(&inst[s_inst].args[parity]);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&sa);
            for (int k = tid; k < (int)(sizeof(StepArgs<T, phase_t<T>>) / 4); k += kThreads) dst[k] = src[k];
        }
        __syncthreads();
        if (tid == 0) sa.flags = flags;
        const uint32_t local = item - inst[s_inst].item_begin;
        __syncthreads();
        int w = (int)local;
        const int bx = w % sa.tiles_x;
        w /= sa.tiles_x;
        const int by = w % sa.tiles_y;
        const int bz = w / sa.tiles_y;
        const int zs = sa.geo.z_lo + bz * sa.zchunk;
        const int ze = min(zs + sa.zchunk, sa.geo.z_hi + 1);
        B::template run_gather<false>(sa, S, bx * kTX, by * kTY, zs, ze, tx, ty, tid);
    }
}

// Boundary kind K of every instance: thread (i0, i1) of face plane, blockIdx.z = instance.
enum : int { BK_WATER_IN = 0, BK_OIL_IN, BK_OUT_Y, BK_OUT_Z, BK_COPY_X, BK_COPY_Y };

template <int Q, class T, int K>
__global__ void bc_batch_kernel(const BatchInst<T> *inst, int parity) {
    const StepArgs<T, phase_t<T>> &a = inst[blockIdx.z].args[parity];
    const int i0 = threadIdx.x + blockIdx.x * blockDim.x, i1 = threadIdx.y + blockIdx.y * blockDim.y;
    const Geometry &G = a.geo;
    if constexpr (K == BK_WATER_IN) { if (G.bcy == BC_JET) bc_water_inflow_at<Q>(a, i0, i1); }
    if constexpr (K == BK_OIL_IN) { if (G.bcz == BC_JET) bc_oil_inflow_at<Q>(a, i0, i1); }
    if constexpr (K == BK_OUT_Y) { if (G.bcy == BC_JET) bc_outflow_y_at<Q>(a, i0, i1); }
    if constexpr (K == BK_OUT_Z) { if (G.bcz == BC_JET) bc_outflow_z_at<Q>(a, i0, i1); }
    if constexpr (K == BK_COPY_X) { if (G.bcx == BC_COPY) bc_copy_x_at<Q>(a, i0, i1); }
    if constexpr (K == BK_COPY_Y) { if (G.bcy == BC_COPY) bc_copy_y_at<Q>(a, i0, i1); }
}

} // namespace ssmd
