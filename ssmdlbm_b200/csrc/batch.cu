// batch.cu — C ABI of the batched sweep (many lattices, one persistent launch).
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "batch.cuh"
#include "host.cuh"

using namespace ssmd;
using namespace ssmd::host;

namespace {

constexpr int kMaxBatch = 4096;

// Resident blocks of the batched bulk kernel per SM, and the SM count.
template <int Q, class T>
void batch_slots(int &per_sm, int &sms) {
    static thread_local int dev_cached = -1, n_cached = 1, m_cached = 148;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != dev_cached) {
        int n = 0, m = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bulk_batch_kernel<Q, T>, kThreads, 0) != cudaSuccess) n = 1;
        if (cudaDeviceGetAttribute(&m, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) m = 148;
        dev_cached = dev;
        n_cached = n > 0 ? n : 1;
        m_cached = m > 0 ? m : 1;
    }
    per_sm = n_cached;
    sms = m_cached;
}

template <class T>
size_t table_bytes(int32_t count) {
    return sizeof(BatchHeader) + (size_t)count * sizeof(BatchInst<T>);
}

size_t table_bytes_for(int storage, int32_t count) {
    return storage == SSMD_STORAGE_F32 ? table_bytes<float>(count) : table_bytes<__half>(count);
}

int check_batch(const ssmd_params *params, const LBMFields *fields, int32_t count) {
    if (!params || !fields || count <= 0 || count > kMaxBatch)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "batch of %d lattices (1..%d)", count, kMaxBatch);
    for (int32_t i = 0; i < count; ++i) {
        if (int e = ssmd_validate(&params[i])) return e;
        if (int e = check_fields(params[i], &fields[i])) return e;
        if (params[i].velocity_set != params[0].velocity_set || params[i].storage != params[0].storage)
            return fail(SSMD_ERR_INVALID_ARGUMENT, "all lattices of a batch share velocity set and storage");
    }
    return SSMD_OK;
}

template <int Q, class T>
int prepare(const ssmd_params *params, const LBMFields *fields, int32_t count, void *table, cudaStream_t st) {
    std::vector<char> host(table_bytes<T>(count), 0);
    auto *hdr = reinterpret_cast<BatchHeader *>(host.data());
    auto *inst = reinterpret_cast<BatchInst<T> *>(host.data() + sizeof(BatchHeader));
    int per_sm = 1, sms = 1;
    batch_slots<Q, T>(per_sm, sms);
    uint32_t begin = 0;
    for (int32_t i = 0; i < count; ++i) {
        const ssmd_params &p = params[i];
        const LBMFields &fl = fields[i];
        for (int par = 0; par < 2; ++par) {
            StepArgs<T, phase_t<T>> &a = inst[i].args[par];
            a.geo = make_geometry(p);
            a.phys = make_physics(p);
            a.fld = make_fields(fl);
            const bool even = par == 0;
            a.f_src = static_cast<const T *>(even ? fl.f : p.f_alt);
            a.f_dst = static_cast<T *>(even ? p.f_alt : fl.f);
            a.g_src = static_cast<const phase_t<T> *>(even ? fl.g : p.g_alt);
            a.g_dst = static_cast<phase_t<T> *>(even ? p.g_alt : fl.g);
            set_bases(a, Q);
            a.status = status_of(p);
            set_closure(a, p);
            a.flags = 0;
            // batch items: a fixed z chunk (tile_z, default 16) keeps items of
            // different lattices comparable in work
            ssmd_params q = p;
            if (q.tile_z == 0) q.tile_z = 16;
            tiling(q, a.geo, per_sm * sms, a.tiles_x, a.tiles_y, a.zchunk, a.nzchunks);
            a.halo_mod = (a.geo.bcx == BC_PERIODIC && a.geo.nx < (uint32_t)(kTX + 4)) ||
                         (a.geo.bcy == BC_PERIODIC && a.geo.ny < (uint32_t)(kTY + 4)) ||
                         (a.geo.bcz == BC_PERIODIC && a.geo.nz < 6u);
        }
        inst[i].item_begin = begin;
        inst[i].items = (uint32_t)(inst[i].args[0].tiles_x * inst[i].args[0].tiles_y * inst[i].args[0].nzchunks);
        begin += inst[i].items;
    }
    hdr->count = (uint32_t)count;
    hdr->total_items = begin;
    if (int e = cuda_check(cudaMemcpyAsync(table, host.data(), host.size(), cudaMemcpyHostToDevice, st),
                           "batch table upload"))
        return e;
    return cuda_check(cudaStreamSynchronize(st), "batch table sync");
}

template <int Q, class T>
int step(const ssmd_params *params, int32_t count, uint64_t step_index, uint32_t flags, void *table,
         cudaStream_t st) {
    auto *hdr = static_cast<BatchHeader *>(table);
    auto *inst = reinterpret_cast<BatchInst<T> *>(static_cast<char *>(table) + sizeof(BatchHeader));
    const int parity = (int)(step_index & 1ull);
    int per_sm = 1, sms = 1;
    batch_slots<Q, T>(per_sm, sms);
    uint32_t max_n[3] = {0, 0, 0};
    bool jet_y = false, jet_z = false, copy_x = false, copy_y = false;
    for (int32_t i = 0; i < count; ++i) {
        const ssmd_params &p = params[i];
        max_n[0] = p.nx > max_n[0] ? p.nx : max_n[0];
        max_n[1] = p.ny > max_n[1] ? p.ny : max_n[1];
        max_n[2] = p.nz > max_n[2] ? p.nz : max_n[2];
        jet_y |= p.bc_y == SSMD_BC_JET;
        jet_z |= p.bc_z == SSMD_BC_JET;
        copy_x |= p.bc_x == SSMD_BC_PERIODIC_COPY;
        copy_y |= p.bc_y == SSMD_BC_PERIODIC_COPY;
    }
    bulk_batch_kernel<Q, T><<<(unsigned)(per_sm * sms), dim3(kTX, kTY), 0, st>>>(hdr, inst, parity, flags);
    if (int e = cuda_check(cudaGetLastError(), "batched bulk launch")) return e;
    // one launch per boundary kind that some lattice uses, in the single-lattice order
    const dim3 b2(32, 4);
    auto grid = [&](uint32_t n0, uint32_t n1) {
        return dim3((n0 + 31) / 32, (n1 + 3) / 4, (unsigned)count);
    };
    if (jet_y) bc_batch_kernel<Q, T, BK_WATER_IN><<<grid(max_n[0], max_n[2]), b2, 0, st>>>(inst, parity);
    if (jet_z) bc_batch_kernel<Q, T, BK_OIL_IN><<<grid(max_n[0], max_n[1]), b2, 0, st>>>(inst, parity);
    if (jet_y) bc_batch_kernel<Q, T, BK_OUT_Y><<<grid(max_n[0], max_n[2]), b2, 0, st>>>(inst, parity);
    if (jet_z) bc_batch_kernel<Q, T, BK_OUT_Z><<<grid(max_n[0], max_n[1]), b2, 0, st>>>(inst, parity);
    if (copy_x) bc_batch_kernel<Q, T, BK_COPY_X><<<grid(max_n[1], max_n[2]), b2, 0, st>>>(inst, parity);
    if (copy_y) bc_batch_kernel<Q, T, BK_COPY_Y><<<grid(max_n[0], max_n[2]), b2, 0, st>>>(inst, parity);
    return cuda_check(cudaGetLastError(), "batched boundary launch");
}

template <class F>
int dispatch(int q, int storage, F &&f) {
    switch (q * 4 + storage) {
    case 19 * 4 + SSMD_STORAGE_F32: return f(std::integral_constant<int, 19>{}, float{});
    case 19 * 4 + SSMD_STORAGE_F16: return f(std::integral_constant<int, 19>{}, __half{});
    case 19 * 4 + SSMD_STORAGE_BF16: return f(std::integral_constant<int, 19>{}, __nv_bfloat16{});
    case 27 * 4 + SSMD_STORAGE_F32: return f(std::integral_constant<int, 27>{}, float{});
    case 27 * 4 + SSMD_STORAGE_F16: return f(std::integral_constant<int, 27>{}, __half{});
    case 27 * 4 + SSMD_STORAGE_BF16: return f(std::integral_constant<int, 27>{}, __nv_bfloat16{});
    default: return fail(SSMD_ERR_UNSUPPORTED, "unsupported velocity set / storage (batches: F32, F16, BF16)");
    }
}

} // namespace

extern "C" size_t ssmd_batch_table_bytes(const ssmd_params *params, int32_t count) {
    if (!params || count <= 0) return 0;
    return table_bytes_for(params[0].storage, count);
}

extern "C" int ssmd_batch_prepare(const ssmd_params *params, const LBMFields *fields, int32_t count, void *table,
                                  size_t table_bytes_given, ssmd_stream_t stream) {
    if (int e = check_batch(params, fields, count)) return e;
    if (!table || table_bytes_given < table_bytes_for(params[0].storage, count))
        return fail(SSMD_ERR_INVALID_ARGUMENT, "batch table too small (%zu < %zu)", table_bytes_given,
                    table_bytes_for(params[0].storage, count));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    return dispatch(params[0].velocity_set, params[0].storage, [&](auto q, auto t) {
        return prepare<decltype(q)::value, decltype(t)>(params, fields, count, table, st);
    });
}

extern "C" int ssmd_batch_step(const ssmd_params *params, int32_t count, uint64_t step_index, uint32_t flags,
                               void *table, ssmd_stream_t stream) {
    if (!params || count <= 0 || count > kMaxBatch || !table)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument or bad batch size");
    if (flags & ~SSMD_STEP_STORE_MACROS)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "batched steps take SSMD_STEP_STORE_MACROS only (0x%x)", flags);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    return dispatch(params[0].velocity_set, params[0].storage, [&](auto q, auto t) {
        return step<decltype(q)::value, decltype(t)>(params, count, step_index, flags, table, st);
    });
}

extern "C" int ssmd_batch_capture_graph(const ssmd_params *params, int32_t count, uint64_t first_step,
                                        int32_t steps, uint32_t flags, void *table, ssmd_stream_t stream,
                                        ssmd_graph_exec_t *out) {
    if (!out || steps <= 0 || (steps & 1))
        return fail(SSMD_ERR_INVALID_ARGUMENT, "steps must be a positive even number and out non-null");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int e = cuda_check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture")) return e;
    int err = SSMD_OK;
    for (int32_t i = 0; i < steps && !err; ++i) err = ssmd_batch_step(params, count, first_step + i, flags, table, stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (err) {
        if (graph) cudaGraphDestroy(graph);
        return err;
    }
    if (int e = cuda_check(ce, "end capture")) return e;
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (int e = cuda_check(ie, "graph instantiate")) return e;
    *out = reinterpret_cast<ssmd_graph_exec_t>(exec);
    return SSMD_OK;
}
