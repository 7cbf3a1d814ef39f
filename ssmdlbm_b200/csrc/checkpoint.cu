// checkpoint.cu — bit-exact save / resume of a lattice.
//
// The reference dumps phi and rho only (src/main.cu:126-129), which cannot
// restart a run.  A checkpoint here holds everything the next step reads:
// the current populations (pull layout), all eleven macroscopic arrays (the
// boundaries read rho, u, Pi and phi on faces and boundary planes) and the
// device step counter (inlet noise).  Loading writes the populations into
// both buffers: slots no kernel writes are identical in the two, every other
// slot is rewritten before it is read.
//
// File: 64-byte header {magic "SSMDCKP2", abi, sizeof(ssmd_params),
// steps_done, device step, cells, Q, storage} + ssmd_params (pointers
// cleared) + 11 FP32 arrays (rho ux uy uz pxx pyy pzz pxy pxz pyz phi) + f + g.
// Format 2 stores g of BF16-storage lattices as IEEE half (format 1 stored
// bfloat16); loading refuses format-1 files and any header whose ABI version,
// cell count, velocity set or storage differs from the caller's parameters,
// so a file is never read with the wrong element types.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "host.cuh"

using namespace ssmd;
using namespace ssmd::host;

namespace {

struct Header {
    char magic[8];
    uint32_t abi;
    uint32_t params_bytes;
    uint64_t steps_done;
    uint64_t device_step;
    uint64_t cells;
    int32_t q;
    int32_t storage;
    uint64_t reserved[2];
};
static_assert(sizeof(Header) == 64, "checkpoint header is 64 bytes");
constexpr char kMagic[9] = "SSMDCKP2";

float *const *scalar_list(const LBMFields *f, float *(&out)[11]) {
    float *v[11] = {f->rho, f->ux, f->uy, f->uz, f->pxx, f->pyy, f->pzz, f->pxy, f->pxz, f->pyz, f->phi};
    for (int i = 0; i < 11; ++i) out[i] = v[i];
    return out;
}

bool same_problem(const ssmd_params &a, const ssmd_params &b) {
    return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.velocity_set == b.velocity_set &&
           a.storage == b.storage && a.bc_x == b.bc_x && a.bc_y == b.bc_y && a.bc_z == b.bc_z;
}

} // namespace

extern "C" int ssmd_checkpoint_save(const ssmd_params *p, const LBMFields *fields, uint64_t steps_done,
                                    const char *path, ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (int e = check_fields(*p, fields)) return e;
    if (!path) return fail(SSMD_ERR_INVALID_ARGUMENT, "path is null");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int e = cuda_check(cudaStreamSynchronize(st), "checkpoint sync")) return e;
    DeviceStatus ds{};
    if (int e = cuda_check(cudaMemcpy(&ds, status_of(*p), sizeof ds, cudaMemcpyDeviceToHost), "status read")) return e;
    std::FILE *fp = std::fopen(path, "wb");
    if (!fp) return fail(SSMD_ERR_INVALID_ARGUMENT, "cannot open %s", path);
    Header h{};
    std::memcpy(h.magic, kMagic, 8);
    h.abi = SSMD_ABI_VERSION;
    h.params_bytes = sizeof(ssmd_params);
    h.steps_done = steps_done;
    h.device_step = ds.step;
    h.cells = (uint64_t)p->nx * p->ny * p->nz;
    h.q = p->velocity_set;
    h.storage = p->storage;
    ssmd_params pc = *p;
    pc.f_alt = pc.g_alt = pc.workspace = nullptr;
    bool ok = std::fwrite(&h, sizeof h, 1, fp) == 1 && std::fwrite(&pc, sizeof pc, 1, fp) == 1;
    const size_t sb = ssmd_scalar_bytes(p);
    std::vector<char> buf(sb > ssmd_f_bytes(p) ? sb : ssmd_f_bytes(p));
    float *sc[11];
    scalar_list(fields, sc);
    for (int i = 0; ok && i < 11; ++i) {
        ok = cudaMemcpy(buf.data(), sc[i], sb, cudaMemcpyDeviceToHost) == cudaSuccess &&
             std::fwrite(buf.data(), 1, sb, fp) == sb;
    }
    const bool even = (steps_done & 1ull) == 0ull;
    const void *pops[2] = {even ? fields->f : p->f_alt, even ? fields->g : p->g_alt};
    const size_t pb[2] = {ssmd_f_bytes(p), ssmd_g_bytes(p)};
    for (int i = 0; ok && i < 2; ++i) {
        ok = cudaMemcpy(buf.data(), pops[i], pb[i], cudaMemcpyDeviceToHost) == cudaSuccess &&
             std::fwrite(buf.data(), 1, pb[i], fp) == pb[i];
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? SSMD_OK : fail(SSMD_ERR_CUDA, "checkpoint write to %s failed", path);
}

extern "C" int ssmd_checkpoint_load(const ssmd_params *p, LBMFields *fields, const char *path,
                                    uint64_t *steps_done, ssmd_stream_t stream) {
    if (int e = ssmd_validate(p)) return e;
    if (int e = check_fields(*p, fields)) return e;
    if (!path || !steps_done) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    std::FILE *fp = std::fopen(path, "rb");
    if (!fp) return fail(SSMD_ERR_INVALID_ARGUMENT, "cannot open %s", path);
    Header h{};
    ssmd_params pc{};
    bool ok = std::fread(&h, sizeof h, 1, fp) == 1;
    if (ok && std::memcmp(h.magic, "SSMDCKP", 7) == 0 && std::memcmp(h.magic, kMagic, 8) != 0) {
        std::fclose(fp);
        return fail(SSMD_ERR_INVALID_ARGUMENT, "%s is a checkpoint of an older format (%.8s, this library reads %.8s)",
                    path, h.magic, kMagic);
    }
    ok = ok && std::memcmp(h.magic, kMagic, 8) == 0 && h.abi == SSMD_ABI_VERSION &&
         h.params_bytes == sizeof(ssmd_params) && h.cells == (uint64_t)p->nx * p->ny * p->nz &&
         h.q == p->velocity_set && h.storage == p->storage && std::fread(&pc, sizeof pc, 1, fp) == 1;
    if (!ok || !same_problem(pc, *p)) {
        std::fclose(fp);
        return fail(SSMD_ERR_INVALID_ARGUMENT, "%s is not a checkpoint of this lattice / storage / ABI", path);
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int e = cuda_check(cudaStreamSynchronize(st), "checkpoint sync")) {
        std::fclose(fp);
        return e;
    }
    const size_t sb = ssmd_scalar_bytes(p);
    std::vector<char> buf(sb > ssmd_f_bytes(p) ? sb : ssmd_f_bytes(p));
    float *sc[11];
    scalar_list(fields, sc);
    for (int i = 0; ok && i < 11; ++i)
        ok = std::fread(buf.data(), 1, sb, fp) == sb &&
             cudaMemcpy(sc[i], buf.data(), sb, cudaMemcpyHostToDevice) == cudaSuccess;
    void *dst[2][2] = {{fields->f, p->f_alt}, {fields->g, p->g_alt}};
    const size_t pb[2] = {ssmd_f_bytes(p), ssmd_g_bytes(p)};
    for (int i = 0; ok && i < 2; ++i) {
        ok = std::fread(buf.data(), 1, pb[i], fp) == pb[i];
        for (int k = 0; ok && k < 2; ++k)
            ok = cudaMemcpy(dst[i][k], buf.data(), pb[i], cudaMemcpyHostToDevice) == cudaSuccess;
    }
    std::fclose(fp);
    if (!ok) return fail(SSMD_ERR_INVALID_ARGUMENT, "checkpoint %s is truncated or unreadable", path);
    DeviceStatus ds{};
    ds.step = h.device_step;
    if (int e = cuda_check(cudaMemcpy(status_of(*p), &ds, sizeof ds, cudaMemcpyHostToDevice), "status write"))
        return e;
    // the file's populations are those of step steps_done; keep the parity by
    // placing them in the buffer that step reads
    *steps_done = h.steps_done;
    return SSMD_OK;
}
