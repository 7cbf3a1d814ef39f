// main.cpp — the simulation driver of the reference (src/main.cu:35-213) on the
// ssmd C ABI: same command line, same directory layout and output files.
//
//   <exe> <VELOCITY_SET> <ID> <any> [--key value ...]
//
// Writes ./bin/<VELOCITY_SET>/<ID>/<ID>_info.txt, phi<step:06>.bin,
// rho<step:06>.bin and step_<step:06>.vti every `save` steps and at the last
// step, and prints the MLUPS of the run (all nx*ny*nz cells per step, as the
// reference counts, main.cu:199-208).  Defaults are the reference's
// constants (constants.cuh:53-101): 128 x 256 x 256 cells, two jets of
// diameter 13, u = 0.05, Re 1400 / 450, We 500, W = 4, 100000 steps, output
// every 1000.  Options override them (see usage()).
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "../../include/ssmd.h"

namespace {

struct Options {
    uint32_t nx = 128, ny = 256, nz = 256;
    int diam_water = 13, diam_oil = 13, radius_water = -1, radius_oil = -1;
    float u_water = 0.05f, u_oil = 0.05f;
    double re_water = 1400, re_oil = 450, weber = 500;
    float width = 4.0f;
    long nsteps = 100000, save = 1000;
    int storage = SSMD_STORAGE_F32;
    int bc_y = SSMD_BC_JET;
    bool benchmark = false;
};

void usage(const char *exe) {
    std::fprintf(stderr,
                 "Usage: %s <velocity set D3Q19|D3Q27> <ID> <any>\n"
                 "  [--nx N --ny N --nz N] [--steps N] [--save N] [--benchmark]\n"
                 "  [--diam-water D --diam-oil D --radius-water R --radius-oil R]\n"
                 "  [--u-water U --u-oil U --re-water R --re-oil R --weber W --width W]\n"
                 "  [--storage f32|f16|bf16] [--periodic-y]\n",
                 exe);
}

bool parse(int argc, char **argv, Options &o) {
    for (int i = 4; i < argc; ++i) {
        const std::string k = argv[i];
        auto val = [&]() -> const char * {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", k.c_str());
                std::exit(1);
            }
            return argv[++i];
        };
        if (k == "--nx") o.nx = std::strtoul(val(), nullptr, 10);
        else if (k == "--ny") o.ny = std::strtoul(val(), nullptr, 10);
        else if (k == "--nz") o.nz = std::strtoul(val(), nullptr, 10);
        else if (k == "--steps") o.nsteps = std::strtol(val(), nullptr, 10);
        else if (k == "--save") o.save = std::strtol(val(), nullptr, 10);
        else if (k == "--benchmark") o.benchmark = true;
        else if (k == "--diam-water") o.diam_water = std::atoi(val());
        else if (k == "--diam-oil") o.diam_oil = std::atoi(val());
        else if (k == "--radius-water") o.radius_water = std::atoi(val());
        else if (k == "--radius-oil") o.radius_oil = std::atoi(val());
        else if (k == "--u-water") o.u_water = std::strtof(val(), nullptr);
        else if (k == "--u-oil") o.u_oil = std::strtof(val(), nullptr);
        else if (k == "--re-water") o.re_water = std::strtod(val(), nullptr);
        else if (k == "--re-oil") o.re_oil = std::strtod(val(), nullptr);
        else if (k == "--weber") o.weber = std::strtod(val(), nullptr);
        else if (k == "--width") o.width = std::strtof(val(), nullptr);
        else if (k == "--periodic-y") o.bc_y = SSMD_BC_PERIODIC_COPY;
        else if (k == "--storage") {
            const std::string s = val();
            o.storage = s == "f16" ? SSMD_STORAGE_F16 : (s == "bf16" ? SSMD_STORAGE_BF16 : SSMD_STORAGE_F32);
        } else {
            std::fprintf(stderr, "unknown option %s\n", k.c_str());
            return false;
        }
    }
    return o.save > 0 && o.nsteps >= 0;
}

// GPU_INDEX environment variable, as the reference (hostFunctions.cuh:139-172).
int device_from_env() {
    int dev = 0;
    if (const char *env = std::getenv("GPU_INDEX")) {
        char *end = nullptr;
        const long v = std::strtol(env, &end, 10);
        if (end != env && v >= 0) dev = static_cast<int>(v);
    }
    if (cudaSetDevice(dev) != cudaSuccess) {
        std::fprintf(stderr, "cudaSetDevice(%d) failed\n", dev);
        return -1;
    }
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
        std::printf("Using GPU %d: %s (SM %d.%d)\n", dev, prop.name, prop.major, prop.minor);
    return dev;
}

// Device buffers of one lattice, zero-initialised, freed on destruction
// (the role of host::FieldAllocate, src/fieldAllocate/FieldAllocate.cuh:42-162).
class Fields {
  public:
    Fields(ssmd_params &p) : p_(p) {
        const size_t sb = ssmd_scalar_bytes(&p);
        float **scalars[] = {&f_.rho, &f_.ux, &f_.uy, &f_.uz, &f_.pxx, &f_.pyy, &f_.pzz, &f_.pxy,
                             &f_.pxz, &f_.pyz, &f_.phi, &f_.fsx, &f_.fsy, &f_.fsz};
        for (float **s : scalars) ok_ &= alloc(reinterpret_cast<void **>(s), sb);
        ok_ &= alloc(&f_.f, ssmd_f_bytes(&p));
        ok_ &= alloc(&f_.g, ssmd_g_bytes(&p));
        ok_ &= alloc(&p.f_alt, ssmd_f_bytes(&p));
        ok_ &= alloc(&p.g_alt, ssmd_g_bytes(&p));
        p.workspace_bytes = ssmd_workspace_bytes(&p);
        ok_ &= alloc(&p.workspace, p.workspace_bytes);
    }
    ~Fields() {
        for (void *q : owned_) cudaFree(q);
    }
    Fields(const Fields &) = delete;
    Fields &operator=(const Fields &) = delete;
    bool ok() const { return ok_; }
    LBMFields *get() { return &f_; }

  private:
    bool alloc(void **ptr, size_t bytes) {
        if (cudaMalloc(ptr, bytes) != cudaSuccess) return false;
        owned_.push_back(*ptr);
        return cudaMemset(*ptr, 0, bytes) == cudaSuccess;
    }
    ssmd_params &p_;
    LBMFields f_{};
    std::vector<void *> owned_;
    bool ok_ = true;
};

int check(int rc, const char *what) {
    if (rc != SSMD_OK) std::fprintf(stderr, "%s failed: %s\n", what, ssmd_last_error());
    return rc;
}

} // namespace

int main(int argc, char **argv) {
    if (argc < 4) {
        usage(argv[0]);
        return 1;
    }
    const std::string vs = argv[1], id = argv[2];
    Options o;
    if ((vs != "D3Q19" && vs != "D3Q27") || !parse(argc, argv, o)) {
        usage(argv[0]);
        return 1;
    }
    const std::filesystem::path dir = std::filesystem::current_path() / "bin" / vs / id;
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (device_from_env() < 0) return 1;

    ssmd_params p{};
    if (check(ssmd_params_reference(&p, o.nx, o.ny, o.nz, vs == "D3Q19" ? 19 : 27, o.u_water, o.u_oil,
                                    o.diam_water, o.diam_oil, o.radius_water, o.radius_oil, o.re_water,
                                    o.re_oil, o.weber, o.width),
              "ssmd_params_reference"))
        return 1;
    p.storage = o.storage;
    p.bc_y = o.bc_y;
    if (check(ssmd_validate(&p), "ssmd_validate")) return 1;
    Fields fields(p);
    if (!fields.ok()) {
        std::fprintf(stderr, "device allocation failed\n");
        return 1;
    }
    cudaStream_t queue{};
    cudaStreamCreate(&queue);
    const ssmd_stream_t st = reinterpret_cast<ssmd_stream_t>(queue);
    if (check(ssmd_init(&p, fields.get(), st), "ssmd_init")) return 1;
    cudaStreamSynchronize(queue);

    const std::string sdir = dir.string() + "/";
    check(ssmd_output_info(sdir.c_str(), id.c_str(), vs.c_str(), o.u_water, o.u_oil, o.re_water, o.re_oil,
                           o.weber, o.nx, o.ny, o.nz, o.diam_water, o.diam_oil, o.nsteps, o.save),
          "info file");
    std::printf("\nVelocity set: %s  NX=%u NY=%u NZ=%u  cells=%llu  steps=%ld  save every %ld\n\n", vs.c_str(),
                o.nx, o.ny, o.nz, (unsigned long long)o.nx * o.ny * o.nz, o.nsteps, o.save);

    const size_t n = (size_t)o.nx * o.ny * o.nz;
    std::vector<float> host(n);
    const char *names[] = {"phi", "rho"};
    float *dev_fields[] = {fields.get()->phi, fields.get()->rho};

    const auto t0 = std::chrono::high_resolution_clock::now();
    for (long step = 0; step <= o.nsteps; ++step) { // main.cu:159
        const bool save = !o.benchmark && (step % o.save == 0 || step == o.nsteps);
        if (check(ssmd_step(fields.get(), &p, (uint64_t)step, save ? SSMD_STEP_STORE_MACROS : 0u, st), "ssmd_step"))
            return 1;
        if (save) {
            cudaStreamSynchronize(queue);
            std::printf("Step %ld: bins in %s\n", step, sdir.c_str());
            for (int k = 0; k < 2; ++k) {
                if (cudaMemcpy(host.data(), dev_fields[k], n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
                    return 1;
                check(ssmd_output_bin(sdir.c_str(), names[k], (uint64_t)step, host.data(), n), "bin");
            }
            check(ssmd_output_vti(sdir.c_str(), (uint64_t)step, o.nx, o.ny, o.nz, names, 2), "vti");
        }
    }
    cudaStreamSynchronize(queue);
    const auto t1 = std::chrono::high_resolution_clock::now();
    uint32_t status = 0;
    if (check(ssmd_check_status(&p, &status, st), "status") || status != 0) {
        std::fprintf(stderr, "device status 0x%x (non-finite density)\n", status);
        return 1;
    }
    const double secs = std::chrono::duration<double>(t1 - t0).count();
    const double mlups = (double)n * (double)(o.nsteps + 1) / (secs * 1e6);
    std::printf("\n// =============================================== //\n");
    std::printf("     Total execution time    : %g s\n", secs);
    std::printf("     Performance             : %g MLUPS\n", mlups);
    std::printf("// =============================================== //\n\n");
    cudaStreamDestroy(queue);
    return 0;
}
