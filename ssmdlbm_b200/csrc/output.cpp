// output.cpp — the reference's output files, written from host buffers.
//
// Formats kept byte for byte so post-processing (ParaView, scripts) is
// unchanged:
//   <dir>/<name><step:06>.bin  raw FP32, nx*ny*nz values, x fastest
//                              (src/postProcess/PostProcess.cuh:44-98)
//   <dir>/step_<step:06>.vti   VTK ImageData, appended raw arrays, each with a
//                              4-byte length header (PostProcess.cuh:100-262)
//   <dir>/<id>_info.txt        run metadata (src/functions/hostFunctions.cuh:47-87)
// Host code only: usable without a GPU.
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ssmd.h"

namespace {

std::string step6(uint64_t step) {
    std::ostringstream ss;
    ss << std::setw(6) << std::setfill('0') << step;
    return ss.str();
}

} // namespace

namespace ssmd {
namespace host {
int fail(int code, const char *fmt, ...);
}
} // namespace ssmd

using ssmd::host::fail;

extern "C" int ssmd_output_bin(const char *dir, const char *name, uint64_t step, const float *values,
                               uint64_t count) {
    if (!dir || !name || (!values && count)) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    const std::filesystem::path path = std::filesystem::path(dir) / (std::string(name) + step6(step) + ".bin");
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    if (!out) return fail(SSMD_ERR_INVALID_ARGUMENT, "cannot open %s", path.string().c_str());
    out.write(reinterpret_cast<const char *>(values), static_cast<std::streamsize>(count * sizeof(float)));
    return out ? SSMD_OK : fail(SSMD_ERR_INVALID_ARGUMENT, "write failed: %s", path.string().c_str());
}

extern "C" int ssmd_output_vti(const char *dir, uint64_t step, uint32_t nx, uint32_t ny, uint32_t nz,
                               const char *const *names, int32_t count) {
    if (!dir || !names || count <= 0) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    struct Array {
        std::string name;
        std::filesystem::path path;
        uint64_t nbytes, offset;
    };
    const uint64_t node_bytes = (uint64_t)nx * ny * nz * sizeof(float);
    const std::string suffix = step6(step);
    std::vector<Array> arrays;
    uint64_t offset = 0;
    for (int32_t i = 0; i < count; ++i) {
        const std::filesystem::path bin = std::filesystem::path(dir) / (std::string(names[i]) + suffix + ".bin");
        std::error_code ec;
        if (!std::filesystem::exists(bin, ec) || ec) continue; // as the reference: skip missing arrays
        const uint64_t fs = std::filesystem::file_size(bin, ec);
        if (ec || fs != node_bytes) continue;
        arrays.push_back({names[i], bin, fs, offset});
        offset += sizeof(uint32_t) + fs;
    }
    if (arrays.empty()) return fail(SSMD_ERR_INVALID_ARGUMENT, "no .bin arrays found for step %llu",
                                    (unsigned long long)step);
    const std::filesystem::path vti = std::filesystem::path(dir) / ("step_" + suffix + ".vti");
    std::ofstream out(vti, std::ios::binary | std::ios::trunc);
    if (!out) return fail(SSMD_ERR_INVALID_ARGUMENT, "cannot open %s", vti.string().c_str());
    const double o = 0.0, sp = 1.0;
    out << R"(<?xml version="1.0"?>)" << '\n';
    out << R"(<VTKFile type="ImageData" version="0.1" byte_order="LittleEndian">)" << '\n';
    out << "  <ImageData WholeExtent=\"0 " << (nx - 1) << " 0 " << (ny - 1) << " 0 " << (nz - 1)
        << "\" Origin=\"" << o << " " << o << " " << o << "\" Spacing=\"" << sp << " " << sp << " " << sp
        << "\">\n";
    out << "    <Piece Extent=\"0 " << (nx - 1) << " 0 " << (ny - 1) << " 0 " << (nz - 1) << "\">\n";
    out << "      <PointData Scalars=\"" << arrays.front().name << "\">\n";
    for (const Array &a : arrays)
        out << "        <DataArray type=\"Float32\" Name=\"" << a.name
            << "\" NumberOfComponents=\"1\" format=\"appended\" offset=\"" << a.offset << "\"/>\n";
    out << "      </PointData>\n";
    out << "      <CellData/>\n";
    out << "    </Piece>\n";
    out << "  </ImageData>\n";
    out << "  <AppendedData encoding=\"raw\">\n";
    out << '_';
    std::vector<char> buf(1 << 20);
    for (const Array &a : arrays) {
        const uint32_t n32 = static_cast<uint32_t>(a.nbytes);
        out.write(reinterpret_cast<const char *>(&n32), sizeof n32);
        std::ifstream in(a.path, std::ios::binary);
        while (in) {
            in.read(buf.data(), static_cast<std::streamsize>(buf.size()));
            const std::streamsize got = in.gcount();
            if (got > 0) out.write(buf.data(), got);
        }
    }
    out << "\n  </AppendedData>\n";
    out << "</VTKFile>\n";
    return out ? SSMD_OK : fail(SSMD_ERR_INVALID_ARGUMENT, "write failed: %s", vti.string().c_str());
}

extern "C" int ssmd_output_info(const char *dir, const char *id, const char *velocity_set, float u_water,
                                float u_oil, double reynolds_water, double reynolds_oil, double weber,
                                uint32_t nx, uint32_t ny, uint32_t nz, int32_t diam_water, int32_t diam_oil,
                                int64_t nsteps, int64_t macro_save) {
    if (!dir || !id || !velocity_set) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    const std::filesystem::path path = std::filesystem::path(dir) / (std::string(id) + "_info.txt");
    std::ofstream file(path, std::ios::out | std::ios::trunc);
    if (!file) return fail(SSMD_ERR_INVALID_ARGUMENT, "cannot open %s", path.string().c_str());
    file << "---------------------------- SIMULATION METADATA ----------------------------\n"
         << "ID:                 " << id << '\n'
         << "Velocity set:       " << velocity_set << '\n'
         << "Water velocity:     " << u_water << '\n'
         << "Oil velocity:       " << u_oil << '\n'
         << "Water Reynolds:     " << reynolds_water << '\n'
         << "Oil Reynolds:       " << reynolds_oil << '\n'
         << "Weber number:       " << weber << "\n\n"
         << "Domain size:        NX=" << nx << ", NY=" << ny << ", NZ=" << nz << '\n'
         << "Water diameter:     D=" << diam_water << '\n'
         << "Oil diameter:       D=" << diam_oil << '\n'
         << "Timesteps:          " << nsteps << '\n'
         << "Output interval:    " << macro_save << "\n\n"
         << "-----------------------------------------------------------------------------\n";
    return file ? SSMD_OK : fail(SSMD_ERR_INVALID_ARGUMENT, "write failed: %s", path.string().c_str());
}
