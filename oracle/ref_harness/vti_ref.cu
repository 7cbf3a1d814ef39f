// vti_ref.cu — the reference's own .vti writer, host only.  TEST INFRASTRUCTURE.
//
// Built by oracle/build.py against the reference's sources (with a case's
// constants.cuh first on the include path, which fixes nx, ny, nz).  Usage:
//   vti_ref DIR STEP
// reads DIR/phi<STEP>.bin and DIR/rho<STEP>.bin and writes DIR/step_<STEP>.vti
// through host::PostProcess::vti (src/postProcess/PostProcess.cuh:100-262)
// with the field list of src/main.cu:126-129.  No device code runs.
#include "functions/deviceFunctions.cuh"
#include "fileIO/fields.cuh"
#include "postProcess/PostProcess.cuh"

int main(int argc, char **argv)
{
    if (argc < 3)
    {
        std::fprintf(stderr, "usage: %s DIR STEP\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const label_t step = static_cast<label_t>(std::stoul(argv[2]));
    static constexpr auto fieldsCfg = std::to_array<host::FieldConfig>({
        {host::FieldID::Phi, "phi", host::FieldDumpShape::Grid3D, true},
        {host::FieldID::Rho, "rho", host::FieldDumpShape::Grid3D, true},
    });
    host::PostProcess write;
    return write.vti(fieldsCfg, dir, step) ? 0 : 1;
}
