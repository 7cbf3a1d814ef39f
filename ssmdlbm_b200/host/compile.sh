#!/bin/bash
# compile.sh — build the driver like the reference's compile.sh (same arguments,
# same executable path): ./compile.sh <VELOCITY_SET> <ID>
# -> <root>/bin/<VELOCITY_SET>/<ID>sim_<VELOCITY_SET>_sm<CC>
# The velocity set is a run-time choice here; it only names the executable.
set -euo pipefail

GPU_INDEX=${GPU_INDEX:-0}
if [ -n "${GPU_ARCH:-}" ]; then
    CC="${GPU_ARCH}"
else
    CC=""
    if command -v nvidia-smi >/dev/null 2>&1; then
        CC=$(nvidia-smi --query-gpu=compute_cap --format=csv,noheader -i "${GPU_INDEX}" 2>/dev/null | head -n1 | tr -d '.')
    fi
    CC=${CC:-100}
fi

VELOCITY_SET=${1:-}
ID=${2:-}
if [ -z "$VELOCITY_SET" ] || [ -z "$ID" ]; then
    echo "Usage: ./compile.sh <VELOCITY_SET> <ID>"
    echo "Example: ./compile.sh D3Q19 000"
    exit 1
fi
if [ "$VELOCITY_SET" != "D3Q19" ] && [ "$VELOCITY_SET" != "D3Q27" ]; then
    echo "Invalid VELOCITY_SET. Use 'D3Q19' or 'D3Q27'."
    exit 1
fi

HOST_DIR="$(cd -- "$(dirname -- "${BASH_SOURCE[0]}")" &>/dev/null && pwd)"
PKG_DIR="$(dirname "${HOST_DIR}")"
ROOT="$(dirname "${PKG_DIR}")"
OUTPUT_DIR="${ROOT}/bin/${VELOCITY_SET}"
EXECUTABLE="${OUTPUT_DIR}/${ID}sim_${VELOCITY_SET}_sm${CC}"
mkdir -p "${OUTPUT_DIR}"

PYTHON=${PYTHON:-python3}
(cd "${ROOT}" && "${PYTHON}" -m ssmdlbm_b200.build)

CUDA_HOME=${CUDA_HOME:-/usr/local/cuda}
g++ -O2 -std=c++17 "${HOST_DIR}/main.cpp" -I"${CUDA_HOME}/include" \
    -L"${PKG_DIR}" -lssmd -L"${CUDA_HOME}/lib64" -lcudart \
    -Wl,-rpath,'$ORIGIN/../../ssmdlbm_b200' -Wl,-rpath,"${CUDA_HOME}/lib64" \
    -o "${EXECUTABLE}"
echo "Compilation completed successfully: ${EXECUTABLE}"
