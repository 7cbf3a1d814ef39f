#!/bin/bash
# pipeline.sh — compile -> simulate -> output, with the reference's interface:
#   ./pipeline.sh <velocity_set> <id> [driver options ...]
# Cleans <root>/bin/<velocity_set>/<id>/, builds the driver (compile.sh) and
# runs it there; outputs are the reference's files (phi/rho .bin, .vti, info).
set -euo pipefail

GPU_INDEX=${GPU_INDEX:-0}
detect_sm() {
    local cc=""
    if command -v nvidia-smi >/dev/null 2>&1; then
        cc=$(nvidia-smi --query-gpu=compute_cap --format=csv,noheader -i "${GPU_INDEX}" 2>/dev/null | head -n1 | tr -d '.')
    fi
    echo "${cc}"
}
GPU_ARCH="$(detect_sm)"; GPU_ARCH="${GPU_ARCH:-100}"

VELOCITY_SET=${1:-}
ID=${2:-}
if [ -z "$VELOCITY_SET" ] || [ -z "$ID" ]; then
    echo "Usage: ./pipeline.sh <velocity_set> <id> [options]"
    echo "Example: ./pipeline.sh D3Q19 000"
    exit 1
fi
shift 2

HOST_DIR="$(cd -- "$(dirname -- "${BASH_SOURCE[0]}")" &>/dev/null && pwd)"
ROOT="$(dirname "$(dirname "${HOST_DIR}")")"
SIMULATION_DIR="${ROOT}/bin/${VELOCITY_SET}/${ID}"
mkdir -p "${SIMULATION_DIR}"
find "${SIMULATION_DIR}" -mindepth 1 ! -name ".gitkeep" -exec rm -rf {} +

GPU_INDEX="${GPU_INDEX}" GPU_ARCH="${GPU_ARCH}" bash "${HOST_DIR}/compile.sh" "${VELOCITY_SET}" "${ID}"
EXECUTABLE="${ROOT}/bin/${VELOCITY_SET}/${ID}sim_${VELOCITY_SET}_sm${GPU_ARCH}"
export GPU_INDEX
cd "${ROOT}"
"${EXECUTABLE}" "${VELOCITY_SET}" "${ID}" 1 "$@"
echo "Process completed successfully!"
