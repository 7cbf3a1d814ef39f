// mlp.cu — the learned closure's per-cell network on the 5th-generation tensor cores.
//
// Network: 12 features -> 64 -> 64 -> 2 outputs, GELU (erf form) after the
// two hidden layers, features standardised by stored mean / inverse std,
// outputs  p = scale * r + offset  with r the last layer's raw output.
// A persistent CTA of 128 threads per SM loops over tiles of 128 cells
// (thread i <-> cell row i of the tile), weights staged once per CTA:
//   X [128 x 16] (bf16, K padded 12 -> 16)   z1 = X W1^T      (tcgen05, N = 64, K = 16)
//   H1 = gelu(z1 + b1) [128 x 64] bf16        z2 = H1 W2^T     (4 MMAs of K = 16)
//   H2 = gelu(z2 + b2) [128 x 64] bf16        r  = H2 W3^T     (N padded 2 -> 16)
// Accumulators live in TMEM (z1: columns 0-63, z2: 64-127, r: 128-143 when
// training, 0-15 otherwise); the
// epilogues read them back with tcgen05.ld, add the bias, apply GELU and
// write the next layer's bf16 operand into shared memory.
// Training (ssmd_mlp_grad) continues in the same CTA with the loss
//   L = (1/n) sum_i sum_k w_ik (r_ik - (t_ik - offset_k) / scale_k)^2
// and its backward pass: dH2 = dR W3 and dZ2 = dH2 gelu'(z2 + b2) on the CUDA
// cores (N = 2 is too narrow for an MMA), dH1 = dZ2 W2 on the tensor cores
// (TMEM columns 192-255), dZ1 = dH1 gelu'(z1 + b1); the weight and bias
// gradients (sums over a tile's 128 rows) on the CUDA cores in FP32,
// carried in registers across the CTA's tiles and added across CTAs with
// atomics once at the end.  Every wait on an MMA is bounded:
// on timeout the CTA records bit 0 of the status word, frees its TMEM and
// returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "host.cuh"
#include "umma.cuh"

using namespace ssmd;
using namespace ssmd::host;

namespace {

constexpr int kIn = SSMD_MLP_IN, kK1 = 16, kH = SSMD_MLP_HIDDEN, kOut = SSMD_MLP_OUT, kN3 = 16;
constexpr int kRows = 128, kThreadsMlp = 128;
constexpr int oW1 = 0, oB1 = oW1 + kH * kK1, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH, kParams = oB3 + kOut;
constexpr int oMean = kParams, oInvStd = oMean + kIn, oScale = oInvStd + kIn, oOffset = oScale + kOut,
              kNet = oOffset + kOut;
static_assert(kParams == SSMD_MLP_PARAMS, "parameter layout");
static_assert(kNet == SSMD_MLP_NET_FLOATS, "network layout");

// TMEM columns: training keeps z1 and z2 for the backward pass (256 columns);
// inference writes the last layer over z1, which is dead by then (128
// columns), so four inference CTAs fit on an SM's 512 columns.
template <bool TRAIN>
constexpr uint32_t tmem_cols() { return TRAIN ? 256u : 128u; }
template <bool TRAIN>
constexpr uint32_t col_r() { return TRAIN ? 128u : 0u; }
constexpr uint32_t cZ1 = 0, cZ2 = 64, cDH1 = 192;
constexpr int kFwdCtasPerSm = 4;
constexpr uint64_t kMmaWaitNs = 1000000000ull;
constexpr int kLd = 65; // fp32 row stride of the dZ staging arrays (bank-conflict free)

// shared-memory map (bytes from a 1024-aligned base)
constexpr uint32_t sX = 0, sW1 = 4096, sW3 = 6144, sH1 = 8192, sW2 = 24576, sH2 = 32768, sFwdEnd = 49152;
constexpr uint32_t sW2T = 49152, sDZ2 = 57344, sDZ2F = 73728, sDZ1F = sDZ2F + kRows * kLd * 4,
                   sDY = sDZ1F + kRows * kLd * 4, sTrainEnd = sDY + kRows * kOut * 4;

template <bool TRAIN>
struct Layout {
    static constexpr uint32_t small = TRAIN ? sTrainEnd : sFwdEnd;
    static constexpr uint32_t b1 = small, b2 = b1 + kH * 4, b3 = b2 + kH * 4, w3f = b3 + 16,
                              norm = w3f + kOut * kH * 4, bar = norm + 32 * 4, slot = bar + 8, abort = slot + 4,
                              end = abort + 4;
    static constexpr size_t bytes = end + 1024; // + alignment slack of the dynamic base
};

__device__ unsigned int g_mlp_status;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}

// Store 8 consecutive values (k0 .. k0 + 7) of row r of an R x K bf16 tile.
__device__ __forceinline__ void st8(unsigned char *tile, int r, int k0, int K, const float *v) {
    uint4 u;
    u.x = pack2(v[0], v[1]);
    u.y = pack2(v[2], v[3]);
    u.z = pack2(v[4], v[5]);
    u.w = pack2(v[6], v[7]);
    *reinterpret_cast<uint4 *>(tile + umma::kmajor_offset(r, k0, K)) = u;
}

__device__ __forceinline__ float ldbf(const unsigned char *tile, int r, int k, int K) {
    return __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(tile + umma::kmajor_offset(r, k, K)));
}

// Copy a [rows x K] block of fp32 weights (row stride K) into a bf16 tile
// of rows_pad rows (extra rows zero); transpose: element (r, k) = src[k * rows + r].
__device__ void load_weights(unsigned char *tile, const float *src, int rows, int rows_pad, int K, bool transpose,
                             int tid) {
    for (int e = tid; e < rows_pad * K; e += kThreadsMlp) {
        const int r = e / K, k = e % K;
        float v = 0.f;
        if (r < rows) v = transpose ? src[k * rows + r] : src[r * K + k];
        *reinterpret_cast<__nv_bfloat16 *>(tile + umma::kmajor_offset(r, k, K)) = __float2bfloat16_rn(v);
    }
}

// Bounded wait on the MMA barrier by every thread, then a block-wide vote.
__device__ __forceinline__ bool wait_mma(uint64_t *bar, uint32_t phase, volatile uint32_t *abort_flag) {
    if (!mbar_wait_bounded(bar, phase, kMmaWaitNs)) *abort_flag = 1u;
    __syncthreads();
    const bool ok = *abort_flag == 0u;
    if (ok) umma::fence_after_sync();
    return ok;
}

// Bias + GELU epilogue of a 64-column accumulator into a [128 x 64] bf16 tile.
__device__ __forceinline__ void hidden_epilogue(uint32_t taddr, const float *bias, unsigned char *tile, int r) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float v[16];
        umma::tmem_ld16(taddr + 16 * c, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = gelu(v[i] + bias[16 * c + i]);
        st8(tile, r, 16 * c, kH, v);
        st8(tile, r, 16 * c + 8, kH, v + 8);
    }
}

template <bool TRAIN>
__global__ void __launch_bounds__(kThreadsMlp, TRAIN ? 1 : kFwdCtasPerSm)
    mlp_kernel(const float *__restrict__ net, const float *__restrict__ feat, const float *__restrict__ target,
               const float *__restrict__ weight, int64_t n, float *__restrict__ out, float *__restrict__ grad,
               double *__restrict__ loss) {
    using L = Layout<TRAIN>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                          ~(uintptr_t)1023);
    const int tid = threadIdx.x, warp = tid >> 5;
    float *b1 = reinterpret_cast<float *>(sm + L::b1);
    float *b2 = reinterpret_cast<float *>(sm + L::b2);
    float *b3 = reinterpret_cast<float *>(sm + L::b3);
    float *w3f = reinterpret_cast<float *>(sm + L::w3f);
    float *norm = reinterpret_cast<float *>(sm + L::norm);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L::bar);
    uint32_t *slot = reinterpret_cast<uint32_t *>(sm + L::slot);
    volatile uint32_t *abort_flag = reinterpret_cast<volatile uint32_t *>(sm + L::abort);

    // ---- set-up: TMEM, barrier, weights, this CTA's features
    if (warp == 0) umma::tmem_alloc(slot, tmem_cols<TRAIN>());
    if (tid == 0) {
        mbar_init(bar, 1);
        *abort_flag = 0u;
        fence_barrier_init();
    }
    load_weights(sm + sW1, net + oW1, kH, kH, kK1, false, tid);
    load_weights(sm + sW2, net + oW2, kH, kH, kH, false, tid);
    load_weights(sm + sW3, net + oW3, kOut, kN3, kH, false, tid);
    if constexpr (TRAIN) load_weights(sm + sW2T, net + oW2, kH, kH, kH, true, tid); // (i, o) = W2[o][i]
    for (int e = tid; e < kH; e += kThreadsMlp) {
        b1[e] = net[oB1 + e];
        b2[e] = net[oB2 + e];
    }
    for (int e = tid; e < kOut * kH; e += kThreadsMlp) w3f[e] = net[oW3 + e];
    if (tid < kOut) b3[tid] = net[oB3 + tid];
    if (tid < kNet - kParams) norm[tid] = net[kParams + tid];
    __syncthreads();

    const int r = tid;
    const uint32_t sbase = smem_addr(sm);
    uint32_t phase = 0;
    bool ok = true;
    // weight-gradient partial sums of this CTA, carried across its tiles
    float gw2[32], gw1[8], gw3 = 0.f, gb = 0.f, gb3 = 0.f;
    if constexpr (TRAIN) {
#pragma unroll
        for (int i = 0; i < 32; ++i) gw2[i] = 0.f;
#pragma unroll
        for (int i = 0; i < 8; ++i) gw1[i] = 0.f;
    }
    float lsum = 0.f;
    const int64_t tiles = (n + kRows - 1) / kRows;
    uint32_t tmem = 0, lane_base = 0;

    for (int64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int64_t row = tile * kRows + r;
        const bool valid = row < n;
        {
            float x[kK1];
#pragma unroll
            for (int i = 0; i < kK1; ++i) {
                float v = 0.f;
                if (i < kIn && valid) v = (feat[row * kIn + i] - norm[i]) * norm[kIn + i];
                x[i] = v;
            }
            st8(sm + sX, r, 0, kK1, x);
            st8(sm + sX, r, 8, kK1, x + 8);
        }
        fence_proxy_async(); // generic-proxy smem writes -> visible to the tensor core
        umma::fence_before_sync();
        __syncthreads(); // also: every TMEM read and MMA of the previous tile is complete
        tmem = *slot;
        lane_base = tmem + ((uint32_t)(warp * 32) << 16);

        // ---- layer 1
        if (tid == 0) {
            umma::fence_after_sync();
            umma::mma_bf16(tmem + cZ1, umma::smem_desc(sbase + sX, 128, 256),
                           umma::smem_desc(sbase + sW1, 128, 256), umma::idesc_bf16(128, kH), false);
            umma::commit(bar);
        }
        ok = wait_mma(bar, phase, abort_flag);
        phase ^= 1u;
        if (!ok) break;
        hidden_epilogue(lane_base + cZ1, b1, sm + sH1, r);
        fence_proxy_async();
        umma::fence_before_sync();
        __syncthreads();

        // ---- layer 2
        if (tid == 0) {
            umma::fence_after_sync();
            for (int ks = 0; ks < kH / 16; ++ks)
                umma::mma_bf16(tmem + cZ2, umma::smem_desc(sbase + sH1 + 256 * ks, 128, 1024),
                               umma::smem_desc(sbase + sW2 + 256 * ks, 128, 1024), umma::idesc_bf16(128, kH),
                               ks > 0);
            umma::commit(bar);
        }
        ok = wait_mma(bar, phase, abort_flag);
        phase ^= 1u;
        if (!ok) break;
        hidden_epilogue(lane_base + cZ2, b2, sm + sH2, r);
        fence_proxy_async();
        umma::fence_before_sync();
        __syncthreads();

        // ---- layer 3 (N padded to 16; rows 2..15 of W3 are zero)
        if (tid == 0) {
            umma::fence_after_sync();
            for (int ks = 0; ks < kH / 16; ++ks)
                umma::mma_bf16(tmem + col_r<TRAIN>(), umma::smem_desc(sbase + sH2 + 256 * ks, 128, 1024),
                               umma::smem_desc(sbase + sW3 + 256 * ks, 128, 1024), umma::idesc_bf16(128, kN3),
                               ks > 0);
            umma::commit(bar);
        }
        ok = wait_mma(bar, phase, abort_flag);
        phase ^= 1u;
        if (!ok) break;
        float rr[kOut];
        {
            float v[16];
            umma::tmem_ld16(lane_base + col_r<TRAIN>(), v);
            rr[0] = v[0] + b3[0];
            rr[1] = v[1] + b3[1];
        }
        if constexpr (!TRAIN) {
            if (valid) {
                out[row * kOut + 0] = fmaf(norm[2 * kIn + 0], rr[0], norm[2 * kIn + 2]);
                out[row * kOut + 1] = fmaf(norm[2 * kIn + 1], rr[1], norm[2 * kIn + 3]);
            }
        } else {
            float *dzf2 = reinterpret_cast<float *>(sm + sDZ2F);
            float *dzf1 = reinterpret_cast<float *>(sm + sDZ1F);
            float *dy = reinterpret_cast<float *>(sm + sDY);
            // ---- loss and dL/dr
            float d0 = 0.f, d1 = 0.f;
            if (valid) {
                const float inv_n = 1.0f / (float)n;
                const float t0 = (target[row * kOut + 0] - norm[2 * kIn + 2]) / norm[2 * kIn + 0];
                const float t1 = (target[row * kOut + 1] - norm[2 * kIn + 3]) / norm[2 * kIn + 1];
                const float w0 = weight ? weight[row * kOut + 0] : 1.0f;
                const float w1 = weight ? weight[row * kOut + 1] : 1.0f;
                const float e0 = rr[0] - t0, e1 = rr[1] - t1;
                lsum += w0 * e0 * e0 + w1 * e1 * e1;
                d0 = 2.0f * w0 * e0 * inv_n;
                d1 = 2.0f * w1 * e1 * inv_n;
            }
            dy[r * kOut + 0] = d0;
            dy[r * kOut + 1] = d1;
            // ---- dZ2 = (dR W3) * gelu'(z2 + b2)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float v[16];
                umma::tmem_ld16(lane_base + cZ2 + 16 * c, v);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int j = 16 * c + i;
                    const float dh = fmaf(d0, w3f[j], d1 * w3f[kH + j]);
                    v[i] = dh * gelu_grad(v[i] + b2[j]);
                    dzf2[r * kLd + j] = v[i];
                }
                st8(sm + sDZ2, r, 16 * c, kH, v);
                st8(sm + sDZ2, r, 16 * c + 8, kH, v + 8);
            }
            fence_proxy_async();
            umma::fence_before_sync();
            __syncthreads();
            // ---- dH1 = dZ2 W2 (B = W2^T, K-major)
            if (tid == 0) {
                umma::fence_after_sync();
                for (int ks = 0; ks < kH / 16; ++ks)
                    umma::mma_bf16(tmem + cDH1, umma::smem_desc(sbase + sDZ2 + 256 * ks, 128, 1024),
                                   umma::smem_desc(sbase + sW2T + 256 * ks, 128, 1024), umma::idesc_bf16(128, kH),
                                   ks > 0);
                umma::commit(bar);
            }
            ok = wait_mma(bar, phase, abort_flag);
            phase ^= 1u;
            if (!ok) break;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float dh[16], z[16];
                umma::tmem_ld16(lane_base + cDH1 + 16 * c, dh);
                umma::tmem_ld16(lane_base + cZ1 + 16 * c, z);
#pragma unroll
                for (int i = 0; i < 16; ++i) dzf1[r * kLd + 16 * c + i] = dh[i] * gelu_grad(z[i] + b1[16 * c + i]);
            }
            __syncthreads();
            // ---- weight and bias gradients of this tile: sums over its 128 rows
            {   // dW2[o][i] = sum_r dZ2[r][o] H1[r][i]: thread -> (o, 32 i)
                const int o = tid >> 1, i0 = (tid & 1) * 32;
                for (int rr2 = 0; rr2 < kRows; ++rr2) {
                    const float d = dzf2[rr2 * kLd + o];
#pragma unroll
                    for (int ch = 0; ch < 4; ++ch) {
                        const uint4 u = *reinterpret_cast<const uint4 *>(sm + sH1 +
                                                                         umma::kmajor_offset(rr2, i0 + 8 * ch, kH));
                        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float2 f2 = __bfloat1622float2(h[e]);
                            gw2[8 * ch + 2 * e] = fmaf(d, f2.x, gw2[8 * ch + 2 * e]);
                            gw2[8 * ch + 2 * e + 1] = fmaf(d, f2.y, gw2[8 * ch + 2 * e + 1]);
                        }
                    }
                }
            }
            {   // dW1[o][i] = sum_r dZ1[r][o] X[r][i]: thread -> (o, 8 i)
                const int o = tid >> 1, i0 = (tid & 1) * 8;
                for (int rr2 = 0; rr2 < kRows; ++rr2) {
                    const float d = dzf1[rr2 * kLd + o];
                    const uint4 u = *reinterpret_cast<const uint4 *>(sm + sX + umma::kmajor_offset(rr2, i0, kK1));
                    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float2 f2 = __bfloat1622float2(h[e]);
                        gw1[2 * e] = fmaf(d, f2.x, gw1[2 * e]);
                        gw1[2 * e + 1] = fmaf(d, f2.y, gw1[2 * e + 1]);
                    }
                }
            }
            {   // dW3[k][j] = sum_r dR[r][k] H2[r][j]; db2 (k = 0 threads), db1 (k = 1); db3
                const int k = tid >> 6, j = tid & 63;
                for (int rr2 = 0; rr2 < kRows; ++rr2) {
                    gw3 = fmaf(dy[rr2 * kOut + k], ldbf(sm + sH2, rr2, j, kH), gw3);
                    gb += k == 0 ? dzf2[rr2 * kLd + j] : dzf1[rr2 * kLd + j];
                }
                if (tid < kOut)
                    for (int rr2 = 0; rr2 < kRows; ++rr2) gb3 += dy[rr2 * kOut + tid];
            }
            __syncthreads(); // the next tile overwrites X, H1, H2 and the dZ staging
        }
    }

    if constexpr (TRAIN) {
        if (ok) {
            const int o = tid >> 1;
            const int i0 = (tid & 1) * 32, i1 = (tid & 1) * 8;
#pragma unroll
            for (int i = 0; i < 32; ++i) atomicAdd(&grad[oW2 + o * kH + i0 + i], gw2[i]);
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (i1 + i < kIn) atomicAdd(&grad[oW1 + o * kK1 + i1 + i], gw1[i]);
            const int k = tid >> 6, j = tid & 63;
            atomicAdd(&grad[oW3 + k * kH + j], gw3);
            atomicAdd(&grad[(k == 0 ? oB2 : oB1) + j], gb);
            if (tid < kOut) atomicAdd(&grad[oB3 + tid], gb3);
            float l = lsum;
            for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
            if ((tid & 31) == 0) atomicAdd(loss, (double)l / (double)n);
        }
    }

    // ---- tear-down: every TMEM read is complete before the warp frees it
    umma::fence_before_sync();
    __syncthreads();
    if (!ok && tid == 0) atomicOr(&g_mlp_status, 1u);
    if (warp == 0) umma::tmem_dealloc(*slot, tmem_cols<TRAIN>());
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int count, float lr, float beta1, float beta2, float eps,
                            float corr1, float corr2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
    const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / corr1) / (sqrtf(vi / corr2) + eps);
}

template <bool TRAIN>
int launch(const float *net, const float *feat, const float *target, const float *weight, int64_t n, float *out,
           float *grad, double *loss, cudaStream_t st) {
    // shared memory sized so that at most 512 / tmem_cols CTAs share an SM:
    // every resident CTA then holds its TMEM columns without waiting in
    // tcgen05.alloc (training: 1 per SM, inference: 4 per SM)
    const size_t floor_bytes = TRAIN ? (size_t)120 * 1024 : (size_t)52 * 1024;
    const size_t smem = Layout<TRAIN>::bytes > floor_bytes ? Layout<TRAIN>::bytes : floor_bytes;
    static bool attr_set = false;
    if (!attr_set) {
        if (int e = cuda_check(cudaFuncSetAttribute(mlp_kernel<TRAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)smem),
                               "mlp smem attribute"))
            return e;
        attr_set = true;
    }
    // persistent: one CTA per SM, each loops over 128-row tiles
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    const int64_t tiles = (n + kRows - 1) / kRows;
    const int64_t slots = (int64_t)sms * (TRAIN ? 1 : kFwdCtasPerSm);
    const unsigned blocks = (unsigned)(tiles < slots ? tiles : slots);
    mlp_kernel<TRAIN><<<blocks, kThreadsMlp, smem, st>>>(net, feat, target, weight, n, out, grad, loss);
    return cuda_check(cudaGetLastError(), "mlp launch");
}

} // namespace

extern "C" int ssmd_mlp_forward(const float *net, const float *features, int64_t n, float *out,
                                ssmd_stream_t stream) {
    if (!net || !features || !out || n < 0) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument or n < 0");
    if (n == 0) return SSMD_OK;
    if (n > (int64_t)0x7FFFFFFF * kRows) return fail(SSMD_ERR_INVALID_ARGUMENT, "too many rows");
    return launch<false>(net, features, nullptr, nullptr, n, out, nullptr, nullptr,
                         reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ssmd_mlp_grad(const float *net, const float *features, const float *targets, const float *weights,
                             int64_t n, float *grad, double *loss, ssmd_stream_t stream) {
    if (!net || !features || !targets || !grad || !loss || n <= 0)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument or n <= 0");
    if (n > (int64_t)0x7FFFFFFF * kRows) return fail(SSMD_ERR_INVALID_ARGUMENT, "too many rows");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int e = cuda_check(cudaMemsetAsync(grad, 0, sizeof(float) * kParams, st), "grad clear")) return e;
    if (int e = cuda_check(cudaMemsetAsync(loss, 0, sizeof(double), st), "loss clear")) return e;
    return launch<true>(net, features, targets, weights, n, nullptr, grad, loss, st);
}

extern "C" int ssmd_mlp_adam(float *net, const float *grad, float *m, float *v, int64_t t, float lr, float beta1,
                             float beta2, float eps, ssmd_stream_t stream) {
    if (!net || !grad || !m || !v || t <= 0) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument or t <= 0");
    const float corr1 = (float)(1.0 - pow((double)beta1, (double)t));
    const float corr2 = (float)(1.0 - pow((double)beta2, (double)t));
    adam_kernel<<<(kParams + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        net, grad, m, v, kParams, lr, beta1, beta2, eps, corr1, corr2);
    return cuda_check(cudaGetLastError(), "adam launch");
}

extern "C" int ssmd_mlp_status(uint32_t *status) {
    if (!status) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    unsigned int v = 0;
    if (int e = cuda_check(cudaMemcpyFromSymbol(&v, g_mlp_status, sizeof v), "mlp status")) return e;
    *status = v;
    return SSMD_OK;
}
