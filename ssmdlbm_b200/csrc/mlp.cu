// mlp.cu — the learned closure's per-cell network on the 5th-generation tensor cores.
//
// Network: 12 features -> 64 -> 64 -> 2 outputs, GELU after the two hidden
// layers in its tanh form, gelu(z) = z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715
// z^3))) (Hendrycks & Gimpel, "Gaussian Error Linear Units", 2016), with
// tanh from the SFU (tanh.approx.f32, absolute error about 2^-11, below the
// bf16 rounding of the hidden activations that follows), features
// standardised by stored mean / inverse std, outputs p = scale * r + offset
// with r the last layer's raw output.  A persistent CTA of 128 threads loops
// over tiles of 128 cells (thread i <-> cell row i of the tile), weights
// staged once per CTA:
//   X [128 x 16] (bf16, K padded 12 -> 16)   z1 = X W1^T      (tcgen05, N = 64, K = 16)
//   H1 = gelu(z1 + b1) [128 x 64] bf16        z2 = H1 W2^T     (4 MMAs of K = 16)
//   H2 = gelu(z2 + b2) [128 x 64] bf16        r  = H2 W3^T     (N padded 2 -> 16)
// The epilogues read the accumulators back with tcgen05.ld (the next 16
// columns in flight while the current 16 are processed), add the bias,
// apply GELU on pairs of columns with packed FP32 arithmetic (fma.rn.f32x2
// and friends, sm_100) and write the next layer's bf16 operand.  Inference
// stages W2 and W3 halved and its epilogues write 2 gelu(z), one multiply
// fewer per value: the products, hence every result, are the same bit for
// bit (scaling by 2 commutes with each rounding).
// Inference (forward, and the fused closure refresh that computes the
// features from the macroscopic fields and applies the outputs) keeps one
// 64-column accumulator (z1, z2 and r in turn: each is dead once its
// epilogue has read it) and one activation tile (X, H1, H2 in turn: each is
// dead once the MMA reading it has completed), 29 KB of shared memory and 64
// TMEM columns per CTA, so seven CTAs share an SM and hide each other's MMA
// round trips.
// Training (ssmd_mlp_grad) keeps z1 and z2 for the backward pass:
//   L = (1/n) sum_i sum_k w_ik (r_ik - (t_ik - offset_k) / scale_k)^2,
// dH2 = dR W3 and dZ2 = dH2 gelu'(z2 + b2) on the CUDA cores (N = 2 is too
// narrow for an MMA), dH1 = dZ2 W2 on the tensor cores, dZ1 = dH1 gelu'(z1 +
// b1); the weight and bias gradients (sums over a tile's 128 rows) on the
// tensor cores too: the epilogues also write H1, H2, X, dZ1, dZ2 and dR
// transposed (bf16, K = the tile's rows), and two MMAs per tile accumulate
// dW2^T, dW3^T (G1) and dW1^T with the bias gradients (G2, through a row of
// ones) in TMEM across the CTA's tiles; they run while the next tile's
// features load.  The CTA's sums are then either added across CTAs with
// atomics (ssmd_mlp_grad) or written as one row per CTA and summed in CTA
// order by a second kernel (ssmd_mlp_grad_ws: the same bits on every run).  Every wait on an MMA is bounded: on timeout
// the CTA records bit 0 of the status word, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "closure.cuh"
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

enum : int { kFwd = 0, kTrain = 1, kRefresh = 2 };

// TMEM columns: training keeps z1 (0-63) and z2 (64-127) for the backward
// pass, r at 128-143, dH1 at 192-255 and the CTA's weight-gradient sums
// across its tiles at 256-335 (G1) and 336-479 (G2); inference puts z1, z2
// and r in turn on columns 0-63.
template <int MODE>
constexpr uint32_t tmem_cols() { return MODE == kTrain ? 512u : 64u; }
template <int MODE>
constexpr uint32_t col_z2() { return MODE == kTrain ? 64u : 0u; }
template <int MODE>
constexpr uint32_t col_r() { return MODE == kTrain ? 128u : 0u; }
constexpr uint32_t cZ1 = 0, cDH1 = 192, cG1 = 256, cG2 = 336;
constexpr int kGK = kRows;         // K of the weight-gradient MMAs: the tile's rows
constexpr int kGB = 2 * kH + 16;   // rows of the gradient B tile: dZ1^T, dZ2^T, dR^T (2 of 16)
constexpr uint64_t kMmaWaitNs = 1000000000ull;
constexpr int kMaxGradCtas = 256; // rows of the deterministic gradient workspace

// shared-memory map (bytes from an aligned base: 1024 bytes for training,
// 128 for inference; the no-swizzle operand layout needs 16); training-only
// tiles: W2^T, bf16 dZ2, and the operands of the weight-gradient MMAs, all
// K-major with K = the tile's 128 rows:
//   GA2 [16 x 128]: X^T (rows 0-11), a row of ones (12), zeros (13-15); the
//       M = 128 MMA reads rows 16-127 from GA1 that follows (their products
//       land in accumulator rows nobody reads)
//   GA1 [128 x 128]: H1^T (rows 0-63), H2^T (rows 64-127)
//   GB  [144 x 128]: dZ1^T (rows 0-63), dZ2^T (64-127), dR^T (128-129), zeros
// so that G1 = GA1 GB[64..143]^T holds dW2^T and dW3^T, and G2 = GA2 GB^T
// holds dW1^T and, in its ones row, the three bias gradients; then a small
// scratch for the per-warp losses
constexpr uint32_t sW2T = 49152, sDZ2 = 57344, sGA2 = 73728, sGA1 = sGA2 + 16 * kGK * 2,
                   sGB = sGA1 + kRows * kGK * 2, sDY = sGB + kGB * kGK * 2;
static_assert(sGA2 + (uint32_t)kRows * kGK * 2 <= sGB, "the M = 128 read of GA2 stays inside GA2 + GA1");
template <int MODE>
struct Layout {
    static constexpr bool T = MODE == kTrain;
    // inference: W1, W3, W2, then one activation tile that holds X, H1, H2 in turn
    static constexpr uint32_t sW1 = T ? 4096 : 0, sW3 = T ? 6144 : 2048, sH1 = T ? 8192 : 12288,
                              sW2 = T ? 24576 : 4096, sH2 = T ? 32768 : sH1, sX = T ? 0 : sH1;
    static constexpr uint32_t big = T ? sDY + kRows * kOut * 4 : sH1 + kRows * kH * 2;
    static constexpr uint32_t b1 = big, b2 = b1 + kH * 4, b3 = b2 + kH * 4, w3f = b3 + 16,
                              norm = w3f + (T ? kOut * kH * 4 : 0), bar = norm + 32 * 4, slot = bar + 8,
                              abort = slot + 4, end = abort + 4;
    static constexpr uint32_t align = T ? 1024 : 128;
    static constexpr size_t bytes = end + align; // + alignment slack of the dynamic base
};

// Everything a launch needs (one struct for the three modes).
struct MlpArgs {
    const float *net;
    const float *feat;   // kFwd, kTrain: n x 12 features
    const float *target; // kTrain
    const float *weight; // kTrain (may be null)
    int64_t n;
    float *out;          // kFwd: n x 2
    float *grad;         // kTrain: atomics into grad, or null with partials
    float *partials;     // kTrain deterministic: one row of kParams + 1 per CTA
    double *loss;        // kTrain (atomic path)
    closure::Grid g;     // kRefresh: the lattice and its macroscopic fields
    const float *rho, *ux, *uy, *uz, *phi;
    float nu_w, nu_dow, nut_max;
    float *nut, *cs;     // kRefresh outputs
};

__device__ unsigned int g_mlp_status;

// GELU, tanh form: u = sqrt(2/pi) z (1 + 0.044715 z^2), gelu = z/2 + z/2 tanh(u)
constexpr float kG0 = 0.7978845608028654f;           // sqrt(2 / pi)
constexpr float kG1 = 0.7978845608028654f * 0.044715f;

__device__ __forceinline__ float tanh_sfu(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// gelu of two columns at once: u = z fma(kG1, z^2, kG0), h = z/2,
// gelu = fma(h, tanh(u), h), elementwise with packed FP32 (fma.rn.f32x2 etc.);
// TWICE: 2 gelu(z) = fma(z, tanh(u), z).
template <bool TWICE = false>
__device__ __forceinline__ float2 gelu2(float2 z) {
    const float2 p = __ffma2_rn(__fmul2_rn(z, z), make_float2(kG1, kG1), make_float2(kG0, kG0));
    const float2 u = __fmul2_rn(z, p);
    const float2 t = make_float2(tanh_sfu(u.x), tanh_sfu(u.y));
    if constexpr (TWICE) return __ffma2_rn(z, t, z);
    const float2 hz = __fmul2_rn(z, make_float2(0.5f, 0.5f));
    return __ffma2_rn(hz, t, hz);
}
// d gelu / dz = (1 + t)/2 + z/2 (1 - t^2) du/dz,  du/dz = sqrt(2/pi) (1 + 3 * 0.044715 z^2)
__device__ __forceinline__ float gelu_grad(float z) {
    const float z2 = z * z;
    const float t = tanh_sfu(z * fmaf(kG1, z2, kG0));
    const float du = fmaf(3.0f * kG1, z2, kG0);
    return fmaf(0.5f * z * du, fmaf(-t, t, 1.0f), fmaf(0.5f, t, 0.5f));
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


// Copy a [rows x K] block of fp32 weights (row stride K), times `scale` (a
// power of two), into a bf16 tile of rows_pad rows (extra rows zero);
// transpose: element (r, k) = src[k * rows + r].
__device__ void load_weights(unsigned char *tile, const float *src, int rows, int rows_pad, int K, bool transpose,
                             int tid, float scale = 1.0f) {
    for (int e = tid; e < rows_pad * K; e += kThreadsMlp) {
        const int r = e / K, k = e % K;
        float v = 0.f;
        if (r < rows) v = transpose ? src[k * rows + r] : src[r * K + k];
        *reinterpret_cast<__nv_bfloat16 *>(tile + umma::kmajor_offset(r, k, K)) = __float2bfloat16_rn(v * scale);
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

// Element (m, k) of a K-major bf16 tile with K = kGK (the weight-gradient
// operands: the tile's rows r are their K).
__device__ __forceinline__ void st_g(unsigned char *tile, int m, int k, uint16_t bits) {
    *reinterpret_cast<uint16_t *>(tile + umma::kmajor_offset(m, k, kGK)) = bits;
}
__device__ __forceinline__ uint16_t bf16_bits(float v) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    return *reinterpret_cast<const uint16_t *>(&h);
}

// Bias + GELU epilogue of a 64-column accumulator into a [128 x 64] bf16 tile
// (TWICE: 2 gelu, for a next layer staged with halved weights; TRANS: the
// same bf16 values also into column r, rows trow0 .. trow0 + 63, of a
// weight-gradient operand tile).  The TMEM load of columns 16 (c + 1) ..
// 16 c + 31 is in flight while columns 16 c .. 16 c + 15 are processed.
template <bool TWICE = false, bool TRANS = false>
__device__ __forceinline__ void hidden_epilogue(uint32_t taddr, const float *bias, unsigned char *tile, int r,
                                                unsigned char *ttile = nullptr, int trow0 = 0) {
    uint32_t nxt[16];
    umma::tmem_ld16_issue(taddr, nxt);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float v[16];
        umma::tmem_ld_wait16(nxt);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(nxt[i]);
        if (c < 3) umma::tmem_ld16_issue(taddr + 16 * (c + 1), nxt);
        uint32_t pk[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float4 b = *reinterpret_cast<const float4 *>(bias + 16 * c + 4 * i);
            const float2 g0 = gelu2<TWICE>(__fadd2_rn(make_float2(v[4 * i], v[4 * i + 1]), make_float2(b.x, b.y)));
            const float2 g1 = gelu2<TWICE>(__fadd2_rn(make_float2(v[4 * i + 2], v[4 * i + 3]), make_float2(b.z, b.w)));
            pk[2 * i] = pack2(g0.x, g0.y);
            pk[2 * i + 1] = pack2(g1.x, g1.y);
        }
        if constexpr (TRANS) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                st_g(ttile, trow0 + 16 * c + 2 * i, r, (uint16_t)(pk[i] & 0xFFFFu));
                st_g(ttile, trow0 + 16 * c + 2 * i + 1, r, (uint16_t)(pk[i] >> 16));
            }
        }
        *reinterpret_cast<uint4 *>(tile + umma::kmajor_offset(r, 16 * c, kH)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        *reinterpret_cast<uint4 *>(tile + umma::kmajor_offset(r, 16 * c + 8, kH)) =
            make_uint4(pk[4], pk[5], pk[6], pk[7]);
    }
}

// The 12 standardised features of one row into x[16] (columns 12-15 zero);
// kRefresh also returns feature 11, nu(phi), for the bound on nu_t.
template <int MODE>
__device__ __forceinline__ void load_row(const MlpArgs &a, const float *norm, int64_t row, bool valid, float (&x)[kK1],
                                         float &nu_phi) {
#pragma unroll
    for (int i = 0; i < kK1; ++i) x[i] = 0.f;
    nu_phi = 0.f;
    if (!valid) return;
    float f[kIn];
    if constexpr (MODE == kRefresh) {
        closure::cell_features(a.g, a.rho, a.ux, a.uy, a.uz, a.phi, a.nu_w, a.nu_dow, row, f);
    } else if ((reinterpret_cast<uintptr_t>(a.feat) & 15u) == 0) {
        const float4 *p = reinterpret_cast<const float4 *>(a.feat + row * kIn); // 48-byte rows: 16-byte aligned
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const float4 v = __ldg(p + q);
            f[4 * q] = v.x;
            f[4 * q + 1] = v.y;
            f[4 * q + 2] = v.z;
            f[4 * q + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < kIn; ++i) f[i] = __ldg(a.feat + row * kIn + i);
    }
    nu_phi = f[11];
#pragma unroll
    for (int i = 0; i < kIn; ++i) x[i] = (f[i] - norm[i]) * norm[kIn + i];
}

template <int MODE>
__global__ void __launch_bounds__(kThreadsMlp, MODE == kTrain ? 1 : 7) mlp_kernel(const MlpArgs a) {
    constexpr bool TRAIN = MODE == kTrain;
    using L = Layout<MODE>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + (L::align - 1)) &
                                                          ~(uintptr_t)(L::align - 1));
    const int tid = threadIdx.x, warp = tid >> 5;
    const float *net = a.net;
    const int64_t n = a.n;
    float *b1 = reinterpret_cast<float *>(sm + L::b1);
    float *b2 = reinterpret_cast<float *>(sm + L::b2);
    float *b3 = reinterpret_cast<float *>(sm + L::b3);
    float *w3f = reinterpret_cast<float *>(sm + L::w3f);
    float *norm = reinterpret_cast<float *>(sm + L::norm);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L::bar);
    uint32_t *slot = reinterpret_cast<uint32_t *>(sm + L::slot);
    volatile uint32_t *abort_flag = reinterpret_cast<volatile uint32_t *>(sm + L::abort);

    // ---- set-up: TMEM, barrier, weights
    if (warp == 0) umma::tmem_alloc(slot, tmem_cols<MODE>());
    if (tid == 0) {
        mbar_init(bar, 1);
        *abort_flag = 0u;
        fence_barrier_init();
    }
    load_weights(sm + L::sW1, net + oW1, kH, kH, kK1, false, tid);
    // inference feeds W2 and W3 with 2 gelu(z): halved weights, the same products
    load_weights(sm + L::sW2, net + oW2, kH, kH, kH, false, tid, TRAIN ? 1.0f : 0.5f);
    load_weights(sm + L::sW3, net + oW3, kOut, kN3, kH, false, tid, TRAIN ? 1.0f : 0.5f);
    if constexpr (TRAIN) load_weights(sm + sW2T, net + oW2, kH, kH, kH, true, tid); // (i, o) = W2[o][i]
    for (int e = tid; e < kH; e += kThreadsMlp) {
        b1[e] = net[oB1 + e];
        b2[e] = net[oB2 + e];
    }
    if constexpr (TRAIN)
        for (int e = tid; e < kOut * kH; e += kThreadsMlp) w3f[e] = net[oW3 + e];
    if (tid < kOut) b3[tid] = net[oB3 + tid];
    if (tid < kNet - kParams) norm[tid] = net[kParams + tid];
    if constexpr (TRAIN) {
        // the rows of the gradient operands that no tile writes: GA2 row 12
        // all ones (its products are the column sums, the bias gradients),
        // rows 13-15 and GB rows 130-143 zero
        const uint16_t one = bf16_bits(1.0f);
        st_g(sm + sGA2, 12, tid, one);
        for (int m = 13; m < 16; ++m) st_g(sm + sGA2, m, tid, 0);
        for (int m = 2 * kH + kOut; m < kGB; ++m) st_g(sm + sGB, m, tid, 0);
    }
    __syncthreads();

    const int r = tid;
    const uint32_t sbase = smem_addr(sm);
    uint32_t phase = 0;
    bool ok = true;
    // training: the weight-gradient MMAs of a tile run while the next tile's
    // features load; gpend says they are in flight (waited for before the
    // next tile writes their operands, and after the last tile)
    bool gpend = false, gfirst = true;
    float lsum = 0.f;
    const int64_t tiles = (n + kRows - 1) / kRows;
    uint32_t tmem = 0, lane_base = 0;

    for (int64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int64_t row = tile * kRows + r;
        const bool valid = row < n;
        float nu_phi;
        {
            float x[kK1];
            load_row<MODE>(a, norm, row, valid, x, nu_phi);
            st8(sm + L::sX, r, 0, kK1, x);
            st8(sm + L::sX, r, 8, kK1, x + 8);
            if constexpr (TRAIN) {
                if (gpend) { // the previous tile's gradient MMAs read GA2, GA1, GB
                    ok = wait_mma(bar, phase, abort_flag);
                    phase ^= 1u;
                    gpend = false;
                    if (!ok) break;
                }
#pragma unroll
                for (int k = 0; k < kIn; ++k) st_g(sm + sGA2, k, r, bf16_bits(x[k])); // X^T
            }
        }
        fence_proxy_async(); // generic-proxy smem writes -> visible to the tensor core
        umma::fence_before_sync();
        __syncthreads(); // also: every TMEM read and MMA of the previous tile is complete
        tmem = *slot;
        lane_base = tmem + ((uint32_t)(warp * 32) << 16);

        // ---- layer 1
        if (tid == 0) {
            umma::fence_after_sync();
            umma::mma_bf16(tmem + cZ1, umma::smem_desc(sbase + L::sX, 128, 256),
                           umma::smem_desc(sbase + L::sW1, 128, 256), umma::idesc_bf16(128, kH), false);
            umma::commit(bar);
        }
        ok = wait_mma(bar, phase, abort_flag);
        phase ^= 1u;
        if (!ok) break;
        hidden_epilogue<!TRAIN, TRAIN>(lane_base + cZ1, b1, sm + L::sH1, r, sm + sGA1, 0); // (H1^T)
        fence_proxy_async();
        umma::fence_before_sync();
        __syncthreads();

        // ---- layer 2
        if (tid == 0) {
            umma::fence_after_sync();
            for (int ks = 0; ks < kH / 16; ++ks)
                umma::mma_bf16(tmem + col_z2<MODE>(), umma::smem_desc(sbase + L::sH1 + 256 * ks, 128, 1024),
                               umma::smem_desc(sbase + L::sW2 + 256 * ks, 128, 1024), umma::idesc_bf16(128, kH),
                               ks > 0);
            umma::commit(bar);
        }
        ok = wait_mma(bar, phase, abort_flag);
        phase ^= 1u;
        if (!ok) break;
        hidden_epilogue<!TRAIN, TRAIN>(lane_base + col_z2<MODE>(), b2, sm + L::sH2, r, sm + sGA1, kH); // (H2^T)
        fence_proxy_async();
        umma::fence_before_sync();
        __syncthreads();

        // ---- layer 3 (N padded to 16; rows 2..15 of W3 are zero)
        if (tid == 0) {
            umma::fence_after_sync();
            for (int ks = 0; ks < kH / 16; ++ks)
                umma::mma_bf16(tmem + col_r<MODE>(), umma::smem_desc(sbase + L::sH2 + 256 * ks, 128, 1024),
                               umma::smem_desc(sbase + L::sW3 + 256 * ks, 128, 1024), umma::idesc_bf16(128, kN3),
                               ks > 0);
            umma::commit(bar);
        }
        ok = wait_mma(bar, phase, abort_flag);
        phase ^= 1u;
        if (!ok) break;
        float rr[kOut];
        {
            float v[2];
            umma::tmem_ld2(lane_base + col_r<MODE>(), v);
            rr[0] = v[0] + b3[0];
            rr[1] = v[1] + b3[1];
        }
        if constexpr (MODE == kFwd) {
            if (valid)
                *reinterpret_cast<float2 *>(a.out + row * kOut) =
                    make_float2(fmaf(norm[2 * kIn + 0], rr[0], norm[2 * kIn + 2]),
                                fmaf(norm[2 * kIn + 1], rr[1], norm[2 * kIn + 3]));
        } else if constexpr (MODE == kRefresh) {
            // the closure's bounds (ssmd_closure_apply): nu_t >= max(-nu(phi)/2, -nut_max)
            if (valid) {
                const float p0 = fmaf(norm[2 * kIn + 0], rr[0], norm[2 * kIn + 2]);
                const float p1 = fmaf(norm[2 * kIn + 1], rr[1], norm[2 * kIn + 3]);
                const float lo = fmaxf(-0.5f * nu_phi, -a.nut_max);
                a.nut[row] = fminf(fmaxf(p0, lo), a.nut_max);
                a.cs[row] = fminf(fmaxf(p1, 0.25f), 4.0f);
            }
        } else {
            // ---- loss and dL/dr
            float d0 = 0.f, d1 = 0.f;
            if (valid) {
                const float inv_n = 1.0f / (float)n;
                const float t0 = (a.target[row * kOut + 0] - norm[2 * kIn + 2]) / norm[2 * kIn + 0];
                const float t1 = (a.target[row * kOut + 1] - norm[2 * kIn + 3]) / norm[2 * kIn + 1];
                const float w0 = a.weight ? a.weight[row * kOut + 0] : 1.0f;
                const float w1 = a.weight ? a.weight[row * kOut + 1] : 1.0f;
                const float e0 = rr[0] - t0, e1 = rr[1] - t1;
                lsum += w0 * e0 * e0 + w1 * e1 * e1;
                d0 = 2.0f * w0 * e0 * inv_n;
                d1 = 2.0f * w1 * e1 * inv_n;
            }
            st_g(sm + sGB, 2 * kH + 0, r, bf16_bits(d0)); // dR^T
            st_g(sm + sGB, 2 * kH + 1, r, bf16_bits(d1));
            // ---- dZ2 = (dR W3) * gelu'(z2 + b2)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float v[16];
                umma::tmem_ld16(lane_base + col_z2<MODE>() + 16 * c, v);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int j = 16 * c + i;
                    const float dh = fmaf(d0, w3f[j], d1 * w3f[kH + j]);
                    v[i] = dh * gelu_grad(v[i] + b2[j]);
                    st_g(sm + sGB, kH + j, r, bf16_bits(v[i])); // dZ2^T
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
                for (int i = 0; i < 16; ++i)
                    st_g(sm + sGB, 16 * c + i, r, bf16_bits(dh[i] * gelu_grad(z[i] + b1[16 * c + i]))); // dZ1^T
            }
            fence_proxy_async();
            umma::fence_before_sync();
            __syncthreads();
            // ---- weight and bias gradients of this tile, summed over its 128
            // rows (the MMAs' K) into the CTA's accumulators G1 and G2:
            //   G1 [128 x 80]  += GA1 GB[64..143]^T: rows 0-63 dW2^T, rows 64-127 cols 64-65 dW3^T
            //   G2 [128 x 144] += GA2 GB^T: rows 0-11 cols 0-63 dW1^T; row 12: db1, db2, db3
            if (tid == 0) {
                umma::fence_after_sync();
                for (int ks = 0; ks < kGK / 16; ++ks)
                    umma::mma_bf16(tmem + cG1, umma::smem_desc(sbase + sGA1 + 256 * ks, 128, 2048),
                                   umma::smem_desc(sbase + sGB + (kH / 8) * 2048 + 256 * ks, 128, 2048),
                                   umma::idesc_bf16(128, kGB - kH), !gfirst || ks > 0);
                for (int ks = 0; ks < kGK / 16; ++ks)
                    umma::mma_bf16(tmem + cG2, umma::smem_desc(sbase + sGA2 + 256 * ks, 128, 2048),
                                   umma::smem_desc(sbase + sGB + 256 * ks, 128, 2048), umma::idesc_bf16(128, kGB),
                                   !gfirst || ks > 0);
                umma::commit(bar);
            }
            gpend = true;
            gfirst = false;
        }
    }
    if constexpr (TRAIN) {
        if (ok && gpend) {
            ok = wait_mma(bar, phase, abort_flag);
            phase ^= 1u;
        }
    }

    if constexpr (TRAIN) {
        if (ok) {
            // atomics into grad, or this CTA's row of the deterministic workspace
            float *dst = a.partials ? a.partials + (size_t)blockIdx.x * (kParams + 1) : a.grad;
            auto put = [&](int k, float v) {
                if (a.partials) dst[k] = v;
                else atomicAdd(&dst[k], v);
            };
            // thread m reads row m of the accumulators (warp w holds lanes 32 w ..)
            const int m = tid;
            if (!gfirst) {
                const uint32_t lb = *slot + ((uint32_t)(warp * 32) << 16);
                float v[16];
                if (m < kH) { // dW2[o][m] = G1[m][o]
#pragma unroll
                    for (int c = 0; c < kH / 16; ++c) {
                        umma::tmem_ld16(lb + cG1 + 16 * c, v);
#pragma unroll
                        for (int i = 0; i < 16; ++i) put(oW2 + (16 * c + i) * kH + m, v[i]);
                    }
                } else { // dW3[k][m - 64] = G1[m][64 + k]
                    umma::tmem_ld16(lb + cG1 + kH, v);
                    put(oW3 + 0 * kH + (m - kH), v[0]);
                    put(oW3 + 1 * kH + (m - kH), v[1]);
                }
                if (warp == 0) { // warp-collective loads: lanes 0-11 dW1, lane 12 the biases
                    for (int c = 0; c < kGB / 16; ++c) {
                        umma::tmem_ld16(lb + cG2 + 16 * c, v);
#pragma unroll
                        for (int i = 0; i < 16; ++i) {
                            const int col = 16 * c + i;
                            if (col < kH && m < kK1) put(oW1 + col * kK1 + m, m < kIn ? v[i] : 0.f); // dW1[o][m]
                            if (m == kIn) {
                                if (col < kH) put(oB1 + col, v[i]);
                                else if (col < 2 * kH) put(oB2 + col - kH, v[i]);
                                else if (col < 2 * kH + kOut) put(oB3 + col - 2 * kH, v[i]);
                            }
                        }
                    }
                }
            } else { // a CTA without tiles adds zeros
                for (int e = tid; e < kParams; e += kThreadsMlp) put(e, 0.f);
            }
            float l = lsum;
            for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
            if (a.partials) {
                float *wl = reinterpret_cast<float *>(sm + sDY); // per-warp losses, summed in warp order
                __syncthreads();
                if ((tid & 31) == 0) wl[warp] = l;
                __syncthreads();
                if (tid == 0) dst[kParams] = ((wl[0] + wl[1]) + wl[2]) + wl[3];
            } else if ((tid & 31) == 0) {
                atomicAdd(a.loss, (double)l / (double)n);
            }
        }
    }

    // ---- tear-down: every TMEM read is complete before the warp frees it
    umma::fence_before_sync();
    __syncthreads();
    if (!ok && tid == 0) atomicOr(&g_mlp_status, 1u);
    if (warp == 0) umma::tmem_dealloc(*slot, tmem_cols<MODE>());
}

// Deterministic reduction of the per-CTA gradient rows: thread k sums column
// k over the CTAs in CTA order (FP32, like the atomic path); the loss column
// in FP64.
__global__ void grad_sum_kernel(const float *__restrict__ partials, int ctas, int64_t n, float *__restrict__ grad,
                                double *__restrict__ loss) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < kParams) {
        float s = 0.f;
        for (int b = 0; b < ctas; ++b) s += partials[(size_t)b * (kParams + 1) + k];
        grad[k] = s;
    } else if (k == kParams) {
        double s = 0.0;
        for (int b = 0; b < ctas; ++b) s += (double)partials[(size_t)b * (kParams + 1) + kParams];
        *loss = s / (double)n;
    }
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

__global__ void average_kernel(float *__restrict__ avg, const float *__restrict__ p, int count, float decay) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    avg[i] = fmaf(decay, avg[i] - p[i], p[i]); // decay avg + (1 - decay) p
}

// Resident CTAs per SM of a mode and the SM count, computed once per mode and
// device from the device's limits: shared memory (with the per-block
// reservation), registers (allocated per warp in multiples of 8 per thread),
// threads, blocks, and TMEM (every resident CTA must get its columns without
// waiting in tcgen05.alloc).  On sm_100a with CUDA 12.9 the occupancy query
// returns 1 for these kernels, where the hardware holds 7 (ncu's
// launch__occupancy_limit_shared_mem), so it is not used.
template <int MODE>
int launch_shape(size_t smem, int &per_sm, int &sms) {
    static thread_local int cached_dev = -1, c_per_sm = 1, c_sms = 148;
    int dev = 0;
    if (int e = cuda_check(cudaGetDevice(&dev), "cudaGetDevice")) return e;
    if (dev != cached_dev) {
        if (int e = cuda_check(cudaFuncSetAttribute(mlp_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)smem),
                               "mlp smem attribute"))
            return e;
        cudaFuncAttributes fa{};
        if (int e = cuda_check(cudaFuncGetAttributes(&fa, mlp_kernel<MODE>), "mlp attributes")) return e;
        auto attr = [&](cudaDeviceAttr a, int fallback) {
            int v = 0;
            return (cudaDeviceGetAttribute(&v, a, dev) == cudaSuccess && v > 0) ? v : fallback;
        };
        const int m = attr(cudaDevAttrMultiProcessorCount, 148);
        const int smem_sm = attr(cudaDevAttrMaxSharedMemoryPerMultiprocessor, 233472);
        const int reserved = attr(cudaDevAttrReservedSharedMemoryPerBlock, 1024);
        const int regs_sm = attr(cudaDevAttrMaxRegistersPerMultiprocessor, 65536);
        const int threads_sm = attr(cudaDevAttrMaxThreadsPerMultiProcessor, 2048);
        const int blocks_sm = attr(cudaDevAttrMaxBlocksPerMultiprocessor, 32);
        const int regs_warp = ((fa.numRegs + 7) / 8) * 8 * 32;
        const int warps = kThreadsMlp / 32;
        int n = smem_sm / ((int)smem + fa.sharedSizeBytes + reserved);
        n = std::min(n, regs_sm / (regs_warp * warps));
        n = std::min(n, threads_sm / kThreadsMlp);
        n = std::min(n, blocks_sm);
        n = std::min(n, (int)(512u / tmem_cols<MODE>()));
        c_per_sm = n > 0 ? n : 1;
        c_sms = m;
        cached_dev = dev;
    }
    per_sm = c_per_sm;
    sms = c_sms;
    return SSMD_OK;
}

template <int MODE>
int launch(MlpArgs a, cudaStream_t st, int max_ctas = 0) {
    // training: one CTA per SM (its 256 TMEM columns and ~120 KB of shared memory)
    const size_t smem = MODE == kTrain ? (Layout<MODE>::bytes > (size_t)120 * 1024 ? Layout<MODE>::bytes
                                                                                     : (size_t)120 * 1024)
                                       : Layout<MODE>::bytes;
    int per_sm = 1, sms = 148;
    if (int e = launch_shape<MODE>(smem, per_sm, sms)) return e;
    const int64_t tiles = (a.n + kRows - 1) / kRows;
    int64_t slots = (int64_t)sms * per_sm;
    if (max_ctas > 0 && slots > max_ctas) slots = max_ctas;
    const unsigned blocks = (unsigned)(tiles < slots ? tiles : slots);
    mlp_kernel<MODE><<<blocks, kThreadsMlp, smem, st>>>(a);
    if (int e = cuda_check(cudaGetLastError(), "mlp launch")) return e;
    if (MODE == kTrain && a.partials) {
        grad_sum_kernel<<<(kParams + 1 + 255) / 256, 256, 0, st>>>(a.partials, (int)blocks, a.n, a.grad, a.loss);
        return cuda_check(cudaGetLastError(), "gradient sum launch");
    }
    return SSMD_OK;
}

} // namespace

extern "C" int ssmd_mlp_forward(const float *net, const float *features, int64_t n, float *out,
                                ssmd_stream_t stream) {
    if (!net || !features || !out || n < 0) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument or n < 0");
    if (n == 0) return SSMD_OK;
    if (n > (int64_t)0x7FFFFFFF * kRows) return fail(SSMD_ERR_INVALID_ARGUMENT, "too many rows");
    if ((reinterpret_cast<uintptr_t>(out) & 7u) != 0) return fail(SSMD_ERR_INVALID_ARGUMENT, "out must be 8-byte aligned");
    MlpArgs a{};
    a.net = net;
    a.feat = features;
    a.n = n;
    a.out = out;
    return launch<kFwd>(a, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ssmd_mlp_grad(const float *net, const float *features, const float *targets, const float *weights,
                             int64_t n, float *grad, double *loss, ssmd_stream_t stream) {
    if (!net || !features || !targets || !grad || !loss || n <= 0)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument or n <= 0");
    if (n > (int64_t)0x7FFFFFFF * kRows) return fail(SSMD_ERR_INVALID_ARGUMENT, "too many rows");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int e = cuda_check(cudaMemsetAsync(grad, 0, sizeof(float) * kParams, st), "grad clear")) return e;
    if (int e = cuda_check(cudaMemsetAsync(loss, 0, sizeof(double), st), "loss clear")) return e;
    MlpArgs a{};
    a.net = net;
    a.feat = features;
    a.target = targets;
    a.weight = weights;
    a.n = n;
    a.grad = grad;
    a.loss = loss;
    return launch<kTrain>(a, st);
}

extern "C" size_t ssmd_mlp_grad_workspace_bytes(void) {
    return sizeof(float) * (size_t)kMaxGradCtas * (kParams + 1);
}

extern "C" int ssmd_mlp_grad_ws(const float *net, const float *features, const float *targets, const float *weights,
                                int64_t n, float *grad, double *loss, float *workspace, size_t workspace_bytes,
                                ssmd_stream_t stream) {
    if (!net || !features || !targets || !grad || !loss || !workspace || n <= 0)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument or n <= 0");
    if (n > (int64_t)0x7FFFFFFF * kRows) return fail(SSMD_ERR_INVALID_ARGUMENT, "too many rows");
    if (workspace_bytes < ssmd_mlp_grad_workspace_bytes())
        return fail(SSMD_ERR_INVALID_ARGUMENT, "workspace_bytes %zu < required %zu", workspace_bytes,
                    ssmd_mlp_grad_workspace_bytes());
    MlpArgs a{};
    a.net = net;
    a.feat = features;
    a.target = targets;
    a.weight = weights;
    a.n = n;
    a.grad = grad;
    a.loss = loss;
    a.partials = workspace;
    return launch<kTrain>(a, reinterpret_cast<cudaStream_t>(stream), kMaxGradCtas);
}

extern "C" int ssmd_closure_refresh(const ssmd_params *coarse, const LBMFields *fields, const float *net,
                                    float nut_max, float *nut, float *sigma_scale, ssmd_stream_t stream) {
    if (int e = ssmd_validate(coarse)) return e;
    if (!fields || !fields->rho || !fields->ux || !fields->uy || !fields->uz || !fields->phi || !net || !nut ||
        !sigma_scale)
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    MlpArgs a{};
    a.net = net;
    a.n = (int64_t)coarse->nx * coarse->ny * coarse->nz;
    a.g = closure::grid_of(*coarse);
    a.rho = fields->rho;
    a.ux = fields->ux;
    a.uy = fields->uy;
    a.uz = fields->uz;
    a.phi = fields->phi;
    a.nu_w = coarse->nu_water;
    a.nu_dow = coarse->nu_oil - coarse->nu_water;
    a.nut_max = nut_max;
    a.nut = nut;
    a.cs = sigma_scale;
    return launch<kRefresh>(a, reinterpret_cast<cudaStream_t>(stream));
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

extern "C" int ssmd_mlp_average(float *avg, const float *net, float decay, ssmd_stream_t stream) {
    if (!avg || !net || !(decay >= 0.0f && decay <= 1.0f))
        return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument or decay outside [0, 1]");
    average_kernel<<<(kParams + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(avg, net, kParams,
                                                                                              decay);
    return cuda_check(cudaGetLastError(), "average launch");
}

extern "C" int ssmd_mlp_status(uint32_t *status) {
    if (!status) return fail(SSMD_ERR_INVALID_ARGUMENT, "null argument");
    unsigned int v = 0;
    if (int e = cuda_check(cudaMemcpyFromSymbol(&v, g_mlp_status, sizeof v), "mlp status")) return e;
    *status = v;
    return SSMD_OK;
}
