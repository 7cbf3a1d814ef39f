// lattice.cuh — velocity sets and the per-cell regularized collision.
//
// Direction order is the reference's (src/velocitySet/D3Q19.cuh:82-131,
// D3Q27.cuh:91-140, D3Q7.cuh:73-122): q = 0 is rest and q = 2k-1, 2k are
// opposite directions.  That order is part of the population data format
// (LBMFields.f is [q][cell]), so it is kept.
//
// The arithmetic is organised by opposite pairs: for c and -c the
// equilibrium, regularized non-equilibrium and Guo forcing terms split into an
// even part E (shared) and an odd part O, and f(+c) = w (E + O),
// f(-c) = w (E - O).  Moments use closed forms of sum_q f_eq c c and
// sum_q F_q c c (4th-order isotropy of D3Q19/D3Q27), which equal the
// reference's per-direction sums (src/lbm.cu:91-120) exactly in real
// arithmetic.
#pragma once

#include <cstdint>
#include <utility>

namespace ssmd {

template <int I>
using ic = std::integral_constant<int, I>;

// Compile-time unrolled loop: f(ic<B>{}), ..., f(ic<E-1>{}).
template <int B, int E, class F>
__host__ __device__ __forceinline__ void unroll(F &&f) {
    if constexpr (B < E) {
        f(ic<B>{});
        unroll<B + 1, E>(static_cast<F &&>(f));
    }
}

// ------------------------------------------------------------------ D3Q27
// (D3Q19 is its first 19 entries.)
__host__ __device__ constexpr int cx27(int q) {
    constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1,
                           1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
    return t[q];
}
__host__ __device__ constexpr int cy27(int q) {
    constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1,
                           0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
    return t[q];
}
__host__ __device__ constexpr int cz27(int q) {
    constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0,
                           -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
    return t[q];
}
// D3Q7 is the first 7 entries of the same table.

template <int Q>
struct VS;

template <>
struct VS<19> {
    static constexpr int Q = 19;
    __host__ __device__ static constexpr float w(int q) {
        return q == 0 ? float(1.0 / 3.0) : (q <= 6 ? float(1.0 / 18.0) : float(1.0 / 36.0));
    }
    // stencil weights used by the gradient / curvature operators
    static constexpr float w1 = float(1.0 / 18.0);
    static constexpr float w2 = float(1.0 / 36.0);
    static constexpr float w3 = 0.0f;
};

template <>
struct VS<27> {
    static constexpr int Q = 27;
    __host__ __device__ static constexpr float w(int q) {
        return q == 0 ? float(8.0 / 27.0)
                      : (q <= 6 ? float(2.0 / 27.0)
                                : (q <= 18 ? float(1.0 / 54.0) : float(1.0 / 216.0)));
    }
    static constexpr float w1 = float(2.0 / 27.0);
    static constexpr float w2 = float(1.0 / 54.0);
    static constexpr float w3 = float(1.0 / 216.0);
};

constexpr float kCs2 = float(1.0 / 3.0);
constexpr float kW7_0 = 0.25f;
constexpr float kW7_1 = 0.125f;

// Macroscopic state of one cell after the moment pass.
struct Moments {
    float rho, ux, uy, uz;
    float pxx, pyy, pzz, pxy, pxz, pyz; // traceless non-equilibrium stress
};

// rho, force-corrected u and traceless Pi_neq from shifted populations f - w
// (reference computeMoments, src/lbm.cu:46-127).
template <int Q>
__device__ __forceinline__ Moments moments(const float (&f)[Q], float fx, float fy, float fz) {
    float s = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
    float sxx = 0.f, syy = 0.f, szz = 0.f, sxy = 0.f, sxz = 0.f, syz = 0.f;
    s = f[0];
    unroll<0, (Q - 1) / 2>([&](auto k) {
        constexpr int qp = 2 * k + 1, qm = 2 * k + 2;
        constexpr int cx = cx27(qp), cy = cy27(qp), cz = cz27(qp);
        const float a = f[qp] + f[qm]; // even combination
        const float d = f[qp] - f[qm]; // odd combination
        s += a;
        if constexpr (cx != 0) jx += cx > 0 ? d : -d;
        if constexpr (cy != 0) jy += cy > 0 ? d : -d;
        if constexpr (cz != 0) jz += cz > 0 ? d : -d;
        if constexpr (cx != 0) sxx += a;
        if constexpr (cy != 0) syy += a;
        if constexpr (cz != 0) szz += a;
        if constexpr (cx * cy != 0) sxy += cx * cy > 0 ? a : -a;
        if constexpr (cx * cz != 0) sxz += cx * cz > 0 ? a : -a;
        if constexpr (cy * cz != 0) syz += cy * cz > 0 ? a : -a;
    });
    Moments m;
    m.rho = s + 1.0f;
    const float inv = __frcp_rn(m.rho); // = 1 / rho, correctly rounded
    const float hinv = 0.5f * inv;
    m.ux = jx * inv + fx * hinv;
    m.uy = jy * inv + fy * hinv;
    m.uz = jz * inv + fz * hinv;
    // T = sum f c c - rho u u + (u F + F u)/2; the (rho - 1) cs2 delta term
    // of sum f_eq c c drops out of the traceless part.
    const float txx = sxx - m.rho * m.ux * m.ux + m.ux * fx;
    const float tyy = syy - m.rho * m.uy * m.uy + m.uy * fy;
    const float tzz = szz - m.rho * m.uz * m.uz + m.uz * fz;
    m.pxy = sxy - m.rho * m.ux * m.uy + 0.5f * (m.ux * fy + m.uy * fx);
    m.pxz = sxz - m.rho * m.ux * m.uz + 0.5f * (m.ux * fz + m.uz * fx);
    m.pyz = syz - m.rho * m.uy * m.uz + 0.5f * (m.uy * fz + m.uz * fy);
    const float tr = (txx + tyy + tzz) * kCs2;
    m.pxx = txx - tr;
    m.pyy = tyy - tr;
    m.pzz = tzz - tr;
    return m;
}

// Post-collision shifted populations:
//   f_q = f_eq(rho, u) + (1 - omega) f_neq^H(Pi, u) + F_q / 2
// with the 2nd-order (D3Q19) or 3rd-order (D3Q27) Hermite forms of the
// reference (D3Q19.cuh:133-177, D3Q27.cuh:147-201).  omco = 1 - omega.
template <int Q>
__device__ __forceinline__ void collide(const Moments &m, float omco, float fx, float fy, float fz,
                                        float (&out)[Q]) {
    const float ux = m.ux, uy = m.uy, uz = m.uz, rho = m.rho;
    const float uu = 1.5f * (ux * ux + uy * uy + uz * uz);
    const float uF = ux * fx + uy * fy + uz * fz;
    const float trP = m.pxx + m.pyy + m.pzz; // ~0, kept for fidelity
    const float k45 = 4.5f * omco;
    // part shared by every direction
    const float A0 = rho * (1.0f - uu) - 1.0f - 1.5f * uF - k45 * kCs2 * trP;
    out[0] = VS<Q>::w(0) * A0;

    // 3rd-order Hermite coefficients of u (x) Pi (D3Q27.cuh:178-184)
    float axxy = 0.f, axxz = 0.f, ayyx = 0.f, ayyz = 0.f, azzx = 0.f, azzy = 0.f, axyz = 0.f;
    if constexpr (Q == 27) {
        axxy = m.pxx * uy + 2.0f * ux * m.pxy;
        axxz = m.pxx * uz + 2.0f * ux * m.pxz;
        ayyx = m.pyy * ux + 2.0f * uy * m.pxy;
        ayyz = m.pyy * uz + 2.0f * uy * m.pyz;
        azzx = m.pzz * ux + 2.0f * uz * m.pxz;
        azzy = m.pzz * uy + 2.0f * uz * m.pyz;
        axyz = ux * m.pyz + uy * m.pxz + uz * m.pxy;
    }

    unroll<0, (Q - 1) / 2>([&](auto k) {
        constexpr int qp = 2 * k + 1, qm = 2 * k + 2;
        constexpr int cx = cx27(qp), cy = cy27(qp), cz = cz27(qp);
        constexpr float w = VS<Q>::w(qp);
        // c.u and c.F with the constant c folded
        float cu = 0.f, cF = 0.f, pcc = 0.f;
        if constexpr (cx != 0) { cu += cx > 0 ? ux : -ux; cF += cx > 0 ? fx : -fx; }
        if constexpr (cy != 0) { cu += cy > 0 ? uy : -uy; cF += cy > 0 ? fy : -fy; }
        if constexpr (cz != 0) { cu += cz > 0 ? uz : -uz; cF += cz > 0 ? fz : -fz; }
        // c c : Pi
        if constexpr (cx != 0) pcc += m.pxx;
        if constexpr (cy != 0) pcc += m.pyy;
        if constexpr (cz != 0) pcc += m.pzz;
        if constexpr (cx * cy != 0) pcc += (cx * cy > 0 ? 2.0f : -2.0f) * m.pxy;
        if constexpr (cx * cz != 0) pcc += (cx * cz > 0 ? 2.0f : -2.0f) * m.pxz;
        if constexpr (cy * cz != 0) pcc += (cy * cz > 0 ? 2.0f : -2.0f) * m.pyz;
        const float cu3 = 3.0f * cu; // reference "cu" = as2 (c.u)
        float E = A0 + 0.5f * rho * cu3 * cu3 + k45 * pcc + 1.5f * cu3 * cF;
        float O = rho * cu3 + 1.5f * cF;
        if constexpr (Q == 27) {
            O += rho * (cu3 * cu3 * cu3 * float(1.0 / 6.0) - uu * cu3);
            float h3 = 0.f;
            constexpr float t = 1.0f / 3.0f;
            // (cx^2 cy - cy/3) etc., constant-folded per direction
            constexpr float cxxy = float(cx * cx * cy) - float(cy) * t;
            constexpr float cxxz = float(cx * cx * cz) - float(cz) * t;
            constexpr float cyyx = float(cx * cy * cy) - float(cx) * t;
            constexpr float cyyz = float(cy * cy * cz) - float(cz) * t;
            constexpr float czzx = float(cx * cz * cz) - float(cx) * t;
            constexpr float czzy = float(cy * cz * cz) - float(cy) * t;
            constexpr float cxyz = float(cx * cy * cz);
            if constexpr (cxxy != 0.f) h3 += cxxy * axxy;
            if constexpr (cxxz != 0.f) h3 += cxxz * axxz;
            if constexpr (cyyx != 0.f) h3 += cyyx * ayyx;
            if constexpr (cyyz != 0.f) h3 += cyyz * ayyz;
            if constexpr (czzx != 0.f) h3 += czzx * azzx;
            if constexpr (czzy != 0.f) h3 += czzy * azzy;
            float odd3 = 3.0f * h3;
            if constexpr (cxyz != 0.f) odd3 += 6.0f * cxyz * axyz;
            O += k45 * odd3;
        }
        out[qp] = w * (E + O);
        out[qm] = w * (E - O);
    });
}

} // namespace ssmd
