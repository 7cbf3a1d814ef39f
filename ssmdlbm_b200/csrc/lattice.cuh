// lattice.cuh — velocity sets and the per-cell regularized collision.
//
// Direction order is the reference's (src/velocitySet/D3Q19.cuh:82-131,
// D3Q27.cuh:91-140, D3Q7.cuh:73-122): q = 0 is rest and q = 2k-1, 2k are
// opposite directions.  That order is part of the population data format
// (LBMFields.f is [q][cell]), so it is kept.
//
// D3Q19 arithmetic is organised by opposite pairs: for c and -c the
// equilibrium, regularized non-equilibrium and Guo forcing terms split into an
// even part E (shared) and an odd part O, and f(+c) = w (E + O),
// f(-c) = w (E - O).  D3Q27, the tensor product of three 3-point axes, is
// evaluated by axis sweeps instead (raw moments by 3-point sums and
// differences, populations from the polynomial coefficients of the collision
// in c).  Moments use closed forms of sum_q f_eq c c and sum_q F_q c c
// (4th-order isotropy of D3Q19/D3Q27), which equal the reference's
// per-direction sums (src/lbm.cu:91-120) exactly in real arithmetic.
#pragma once

#include <cstdint>
#include <utility>

namespace ssmd {

// Reciprocal and square root on the SFU (rcp.approx / sqrt.approx: at most 1
// ulp / 2^-23 relative error, subnormal inputs and results flushed to 0).
// The reference divides with IEEE rounding; the step stays within FP32
// rounding of it (the parity tests hold 1e-5 after 100 steps against its own
// kernels), and the correctly rounded forms cost 6-8 more instructions each,
// three to four times per cell: 1.8-6 % of the bulk kernel's time on B200.
__device__ __forceinline__ float rcp_sfu(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sqrt_sfu(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

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

// D3Q27 index of the velocity (cx, cy, cz).
__host__ __device__ constexpr int q27(int cx, int cy, int cz) {
    for (int q = 0; q < 27; ++q)
        if (cx27(q) == cx && cy27(q) == cy && cz27(q) == cz) return q;
    return -1;
}

// One-axis D3Q27 weight factor: w_q = w1(cx) w1(cy) w1(cz).
__host__ __device__ constexpr double w1d(int c) { return c == 0 ? 2.0 / 3.0 : 1.0 / 6.0; }

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
    if constexpr (Q == 27) {
        // D3Q27 is the tensor product of three 3-point axes: the raw moments
        // sum_q f c_x^a c_y^b c_z^c (a + b + c <= 2) follow from three sweeps of
        // 3-point sums (0th moment), differences (1st) and outer sums (2nd).
        float X0[3][3], X1[3][3], X2[3][3]; // x sweep, [cy + 1][cz + 1]
        unroll<0, 9>([&](auto l) {
            constexpr int cy = l % 3 - 1, cz = l / 3 - 1;
            const float fm = f[q27(-1, cy, cz)], f0 = f[q27(0, cy, cz)], fp = f[q27(1, cy, cz)];
            X2[cy + 1][cz + 1] = fp + fm;
            X1[cy + 1][cz + 1] = fp - fm;
            X0[cy + 1][cz + 1] = X2[cy + 1][cz + 1] + f0;
        });
        float Y00[3], Y01[3], Y02[3], Y10[3], Y11[3], Y20[3]; // y sweep, [cz + 1]
        unroll<0, 3>([&](auto c) {
            Y02[c] = X0[2][c] + X0[0][c];
            Y00[c] = Y02[c] + X0[1][c];
            Y01[c] = X0[2][c] - X0[0][c];
            Y10[c] = (X1[2][c] + X1[0][c]) + X1[1][c];
            Y11[c] = X1[2][c] - X1[0][c];
            Y20[c] = (X2[2][c] + X2[0][c]) + X2[1][c];
        });
        szz = Y00[2] + Y00[0];
        s = szz + Y00[1];
        jz = Y00[2] - Y00[0];
        jy = (Y01[2] + Y01[0]) + Y01[1];
        syz = Y01[2] - Y01[0];
        syy = (Y02[2] + Y02[0]) + Y02[1];
        jx = (Y10[2] + Y10[0]) + Y10[1];
        sxz = Y10[2] - Y10[0];
        sxy = (Y11[2] + Y11[0]) + Y11[1];
        sxx = (Y20[2] + Y20[0]) + Y20[1];
    } else {
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
    }
    Moments m;
    m.rho = s + 1.0f;
    const float inv = rcp_sfu(m.rho);
    const float hinv = 0.5f * inv;
    m.ux = fmaf(jx, inv, fx * hinv);
    m.uy = fmaf(jy, inv, fy * hinv);
    m.uz = fmaf(jz, inv, fz * hinv);
    // T = sum f c c - rho u u + (u F + F u)/2; the (rho - 1) cs2 delta term
    // of sum f_eq c c drops out of the traceless part.  (Here and below every
    // multiply-add is written as an explicit fma, so that each instantiation
    // of this code rounds alike.)
    const float nrux = -m.rho * m.ux, nruy = -m.rho * m.uy;
    const float txx = fmaf(m.ux, fx, fmaf(nrux, m.ux, sxx));
    const float tyy = fmaf(m.uy, fy, fmaf(nruy, m.uy, syy));
    const float tzz = fmaf(m.uz, fz, fmaf(-m.rho * m.uz, m.uz, szz));
    m.pxy = fmaf(0.5f, fmaf(m.ux, fy, m.uy * fx), fmaf(nrux, m.uy, sxy));
    m.pxz = fmaf(0.5f, fmaf(m.ux, fz, m.uz * fx), fmaf(nrux, m.uz, sxz));
    m.pyz = fmaf(0.5f, fmaf(m.uy, fz, m.uz * fy), fmaf(nruy, m.uz, syz));
    const float tr = (txx + tyy + tzz) * kCs2;
    m.pxx = txx - tr;
    m.pyy = tyy - tr;
    m.pzz = tzz - tr;
    return m;
}

// D3Q27 collide(): the post-collision populations evaluated as a polynomial in the
// velocity components.  f_q - w_q = w_q P(c_q) with
//   P(c) = sum_{a,b,c <= 2} p_abc c_x^a c_y^b c_z^c
// (c_i^3 = c_i on the lattice), whose 17 nonzero coefficients collect the
// equilibrium, the regularized 2nd- and 3rd-order non-equilibrium parts and
// the Guo term of collide() below; the 27 values then follow from three
// 3-point sweeps along z, y and x, the product weights w1(c_x) w1(c_y) w1(c_z)
// folded into the last one.
__device__ __forceinline__ void collide27_tensor(const Moments &m, float omco, float fx, float fy, float fz,
                                                 float (&out)[27]) {
    const float ux = m.ux, uy = m.uy, uz = m.uz, rho = m.rho;
    const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    const float uu = 1.5f * (ux2 + uy2 + uz2);
    const float uF = fmaf(ux, fx, fmaf(uy, fy, uz * fz));
    const float trP = m.pxx + m.pyy + m.pzz; // ~0, kept for fidelity
    const float k45 = 4.5f * omco, k3 = 3.0f * k45;
    const float rux = rho * ux, ruy = rho * uy, ruz = rho * uz;
    // 3rd-order Hermite coefficients of u (x) Pi (D3Q27.cuh:178-184)
    const float axxy = fmaf(m.pxx, uy, 2.0f * ux * m.pxy);
    const float axxz = fmaf(m.pxx, uz, 2.0f * ux * m.pxz);
    const float ayyx = fmaf(m.pyy, ux, 2.0f * uy * m.pxy);
    const float ayyz = fmaf(m.pyy, uz, 2.0f * uy * m.pyz);
    const float azzx = fmaf(m.pzz, ux, 2.0f * uz * m.pxz);
    const float azzy = fmaf(m.pzz, uy, 2.0f * uz * m.pyz);
    const float axyz = fmaf(ux, m.pyz, fmaf(uy, m.pxz, uz * m.pxy));
    // coefficients: constant, linear (equilibrium + Guo + the linear parts of
    // the cubic terms), quadratic, mixed quadratic, cubic
    const float p000 = fmaf(rho, 1.0f - uu, -1.0f) - fmaf(1.5f, uF, k45 * kCs2 * trP);
    const float p100 = fmaf(3.0f, rux, 1.5f * fx) - fmaf(4.5f * rux, uy2 + uz2, k45 * (ayyx + azzx));
    const float p010 = fmaf(3.0f, ruy, 1.5f * fy) - fmaf(4.5f * ruy, ux2 + uz2, k45 * (axxy + azzy));
    const float p001 = fmaf(3.0f, ruz, 1.5f * fz) - fmaf(4.5f * ruz, ux2 + uy2, k45 * (axxz + ayyz));
    const float p200 = fmaf(4.5f * ux, rux + fx, k45 * m.pxx);
    const float p020 = fmaf(4.5f * uy, ruy + fy, k45 * m.pyy);
    const float p002 = fmaf(4.5f * uz, ruz + fz, k45 * m.pzz);
    const float p110 = fmaf(9.0f * rux, uy, fmaf(2.0f * k45, m.pxy, 4.5f * fmaf(ux, fy, uy * fx)));
    const float p101 = fmaf(9.0f * rux, uz, fmaf(2.0f * k45, m.pxz, 4.5f * fmaf(ux, fz, uz * fx)));
    const float p011 = fmaf(9.0f * ruy, uz, fmaf(2.0f * k45, m.pyz, 4.5f * fmaf(uy, fz, uz * fy)));
    const float p210 = fmaf(13.5f * rux * ux, uy, k3 * axxy); // c_x^2 c_y
    const float p201 = fmaf(13.5f * rux * ux, uz, k3 * axxz); // c_x^2 c_z
    const float p120 = fmaf(13.5f * ruy * uy, ux, k3 * ayyx); // c_x c_y^2
    const float p021 = fmaf(13.5f * ruy * uy, uz, k3 * ayyz); // c_y^2 c_z
    const float p102 = fmaf(13.5f * ruz * uz, ux, k3 * azzx); // c_x c_z^2
    const float p012 = fmaf(13.5f * ruz * uz, uy, k3 * azzy); // c_y c_z^2
    const float p111 = fmaf(27.0f * rux * uy, uz, 2.0f * k3 * axyz);

    // z sweep: L_ab(cz) = sum_c p_abc cz^c, [cz + 1]
    float L00[3], L10[3], L01[3], L20[3], L02[3], L11[3];
    auto line3 = [](float c0, float c1, float c2, float (&L)[3]) {
        const float e = c0 + c2;
        L[0] = e - c1;
        L[1] = c0;
        L[2] = e + c1;
    };
    auto line2 = [](float c0, float c1, float (&L)[3]) {
        L[0] = c0 - c1;
        L[1] = c0;
        L[2] = c0 + c1;
    };
    line3(p000, p001, p002, L00);
    line3(p100, p101, p102, L10);
    line3(p010, p011, p012, L01);
    line2(p200, p201, L20);
    line2(p020, p021, L02);
    line2(p110, p111, L11);
    // y sweep, then the x sweep with the weights
    unroll<0, 3>([&](auto zc) {
        constexpr int cz = zc - 1;
        float M0[3], M1[3], M2[3]; // [cy + 1]
        line3(L00[zc], L01[zc], L02[zc], M0);
        line3(L10[zc], L11[zc], p120, M1);
        line2(L20[zc], p210, M2);
        unroll<0, 3>([&](auto yc) {
            constexpr int cy = yc - 1;
            constexpr float W0 = float(w1d(0) * w1d(cy) * w1d(cz));
            constexpr float W1 = float(w1d(1) * w1d(cy) * w1d(cz));
            const float e = M0[yc] + M2[yc];
            const float t = W1 * M1[yc];
            out[q27(0, cy, cz)] = W0 * M0[yc];
            out[q27(1, cy, cz)] = fmaf(W1, e, t);
            out[q27(-1, cy, cz)] = fmaf(W1, e, -t);
        });
    });
}

// D3Q19 collide(), by opposite pairs.
__device__ __forceinline__ void collide19_pairs(const Moments &m, float omco, float fx, float fy, float fz,
                                                float (&out)[19]) {
    constexpr int Q = 19;
    const float ux = m.ux, uy = m.uy, uz = m.uz, rho = m.rho;
    const float uu = 1.5f * fmaf(ux, ux, fmaf(uy, uy, uz * uz));
    const float uF = fmaf(ux, fx, fmaf(uy, fy, uz * fz));
    const float trP = m.pxx + m.pyy + m.pzz; // ~0, kept for fidelity
    const float k45 = 4.5f * omco;
    // part shared by every direction
    const float A0 = fmaf(rho, 1.0f - uu, -1.0f) - fmaf(1.5f, uF, k45 * kCs2 * trP);
    out[0] = VS<Q>::w(0) * A0;
    const float hrho = 0.5f * rho;

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
        if constexpr (cx * cy != 0) pcc = fmaf(cx * cy > 0 ? 2.0f : -2.0f, m.pxy, pcc);
        if constexpr (cx * cz != 0) pcc = fmaf(cx * cz > 0 ? 2.0f : -2.0f, m.pxz, pcc);
        if constexpr (cy * cz != 0) pcc = fmaf(cy * cz > 0 ? 2.0f : -2.0f, m.pyz, pcc);
        const float cu3 = 3.0f * cu; // reference "cu" = as2 (c.u)
        const float cF15 = 1.5f * cF;
        // E = A0 + 0.5 rho cu3^2 + k45 pcc + 1.5 cu3 cF, O = rho cu3 + 1.5 cF
        const float E = fmaf(cu3, fmaf(hrho, cu3, cF15), fmaf(k45, pcc, A0));
        const float O = fmaf(rho, cu3, cF15);
        out[qp] = w * (E + O);
        out[qm] = w * (E - O);
    });
}

// Post-collision shifted populations:
//   f_q = f_eq(rho, u) + (1 - omega) f_neq^H(Pi, u) + F_q / 2
// with the 2nd-order (D3Q19) or 3rd-order (D3Q27) Hermite forms of the
// reference (D3Q19.cuh:133-177, D3Q27.cuh:147-201).  omco = 1 - omega.
template <int Q>
__device__ __forceinline__ void collide(const Moments &m, float omco, float fx, float fy, float fz,
                                        float (&out)[Q]) {
    if constexpr (Q == 27) collide27_tensor(m, omco, fx, fy, fz, out);
    else collide19_pairs(m, omco, fx, fy, fz, out);
}

} // namespace ssmd
