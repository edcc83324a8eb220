// Point physics of the SRHD update, templated on the arithmetic type.
//
// Each function follows Wesenheit/Verona's Julia source (file:line cited) in
// the same evaluation order: a + b + c is (a + b) + c, x^2 is x*x, x^3 is
// x*x*x, min/max propagate NaN, and only the explicit fma() calls of
// src/2dim/structs.jl:192,205,212 are fused. The FP64 translation unit is
// compiled with -fmad=false, so for T = double every result is bit-identical
// to the reference's rounding (IEEE +,-,*,/,sqrt are correctly rounded on
// sm_100a). The FP32-bulk units use the same code with FP32 constants, except
// for the reconstructions, which have FP32 forms of their own (minmod32,
// ppm32, wenoz32: the same schemes with sign-bit tests, shared differences
// and approximate reciprocals).
#pragma once
#include "vb_ns.h"
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#define VB_HD __host__ __device__ __forceinline__

namespace VB_NS {

enum { REC_MINMOD = 0, REC_PPM = 1, REC_WENOZ = 2 };
enum { RS_HLL = 0, RS_HLLC = 1 };

template <typename T> VB_HD T sq(T x) { return x * x; }

// Base.max / Base.min for IEEE floats: NaN-propagating, +0 > -0.
template <typename T> VB_HD T jmax(T x, T y) {
    T d = x - y;
    if (isnan(x) || isnan(y)) return d;
    return signbit(d) ? y : x;
}
template <typename T> VB_HD T jmin(T x, T y) {
    T d = x - y;
    if (isnan(x) || isnan(y)) return d;
    return signbit(d) ? x : y;
}
// Base.sign: +-1, keeps signed zero, NaN stays NaN.
template <typename T> VB_HD T jsign(T x) { return x > T(0) ? T(1) : (x < T(0) ? T(-1) : x); }

// FP64 a / b with a zero dividend kept out of the divide. Measured on B200,
// an FP64 divide of an exact zero costs several times a regular one (a WENOZ
// reconstruction of equal values took 1.5x, of zeros 1.8x, the time of one
// of varied values), and a static uniform region (v = 0, equal neighbours)
// puts exact zeros into every smoothness difference, velocity and flux of
// its cells. So the divide always receives a nonzero dividend (1 in place of
// a zero, passed through an opaque move that the compiler cannot fold back),
// with no branch around it, and the zero's quotient is formed from it:
//   qdiv:     a * (1 / b), the IEEE quotient of +-0 by any b (signed zero for
//             a finite nonzero or infinite b, NaN for a zero or NaN b), for
//             every b except a subnormal of magnitude at most 2^-1024,
//             whose reciprocal overflows (no divisor of this scheme comes
//             near one);
//   qdiv_pos: a itself, for a b that is positive (or +inf) whenever a is
//             zero, as the caller's algebra guarantees.
// Both are bit-identical to the correctly rounded divide on those domains.
// FP32 keeps the plain operation (its units divide approximately).
VB_HD double opaque(double x) {
#ifdef __CUDA_ARCH__
    asm("mov.f64 %0, %0;" : "+d"(x));
#endif
    return x;
}
template <typename T> VB_HD T qdiv(T a, T b) {
    if constexpr (sizeof(T) == 8) {
        const bool z = a == T(0);
        const T q = opaque(z ? T(1) : a) / b;
        return z ? a * q : q;
    }
    return a / b;
}
template <typename T> VB_HD T qdiv_pos(T a, T b) {
    if constexpr (sizeof(T) == 8) {
        const bool z = a == T(0);
        const T q = opaque(z ? T(1) : a) / b;
        return z ? a : q;
    }
    return a / b;
}
// sqrt(+-0) is the argument itself
template <typename T> VB_HD T qsqrt(T a) {
    if constexpr (sizeof(T) == 8) {
        if (a == T(0)) return a;
    }
    return sqrt(a);
}

// ---- reconstruction (src/fluxlimiter.jl) -----------------------------------
// Every limiter returns (qr_i, ql_ip1): the value of cell i at its left face
// i-1/2 and at its right face i+1/2.

// MINMOD, src/fluxlimiter.jl:1-13
template <typename T> VB_HD void minmod(T qm1, T q, T qp1, T& qr, T& ql) {
    T sp = qp1 - q;
    T sm = q - qm1;
    T ssp = jsign(sp), ssm = jsign(sm);
    T asp = fabs(sp), asm_ = fabs(sm);
    T dU = T(0.25) * (ssp + ssm) * jmin(asp, asm_);
    qr = q - dU;
    ql = q + dU;
}

// WENO-Z epsilon. The reference's 1e-42 is subnormal in FP32 and would
// overflow tau/eps; the FP32 form uses a normal epsilon and caps the
// smoothness indicator (a documented precision-policy choice).
template <typename T> struct WenoEps;
template <> struct WenoEps<double> {
    static VB_HD double eps() { return 1.0e-42; }
    static VB_HD double cap(double x) { return x; }
};
template <> struct WenoEps<float> {
    static VB_HD float eps() { return 1.0e-30f; }
    static VB_HD float cap(float x) { return fminf(x, 1.0e15f); }
};

// WENOZ, src/fluxlimiter.jl:19-71
template <typename T>
VB_HD void wenoz(T q_im2, T q_im1, T q_i, T q_ip1, T q_ip2, T& qr_i, T& ql_ip1) {
    const T c1 = T(13.0) / T(12.0), c2 = T(0.25);
    T b1 = c1 * sq(q_im2 + q_i - T(2) * q_im1) + c2 * sq(q_im2 + T(3) * q_i - T(4) * q_im1);
    T b2 = c1 * sq(q_im1 + q_ip1 - T(2) * q_i) + c2 * sq(q_im1 - q_ip1);
    T b3 = c1 * sq(q_ip2 + q_i - T(2) * q_ip1) + c2 * sq(q_ip2 + T(3) * q_i - T(4) * q_ip1);
    const T epsL = WenoEps<T>::eps();
    T tau5 = fabs(b1 - b3);
    T i1, i2, i3;
    if constexpr (sizeof(T) == 8) {
        // tau5 = 0 (equal smoothness on both sides, every uniform region):
        // each ratio is +0, as b_k + eps > 0 (b_k >= 0 is finite or +inf there)
        const bool z = tau5 == T(0);
        const T tn = opaque(z ? T(1) : tau5);
        const T q1 = tn / (b1 + epsL), q2 = tn / (b2 + epsL), q3 = tn / (b3 + epsL);
        i1 = z ? tau5 : q1;
        i2 = z ? tau5 : q2;
        i3 = z ? tau5 : q3;
    } else {
        i1 = WenoEps<T>::cap(tau5 / (b1 + epsL));
        i2 = WenoEps<T>::cap(tau5 / (b2 + epsL));
        i3 = WenoEps<T>::cap(tau5 / (b3 + epsL));
    }

    T f1 = T(2) * q_im2 - T(7) * q_im1 + T(11) * q_i;
    T f2 = -q_im1 + T(5) * q_i + T(2) * q_ip1;
    T f3 = T(2) * q_i + T(5) * q_ip1 - q_ip2;
    T a1 = T(0.1) * (T(1) + sq(i1)), a2 = T(0.6) * (T(1) + sq(i2)), a3 = T(0.3) * (T(1) + sq(i3));
    T asum = T(6) * (a1 + a2 + a3);
    ql_ip1 = qdiv_pos(f1 * a1 + f2 * a2 + f3 * a3, asum);  // asum >= 6

    f1 = T(2) * q_ip2 - T(7) * q_ip1 + T(11) * q_i;
    f2 = -q_ip1 + T(5) * q_i + T(2) * q_im1;
    f3 = T(2) * q_i + T(5) * q_im1 - q_im2;
    a1 = T(0.1) * (T(1) + sq(i3));
    a2 = T(0.6) * (T(1) + sq(i2));
    a3 = T(0.3) * (T(1) + sq(i1));
    asum = T(6) * (a1 + a2 + a3);
    qr_i = qdiv_pos(f1 * a1 + f2 * a2 + f3 * a3, asum);
}

// PPM, src/fluxlimiter.jl:74-180
template <typename T>
VB_HD void ppm(T q_im2, T q_im1, T q_i, T q_ip1, T q_ip2, T& qr_out, T& ql_out) {
    const T C2 = T(1.25);
    T qa = q_i - q_im1;
    T qb = q_ip1 - q_i;
    T dd_im1 = T(0.5) * qa + T(0.5) * (q_im1 - q_im2);
    T dd = T(0.5) * qb + T(0.5) * qa;
    T dd_ip1 = T(0.5) * (q_ip2 - q_ip1) + T(0.5) * qb;

    T dph = T(0.5) * (q_im1 + q_i) + qdiv_pos(dd_im1 - dd, T(6));
    T dph_ip1 = T(0.5) * (q_i + q_ip1) + qdiv_pos(dd - dd_ip1, T(6));

    T d2qc_im1 = q_im2 + q_i - T(2) * q_im1;
    T d2qc = q_im1 + q_ip1 - T(2) * q_i;
    T d2qc_ip1 = q_i + q_ip2 - T(2) * q_ip1;

    T qa_tmp = dph - q_im1;
    T qb_tmp = q_i - dph;
    qa = T(3) * (q_im1 + q_i - T(2) * dph);
    qb = d2qc_im1;
    T qc = d2qc;
    T qd = T(0);
    if (jsign(qa) == jsign(qb) && jsign(qa) == jsign(qc))
        qd = jsign(qa) * jmin(C2 * fabs(qb), jmin(C2 * fabs(qc), fabs(qa)));
    T dph_tmp = T(0.5) * (q_im1 + q_i) - qdiv_pos(qd, T(6));
    if (qa_tmp * qb_tmp < T(0)) dph = dph_tmp;

    qa_tmp = dph_ip1 - q_i;
    qb_tmp = q_ip1 - dph_ip1;
    qa = T(3) * (q_i + q_ip1 - T(2) * dph_ip1);
    qb = d2qc;
    qc = d2qc_ip1;
    qd = T(0);
    if (jsign(qa) == jsign(qb) && jsign(qa) == jsign(qc))
        qd = jsign(qa) * jmin(C2 * fabs(qb), jmin(C2 * fabs(qc), fabs(qa)));
    T dphip1_tmp = T(0.5) * (q_i + q_ip1) - qdiv_pos(qd, T(6));
    if (qa_tmp * qb_tmp < T(0)) dph_ip1 = dphip1_tmp;

    T d2qf = T(6) * (dph + dph_ip1 - T(2) * q_i);
    T qr_i = dph;
    T ql_ip1 = dph_ip1;
    T dqf_minus = q_i - qr_i;
    T dqf_plus = ql_ip1 - q_i;

    qa_tmp = dqf_minus * dqf_plus;
    qb_tmp = (q_ip1 - q_i) * (q_i - q_im1);
    qa = d2qc_im1;
    qb = d2qc;
    qc = d2qc_ip1;
    qd = d2qf;
    T qe = T(0);
    if (jsign(qa) == jsign(qb) && jsign(qa) == jsign(qc) && jsign(qa) == jsign(qd))
        qe = jsign(qd) * jmin(jmin(C2 * fabs(qa), C2 * fabs(qb)), jmin(C2 * fabs(qc), fabs(qd)));

    qa = jmax(T(fabs(q_im1)), T(fabs(q_im2)));
    qb = jmax(jmax(T(fabs(q_i)), T(fabs(q_ip1))), T(fabs(q_ip2)));
    T rho = T(0);
    if (fabs(qd) > T(1.0e-12) * jmax(qa, qb)) rho = qe / qd;

    T tmp_m = q_i - rho * dqf_minus;
    T tmp_p = q_i + rho * dqf_plus;
    T tmp2_m = q_i - T(2) * dqf_plus;
    T tmp2_p = q_i + T(2) * dqf_minus;
    if (qa_tmp <= T(0) || qb_tmp <= T(0)) {
        if (rho <= T(1) - T(1.0e-12)) {
            qr_i = tmp_m;
            ql_ip1 = tmp_p;
        }
    } else {
        if (fabs(dqf_minus) >= T(2) * fabs(dqf_plus)) qr_i = tmp2_m;
        if (fabs(dqf_plus) >= T(2) * fabs(dqf_minus)) ql_ip1 = tmp2_p;
    }
    qr_out = qr_i;
    ql_out = ql_ip1;
}

// ---- FP32 forms of MINMOD and PPM --------------------------------------------
// The FP32-bulk kernels test signs by their sign bits with integer operations
// instead of the reference's three-valued sign(): where an operand is zero
// the reference's result is 0 and the minimum that the test selects is that
// zero too, so the values differ only for NaN operands (a NaN state).
VB_HD int f32_bits(float x) {
#ifdef __CUDA_ARCH__
    return __float_as_int(x);
#else
    int i;
    memcpy(&i, &x, 4);
    return i;
#endif
}
VB_HD bool same_sign3(float a, float b, float c) {
    const int ia = f32_bits(a);
    return ((ia ^ f32_bits(b)) | (ia ^ f32_bits(c))) >= 0;
}
// NaN-propagating minimum (Julia's min on floats)
VB_HD float fmin_nan(float a, float b) {
#ifdef __CUDA_ARCH__
    float r;
    asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
#else
    return (a != a || b != b) ? a + b : fminf(a, b);
#endif
}
VB_HD void minmod32(float qm1, float q, float qp1, float& qr, float& ql) {
    const float sp = qp1 - q, sm = q - qm1;
    const float du = same_sign3(sp, sm, sm) ? copysignf(0.5f * fmin_nan(fabsf(sp), fabsf(sm)), sp) : 0.0f;
    qr = q - du;
    ql = q + du;
}
VB_HD float ppm_limit32(float a, float b, float c) {  // sign(a) min(1.25|b|, 1.25|c|, |a|) or 0
    return same_sign3(a, b, c) ? copysignf(fmin_nan(1.25f * fabsf(b), fmin_nan(1.25f * fabsf(c), fabsf(a))), a)
                               : 0.0f;
}
VB_HD void ppm32(float qm2, float qm1, float q, float qp1, float qp2, float& qr_out, float& ql_out) {
    const float qa = q - qm1, qb = qp1 - q, sm = qm1 + q, sp = q + qp1;
    float dph = 0.5f * sm + (0.5f / 6.0f) * ((qm1 - qm2) - qb);
    float dphp = 0.5f * sp + (0.5f / 6.0f) * (qa - (qp2 - qp1));
    const float d2m = qm2 + q - 2.0f * qm1, d2c = qm1 + qp1 - 2.0f * q, d2p = q + qp2 - 2.0f * qp1;
    const float qdl = ppm_limit32(3.0f * (sm - 2.0f * dph), d2m, d2c);
    if ((dph - qm1) * (q - dph) < 0.0f) dph = 0.5f * sm - qdl * (1.0f / 6.0f);
    const float qdr = ppm_limit32(3.0f * (sp - 2.0f * dphp), d2c, d2p);
    if ((dphp - q) * (qp1 - dphp) < 0.0f) dphp = 0.5f * sp - qdr * (1.0f / 6.0f);
    const float d2qf = 6.0f * (dph + dphp - 2.0f * q);
    const float dqm = q - dph, dqp = dphp - q;
    const bool same = same_sign3(d2m, d2c, d2p) && same_sign3(d2m, d2qf, d2qf);
    const float qe =
        same ? copysignf(fmin_nan(fmin_nan(1.25f * fabsf(d2m), 1.25f * fabsf(d2c)), fmin_nan(1.25f * fabsf(d2p), fabsf(d2qf))),
                         d2qf)
             : 0.0f;
    const float qmax = fmaxf(fmaxf(fabsf(qm1), fabsf(qm2)), fmaxf(fmaxf(fabsf(q), fabsf(qp1)), fabsf(qp2)));
    const float rho = fabsf(d2qf) > 1.0e-12f * qmax ? qe / d2qf : 0.0f;
    float qr = dph, ql = dphp;
    if (dqm * dqp <= 0.0f || qb * qa <= 0.0f) {
        if (rho <= 1.0f - 1.0e-12f) {
            qr = q - rho * dqm;
            ql = q + rho * dqp;
        }
    } else {
        if (fabsf(dqm) >= 2.0f * fabsf(dqp)) qr = q - 2.0f * dqp;
        if (fabsf(dqp) >= 2.0f * fabsf(dqm)) ql = q + 2.0f * dqm;
    }
    qr_out = qr;
    ql_out = ql;
}

// FP32 WENOZ on the one-sided differences D1..D4 of the five values, which
// the smoothness indicators and the three stencils share:
//   beta_k * 12/13 = t_k^2 + (3/13) u_k^2 (t: the second difference, u: the
//   one-sided combination of each sub-stencil); face value = q_i +
//   sum_k d_k s_k g_k / sum_k d_k s_k with g_k = f_k - q_i and
//   s_k = 1 + (tau5 / (beta_k + eps))^2, d = (0.1, 0.6, 0.3).
// The factor 13/12 cancels in tau5 / beta except against eps (1e-30); the
// smoothness ratio is capped at 1e9 so that the two faces' denominators
// (each <= 1e18) share one reciprocal of their product. Same scheme as the
// reference's WENOZ (src/fluxlimiter.jl:19-71), different FP32 rounding.
VB_HD float rcp32(float x) {
#ifdef __CUDA_ARCH__
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return 1.0f / x;
#endif
}
VB_HD void wenoz32(float qm2, float qm1, float q0, float qp1, float qp2, float& qr, float& ql) {
    const float D1 = qm1 - qm2, D2 = q0 - qm1, D3 = qp1 - q0, D4 = qp2 - qp1;
    const float r = 3.0f / 13.0f;
    float t = D2 - D1, u = fmaf(2.0f, D2, t);
    const float b1 = fmaf(r * u, u, t * t);
    t = D3 - D2;
    u = D2 + D3;
    const float b2 = fmaf(r * u, u, t * t);
    t = D4 - D3;
    u = fmaf(-2.0f, D3, t);
    const float b3 = fmaf(r * u, u, t * t);
    const float tau = fabsf(b1 - b3);
    const float i1 = fminf(tau * rcp32(b1 + 1.0e-30f), 1.0e9f);
    const float i2 = fminf(tau * rcp32(b2 + 1.0e-30f), 1.0e9f);
    const float i3 = fminf(tau * rcp32(b3 + 1.0e-30f), 1.0e9f);
    const float s1 = fmaf(i1, i1, 1.0f), s2 = fmaf(i2, i2, 1.0f), s3 = fmaf(i3, i3, 1.0f);
    const float numl = fmaf(s3, fmaf(1.2f / 6.0f, D3, (-0.3f / 6.0f) * D4),
                            fmaf(s2, fmaf(1.2f / 6.0f, D3, (0.6f / 6.0f) * D2), s1 * fmaf(0.5f / 6.0f, D2, (-0.2f / 6.0f) * D1)));
    const float denl = fmaf(0.3f, s3, fmaf(0.6f, s2, 0.1f * s1));
    const float numr = fmaf(s1, fmaf(-1.2f / 6.0f, D2, (0.3f / 6.0f) * D1),
                            fmaf(s2, fmaf(-1.2f / 6.0f, D2, (-0.6f / 6.0f) * D3), s3 * fmaf(0.2f / 6.0f, D4, (-0.5f / 6.0f) * D3)));
    const float denr = fmaf(0.3f, s1, fmaf(0.6f, s2, 0.1f * s3));
    const float rd = rcp32(denl * denr);
    ql = fmaf(numl * denr, rd, q0);
    qr = fmaf(numr * denl, rd, q0);
}

// reconstruction(::Val{M}, ...), src/fluxlimiter.jl:183-200; the FP32-bulk
// kernels take the FP32 forms of MINMOD, PPM and WENOZ above
template <int REC, typename T>
VB_HD void recon(T q_im2, T q_im1, T q_i, T q_ip1, T q_ip2, T& qr, T& ql) {
    if constexpr (sizeof(T) == 4 && REC == REC_MINMOD)
        minmod32(q_im1, q_i, q_ip1, qr, ql);
    else if constexpr (sizeof(T) == 4 && REC == REC_PPM)
        ppm32(q_im2, q_im1, q_i, q_ip1, q_ip2, qr, ql);
    else if constexpr (sizeof(T) == 4)
        wenoz32(q_im2, q_im1, q_i, q_ip1, q_ip2, qr, ql);
    else if constexpr (REC == REC_MINMOD)
        minmod(q_im1, q_i, q_ip1, qr, ql);
    else if constexpr (REC == REC_PPM)
        ppm(q_im2, q_im1, q_i, q_ip1, q_ip2, qr, ql);
    else
        wenoz(q_im2, q_im1, q_i, q_ip1, q_ip2, qr, ql);
}

// a[i] for a runtime axis i < N, as an unrolled select: the arrays of a face
// state stay in registers, and no access depends on a runtime index (a
// runtime-indexed local array read back a stale element in one kernel).
template <int N, typename T> VB_HD T pick(const T* a, int i) {
    T r = a[0];
#pragma unroll
    for (int k = 1; k < N; ++k)
        if (k == i) r = a[k];
    return r;
}

// ---- EOS and state conversions ---------------------------------------------
// SoundSpeed, src/eos.jl:15-21
template <typename T> VB_HD T sound_speed(T rho, T u, T g) {
    return sqrt((g * (g - T(1)) * u) / (rho + g * u));
}

// gam = sqrt(ux^2 + uy^2 + uz^2 + 1), src/3dim/structs.jl:89
template <int DIM, typename T> VB_HD T lorentz(const T* P) {
    T s = sq(P[2]);
    if (DIM > 1) s = s + sq(P[3]);
    if (DIM > 2) s = s + sq(P[4]);
    return sqrt(s + T(1));
}

// function_PtoU, src/3dim/structs.jl:84-96 (2D: src/2dim/structs.jl:87-98)
template <int DIM, typename T> VB_HD void prim2con(T g, const T* P, T* U) {
    T gam = lorentz<DIM>(P);
    T w = g * P[1] + P[0];
    U[0] = gam * P[0];
    U[1] = (g - T(1)) * P[1] - sq(gam) * w;
#pragma unroll
    for (int m = 0; m < DIM; ++m) U[2 + m] = P[2 + m] * gam * w;
}

// function_PtoFx/Fy/Fz, src/3dim/structs.jl:99-142
template <int DIM, typename T> VB_HD void prim2flux(int d, T g, const T* P, T* F) {
    T gam = lorentz<DIM>(P);
    T w = g * P[1] + P[0];
    T un = pick<DIM>(P + 2, d);
    F[0] = P[0] * un;
    F[1] = -w * un * gam;
#pragma unroll
    for (int m = 0; m < DIM; ++m) {
        if (m == d)
            F[2 + m] = sq(un) * w + (g - T(1)) * P[1];
        else
            F[2 + m] = P[2 + m] * un * w;
    }
}

// HARM signal speeds of one state, src/3dim/algos.jl:130-157
template <int DIM, typename T> VB_HD void harm_speeds(int d, T g, const T* P, T& lp, T& lm) {
    T lor = lorentz<DIM>(P);
    T v = qdiv(pick<DIM>(P + 2, d), lor);
    T C = sound_speed(P[0], P[1], g);
    T sig = sq(C) / (sq(lor) * (T(1) - sq(C)));
    T r = sqrt(sig * (T(1) - sq(v) + sig));
    lp = (v + r) / (T(1) + sig);
    lm = (v - r) / (T(1) + sig);
}

// Everything the Riemann solvers need from one face state, computed once:
// conserved vector and flux along d (function_PtoU / function_PtoFx..z),
// Lorentz factor, normal velocity, pressure and the HARM signal speeds
// (src/3dim/algos.jl:117-157). Same expressions as the separate functions
// above, so the values are identical.
template <int DIM, typename T> struct FaceState {
    static constexpr int NV = 2 + DIM;
    T U[NV], F[NV];
    T vn, p, lp, lm;
    VB_HD void make(int d, T g, const T* P) {
        T gam = lorentz<DIM>(P);
        T w = g * P[1] + P[0];
        T un = pick<DIM>(P + 2, d);
        U[0] = gam * P[0];
        U[1] = (g - T(1)) * P[1] - sq(gam) * w;
        F[0] = P[0] * un;
        F[1] = -w * un * gam;
#pragma unroll
        for (int m = 0; m < DIM; ++m) {
            U[2 + m] = P[2 + m] * gam * w;
            if (m == d)
                F[2 + m] = sq(un) * w + (g - T(1)) * P[1];
            else
                F[2 + m] = P[2 + m] * un * w;
        }
        vn = qdiv(un, gam);
        p = (g - T(1)) * P[1];
        T C = sound_speed(P[0], P[1], g);
        T sig = sq(C) / (sq(gam) * (T(1) - sq(C)));
        T r = sqrt(sig * (T(1) - sq(vn) + sig));
        lp = (vn + r) / (T(1) + sig);
        lm = (vn - r) / (T(1) + sig);
    }
};

// HLL face flux, src/3dim/algos.jl:117-174 (states already floored)
template <int DIM, typename T>
VB_HD void hll_flux(int d, T g, const T* PL, const T* PR, T* Fo) {
    constexpr int NV = 2 + DIM;
    FaceState<DIM, T> R, L;
    R.make(d, g, PR);
    L.make(d, g, PL);
    T Cmax = jmax(L.lp, R.lp);
    T Cmin = -jmin(L.lm, R.lm);
    if (Cmax < T(0)) {
#pragma unroll
        for (int v = 0; v < NV; ++v) Fo[v] = R.F[v];
    } else if (Cmin < T(0)) {
#pragma unroll
        for (int v = 0; v < NV; ++v) Fo[v] = L.F[v];
    } else {
#pragma unroll
        for (int v = 0; v < NV; ++v)
            Fo[v] = qdiv(R.F[v] * Cmin + L.F[v] * Cmax - Cmax * Cmin * (R.U[v] - L.U[v]), Cmax + Cmin);
    }
}

// HLLC face flux: an extension (the reference is HLL only). Mignone & Bodo
// (2005, MNRAS 364, 126) relativistic HLLC with the HARM/Davis speed bounds
// of the HLL above, falling back to HLL where the star state is unphysical.
// Verona's conserved vector is (D, -E, m) and its flux (D v_n, -m_n, m v_n + p e_n).
template <int DIM, typename T>
VB_HD void hllc_flux(int d, T g, const T* PL, const T* PR, T* Fo) {
    // Branch-free: the HLL flux and the star-state flux are both formed and
    // the result is selected once at the end, with the same conditions (and
    // therefore the same values) as the early-return form of the oracle.
    constexpr int NV = 2 + DIM;
    FaceState<DIM, T> R, L;
    R.make(d, g, PR);
    L.make(d, g, PL);
    const T Cmax = jmax(L.lp, R.lp);
    const T Cmin = -jmin(L.lm, R.lm);
    T Fh[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v)
        Fh[v] = qdiv(R.F[v] * Cmin + L.F[v] * Cmax - Cmax * Cmin * (R.U[v] - L.U[v]), Cmax + Cmin);
    const T lL = -Cmin, lR = Cmax;
    const T idl = T(1) / (lR - lL);
    const T E_L = -L.U[1], E_R = -R.U[1];
    const T m_L = pick<DIM>(L.U + 2, d), m_R = pick<DIM>(R.U + 2, d);
    const T FE_L = -L.F[1], FE_R = -R.F[1];
    const T Fm_L = pick<DIM>(L.F + 2, d), Fm_R = pick<DIM>(R.F + 2, d);
    const T E_h = (lR * E_R - lL * E_L - (FE_R - FE_L)) * idl;
    const T m_h = (lR * m_R - lL * m_L - (Fm_R - Fm_L)) * idl;
    const T FE_h = (lR * FE_L - lL * FE_R + lR * lL * (E_R - E_L)) * idl;
    const T Fm_h = (lR * Fm_L - lL * Fm_R + lR * lL * (m_R - m_L)) * idl;
    const T b = E_h + Fm_h;
    T disc = b * b - T(4) * FE_h * m_h;
    if (disc < T(0)) disc = T(0);
    const T ls = qdiv(T(2) * m_h, b + qsqrt(disc));
    const T ps = Fm_h - FE_h * ls;
    // star state of the side the contact leaves behind x/t = 0
    const bool left = ls >= T(0);
    T U[NV], F[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        U[v] = left ? L.U[v] : R.U[v];
        F[v] = left ? L.F[v] : R.F[v];
    }
    const T lK = left ? lL : lR;
    const T vn = left ? L.vn : R.vn;
    const T p = left ? L.p : R.p;
    const T E = -U[1];
    const T fac = (lK - vn) / (lK - ls);
    T Us[NV];
    Us[0] = U[0] * fac;
#pragma unroll
    for (int m = 0; m < DIM; ++m)
        Us[2 + m] = m == d ? qdiv(U[2 + m] * (lK - vn) + ps - p, lK - ls) : U[2 + m] * fac;
    const T Es = (E * (lK - vn) + ps * ls - p * vn) / (lK - ls);
    Us[1] = -Es;
    // supersonic right / left, unphysical star state -> HLL, else the star flux
    const bool use_R = Cmax < T(0);
    const bool use_L = !use_R && Cmin < T(0);
    const bool use_hll = !use_R && !use_L && (!(ps > T(0)) || !(ls >= lL && ls <= lR));
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const T fs = F[v] + lK * (Us[v] - U[v]);
        Fo[v] = use_R ? R.F[v] : (use_L ? L.F[v] : (use_hll ? Fh[v] : fs));
    }
}

template <int DIM, int RS, typename T>
VB_HD void face_flux(int d, T g, const T* PL, const T* PR, T* Fo) {
    if (RS == RS_HLLC)
        hllc_flux<DIM>(d, g, PL, PR, Fo);
    else
        hll_flux<DIM>(d, g, PL, PR, Fo);
}

// Largest |lambda| over the axes of one cell-centred state (CFL signal speed;
// an extension -- the reference uses a fixed light-speed dt).
template <int DIM, typename T> VB_HD T max_signal_speed(T g, const T* P) {
    T c = T(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        T lp, lm;
        harm_speeds<DIM>(d, g, P, lp, lm);
        c = fmax(c, fmax(fabs(lp), fabs(lm)));
    }
    return c;
}

}  // namespace vb
