// Z-pair 3D stage kernel of the FP32-bulk form: the z-marching kernel of
// vb_stage_zm.cuh with every thread owning TWO consecutive cells (k, k+1) of
// its (x, y) column, carried as one float2 through the whole stencil.
//
// sm_100a executes FP32 add / multiply / fma on register pairs
// (FADD2 / FMUL2 / FFMA2: __fadd2_rn, __fmul2_rn, __ffma2_rn), so one
// instruction advances both cells. Reconstruction (every limiter), the face floors,
// the Riemann flux (HLL / HLLC), the flux difference and its accumulation are
// written on float2 lanes; reciprocal, square root, min/max and selects stay
// per lane. Each barrier of the plane loop now serves two planes.
//
// Staging (TMA form, the default): every plane of the state, all five
// variables with the 3-cell x/y halo of the CTA's column tile, arrives as one
// TMA tile into a ring of six plane slots; the z window, the x/y stencils and
// the halo reconstructions all read the ring. The other form loads the
// thread's own column into a private z window and brings the x/y halo of each
// pair of planes by 4-byte asynchronous copies into an interleaved buffer.
//
// Arithmetic differs from the scalar FP32 kernel only in rounding (packed
// fma contraction written out by hand, 1/6 folded into the WENOZ stencil
// weights, C^2 formed without the square root and re-square, approximate
// reciprocal / square root); the conserved update U - div and con2prim stay
// FP64 exactly as in k_stage_zm. Same scheme as the reference's 3D kernels
// (src/3dim/algos.jl:14-200, src/fluxlimiter.jl:19-71) plus HLLC.
#pragma once
#include "vb_ns.h"
#include <cuda.h>  // CUtensorMap

#include "vb_stage_zm.cuh"
#include "vb_tc.cuh"

namespace VB_NS {
namespace pk {

using f2 = float2;
__device__ __forceinline__ f2 P2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ f2 S2(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 add(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 mul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
// a - b, exact in the product: b * (-1) + a
__device__ __forceinline__ f2 sub(f2 a, f2 b) { return __ffma2_rn(b, S2(-1.0f), a); }
__device__ __forceinline__ float rcp1(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt1(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// NaN-propagating max / min (Julia's Base.max / Base.min on floats)
__device__ __forceinline__ float maxn(float a, float b) {
    float r;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float minn(float a, float b) {
    float r;
    asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ f2 rcp(f2 a) { return P2(rcp1(a.x), rcp1(a.y)); }
__device__ __forceinline__ f2 vsqrt(f2 a) { return P2(sqrt1(a.x), sqrt1(a.y)); }
__device__ __forceinline__ f2 vmax(f2 a, f2 b) { return P2(maxn(a.x, b.x), maxn(a.y, b.y)); }
__device__ __forceinline__ f2 vmin(f2 a, f2 b) { return P2(minn(a.x, b.x), minn(a.y, b.y)); }
__device__ __forceinline__ f2 vabs(f2 a) { return P2(fabsf(a.x), fabsf(a.y)); }
struct m2 {
    bool x, y;
};
// 4-byte global -> shared copy that bypasses the registers (completes asynchronously)
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(sdst)),
                 "l"(gsrc)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ f2 sel(m2 m, f2 a, f2 b) { return P2(m.x ? a.x : b.x, m.y ? a.y : b.y); }

__device__ __forceinline__ f2 num_scale(f2 num, f2 den_other) { return mul(num, den_other); }

// WENOZ (src/fluxlimiter.jl:19-71) on two cells: returns (qr_i, ql_ip1).
// Written on the one-sided differences D1..D4 of the five values, which the
// smoothness indicators and the three stencils share:
//   beta_k * 12/13 = t_k^2 + (3/13) u_k^2 with the reference's t (second
//   difference) and u (one-sided combination) of each sub-stencil;
//   face value = q_i + sum_k d_k s_k g_k / sum_k d_k s_k, g_k = f_k - q_i,
//   s_k = 1 + (tau5 / (beta_k + eps))^2, d = (0.1, 0.6, 0.3).
// The common factor 13/12 of the betas cancels in tau5 / beta except against
// the FP32 epsilon (1e-30, an effective 1.08e-30). The smoothness ratio is
// capped at 1e9, so every s_k <= 1e18 and the two faces' denominators share
// one reciprocal of their product (<= 1e36, inside the FP32 range): at FP32
// precision a weight ratio beyond 1e8 already acts as infinite, so the cap
// (1e15 in the scalar FP32 form) changes no selected stencil.
__device__ __forceinline__ void wenoz(f2 qm2, f2 qm1, f2 q0, f2 qp1, f2 qp2, f2& qr, f2& ql) {
    const f2 D1 = sub(qm1, qm2), D2 = sub(q0, qm1), D3 = sub(qp1, q0), D4 = sub(qp2, qp1);
    const f2 r = S2(3.0f / 13.0f);
    // beta_k + eps with eps folded into the square term: fma(t, t, eps)
    const f2 eps = S2(1.0e-30f);
    f2 t = sub(D2, D1);           // q_im2 + q_i - 2 q_im1
    f2 u = fma(S2(2.0f), D2, t);  // q_im2 + 3 q_i - 4 q_im1
    const f2 b1 = fma(mul(r, u), u, fma(t, t, eps));
    t = sub(D3, D2);  // q_im1 + q_ip1 - 2 q_i
    u = add(D2, D3);  // q_ip1 - q_im1
    const f2 b2 = fma(mul(r, u), u, fma(t, t, eps));
    t = sub(D4, D3);               // q_ip2 + q_i - 2 q_ip1
    u = fma(S2(-2.0f), D3, t);     // q_ip2 + 3 q_i - 4 q_ip1
    const f2 b3 = fma(mul(r, u), u, fma(t, t, eps));
    const f2 tau = vabs(sub(b1, b3));
    f2 i1 = mul(tau, rcp(b1));
    f2 i2 = mul(tau, rcp(b2));
    f2 i3 = mul(tau, rcp(b3));
    i1 = P2(fminf(i1.x, 1.0e9f), fminf(i1.y, 1.0e9f));
    i2 = P2(fminf(i2.x, 1.0e9f), fminf(i2.y, 1.0e9f));
    i3 = P2(fminf(i3.x, 1.0e9f), fminf(i3.y, 1.0e9f));
    const f2 one = S2(1.0f);
    const f2 s1 = fma(i1, i1, one), s2 = fma(i2, i2, one), s3 = fma(i3, i3, one);
    // right face of cell i (left-biased stencils), weights d_k folded into g_k:
    // 0.1 g1 = 0.1 (5 D2 - 2 D1) / 6, 0.6 g2 = 0.6 (D2 + 2 D3) / 6, 0.3 g3 = 0.3 (4 D3 - D4) / 6
    f2 numl, denl, numr, denr;
    const f2 m6 = mul(S2(0.6f), s2);  // the middle weight's term, common to both denominators
    // (the term 1.2 D3 / 6 of g2 and g3 formed once; on the other face 1.2 D2 / 6)
    {
        const f2 g1 = fma(S2(0.5f / 6.0f), D2, mul(S2(-0.2f / 6.0f), D1));
        const f2 m3 = mul(S2(1.2f / 6.0f), D3);
        const f2 g2 = fma(S2(0.6f / 6.0f), D2, m3);
        const f2 g3 = fma(S2(-0.3f / 6.0f), D4, m3);
        numl = fma(s3, g3, fma(s2, g2, mul(s1, g1)));
        denl = fma(S2(0.3f), s3, fma(S2(0.1f), s1, m6));
    }
    // left face of cell i (right-biased stencils), d = (0.1, 0.6, 0.3) on (s3, s2, s1):
    // 0.1 (2 D4 - 5 D3) / 6, 0.6 (-D3 - 2 D2) / 6, 0.3 (D1 - 4 D2) / 6
    {
        const f2 g1 = fma(S2(0.2f / 6.0f), D4, mul(S2(-0.5f / 6.0f), D3));
        const f2 m2 = mul(S2(-1.2f / 6.0f), D2);
        const f2 g2 = fma(S2(-0.6f / 6.0f), D3, m2);
        const f2 g3 = fma(S2(0.3f / 6.0f), D1, m2);
        numr = fma(s1, g3, fma(s2, g2, mul(s3, g1)));
        denr = fma(S2(0.3f), s1, fma(S2(0.1f), s3, m6));
    }
    // 1 / denl = denr / (denl denr), 1 / denr = denl / (denl denr): one reciprocal
    const f2 rd = rcp(mul(denl, denr));
    ql = fma(num_scale(numl, denr), rd, q0);
    qr = fma(num_scale(numr, denl), rd, q0);
}

// Monotonicity limit of PPM on one lane: the reference's
// sign(a) == sign(b) == sign(c) ? sign(a) min(C2 |b|, C2 |c|, |a|) : 0, with
// C2 |b| and C2 |c| already formed. The sign test compares sign bits with
// integer operations: where one of a, b, c is zero the reference gives 0 and
// the minimum here is that zero too, so only NaN inputs (a NaN state) differ.
__device__ __forceinline__ bool same_sign(float a, float b, float c) {
    const int ia = __float_as_int(a);
    return ((ia ^ __float_as_int(b)) | (ia ^ __float_as_int(c))) >= 0;
}
__device__ __forceinline__ float ppm_mc(float a, float b, float c, float cb, float cc) {
    return same_sign(a, b, c) ? copysignf(minn(cb, minn(cc, fabsf(a))), a) : 0.0f;
}

// PPM (src/fluxlimiter.jl:74-180) on two cells: the interface values, their
// limiting and the parabola's monotonicity fix as packed arithmetic, the
// sign tests, minima and the final choices per lane as selects (the scalar
// form branches on every one of them). Arithmetic differs from the scalar
// FP32 limiter in rounding only: 1/6 and 0.5 folded into fma, the ratio
// qe / d2qf from the approximate reciprocal.
__device__ __forceinline__ void ppm2(f2 qm2, f2 qm1, f2 q0, f2 qp1, f2 qp2, f2& qr, f2& ql) {
    const f2 h = S2(0.5f), c2 = S2(1.25f), mtwo = S2(-2.0f);
    const f2 qa = sub(q0, qm1), qb = sub(qp1, q0);
    const f2 sm = add(qm1, q0), sp = add(q0, qp1);
    // dd_im1 - dd = 0.5 (qm1 - qm2 - qb), dd - dd_ip1 = 0.5 (qa - (qp2 - qp1))
    f2 dph = fma(h, sm, mul(S2(0.5f / 6.0f), sub(sub(qm1, qm2), qb)));
    f2 dphp = fma(h, sp, mul(S2(0.5f / 6.0f), sub(qa, sub(qp2, qp1))));
    const f2 d2m = fma(mtwo, qm1, add(qm2, q0));
    const f2 d2c = fma(mtwo, q0, add(qm1, qp1));
    const f2 d2p = fma(mtwo, qp1, add(q0, qp2));
    const f2 cm = mul(c2, vabs(d2m)), cc = mul(c2, vabs(d2c)), cp = mul(c2, vabs(d2p));
    {  // limit the left interface value
        const f2 A = mul(S2(3.0f), fma(mtwo, dph, sm));
        const f2 qd = P2(ppm_mc(A.x, d2m.x, d2c.x, cm.x, cc.x), ppm_mc(A.y, d2m.y, d2c.y, cm.y, cc.y));
        const f2 cand = fma(S2(-1.0f / 6.0f), qd, mul(h, sm));
        const f2 t = mul(sub(dph, qm1), sub(q0, dph));
        dph = sel(m2{t.x < 0.0f, t.y < 0.0f}, cand, dph);
    }
    {  // and the right one
        const f2 A = mul(S2(3.0f), fma(mtwo, dphp, sp));
        const f2 qd = P2(ppm_mc(A.x, d2c.x, d2p.x, cc.x, cp.x), ppm_mc(A.y, d2c.y, d2p.y, cc.y, cp.y));
        const f2 cand = fma(S2(-1.0f / 6.0f), qd, mul(h, sp));
        const f2 t = mul(sub(dphp, q0), sub(qp1, dphp));
        dphp = sel(m2{t.x < 0.0f, t.y < 0.0f}, cand, dphp);
    }
    const f2 d2qf = mul(S2(6.0f), fma(mtwo, q0, add(dph, dphp)));
    const f2 dqm = sub(q0, dph), dqp = sub(dphp, q0);
    const f2 at = mul(dqm, dqp), bt = mul(qb, qa);
    const f2 qmax = vmax(vmax(vabs(qm1), vabs(qm2)), vmax(vmax(vabs(q0), vabs(qp1)), vabs(qp2)));
    const f2 rq = rcp(d2qf);
    f2 rho;
#pragma unroll
    for (int l = 0; l < 2; ++l) {
        const float a = l ? d2m.y : d2m.x, b = l ? d2c.y : d2c.x, c = l ? d2p.y : d2p.x, d = l ? d2qf.y : d2qf.x;
        const bool same = same_sign(a, b, c) && same_sign(a, d, d);
        const float mn = minn(minn(l ? cm.y : cm.x, l ? cc.y : cc.x), minn(l ? cp.y : cp.x, fabsf(d)));
        const float qe = same ? copysignf(mn, d) : 0.0f;
        const float r = fabsf(d) > 1.0e-12f * (l ? qmax.y : qmax.x) ? qe * (l ? rq.y : rq.x) : 0.0f;
        if (l) rho.y = r; else rho.x = r;
    }
    const f2 tm = fma(mul(S2(-1.0f), rho), dqm, q0), tp = fma(rho, dqp, q0);
    const f2 t2m = fma(mtwo, dqp, q0), t2p = fma(S2(2.0f), dqm, q0);
    const f2 adm = vabs(dqm), adp = vabs(dqp);
#pragma unroll
    for (int l = 0; l < 2; ++l) {
        const bool ext = (l ? at.y : at.x) <= 0.0f || (l ? bt.y : bt.x) <= 0.0f;
        const bool flat = (l ? rho.y : rho.x) <= 1.0f - 1.0e-12f;
        const float am = l ? adm.y : adm.x, ap = l ? adp.y : adp.x;
        const float r0 = l ? dph.y : dph.x, l0 = l ? dphp.y : dphp.x;
        const float rr = ext ? (flat ? (l ? tm.y : tm.x) : r0) : (am >= 2.0f * ap ? (l ? t2m.y : t2m.x) : r0);
        const float ll = ext ? (flat ? (l ? tp.y : tp.x) : l0) : (ap >= 2.0f * am ? (l ? t2p.y : t2p.x) : l0);
        if (l) {
            qr.y = rr;
            ql.y = ll;
        } else {
            qr.x = rr;
            ql.x = ll;
        }
    }
}

// MINMOD (src/fluxlimiter.jl:1-13) on two cells: dU = 0.25 (sign(s+) +
// sign(s-)) min(|s+|, |s-|) is sign(s+) min(...) / 2 where the one-sided
// slopes share a sign bit and 0 elsewhere (a zero slope makes the minimum
// zero), so the sign test is one integer comparison per lane.
__device__ __forceinline__ void minmod2(f2 qm1, f2 q0, f2 qp1, f2& qr, f2& ql) {
    const f2 sp = sub(qp1, q0), sm = sub(q0, qm1);
    const f2 m = mul(S2(0.5f), vmin(vabs(sp), vabs(sm)));
    f2 du;
    du.x = (__float_as_int(sp.x) ^ __float_as_int(sm.x)) >= 0 ? copysignf(m.x, sp.x) : 0.0f;
    du.y = (__float_as_int(sp.y) ^ __float_as_int(sm.y)) >= 0 ? copysignf(m.y, sp.y) : 0.0f;
    qr = sub(q0, du);
    ql = add(q0, du);
}

// Reconstruction of two cells on the packed pairs.
template <int REC>
__device__ __forceinline__ void recon2(f2 qm2, f2 qm1, f2 q0, f2 qp1, f2 qp2, f2& qr, f2& ql) {
    if constexpr (REC == REC_WENOZ) {
        wenoz(qm2, qm1, q0, qp1, qp2, qr, ql);
    } else if constexpr (REC == REC_PPM) {
        ppm2(qm2, qm1, q0, qp1, qp2, qr, ql);
    } else {
        minmod2(qm1, q0, qp1, qr, ql);
    }
}

// One face state along axis D (compile time): the primitive state and what
// the HARM speeds / HLL / HLLC need from it (src/3dim/algos.jl:117-157).
// Sign convention of the energy slot: E = -U[1] > 0 and FE = -F[1].
template <int D> struct Side {
    f2 P[5];
    f2 gam, gw, uw, vn, p, np, lp, lm;
    __device__ __forceinline__ void make(f2 g, f2 gm1, const f2* Pin) {
#pragma unroll
        for (int v = 0; v < 5; ++v) P[v] = Pin[v];
        const f2 one = S2(1.0f);
        gam = vsqrt(fma(P[4], P[4], fma(P[3], P[3], fma(P[2], P[2], one))));
        const f2 w = fma(g, P[1], P[0]);
        const f2 un = P[2 + D];
        gw = mul(gam, w);
        uw = mul(un, w);
        p = mul(gm1, P[1]);
        np = mul(S2(-1.0f), p);
        // C^2 = Gamma (Gamma - 1) u / (rho + Gamma u) = Gamma p / w  (SoundSpeed, src/eos.jl:15-21), so
        // sig = C^2 / (gam^2 (1 - C^2)) = Gamma p / (gam^2 (w - Gamma p)), w - Gamma p > 0. With
        // R = 1 / (gam (w - Gamma p)), one reciprocal: 1 / gam = (w - Gamma p) R, sig = Gamma p R / gam
        const f2 gp = mul(g, p);
        const f2 wgp = sub(w, gp);
        const f2 R = rcp(mul(gam, wgp));
        const f2 igam = mul(wgp, R);
        vn = mul(un, igam);
        const f2 sig = mul(mul(gp, R), igam);
        const f2 r = vsqrt(mul(sig, sub(sig, fma(vn, vn, S2(-1.0f)))));  // sig (1 - vn^2 + sig)
        const f2 inv = rcp(add(one, sig));
        lp = mul(add(vn, r), inv);
        lm = mul(sub(vn, r), inv);
    }
    // conserved component v in the energy-positive convention (slot 1 = E)
    __device__ __forceinline__ f2 U(int v) const {
        if (v == 0) return mul(gam, P[0]);
        if (v == 1) return fma(gam, gw, np);
        return mul(P[v], gw);
    }
    // flux component v along D, energy slot = FE
    __device__ __forceinline__ f2 F(int v) const {
        if (v == 0) return mul(P[0], P[2 + D]);
        if (v == 1) return mul(uw, gam);
        if (v == 2 + D) return fma(P[2 + D], uw, p);
        return mul(P[v], uw);
    }
};

// HLL (RS_HLL, src/3dim/algos.jl:149-174) or HLLC (RS_HLLC: Mignone & Bodo
// 2005 with the HLL fallback for an unphysical star state) flux of two faces.
template <int D, int RS>
__device__ __forceinline__ void face_flux(f2 g, f2 gm1, const f2* PL, const f2* PR, f2* Fo) {
    Side<D> L, R;
    L.make(g, gm1, PL);
    R.make(g, gm1, PR);
    const f2 lR = vmax(L.lp, R.lp);  // Cmax
    const f2 lL = vmin(L.lm, R.lm);  // -Cmin
    const f2 idl = rcp(sub(lR, lL));
    const m2 use_R{lR.x < 0.0f, lR.y < 0.0f};
    const m2 use_L{!use_R.x && lL.x > 0.0f, !use_R.y && lL.y > 0.0f};
    // HLL flux, energy-positive convention: (lR F_L - lL F_R + lR lL (U_R - U_L)) / (lR - lL)
    const f2 nlL = mul(S2(-1.0f), lL);
    const f2 cL = mul(lR, idl), cR = mul(nlL, idl), cU = mul(mul(lR, lL), idl);
    auto hll = [&](int v) { return fma(cU, sub(R.U(v), L.U(v)), fma(cL, L.F(v), mul(cR, R.F(v)))); };
    f2 Fh[5];
#pragma unroll
    for (int v = 0; v < 5; ++v)
        if (RS == RS_HLL || v == 1 || v == 2 + D) Fh[v] = hll(v);
    if (RS == RS_HLL) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            f2 o = sel(use_R, R.F(v), sel(use_L, L.F(v), Fh[v]));
            Fo[v] = v == 1 ? mul(S2(-1.0f), o) : o;
        }
        return;
    }
    // star state: E_h, m_h are the HLL state, FE_h, Fm_h the HLL flux
    const f2 E_h = mul(sub(fma(lR, R.U(1), mul(nlL, L.U(1))), sub(R.F(1), L.F(1))), idl);
    const f2 m_h = mul(sub(fma(lR, R.U(2 + D), mul(nlL, L.U(2 + D))), sub(R.F(2 + D), L.F(2 + D))), idl);
    const f2 FE_h = Fh[1], Fm_h = Fh[2 + D];
    const f2 b = add(E_h, Fm_h);
    f2 disc = fma(S2(-4.0f), mul(FE_h, m_h), mul(b, b));
    disc = P2(disc.x < 0.0f ? 0.0f : disc.x, disc.y < 0.0f ? 0.0f : disc.y);
    const f2 ls = mul(mul(S2(2.0f), m_h), rcp(add(b, vsqrt(disc))));
    const f2 ps = fma(S2(-1.0f), mul(FE_h, ls), Fm_h);
    const m2 left{ls.x >= 0.0f, ls.y >= 0.0f};
    // side K behind the contact
    const f2 lK = sel(left, lL, lR);
    const f2 vn = sel(left, L.vn, R.vn);
    const f2 p = sel(left, L.p, R.p);
    const f2 ilk = rcp(sub(lK, ls));
    const f2 dv = sub(lK, vn);
    const f2 fac = mul(dv, ilk);
    const f2 lkf = mul(lK, sub(fac, S2(1.0f)));  // star flux of a passive component: F + lK (fac - 1) U
    const m2 use_hll{!use_R.x && !use_L.x && (!(ps.x > 0.0f) || !(ls.x >= lL.x && ls.x <= lR.x)),
                     !use_R.y && !use_L.y && (!(ps.y > 0.0f) || !(ls.y >= lL.y && ls.y <= lR.y))};
    // Passive components (density, transverse momenta): U and F of one side S,
    // the upwind side of a supersonic face, else the side behind the contact,
    // selected before the products; a supersonic face gets F_S (lkf -> 0).
    // Their HLL flux is formed only where a lane falls back to HLL.
    const m2 sup{use_R.x || use_L.x, use_R.y || use_L.y};
    const m2 sL{use_L.x || (!use_R.x && left.x), use_L.y || (!use_R.y && left.y)};
    const f2 gS = sel(sL, L.gam, R.gam), gwS = sel(sL, L.gw, R.gw), uwS = sel(sL, L.uw, R.uw);
    const f2 unS = sel(sL, L.P[2 + D], R.P[2 + D]);
    const f2 lkfS = P2(sup.x ? 0.0f : lkf.x, sup.y ? 0.0f : lkf.y);
    const bool any_hll = use_hll.x || use_hll.y;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        f2 o;
        if (v == 1 || v == 2 + D) {
            const f2 UK = sel(left, L.U(v), R.U(v));
            const f2 FK = sel(left, L.F(v), R.F(v));
            f2 fs;
            if (v == 1)  // E* = (E (lK - vn) + p* ls - p vn) / (lK - ls)
                fs = fma(lK, sub(mul(fma(UK, dv, sub(mul(ps, ls), mul(p, vn))), ilk), UK), FK);
            else  // m* = (m (lK - vn) + p* - p) / (lK - ls)
                fs = fma(lK, sub(mul(sub(fma(UK, dv, ps), p), ilk), UK), FK);
            o = sel(use_R, R.F(v), sel(use_L, L.F(v), sel(use_hll, Fh[v], fs)));
        } else {
            const f2 PS = sel(sL, L.P[v], R.P[v]);
            const f2 US = v == 0 ? mul(gS, PS) : mul(PS, gwS);
            const f2 FS = v == 0 ? mul(PS, unS) : mul(PS, uwS);
            o = fma(lkfS, US, FS);  // U* = U fac: F + lK (fac - 1) U
        }
        Fo[v] = v == 1 ? mul(S2(-1.0f), o) : o;
    }
    if (any_hll) {
#pragma unroll
        for (int v = 0; v < 5; ++v)
            if (v != 1 && v != 2 + D) Fo[v] = sel(use_hll, hll(v), Fo[v]);
    }
}

}  // namespace pk

template <int TX, int TY> struct ZpGeom {
    static constexpr int NV = 5, NT = TX * TY;
    static constexpr int EX = TX + 6, EY = TY + 6;
    static constexpr int PLN = EX * EY;
    static constexpr int FXN = (TX + 1) * TY, FYN = TX * (TY + 1);
    static constexpr int FN = FXN > FYN ? FXN : FYN;
    static constexpr int QXN = TX > TY ? TX : TY;
    static constexpr int YHN = 2 * TX;  // y-halo states: ql of the cells of row -1, qr of row TY
    static constexpr int ZR = 6;  // z-window ring: planes k-1 .. k+4
    static constexpr size_t smem_bytes() {
        return sizeof(float2) * NV * (size_t)(PLN + 2 * FN + QXN + YHN) + sizeof(float) * (size_t)ZR * NV * NT;
    }
};

// Ring of the TMA form: plane z of every variable, with its x/y halo, in slot
// z % ZR as one TMA box [NV][EY][BXW] (x fastest). The box starts at
// x = i0 - 3 = TX * blockIdx.x, a multiple of 4 cells (16 bytes, the TMA
// coordinate rule), and is BXW >= TX + 6 cells wide, a multiple of 4.
template <int TX, int TY> struct ZpTmaGeom {
    static constexpr int NV = 5, ZR = 6;
    static constexpr int BXW = (TX + 6 + 3) / 4 * 4, EY = TY + 6;
    static constexpr int VSTR = EY * BXW;                        // floats between variables in a slot
    static constexpr int BOX_BYTES = 4 * NV * VSTR;              // one plane, every variable
    static constexpr int SLOTF = (BOX_BYTES + 127) / 128 * 128 / 4;  // floats per slot (128-byte aligned)
    static constexpr size_t smem_bytes() {
        using G = ZpGeom<TX, TY>;
        return 128 + 4 * (size_t)ZR * SLOTF + sizeof(float2) * NV * (size_t)(2 * G::FN + G::QXN + G::YHN) + 8 * ZR;
    }
};
// the TMA rules and the residency the launch bound assumes (2 CTAs per SM)
static_assert(ZpTmaGeom<32, 8>::BXW >= 32 + 6 && (ZpTmaGeom<32, 8>::BXW * 4) % 16 == 0, "box row");
static_assert((32 * 4) % 16 == 0, "box x start 32 * blockIdx.x is 16-byte aligned");
static_assert(ZpTmaGeom<32, 8>::SLOTF * 4 % 128 == 0 && ZpTmaGeom<32, 8>::BOX_BYTES <= ZpTmaGeom<32, 8>::SLOTF * 4,
              "ring slots hold one box and stay 128-byte aligned");
static_assert(2 * (ZpTmaGeom<32, 8>::smem_bytes() + 1024) <= 228 * 1024, "two CTAs per SM");
constexpr uint32_t ZP_MAX_POLLS = 1u << 22;  // bounded waits for a TMA plane

// What a pair stage kernel leaves behind: con2prim done in the kernel (fused),
// U for k_c2p (split), or the FP32 divergence in Pout for the learned
// con2prim kernel, which forms U itself (div).
enum { ZP_FUSED = 0, ZP_U = 1, ZP_DIV = 2 };

// TMA: the planes come as TMA boxes into a ring of ZR slots (ZpTmaGeom, tm:
// the tensor map of Pin, dims (x, y, z, variable)); otherwise the column's
// z-window is loaded by the thread and the x/y halo of the planes (k, k+1)
// by 4-byte asynchronous copies into an interleaved pair buffer.
template <int REC, int RS, int TX, int TY, int LZ, int MINB, int TAIL, bool TMA>
__global__ void __launch_bounds__(TX * TY, MINB)
    k_stage_zp(StageParams p, StageBufs<float> b, const __grid_constant__ CUtensorMap tm) {
    using namespace pk;
    using G = ZpGeom<TX, TY>;
    using TG = ZpTmaGeom<TX, TY>;
    constexpr int NV = 5, NT = G::NT, FN = G::FN, QXN = G::QXN, ZR = G::ZR;
    constexpr int FXR = TX + 1;
    // plane access: element (v, y, x) of a plane at v * VSTR + (y + 3) * ROW + x + 3
    constexpr int ROW = TMA ? TG::BXW : G::EX, VSTR = TMA ? TG::VSTR : G::PLN, SLOTF = TG::SLOTF;
    static_assert(!TMA || TX % 4 == 0, "TMA boxes start at x = TX * blockIdx.x");
    extern __shared__ __align__(16) unsigned char smem_raw[];  // TMA form: 128-byte base found below
    f2* sPl = nullptr;         // cp.async form: [NV][EY][EX] planes (k, k+1) with x/y halo
    float* sZ = nullptr;       // cp.async form: [ZR][NV][NT] this thread's z-window
    float* sRing = nullptr;    // TMA form: [ZR][SLOTF] plane boxes
    uint64_t* sBar = nullptr;  // TMA form: one mbarrier per ring slot
    f2 *sQL, *sF, *sQX;        // [NV][FN] left states, [NV][FN] fluxes, [NV][QXN] last right states
    f2* sYH;                   // [NV][2 TX]: ql of the cells of row -1, qr of the cells of row TY
    if constexpr (TMA) {
        unsigned char* base = smem_raw + ((128u - (tc::smem_u32(smem_raw) & 127u)) & 127u);
        sRing = reinterpret_cast<float*>(base);
        sQL = reinterpret_cast<f2*>(sRing + ZR * SLOTF);
        sF = sQL + NV * FN;
        sQX = sF + NV * FN;
        sYH = sQX + NV * QXN;
        sBar = reinterpret_cast<uint64_t*>(sYH + NV * G::YHN);
    } else {
        sPl = reinterpret_cast<f2*>(smem_raw);
        sQL = sPl + NV * G::PLN;
        sF = sQL + NV * FN;
        sQX = sF + NV * FN;
        sYH = sQX + NV * QXN;
        sZ = reinterpret_cast<float*>(sYH + NV * G::YHN);
    }

    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int i0 = NG + blockIdx.x * TX, j0 = NG + blockIdx.y * TY;
    const int i = i0 + tx, j = j0 + ty;
    const int z0 = NG + blockIdx.z * LZ;
    const int zend = min(z0 + LZ, p.n[2] - NG);
    const long long sy = p.sy, sz = p.sz, vs = p.vs;
    const long long col = i + sy * j;
    const f2 fl = S2((float)p.floor_);
    const f2 g = S2((float)p.gamma), gm1 = S2((float)(p.gamma - 1.0));
    const f2 cx = S2((float)p.dtdx[0]), cy = S2((float)p.dtdx[1]), cz = S2((float)p.dtdx[2]);

    auto zs = [&](int z, int v) -> float& {
        if constexpr (TMA)
            return sRing[(z % ZR) * SLOTF + v * VSTR + (ty + 3) * ROW + tx + 3];
        else
            return sZ[((z % ZR) * NV + v) * NT + tid];
    };
    auto zload = [&](int z) {
        const bool in = z < p.n[2];
#pragma unroll
        for (int v = 0; v < NV; ++v) zs(z, v) = in ? b.Pin[v * vs + col + sz * z] : 0.0f;
    };
    // reconstruct the cells (c, c+1) along z from the window planes c-2 .. c+3, floored
    auto zrecon = [&](int c, f2* qr, f2* ql) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const float s0 = zs(c - 2, v), s1 = zs(c - 1, v), s2 = zs(c, v), s3 = zs(c + 1, v), s4 = zs(c + 2, v),
                        s5 = zs(c + 3, v);
            recon2<REC>(P2(s0, s1), P2(s1, s2), P2(s2, s3), P2(s3, s4), P2(s4, s5), qr[v], ql[v]);
            if (v < 2) {
                qr[v] = vmax(fl, qr[v]);
                ql[v] = vmax(fl, ql[v]);
            }
        }
    };

    // x/y halo of the planes (kk, kk+1) -> sPl, by asynchronous copies: issued for
    // the next pair once the current pair's x/y reconstructions are done, and
    // waited for at the next pair's first barrier
    constexpr int NXH = 6 * TY, NH = NXH + 6 * TX;
    auto halo_issue = [&](int kk) {
        for (int e = tid; e < NH; e += NT) {
            int hx, hy;
            if (e < NXH) {
                int s6 = e % 6;
                hy = e / 6;
                hx = s6 < 3 ? s6 - 3 : TX + s6 - 3;
            } else {
                int e2 = e - NXH, s6 = e2 / TX;
                hx = e2 % TX;
                hy = s6 < 3 ? s6 - 3 : TY + s6 - 3;
            }
            const long long gc = (i0 + hx) + sy * (j0 + hy) + sz * kk;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                f2* d = &sPl[v * VSTR + (hy + 3) * ROW + hx + 3];
                cp_async4(&d->x, b.Pin + v * vs + gc);
                cp_async4(&d->y, b.Pin + v * vs + gc + sz);
            }
        }
    };
    // TMA form: plane z -> slot z % ZR (one thread issues); plane z is the
    // ((z - z0 + 3) / ZR)-th load of its slot, which fixes the phase parity
    auto plane_issue = [&](int z) {
        uint64_t* bar = &sBar[z % ZR];
        tc::mbar_arrive_expect_tx(bar, TG::BOX_BYTES);
        tc::tma_load_4d(sRing + (z % ZR) * SLOTF, &tm, i0 - NG, j0 - NG, z, 0, bar);
    };
    auto plane_wait = [&](int z) -> bool {
        const uint32_t parity = (uint32_t)((z - z0 + NG) / ZR) & 1u;
        return tc::mbar_wait(&sBar[z % ZR], parity, nullptr, ZP_MAX_POLLS);
    };
    bool stalled = false;  // TMA form: a plane wait ran out (uniform after the next barrier)
    int z_issued = z0 + 2;  // TMA form: last plane issued

    float qlz[NV];  // ql of cell k (left state of face k+1/2)
    float Fzm[NV];  // flux at face k-1/2
    // prologue: window z0-3 .. z0+2, cells (z0-1, z0), the flux at z0-1/2 (both lanes), then z0+3, z0+4
    if constexpr (TMA) {
        if (tid == 0) {
            for (int s = 0; s < ZR; ++s) tc::mbar_init(&sBar[s], 1);
            tc::fence_mbar_init();
        }
        __syncthreads();
        if (tid == 0)
            for (int z = z0 - 3; z <= z0 + 2; ++z) plane_issue(z);
        for (int z = z0 - 3; z <= z0 + 2; ++z) stalled |= !plane_wait(z);
    } else {
        halo_issue(z0);
        for (int z = z0 - 3; z <= z0 + 2; ++z) zload(z);
    }
    {
        f2 qr[NV], ql[NV], L[NV], R[NV], F[NV];
        zrecon(z0 - 1, qr, ql);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            L[v] = S2(ql[v].x);
            R[v] = S2(qr[v].y);
            qlz[v] = ql[v].y;
        }
        face_flux<2, RS>(g, gm1, L, R, F);
#pragma unroll
        for (int v = 0; v < NV; ++v) Fzm[v] = F[v].x;
    }
    if constexpr (!TMA) {
        zload(z0 + 3);
        zload(z0 + 4);
    }

    unsigned long long n_fail = 0, n_fb = 0, n_it = 0, n_cells = 0;
    for (int k = z0; k < zend; k += 2) {
        const bool two = k + 1 < zend;
        const long long c = col + sz * k;
        f2 acc[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = S2(0.0f);

        // stage planes (k, k+1): own column from the window; the halo copies were
        // issued earlier (plane k+1 <= zend <= n2 - 3 exists even when the pair is incomplete).
        // TMA form: planes k, k+1 are in the ring (waited for by the previous z step);
        // once every thread is past the previous step, planes k+3, k+4 replace k-3, k-2
        if constexpr (TMA) {
            if (__syncthreads_or(stalled)) {
                stalled = true;
                break;
            }
            if (tid == 0) {
                tc::fence_proxy_async();
                plane_issue(k + 3);
                plane_issue(k + 4);
            }
            z_issued = k + 4;
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) sPl[v * VSTR + (ty + 3) * ROW + tx + 3] = P2(zs(k, v), zs(k + 1, v));
            cp_async_wait_all();
            __syncthreads();
        }
        // pair of planes (k, k+1) at offset o of a variable's plane
        const int sk = (k % ZR) * SLOTF, sk1 = ((k + 1) % ZR) * SLOTF;
        auto pq = [&](int v, int o) -> f2 {
            if constexpr (TMA)
                return P2(sRing[sk + v * VSTR + o], sRing[sk1 + v * VSTR + o]);
            else
                return sPl[v * VSTR + o];
        };

        // x: reconstruct own cells; halo cells -1 and TX of each row
        f2 qrx[NV];
        {
            const int o = (ty + 3) * ROW + tx + 3;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                f2 qr, ql;
                recon2<REC>(pq(v, o - 2), pq(v, o - 1), pq(v, o), pq(v, o + 1), pq(v, o + 2), qr, ql);
                if (v < 2) {
                    qr = vmax(fl, qr);
                    ql = vmax(fl, ql);
                }
                qrx[v] = qr;
                sQL[v * FN + ty * FXR + tx + 1] = ql;
            }
        }
        // halo cells -1 and TX of every row, one (cell, variable) per thread and
        // XPW per warp, so that every warp adds one reconstruction at most
        {
            constexpr int XH = 2 * TY * NV, NW = NT / 32, XPW = (XH + NW - 1) / NW;
            static_assert(XPW <= 32, "x-halo items per warp");
            const int lane = tid & 31, e = (tid >> 5) * XPW + lane;
            if (lane < XPW && e < XH) {
                const int v = e % NV, cell = e / NV, r = cell >> 1, side = cell & 1;
                const int o = (r + 3) * ROW + (side ? TX : -1) + 3;
                f2 qr, ql;
                recon2<REC>(pq(v, o - 2), pq(v, o - 1), pq(v, o), pq(v, o + 1), pq(v, o + 2), qr, ql);
                if (v < 2) {
                    qr = vmax(fl, qr);
                    ql = vmax(fl, ql);
                }
                if (side)
                    sQX[v * QXN + r] = qr;
                else
                    sQL[v * FN + r * FXR] = ql;
            }
        }
        __syncthreads();
        {
            f2 PL[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) PL[v] = sQL[v * FN + ty * FXR + tx];
            face_flux<0, RS>(g, gm1, PL, qrx, F);
#pragma unroll
            for (int v = 0; v < NV; ++v) sF[v * FN + ty * FXR + tx] = F[v];
        }
        // the last warp computes the TY faces at the tiles' x edge; meanwhile the
        // other warps reconstruct the y halo (cells -1 and TY of every column,
        // one (cell, variable) per thread) from the planes already staged, into
        // buffers of its own, so that the y phase below has no halo work
        static_assert(TY <= 32 && NT > 32, "x-edge faces fit the last warp");
        if (tid >= NT - 32) {
            const int e = NT - 1 - tid;
            if (e < TY) {
                f2 PL[NV], PR[NV], F[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    PL[v] = sQL[v * FN + e * FXR + TX];
                    PR[v] = sQX[v * QXN + e];
                }
                face_flux<0, RS>(g, gm1, PL, PR, F);
#pragma unroll
                for (int v = 0; v < NV; ++v) sF[v * FN + e * FXR + TX] = F[v];
            }
        } else {
            for (int e = tid; e < 2 * TX * NV; e += NT - 32) {
                const int v = e / (2 * TX), cell = e % (2 * TX), cx_ = cell % TX, side = cell / TX;
                const int o = ((side ? TY : -1) + 3) * ROW + cx_ + 3;
                f2 qr, ql;
                recon2<REC>(pq(v, o - 2 * ROW), pq(v, o - ROW), pq(v, o), pq(v, o + ROW), pq(v, o + 2 * ROW), qr,
                            ql);
                if (v < 2) {
                    qr = vmax(fl, qr);
                    ql = vmax(fl, ql);
                }
                sYH[v * (2 * TX) + side * TX + cx_] = side ? qr : ql;
            }
        }
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v)
            acc[v] = fma(cx, sub(sF[v * FN + ty * FXR + tx + 1], sF[v * FN + ty * FXR + tx]), acc[v]);

        // y: reconstruct own cells; halo cells -1 and TY of each column
        f2 qry[NV];
        {
            const int o = (ty + 3) * ROW + tx + 3;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                f2 qr, ql;
                recon2<REC>(pq(v, o - 2 * ROW), pq(v, o - ROW), pq(v, o), pq(v, o + ROW), pq(v, o + 2 * ROW), qr,
                            ql);
                if (v < 2) {
                    qr = vmax(fl, qr);
                    ql = vmax(fl, ql);
                }
                qry[v] = qr;
                sQL[v * FN + (ty + 1) * TX + tx] = ql;
            }
        }
        __syncthreads();
        // every read of sPl for this pair is done: fetch the next pair's halo
        if constexpr (!TMA) {
            if (k + 2 < zend) halo_issue(k + 2);
        }
        {
            f2 PL[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) PL[v] = ty == 0 ? sYH[v * (2 * TX) + tx] : sQL[v * FN + ty * TX + tx];
            face_flux<1, RS>(g, gm1, PL, qry, F);
#pragma unroll
            for (int v = 0; v < NV; ++v) sF[v * FN + ty * TX + tx] = F[v];
        }
        for (int e = NT - 1 - tid; e >= 0 && e < TX; e += NT) {
            f2 PL[NV], PR[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                PL[v] = sQL[v * FN + TY * TX + e];
                PR[v] = sYH[v * (2 * TX) + TX + e];
            }
            face_flux<1, RS>(g, gm1, PL, PR, F);
#pragma unroll
            for (int v = 0; v < NV; ++v) sF[v * FN + TY * TX + e] = F[v];
        }
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v)
            acc[v] = fma(cy, sub(sF[v * FN + (ty + 1) * TX + tx], sF[v * FN + ty * TX + tx]), acc[v]);

        // z: planes k+5, k+6 are fetched now and enter the window after the
        // reconstruction of cells (k+1, k+2) from planes k-1 .. k+4; faces
        // k+1/2 (left ql(k), right qr(k+1)) and k+3/2 (left ql(k+1), right qr(k+2))
        // (TMA form: planes k+3, k+4 were issued at the top of this step)
        float nxt[2 * NV];
        if constexpr (TMA) {
            stalled |= !plane_wait(k + 3);
            stalled |= !plane_wait(k + 4);
        } else {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const bool in = k + 5 + q < p.n[2];
#pragma unroll
                for (int v = 0; v < NV; ++v) nxt[q * NV + v] = in ? b.Pin[v * vs + c + (5 + q) * sz] : 0.0f;
            }
        }
        float Pk[2 * NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            Pk[v] = zs(k, v);
            Pk[NV + v] = zs(k + 1, v);
        }
        {
            f2 qr1[NV], ql1[NV], L[NV], Fz[NV];
            zrecon(k + 1, qr1, ql1);
#pragma unroll
            for (int v = 0; v < NV; ++v) L[v] = P2(qlz[v], ql1[v].x);
            face_flux<2, RS>(g, gm1, L, qr1, Fz);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                acc[v] = fma(cz, sub(Fz[v], P2(Fzm[v], Fz[v].x)), acc[v]);
                Fzm[v] = Fz[v].y;
                qlz[v] = ql1[v].y;
            }
        }
        if constexpr (!TMA) {
#pragma unroll
            for (int q = 0; q < 2; ++q)
#pragma unroll
                for (int v = 0; v < NV; ++v) zs(k + 5 + q, v) = nxt[q * NV + v];
        }

        // ZP_DIV: the FP32 divergence into Pout; ZP_U: the RK combination in FP64
        // (U - div) into Uo; ZP_FUSED: that, then con2prim (guess: this stage's P)
        // and the floors
        if (TAIL == ZP_DIV) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                b.Pout[v * vs + c] = acc[v].x;
                if (two) b.Pout[v * vs + c + sz] = acc[v].y;
            }
        }
#pragma unroll
        for (int q = 0; q < (TAIL == ZP_DIV ? 0 : 2); ++q) {
            if (q == 1 && !two) break;
            const long long cc = c + q * sz;
            double U[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                double u = b.Us[v * vs + cc] - (double)(q ? acc[v].y : acc[v].x);
                if (p.rk_a != 0.0) u = p.rk_a * b.U0[v * vs + cc] + p.rk_b * u;
                U[v] = u;
                b.Uo[v * vs + cc] = u;
            }
            if (TAIL == ZP_FUSED) {
                double P[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) P[v] = (double)Pk[q * NV + v];
                int fb;
                int r = solve_cell<3>(p, U, P, cc, fb);
                n_fail += (r < 0);
                n_fb += fb;
                n_it += (r < 0 ? -r : r);
                n_cells += 1;
                P[0] = jmax(P[0], p.floor_);
                P[1] = jmax(P[1], p.floor_);
#pragma unroll
                for (int v = 0; v < NV; ++v) b.Pout[v * vs + cc] = (float)P[v];
            }
        }
    }

    if constexpr (TMA) {
        // the loop waited for every plane it issued unless a wait ran out: then
        // wait (bounded) for the newest load of each slot before the CTA exits
        if (__syncthreads_or(stalled)) {
            for (int z = z_issued - ZR + 1; z <= z_issued; ++z)
                if (z >= z0 - NG) plane_wait(z);
            if (tid == 0) count_add(p.counters, CNT_TIMEOUT, 1);
        }
    }
    if (n_fail) count_add(p.counters, CNT_C2P_FAIL, n_fail);
    if (p.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            n_fb += __shfl_xor_sync(0xffffffffu, n_fb, o);
            n_it += __shfl_xor_sync(0xffffffffu, n_it, o);
            n_cells += __shfl_xor_sync(0xffffffffu, n_cells, o);
        }
        if ((tid & 31) == 0) {
            count_add(p.counters, CNT_C2P_FALLBACK, n_fb);
            count_add(p.counters, CNT_C2P_ITERS, n_it);
            count_add(p.counters, CNT_C2P_CELLS, n_cells);
        }
    } else if (n_fb) {
        count_add(p.counters, CNT_C2P_FALLBACK, n_fb);
    }
}

// Tile shape of the z-pair kernel: same column tile as the scalar FP32
// z-marching kernel; 2 CTAs of 256 threads per SM (128 registers each).
struct ZpCfg {
    static constexpr int TX = 32, TY = 8, LZ = 64, MINB = 2, MINB_SPLIT = 2;
};

template <int REC, int RS, int TAIL, bool TMA>
cudaError_t launch_stage_zp_t(const StageParams& p, const StageBufs<float>& b, cudaStream_t s) {
    using C = ZpCfg;
    auto kern = k_stage_zp<REC, RS, C::TX, C::TY, C::LZ, TAIL == ZP_FUSED ? C::MINB : C::MINB_SPLIT, TAIL, TMA>;
    constexpr size_t smem = TMA ? ZpTmaGeom<C::TX, C::TY>::smem_bytes() : ZpGeom<C::TX, C::TY>::smem_bytes();
    static unsigned long long attr_set = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(attr_set >> (dev & 63) & 1ULL)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        attr_set |= 1ULL << (dev & 63);
    }
    dim3 grid((p.n[0] - 2 * NG) / C::TX, (p.n[1] - 2 * NG) / C::TY, (p.n[2] - 2 * NG + C::LZ - 1) / C::LZ);
    CUtensorMap tm;
    if (TMA)
        tm = *static_cast<const CUtensorMap*>(p.tmap_in);
    else
        memset(&tm, 0, sizeof tm);
    kern<<<grid, C::TX * C::TY, smem, s>>>(p, b, tm);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || TAIL != ZP_U || p.skip_c2p) return e;
    const long long cells = (long long)(p.n[0] - 2 * NG) * (p.n[1] - 2 * NG) * (p.n[2] - 2 * NG);
    if ((unsigned long long)cells > MAX_CELLS_U32) return cudaErrorInvalidValue;
    if (p.c2p_mode == C2P_GUESS_W)
        k_c2p<float, 2><<<grid_for(cells, 256), 256, 0, s>>>(p, b);
    else
        k_c2p<float, 1><<<grid_for(cells, 256), 256, 0, s>>>(p, b);
    return cudaGetLastError();
}

// Every reconstruction with HLL or HLLC in the FP32-bulk form (zp_available).
// The divergence hand-off (ZP_DIV) is taken when the caller's con2prim kernel
// forms U itself (p.want_div, the fused learned con2prim).
template <int REC, int RS, bool TMA>
cudaError_t dispatch_stage_zp_tail(const StageParams& p, const StageBufs<float>& b, cudaStream_t s) {
    if (!(p.split || p.skip_c2p)) return launch_stage_zp_t<REC, RS, ZP_FUSED, TMA>(p, b, s);
    if (p.skip_c2p && p.want_div) return launch_stage_zp_t<REC, RS, ZP_DIV, TMA>(p, b, s);
    return launch_stage_zp_t<REC, RS, ZP_U, TMA>(p, b, s);
}
// the TMA form where the caller encoded a tensor map of Pin (p.tmap_in)
template <int REC, int RS>
cudaError_t dispatch_stage_zp_rs(const StageParams& p, const StageBufs<float>& b, cudaStream_t s) {
    return p.tmap_in ? dispatch_stage_zp_tail<REC, RS, true>(p, b, s) : dispatch_stage_zp_tail<REC, RS, false>(p, b, s);
}
template <int REC>
cudaError_t dispatch_stage_zp_rec(int rs, const StageParams& p, const StageBufs<float>& b, cudaStream_t s) {
    return rs == RS_HLLC ? dispatch_stage_zp_rs<REC, RS_HLLC>(p, b, s) : dispatch_stage_zp_rs<REC, RS_HLL>(p, b, s);
}
inline cudaError_t dispatch_stage_zp(int rec, int rs, const StageParams& p, const StageBufs<float>& b,
                                     cudaStream_t s) {
    if (rec == REC_MINMOD) return dispatch_stage_zp_rec<REC_MINMOD>(rs, p, b, s);
    if (rec == REC_PPM) return dispatch_stage_zp_rec<REC_PPM>(rs, p, b, s);
    return dispatch_stage_zp_rec<REC_WENOZ>(rs, p, b, s);
}

}  // namespace vb
