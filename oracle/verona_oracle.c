/*
 * verona_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle and the
 * timed CPU baseline). The product library never links or calls this file.
 *
 * A plain-C FP64 restatement of Wesenheit/Verona's SRHD update. Every function
 * follows the Julia source line for line and keeps its evaluation order:
 * Julia evaluates a + b + c as (a + b) + c, x^2 as x*x, x^3 as x*x*x, never
 * contracts a*b + c into an FMA (only the explicit fma() calls of
 * src/2dim/structs.jl:192,205,212 are fused), and min/max propagate NaN.
 * Build with -ffp-contract=off so gcc keeps the same rounding.
 *
 * Extensions beyond the reference (HLLC, SSP-RK3, MINMOD/PPM in 2D/3D, the
 * nozzle and outflow boundary kinds, generic 1D with ghosts) are written in
 * the same style so that the CUDA path can be held to the same numbers.
 *
 * Parity against the reference itself is unpinned (the reference is Julia
 * and does not run here; it has no tests or golden vectors). The restatement
 * is pinned by published known answers and properties in tests/.
 */
#include "verona_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NG 3
#define SQR(x) ((x) * (x))

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---- Julia float semantics ------------------------------------------------ */
/* Base.max / Base.min for IEEE floats: NaN-propagating, +0 > -0. */
static inline double jmax(double x, double y) {
    double d = x - y;
    if (isnan(x) || isnan(y)) return d;
    return signbit(d) ? y : x;
}
static inline double jmin(double x, double y) {
    double d = x - y;
    if (isnan(x) || isnan(y)) return d;
    return signbit(d) ? x : y;
}
/* Base.sign: +-1, keeps signed zero, NaN stays NaN */
static inline double jsign(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : x); }

/* ---- reconstruction: src/fluxlimiter.jl ---------------------------------- */
/* MINMOD, src/fluxlimiter.jl:1-13 */
static inline void minmod(double qm1, double q, double qp1, double* qr, double* ql) {
    double sp = qp1 - q;
    double sm = q - qm1;
    double ssp = jsign(sp), ssm = jsign(sm);
    double asp = fabs(sp), asm_ = fabs(sm);
    double dU = 0.25 * (ssp + ssm) * jmin(asp, asm_);
    *qr = q - dU;
    *ql = q + dU;
}

/* WENOZ, src/fluxlimiter.jl:19-71 */
static inline void wenoz(double q_im2, double q_im1, double q_i, double q_ip1, double q_ip2,
                         double* qr_i, double* ql_ip1) {
    const double c1 = 13.0 / 12.0, c2 = 0.25;
    double b1 = c1 * SQR(q_im2 + q_i - 2.0 * q_im1) + c2 * SQR(q_im2 + 3.0 * q_i - 4.0 * q_im1);
    double b2 = c1 * SQR(q_im1 + q_ip1 - 2.0 * q_i) + c2 * SQR(q_im1 - q_ip1);
    double b3 = c1 * SQR(q_ip2 + q_i - 2.0 * q_ip1) + c2 * SQR(q_ip2 + 3.0 * q_i - 4.0 * q_ip1);
    const double epsL = 1.0e-42;
    double tau5 = fabs(b1 - b3);
    double i1 = tau5 / (b1 + epsL), i2 = tau5 / (b2 + epsL), i3 = tau5 / (b3 + epsL);

    double f1 = 2.0 * q_im2 - 7.0 * q_im1 + 11.0 * q_i;
    double f2 = -q_im1 + 5.0 * q_i + 2.0 * q_ip1;
    double f3 = 2.0 * q_i + 5.0 * q_ip1 - q_ip2;
    double a1 = 0.1 * (1.0 + SQR(i1)), a2 = 0.6 * (1.0 + SQR(i2)), a3 = 0.3 * (1.0 + SQR(i3));
    double asum = 6.0 * (a1 + a2 + a3);
    *ql_ip1 = (f1 * a1 + f2 * a2 + f3 * a3) / asum;

    f1 = 2.0 * q_ip2 - 7.0 * q_ip1 + 11.0 * q_i;
    f2 = -q_ip1 + 5.0 * q_i + 2.0 * q_im1;
    f3 = 2.0 * q_i + 5.0 * q_im1 - q_im2;
    a1 = 0.1 * (1.0 + SQR(i3));
    a2 = 0.6 * (1.0 + SQR(i2));
    a3 = 0.3 * (1.0 + SQR(i1));
    asum = 6.0 * (a1 + a2 + a3);
    *qr_i = (f1 * a1 + f2 * a2 + f3 * a3) / asum;
}

/* PPM, src/fluxlimiter.jl:74-180 */
static inline void ppm(double q_im2, double q_im1, double q_i, double q_ip1, double q_ip2,
                       double* qr_out, double* ql_out) {
    const double C2 = 1.25;
    double qa = q_i - q_im1;
    double qb = q_ip1 - q_i;
    double dd_im1 = 0.5 * qa + 0.5 * (q_im1 - q_im2);
    double dd = 0.5 * qb + 0.5 * qa;
    double dd_ip1 = 0.5 * (q_ip2 - q_ip1) + 0.5 * qb;

    double dph = 0.5 * (q_im1 + q_i) + (dd_im1 - dd) / 6.0;
    double dph_ip1 = 0.5 * (q_i + q_ip1) + (dd - dd_ip1) / 6.0;

    double d2qc_im1 = q_im2 + q_i - 2.0 * q_im1;
    double d2qc = q_im1 + q_ip1 - 2.0 * q_i;
    double d2qc_ip1 = q_i + q_ip2 - 2.0 * q_ip1;

    /* i-1/2 */
    double qa_tmp = dph - q_im1;
    double qb_tmp = q_i - dph;
    qa = 3.0 * (q_im1 + q_i - 2.0 * dph);
    qb = d2qc_im1;
    double qc = d2qc;
    double qd = 0.0;
    if (jsign(qa) == jsign(qb) && jsign(qa) == jsign(qc))
        qd = jsign(qa) * jmin(C2 * fabs(qb), jmin(C2 * fabs(qc), fabs(qa)));
    double dph_tmp = 0.5 * (q_im1 + q_i) - qd / 6.0;
    if (qa_tmp * qb_tmp < 0.0) dph = dph_tmp;

    /* i+1/2 */
    qa_tmp = dph_ip1 - q_i;
    qb_tmp = q_ip1 - dph_ip1;
    qa = 3.0 * (q_i + q_ip1 - 2.0 * dph_ip1);
    qb = d2qc;
    qc = d2qc_ip1;
    qd = 0.0;
    if (jsign(qa) == jsign(qb) && jsign(qa) == jsign(qc))
        qd = jsign(qa) * jmin(C2 * fabs(qb), jmin(C2 * fabs(qc), fabs(qa)));
    double dphip1_tmp = 0.5 * (q_i + q_ip1) - qd / 6.0;
    if (qa_tmp * qb_tmp < 0.0) dph_ip1 = dphip1_tmp;

    double d2qf = 6.0 * (dph + dph_ip1 - 2.0 * q_i);
    double qr_i = dph;
    double ql_ip1 = dph_ip1;

    double dqf_minus = q_i - qr_i;
    double dqf_plus = ql_ip1 - q_i;

    qa_tmp = dqf_minus * dqf_plus;
    qb_tmp = (q_ip1 - q_i) * (q_i - q_im1);

    qa = d2qc_im1;
    qb = d2qc;
    qc = d2qc_ip1;
    qd = d2qf;
    double qe = 0.0;
    if (jsign(qa) == jsign(qb) && jsign(qa) == jsign(qc) && jsign(qa) == jsign(qd))
        qe = jsign(qd) * jmin(jmin(C2 * fabs(qa), C2 * fabs(qb)), jmin(C2 * fabs(qc), fabs(qd)));

    qa = jmax(fabs(q_im1), fabs(q_im2));
    qb = jmax(jmax(fabs(q_i), fabs(q_ip1)), fabs(q_ip2));

    double rho = 0.0;
    if (fabs(qd) > 1.0e-12 * jmax(qa, qb)) rho = qe / qd;

    double tmp_m = q_i - rho * dqf_minus;
    double tmp_p = q_i + rho * dqf_plus;
    double tmp2_m = q_i - 2.0 * dqf_plus;
    double tmp2_p = q_i + 2.0 * dqf_minus;

    if (qa_tmp <= 0.0 || qb_tmp <= 0.0) {
        if (rho <= 1.0 - 1.0e-12) {
            qr_i = tmp_m;
            ql_ip1 = tmp_p;
        }
    } else {
        if (fabs(dqf_minus) >= 2.0 * fabs(dqf_plus)) qr_i = tmp2_m;
        if (fabs(dqf_plus) >= 2.0 * fabs(dqf_minus)) ql_ip1 = tmp2_p;
    }
    *qr_out = qr_i;
    *ql_out = ql_ip1;
}

/* reconstruction(::Val{M}, ...), src/fluxlimiter.jl:183-200 */
static inline void recon(int method, double q_im2, double q_im1, double q_i, double q_ip1,
                         double q_ip2, double* qr, double* ql) {
    if (method == OR_MINMOD)
        minmod(q_im1, q_i, q_ip1, qr, ql);
    else if (method == OR_PPM)
        ppm(q_im2, q_im1, q_i, q_ip1, q_ip2, qr, ql);
    else
        wenoz(q_im2, q_im1, q_i, q_ip1, q_ip2, qr, ql);
}

void or_recon(int method, const double q[5], double out[2]) {
    recon(method, q[0], q[1], q[2], q[3], q[4], &out[0], &out[1]);
}

/* SoundSpeed, src/eos.jl:15-21 */
static inline double sound_speed(double rho, double u, double g) {
    return sqrt((g * (g - 1.0) * u) / (rho + g * u));
}
double or_sound_speed(double rho, double u, double g) { return sound_speed(rho, u, g); }

/* ---- ND point physics: src/3dim/structs.jl:84-142, src/2dim/structs.jl:87-127 */
static inline double lorentz(int dims, const double* P) {
    double s = SQR(P[2]);
    if (dims > 1) s = s + SQR(P[3]);
    if (dims > 2) s = s + SQR(P[4]);
    return sqrt(s + 1.0);
}

/* function_PtoU */
static inline void prim2con(int dims, double g, const double* P, double* U) {
    double gam = lorentz(dims, P);
    double w = g * P[1] + P[0];
    U[0] = gam * P[0];
    U[1] = (g - 1.0) * P[1] - SQR(gam) * w;
    for (int m = 0; m < dims; ++m) U[2 + m] = P[2 + m] * gam * w;
}
void or_prim2con(int dims, double g, const double* P, double* U) { prim2con(dims, g, P, U); }

/* function_PtoFx / PtoFy / PtoFz */
static inline void prim2flux(int dims, int d, double g, const double* P, double* F) {
    double gam = lorentz(dims, P);
    double w = g * P[1] + P[0];
    double un = P[2 + d];
    F[0] = P[0] * un;
    F[1] = -w * un * gam;
    for (int m = 0; m < dims; ++m) {
        if (m == d)
            F[2 + m] = SQR(un) * w + (g - 1.0) * P[1];
        else
            F[2 + m] = P[2 + m] * un * w;
    }
}

/* HARM signal speeds of one state along d: returns lambda+ and lambda-
 * (src/3dim/algos.jl:130-157). */
static inline void harm_speeds(int dims, int d, double g, const double* P, double* lp, double* lm) {
    double lor = lorentz(dims, P);
    double v = P[2 + d] / lor;
    double C = sound_speed(P[0], P[1], g);
    double sig = SQR(C) / (SQR(lor) * (1.0 - SQR(C)));
    double r = sqrt(sig * (1.0 - SQR(v) + sig));
    *lp = (v + r) / (1.0 + sig);
    *lm = (v - r) / (1.0 + sig);
}

/* HLL face flux, src/3dim/algos.jl:117-174 (after the face floor) */
static void hll_flux(int dims, int d, double g, const double* PL, const double* PR, double* Fo) {
    int nv = 2 + dims;
    double UL[5], UR[5], FL[5], FR[5];
    prim2con(dims, g, PR, UR);
    prim2con(dims, g, PL, UL);
    prim2flux(dims, d, g, PR, FR);
    prim2flux(dims, d, g, PL, FL);
    double lpL, lmL, lpR, lmR;
    harm_speeds(dims, d, g, PL, &lpL, &lmL);
    harm_speeds(dims, d, g, PR, &lpR, &lmR);
    double Cmax = jmax(lpL, lpR);
    double Cmin = -jmin(lmL, lmR);
    if (Cmax < 0) {
        for (int v = 0; v < nv; ++v) Fo[v] = FR[v];
    } else if (Cmin < 0) {
        for (int v = 0; v < nv; ++v) Fo[v] = FL[v];
    } else {
        for (int v = 0; v < nv; ++v)
            Fo[v] = (FR[v] * Cmin + FL[v] * Cmax - Cmax * Cmin * (UR[v] - UL[v])) / (Cmax + Cmin);
    }
}

/* HLLC face flux (extension; not in the reference, which is HLL only).
 * Mignone & Bodo (2005, MNRAS 364, 126) SRHD HLLC with the same HARM/Davis
 * speed estimates as the reference HLL, falling back to HLL where the star
 * state is unphysical (p* <= 0, contact outside [lambda_L, lambda_R]). Verona's conserved vector is
 * (D, -E, m_1..m_dims) and its flux (D v, -m_n, m v + p e_n). */
static void hllc_flux(int dims, int d, double g, const double* PL, const double* PR, double* Fo) {
    int nv = 2 + dims;
    double UL[5], UR[5], FL[5], FR[5];
    prim2con(dims, g, PR, UR);
    prim2con(dims, g, PL, UL);
    prim2flux(dims, d, g, PR, FR);
    prim2flux(dims, d, g, PL, FL);
    double lpL, lmL, lpR, lmR;
    harm_speeds(dims, d, g, PL, &lpL, &lmL);
    harm_speeds(dims, d, g, PR, &lpR, &lmR);
    double Cmax = jmax(lpL, lpR);
    double Cmin = -jmin(lmL, lmR);
    if (Cmax < 0) {
        for (int v = 0; v < nv; ++v) Fo[v] = FR[v];
        return;
    }
    if (Cmin < 0) {
        for (int v = 0; v < nv; ++v) Fo[v] = FL[v];
        return;
    }
    double lL = -Cmin, lR = Cmax;
    double idl = 1.0 / (lR - lL);
    /* HLL averages of E (= -U[1]), m_n (= U[2+d]) and their fluxes (m_n, m_n v + p) */
    double E_L = -UL[1], E_R = -UR[1];
    double m_L = UL[2 + d], m_R = UR[2 + d];
    double FE_L = -FL[1], FE_R = -FR[1];
    double Fm_L = FL[2 + d], Fm_R = FR[2 + d];
    double E_h = (lR * E_R - lL * E_L - (FE_R - FE_L)) * idl;
    double m_h = (lR * m_R - lL * m_L - (Fm_R - Fm_L)) * idl;
    double FE_h = (lR * FE_L - lL * FE_R + lR * lL * (E_R - E_L)) * idl;
    double Fm_h = (lR * Fm_L - lL * Fm_R + lR * lL * (m_R - m_L)) * idl;
    /* contact speed: smaller root of FE_h x^2 - (E_h + Fm_h) x + m_h = 0 */
    double b = E_h + Fm_h;
    double disc = b * b - 4.0 * FE_h * m_h;
    if (disc < 0.0) disc = 0.0;
    double ls = 2.0 * m_h / (b + sqrt(disc));
    double ps = Fm_h - FE_h * ls;
    /* unphysical star state: the HLL flux of the same states */
    if (!(ps > 0.0) || !(ls >= lL && ls <= lR)) {
        for (int v = 0; v < nv; ++v)
            Fo[v] = (FR[v] * Cmin + FL[v] * Cmax - Cmax * Cmin * (UR[v] - UL[v])) / (Cmax + Cmin);
        return;
    }
    const double* P;
    const double* U;
    const double* F;
    double lK;
    if (ls >= 0.0) {
        P = PL; U = UL; F = FL; lK = lL;
    } else {
        P = PR; U = UR; F = FR; lK = lR;
    }
    double lor = lorentz(dims, P);
    double vn = P[2 + d] / lor;
    double p = (g - 1.0) * P[1];
    double E = -U[1];
    double fac = (lK - vn) / (lK - ls);
    double Us[5];
    Us[0] = U[0] * fac;
    for (int m = 0; m < dims; ++m) Us[2 + m] = U[2 + m] * fac;
    Us[2 + d] = (U[2 + d] * (lK - vn) + ps - p) / (lK - ls);
    double Es = (E * (lK - vn) + ps * ls - p * vn) / (lK - ls);
    Us[1] = -Es;
    for (int v = 0; v < nv; ++v) Fo[v] = F[v] + lK * (Us[v] - U[v]);
}

void or_face_flux(int dims, int axis, int riemann, double g, const double* PL, const double* PR,
                  double* F) {
    if (riemann == OR_HLLC)
        hllc_flux(dims, axis, g, PL, PR, F);
    else
        hll_flux(dims, axis, g, PL, PR, F);
}

/* ---- con2prim ------------------------------------------------------------ */

/* 3x3 solve used by the 1D Newton (src/1dim/structs.jl:94, StaticArrays 1.9.11
 * `\` for a 3x3 static matrix). StaticArrays is not vendored in the reference;
 * this is the published adjugate (Cramer) formula with the determinant as the
 * triple product of the columns -- parity unpinned at the last bit. A is
 * column-major, A[r + 3c]. */
static void solve3(const double* A, const double* b, double* x) {
#define a(r, c) A[((r)-1) + 3 * ((c)-1)]
    double c1 = a(2, 2) * a(3, 3) - a(3, 2) * a(2, 3);
    double c2 = a(3, 2) * a(1, 3) - a(1, 2) * a(3, 3);
    double c3 = a(1, 2) * a(2, 3) - a(2, 2) * a(1, 3);
    double det = a(1, 1) * c1 + a(2, 1) * c2 + a(3, 1) * c3;
    x[0] = ((a(2, 2) * a(3, 3) - a(2, 3) * a(3, 2)) * b[0] + (a(1, 3) * a(3, 2) - a(1, 2) * a(3, 3)) * b[1] +
            (a(1, 2) * a(2, 3) - a(1, 3) * a(2, 2)) * b[2]) / det;
    x[1] = ((a(2, 3) * a(3, 1) - a(2, 1) * a(3, 3)) * b[0] + (a(1, 1) * a(3, 3) - a(1, 3) * a(3, 1)) * b[1] +
            (a(1, 3) * a(2, 1) - a(1, 1) * a(2, 3)) * b[2]) / det;
    x[2] = ((a(2, 1) * a(3, 2) - a(2, 2) * a(3, 1)) * b[0] + (a(1, 2) * a(3, 1) - a(1, 1) * a(3, 2)) * b[1] +
            (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) * b[2]) / det;
#undef a
}

/* 1D UtoP per cell, src/1dim/structs.jl:78-105 with F_ptoU :48-54 and
 * Jacobian :32-46. Returns the iteration at which it stopped (n_iter if the
 * cap was hit). */
static int c2p_1d(double g, int n_iter, double tol, const double* U, double* P) {
    double x1 = P[0], x2 = P[1], x3 = P[2];
    int it;
    for (it = 1; it <= n_iter; ++it) {
        double gam = sqrt(SQR(x3) + 1.0);
        double w = g * x2 + x1;
        double f[3], J[9], dlt[3];
        f[0] = gam * x1;
        f[1] = (g - 1.0) * x2 - SQR(gam) * w;
        f[2] = x3 * gam * w;
        double gj = sqrt(1.0 + SQR(x3));
        double wj = g * x2 + x1;
        J[0 + 3 * 0] = gj;
        J[0 + 3 * 1] = 0.0;
        J[0 + 3 * 2] = x1 * x3 / gj;
        J[1 + 3 * 0] = -SQR(gj);
        J[1 + 3 * 1] = (g - 1.0) - SQR(gj) * g;
        J[1 + 3 * 2] = -2.0 * x3 * wj;
        J[2 + 3 * 0] = gj * x3;
        J[2 + 3 * 1] = gj * x3 * g;
        J[2 + 3 * 2] = (2.0 * SQR(x3) + 1.0) / gj * wj;
        f[0] = f[0] - U[0];
        f[1] = f[1] - U[1];
        f[2] = f[2] - U[2];
        solve3(J, f, dlt);
        if (sqrt(SQR(dlt[0]) + SQR(dlt[1]) + SQR(dlt[2])) < tol) break;
        x1 = x1 - dlt[0];
        x2 = x2 - dlt[1];
        x3 = x3 - dlt[2];
    }
    P[0] = x1;
    P[1] = x2;
    P[2] = x3;
    return it;
}

/* Row swaps made by lu_pivot4 on this thread since the last or_lu4_swaps_take
 * (instrumentation for the tests that show the pivoting path runs; it does not
 * touch the arithmetic). */
static _Thread_local long long g_lu4_swaps = 0;
long long or_lu4_swaps_take(void) {
    long long n = g_lu4_swaps;
    g_lu4_swaps = 0;
    return n;
}

/* LU_dec_pivot!, src/2dim/structs.jl:121-208 (4x4, scaled partial pivoting,
 * explicit fma). Returns 0 on a row-wise singular matrix (the reference
 * throws there). */
static int lu_pivot4(double* A, double* t, double* x) {
#define I4(i, j) (((j)-1) * 4 + (i)-1)
    double rn[4];
    for (int i = 1; i <= 4; ++i) {
        double am = 0.0;
        for (int j = 1; j <= 4; ++j) {
            double tmp = fabs(A[I4(i, j)]);
            if (tmp > am) am = tmp;
        }
        if (am == 0.0) return 0;
        rn[i - 1] = 1.0 / am;
    }
    for (int k = 1; k <= 4; ++k) {
        int piv = k;
        double pv = fabs(A[I4(k, k)]) * rn[k - 1];
        for (int i = k + 1; i <= 4; ++i) {
            double tmp = fabs(A[I4(i, k)]) * rn[i - 1];
            if (tmp > pv) {
                pv = tmp;
                piv = i;
            }
        }
        if (piv != k) {
            ++g_lu4_swaps;
            for (int j = 1; j <= 4; ++j) {
                double tmp = A[I4(k, j)];
                A[I4(k, j)] = A[I4(piv, j)];
                A[I4(piv, j)] = tmp;
            }
            double tmp = t[k - 1];
            t[k - 1] = t[piv - 1];
            t[piv - 1] = tmp;
            tmp = rn[k - 1];
            rn[k - 1] = rn[piv - 1];
            rn[piv - 1] = tmp;
        }
        for (int i = k + 1; i <= 4; ++i) {
            A[I4(i, k)] /= A[I4(k, k)];
            for (int j = k + 1; j <= 4; ++j) A[I4(i, j)] = fma(-A[I4(i, k)], A[I4(k, j)], A[I4(i, j)]);
        }
    }
    for (int i = 1; i <= 4; ++i) {
        x[i - 1] = t[i - 1];
        for (int j = 1; j <= i - 1; ++j) x[i - 1] = fma(-A[I4(i, j)], x[j - 1], x[i - 1]);
    }
    for (int i = 4; i >= 1; --i) {
        for (int j = i + 1; j <= 4; ++j) x[i - 1] = fma(-A[I4(i, j)], x[j - 1], x[i - 1]);
        x[i - 1] /= A[I4(i, i)];
    }
#undef I4
    return 1;
}

/* 2D function_UtoP per cell, src/2dim/structs.jl:249-330. Returns the
 * iteration at which it stopped, -1 on a singular Jacobian. */
static int c2p_2d(double g, int n_iter, double tol, const double* U, double* P) {
    int it;
    for (it = 1; it <= n_iter; ++it) {
        double gam = sqrt(SQR(P[2]) + SQR(P[3]) + 1.0);
        double w = g * P[1] + P[0];
        double f[4], J[16], o[4];
        f[0] = gam * P[0] - U[0];
        f[1] = (g - 1.0) * P[1] - SQR(gam) * w - U[1];
        f[2] = P[2] * gam * w - U[2];
        f[3] = P[3] * gam * w - U[3];
        J[0] = gam;
        J[4] = 0.0;
        J[8] = P[0] * P[2] / gam;
        J[12] = P[0] * P[3] / gam;
        J[1] = -SQR(gam);
        J[5] = (g - 1.0) - SQR(gam) * g;
        J[9] = -2.0 * P[2] * w;
        J[13] = -2.0 * P[3] * w;
        J[2] = gam * P[2];
        J[6] = gam * P[2] * g;
        J[10] = (2.0 * SQR(P[2]) + SQR(P[3]) + 1.0) / gam * w;
        J[14] = P[2] * P[3] / gam * w;
        J[3] = gam * P[3];
        J[7] = gam * P[3] * g;
        J[11] = P[2] * P[3] / gam * w;
        J[15] = (2.0 * SQR(P[3]) + SQR(P[2]) + 1.0) / gam * w;
        if (!lu_pivot4(J, f, o)) return -1;
        if (sqrt(SQR(o[0]) + SQR(o[1]) + SQR(o[2]) + SQR(o[3])) < tol) break;
        P[0] = P[0] - o[0];
        P[1] = P[1] - o[1];
        P[2] = P[2] - o[2];
        P[3] = P[3] - o[3];
    }
    return it;
}

/* LU_dec_5D! / LU_dec_2D!, src/3dim/structs.jl:144-214 (no pivoting) */
static void lu_plain(int n, double* A, const double* t, double* x) {
#define IX(i, j) (((j)-1) * n + (i)-1)
    for (int k = 1; k <= n; ++k)
        for (int i = k + 1; i <= n; ++i) {
            A[IX(i, k)] /= A[IX(k, k)];
            for (int j = k + 1; j <= n; ++j) A[IX(i, j)] -= A[IX(i, k)] * A[IX(k, j)];
        }
    for (int i = 1; i <= n; ++i) {
        x[i - 1] = t[i - 1];
        for (int j = 1; j <= i - 1; ++j) x[i - 1] -= A[IX(i, j)] * x[j - 1];
    }
    for (int i = n; i >= 1; --i) {
        for (int j = i + 1; j <= n; ++j) x[i - 1] -= A[IX(i, j)] * x[j - 1];
        x[i - 1] /= A[IX(i, i)];
    }
#undef IX
}

/* 3D function_UtoP per cell, src/3dim/structs.jl:258-620: 1DW Newton ->
 * Noble 2D Newton with line search -> 5x5 primitive Newton -> bisection on
 * the 1DW residual. Returns 1..4 for the stage that converged, -1 if none
 * did (the cell is set to NaN, as the reference does). */
static int c2p_3d(double g, int n_iter, double tol, const double* Uc, double* P) {
    const double D = Uc[0], Q_t = Uc[1], Q_x = Uc[2], Q_y = Uc[3], Q_z = Uc[4];
    int conv1 = 0, conv2 = 0, conv5 = 0, convb = 0;
    double S2 = 0, W = 0, v2;

    /* 1DW (:273-343) */
    {
        S2 = Q_x * Q_x + Q_y * Q_y + Q_z * Q_z;
        double gm = sqrt(SQR(P[2]) + SQR(P[3]) + SQR(P[4]) + 1.0);
        double w_small = P[0] + g * P[1];
        W = w_small * SQR(gm);
        double W_max = 1e30;
        double W_min = sqrt(S2) * (1.0 + 1e-15);
        /* the reference loop never ends for W <= 0; 400 passes cover every positive W */
        for (int guard = 0; guard < 400 && S2 / SQR(W) >= 1.0 && W < W_max; ++guard) W *= 10.0;
        v2 = jmin(S2 / SQR(W), 1.0 - 1e-15);
        for (int it = 0; it < n_iter; ++it) {
            if (W < W_min) W = W_min;
            v2 = S2 / SQR(W);
            if (v2 < 0.0)
                v2 = 0.0;
            else if (v2 > 1.0 - 1e-15)
                v2 = 1.0 - 1e-15;
            double k = (g - 1.0) / g;
            double bf = Q_t + W - k * (W * (1.0 - v2) - D * sqrt(1.0 - v2));
            double W3 = W * W * W;
            double bj = 1.0 - ((g - 1.0) / g) * (1.0 - v2) -
                        ((g - 1.0) / g) * (W * (2.0 * S2 / W3) - D * (S2 / (W3 * sqrt(1.0 - v2))));
            double dW = bf / bj;
            double Wp = W - dW;
            if (Wp < W_min)
                W = 0.5 * (W + W_min);
            else
                W = Wp;
            if (dW < 0) dW = -dW;
            if (SQR(dW) < SQR(tol)) {
                conv1 = 1;
                break;
            }
        }
    }

    /* Noble 2D (:345-447) */
    if (!conv1) {
        S2 = Q_x * Q_x + Q_y * Q_y + Q_z * Q_z;
        double gm = sqrt(SQR(P[2]) + SQR(P[3]) + SQR(P[4]) + 1.0);
        double w_small = P[0] + g * P[1];
        W = w_small * SQR(gm);
        double W_max = 1e30;
        /* the reference loop never ends for W <= 0; 400 passes cover every positive W */
        for (int guard = 0; guard < 400 && S2 / SQR(W) >= 1.0 && W < W_max; ++guard) W *= 10.0;
        v2 = jmin(S2 / SQR(W), 1.0 - 1e-15);
        double W_old, v2_old;
        for (int it = 0; it < n_iter; ++it) {
            W_old = W;
            v2_old = v2;
            double k = (g - 1.0) / g;
            double f[2], J[4], o[2];
            f[0] = v2 - S2 / SQR(W);
            f[1] = Q_t + W - k * (W * (1.0 - v2) - D * sqrt(1.0 - v2));
            J[0] = 2.0 * S2 / (W * W * W);
            J[1] = 1.0 - k * (1.0 - v2);
            J[2] = 1.0;
            J[3] = k * (W - D / (2.0 * sqrt(1.0 - v2)));
            lu_plain(2, J, f, o);
            double dW = o[0], dv2 = o[1];
            double alpha = 1.0;
            int ok = 0;
            for (int ls = 0; ls < 10; ++ls) {
                double sq = sqrt(W - alpha * dW);
                double Wc = SQR(sq);
                double v2c = v2 - alpha * dv2;
                if (Wc <= 0 || Wc > W_max) Wc = W_old;
                if (v2c < 0)
                    v2c = 0.0;
                else if (v2c >= 1)
                    v2c = 1.0 - 1e-15;
                double r1 = v2c - S2 / SQR(Wc);
                double r2 = Q_t + Wc - k * (Wc * (1.0 - v2c) - D * sqrt(1.0 - v2c));
                double errc = SQR(r1) + SQR(r2);
                double r1o = v2 - S2 / SQR(W);
                double r2o = Q_t + W - k * (W * (1.0 - v2) - D * sqrt(1.0 - v2));
                double erro = SQR(r1o) + SQR(r2o);
                if (errc <= erro) {
                    W = Wc;
                    v2 = v2c;
                    ok = 1;
                    break;
                } else {
                    alpha *= 0.5;
                }
            }
            if (!ok) {
                W = W_old;
                v2 = v2_old;
            }
            double relW = sqrt(SQR(W - W_old)) / jmax(fabs(W_old), SQR(tol));
            double relv2 = sqrt(SQR(v2 - v2_old)) / jmax(fabs(v2_old), SQR(tol));
            if (relW + relv2 < tol) {
                conv2 = 1;
                break;
            }
        }
    }

    /* 5D primitive Newton (:449-539) */
    if (!conv1 && !conv2) {
        for (int it = 0; it < n_iter; ++it) {
            double gam = sqrt(SQR(P[2]) + SQR(P[3]) + SQR(P[4]) + 1.0);
            double w = g * P[1] + P[0];
            double f[5], J[25], o[5];
            f[0] = gam * P[0] - Uc[0];
            f[1] = (g - 1.0) * P[1] - SQR(gam) * w - Uc[1];
            f[2] = P[2] * gam * w - Uc[2];
            f[3] = P[3] * gam * w - Uc[3];
            f[4] = P[4] * gam * w - Uc[4];
            J[0] = gam;
            J[5] = 0.0;
            J[10] = P[2] * P[0] / gam;
            J[15] = P[3] * P[0] / gam;
            J[20] = P[4] * P[0] / gam;
            J[1] = -SQR(gam);
            J[6] = g * (-SQR(gam)) + g - 1.0;
            J[11] = -2.0 * P[2] * w;
            J[16] = -2.0 * P[3] * w;
            J[21] = -2.0 * P[4] * w;
            J[2] = P[2] * gam;
            J[7] = g * P[2] * gam;
            J[12] = SQR(P[2]) * w / gam + w * gam;
            J[17] = P[2] * P[3] * w / gam;
            J[22] = P[2] * P[4] * w / gam;
            J[3] = P[3] * gam;
            J[8] = g * P[3] * gam;
            J[13] = P[2] * P[3] * w / gam;
            J[18] = SQR(P[3]) * w / gam + w * gam;
            J[23] = P[3] * P[4] * w / gam;
            J[4] = P[4] * gam;
            J[9] = g * P[4] * gam;
            J[14] = P[2] * P[4] * w / gam;
            J[19] = P[3] * P[4] * w / gam;
            J[24] = SQR(P[4]) * w / gam + w * gam;
            lu_plain(5, J, f, o);
            if (SQR(o[0]) + SQR(o[1]) + SQR(o[2]) + SQR(o[3]) + SQR(o[4]) < SQR(tol)) {
                if (isfinite(P[0]) && isfinite(P[1]) && isfinite(P[2]) && isfinite(P[3]) && isfinite(P[4])) {
                    conv5 = 1;
                    P[0] = jmax(1e-8, P[0]);
                    P[1] = jmax(1e-8, P[1]);
                    double gm = sqrt(SQR(P[2]) + SQR(P[3]) + SQR(P[4]) + 1.0);
                    P[2] = P[2] / gm;
                    P[3] = P[3] / gm;
                    P[4] = P[4] / gm;
                    gm = jmin(gm, 50.0);
                    P[2] = P[2] * gm;
                    P[3] = P[3] * gm;
                    P[4] = P[4] * gm;
                }
                break;
            }
            P[0] = P[0] - o[0];
            P[1] = P[1] - o[1];
            P[2] = P[2] - o[2];
            P[3] = P[3] - o[3];
            P[4] = P[4] - o[4];
        }
    }

    /* bisection on the 1DW residual (:541-596) */
    if (!conv1 && !conv2 && !conv5) {
        S2 = Q_x * Q_x + Q_y * Q_y + Q_z * Q_z;
        double k = (g - 1.0) / g;
        double W_min = jmax(1e-15, sqrt(S2));
        double W_max = W_min * 10.0;
#define RES(Wv) (Q_t + (Wv) - k * ((Wv) * (1.0 - S2 / SQR(Wv)) - D * sqrt(jmax(0.0, 1.0 - S2 / SQR(Wv)))))
        double fmin_ = RES(W_min);
        double fmax_ = RES(W_max);
        int count = 0;
        while (fmin_ * fmax_ > 0 && count < 100) {
            W_max *= 10.0;
            fmax_ = RES(W_max);
            count += 1;
        }
        if (fmin_ * fmax_ <= 0) {
            for (int it = 0; it < n_iter * 10; ++it) {
                double Wm = 0.5 * (W_min + W_max);
                double fm = RES(Wm);
                if (SQR(fm) < SQR(1e-6)) {
                    convb = 1;
                    W = Wm;
                    break;
                }
                if (fmin_ * fm < 0) {
                    W_max = Wm;
                    fmax_ = fm;
                } else {
                    W_min = Wm;
                    fmin_ = fm;
                }
                W = Wm;
            }
        }
#undef RES
    }

    if (conv1 || conv2 || convb) {
        v2 = S2 / SQR(W);
        double gm = 1.0 / sqrt(1.0 - v2);
        gm = jmin(gm, 50.0);
        double rho = jmax(1e-8, D / gm);
        double UU = jmax(1e-8, (W / SQR(gm) - D / gm) / g);
        P[0] = rho;
        P[1] = UU;
        P[2] = gm * Q_x / W;
        P[3] = gm * Q_y / W;
        P[4] = gm * Q_z / W;
    }
    if (!conv1 && !conv2 && !conv5 && !convb) {
        for (int v = 0; v < 5; ++v) P[v] = NAN;
        return -1;
    }
    return conv1 ? 1 : conv2 ? 2 : conv5 ? 3 : 4;
}

int or_con2prim(int dims, double g, int n_iter, double tol, const double* U, double* P) {
    if (dims == 1) return c2p_1d(g, n_iter, tol, U, P);
    if (dims == 2) return c2p_2d(g, n_iter, tol, U, P);
    return c2p_3d(g, n_iter, tol, U, P);
}

/* ========================================================================== */
/* 1D reference solver, src/1dim/algos.jl:58-315                             */
/* ========================================================================== */
struct or1d {
    int N;
    double g, tol;
    int rec, n_iter;
    double *P, *Ph, *U, *Uh, *PL, *PR, *F; /* component-major [3][N] */
};

static double* alloc3(int N) { return (double*)calloc((size_t)3 * N, sizeof(double)); }

/* PtoU, src/1dim/structs.jl:58-66 (all cells) */
static void ptou_1dref(int N, double g, const double* P, double* U) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        double p1 = P[i], p2 = P[N + i], p3 = P[2 * N + i];
        double gamma = sqrt(SQR(p3) + 1.0);
        double pressure = (g - 1.0) * p2;
        U[i] = p1 * gamma;
        U[N + i] = -(p2 + pressure + p1) * SQR(gamma) + pressure;
        U[2 * N + i] = (p2 + pressure + p1) * gamma * p3;
    }
}

or1d_t* or1d_create(int N, const double* rho, const double* u, const double* ux, double g, int rec,
                    int n_iter, double tol) {
    or1d_t* s = (or1d_t*)calloc(1, sizeof(or1d_t));
    s->N = N;
    s->g = g;
    s->rec = rec;
    s->n_iter = n_iter;
    s->tol = tol;
    s->P = alloc3(N);
    s->Ph = alloc3(N);
    s->U = alloc3(N);
    s->Uh = alloc3(N);
    s->PL = alloc3(N);
    s->PR = alloc3(N);
    s->F = alloc3(N);
    memcpy(s->P, rho, N * sizeof(double));
    memcpy(s->P + N, u, N * sizeof(double));
    memcpy(s->P + 2 * N, ux, N * sizeof(double));
    /* PR = deepcopy(P); PL = deepcopy(P)  (:182-183) */
    memcpy(s->PR, s->P, 3 * N * sizeof(double));
    memcpy(s->PL, s->P, 3 * N * sizeof(double));
    ptou_1dref(N, g, s->P, s->U); /* :193 */
    memcpy(s->Uh, s->U, 3 * N * sizeof(double)); /* Uhalf = deepcopy(U) :194 */
    memcpy(s->Ph, s->P, 3 * N * sizeof(double));
    return s;
}

/* one stage: reconstruction into PR/PL, HLL fluxes F, update into Uout
 * (src/1dim/algos.jl:91-177 / :184-302) */
static void stage_1dref(or1d_t* s, const double* P, const double* Ubase, double* Uout, double coef) {
    const int N = s->N;
    const double g = s->g;
    for (int v = 0; v < 3; ++v) {
        const double* q = P + v * N;
        double* pr = s->PR + v * N;
        double* pl = s->PL + v * N;
        if (s->rec == OR_MINMOD) {
            /* i = 2:(N-1), 1-based -> 0-based i in [1, N-2] */
#pragma omp parallel for schedule(static)
            for (int i = 1; i <= N - 2; ++i) minmod(q[i - 1], q[i], q[i + 1], &pr[i - 1], &pl[i]);
        } else {
            /* i = 3:(N-2) -> 0-based [2, N-3] */
#pragma omp parallel for schedule(static)
            for (int i = 2; i <= N - 3; ++i) {
                if (s->rec == OR_PPM)
                    ppm(q[i - 2], q[i - 1], q[i], q[i + 1], q[i + 2], &pr[i - 1], &pl[i]);
                else
                    wenoz(q[i - 2], q[i - 1], q[i], q[i + 1], q[i + 2], &pr[i - 1], &pl[i]);
            }
        }
    }
    /* PtoU(PR,UR), PtoU(PL,UL), PtoF(PR,FR), PtoF(PL,FL), then the HLL loop
     * over all faces (:233-282); fused per face here, same arithmetic. */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        double pl1 = s->PL[i], pl2 = s->PL[N + i], pl3 = s->PL[2 * N + i];
        double pr1 = s->PR[i], pr2 = s->PR[N + i], pr3 = s->PR[2 * N + i];
        double UL[3], UR[3], FL[3], FR[3];
        {
            double gamma = sqrt(SQR(pr3) + 1.0), pressure = (g - 1.0) * pr2;
            UR[0] = pr1 * gamma;
            UR[1] = -(pr2 + pressure + pr1) * SQR(gamma) + pressure;
            UR[2] = (pr2 + pressure + pr1) * gamma * pr3;
            FR[0] = pr1 * pr3;
            FR[1] = -(pr2 + pressure + pr1) * gamma * pr3;
            FR[2] = pressure + (pr2 + pressure + pr1) * SQR(pr3);
        }
        {
            double gamma = sqrt(SQR(pl3) + 1.0), pressure = (g - 1.0) * pl2;
            UL[0] = pl1 * gamma;
            UL[1] = -(pl2 + pressure + pl1) * SQR(gamma) + pressure;
            UL[2] = (pl2 + pressure + pl1) * gamma * pl3;
            FL[0] = pl1 * pl3;
            FL[1] = -(pl2 + pressure + pl1) * gamma * pl3;
            FL[2] = pressure + (pl2 + pressure + pl1) * SQR(pl3);
        }
        double vL = pl3 / sqrt(SQR(pl3) + 1.0);
        double vR = pr3 / sqrt(SQR(pr3) + 1.0);
        double CL = sound_speed(pl1, pl2, g);
        double CR = sound_speed(pr1, pr2, g);
        double sL = SQR(CL) / ((SQR(pl3) + 1.0) * (1.0 - SQR(CL)));
        double sR = SQR(CR) / ((SQR(pr3) + 1.0) * (1.0 - SQR(CR)));
        double Cmax = jmax((vL + sqrt(sL * (1.0 - SQR(vL) + sL))) / (1.0 + sL),
                           (vR + sqrt(sR * (1.0 - SQR(vR) + sR))) / (1.0 + sR));
        double Cmin = -jmin((vL - sqrt(sL * (1.0 - SQR(vL) + sL))) / (1.0 + sL),
                            (vR - sqrt(sR * (1.0 - SQR(vR) + sR))) / (1.0 + sR));
        for (int v = 0; v < 3; ++v) {
            double f;
            if (Cmax < 0)
                f = FR[v];
            else if (Cmin < 0)
                f = FL[v];
            else
                f = (FR[v] * Cmin + FL[v] * Cmax - Cmax * Cmin * (UR[v] - UL[v])) / (Cmax + Cmin);
            s->F[v * N + i] = f;
        }
    }
    /* update, i = 2:(N-2) -> 0-based [1, N-3] (:284-288, :409-413) */
    for (int v = 0; v < 3; ++v) {
        const double* F = s->F + v * N;
        const double* Ub = Ubase + v * N;
        double* Uo = Uout + v * N;
#pragma omp parallel for schedule(static)
        for (int i = 1; i <= N - 3; ++i) Uo[i] = Ub[i] - coef * (F[i] - F[i - 1]);
    }
}

static void utop_1dref(or1d_t* s, const double* U, double* P) {
    const int N = s->N;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        double u[3] = {U[i], U[N + i], U[2 * N + i]};
        double p[3] = {P[i], P[N + i], P[2 * N + i]};
        c2p_1d(s->g, s->n_iter, s->tol, u, p);
        P[i] = p[0];
        P[N + i] = p[1];
        P[2 * N + i] = p[2];
    }
}

void or1d_step(or1d_t* s, double dt, double dx, int nsteps) {
    const int N = s->N;
    for (int n = 0; n < nsteps; ++n) {
        stage_1dref(s, s->P, s->U, s->Uh, 0.5 * dt / dx);
        memcpy(s->Ph, s->P, 3 * N * sizeof(double)); /* Phalf = deepcopy(P) :290 */
        utop_1dref(s, s->Uh, s->Ph);
        stage_1dref(s, s->Ph, s->U, s->U, dt / dx);
        utop_1dref(s, s->U, s->P);
    }
}

void or1d_get(const or1d_t* s, double* rho, double* u, double* ux) {
    memcpy(rho, s->P, s->N * sizeof(double));
    memcpy(u, s->P + s->N, s->N * sizeof(double));
    memcpy(ux, s->P + 2 * s->N, s->N * sizeof(double));
}
void or1d_get_cons(const or1d_t* s, double* U1, double* U2, double* U3) {
    memcpy(U1, s->U, s->N * sizeof(double));
    memcpy(U2, s->U + s->N, s->N * sizeof(double));
    memcpy(U3, s->U + 2 * s->N, s->N * sizeof(double));
}
void or1d_destroy(or1d_t* s) {
    if (!s) return;
    free(s->P); free(s->Ph); free(s->U); free(s->Uh); free(s->PL); free(s->PR); free(s->F);
    free(s);
}

/* ========================================================================== */
/* ND solver with ghosts                                                      */
/* ========================================================================== */
struct ornd {
    int dims, nv;
    int n[3];        /* padded sizes */
    long ncell;
    double g, floor_, tol;
    int n_iter, recon, riemann, rk;
    double dx[3];
    double *P, *U0, *U1, *F[3];
    int bc_kind[6];
    double bc_par[6][16];
    double t;
    int64_t c2p_fail;
};

#define CELL(n, i, j, k) ((long)(i) + (long)(n)[0] * ((long)(j) + (long)(n)[1] * (long)(k)))

/* kernel_PtoU on all cells, src/3dim/structs.jl:66-81 */
void ornd_k_ptou(int dims, const int np[3], const double* P, double* U, double g) {
    const int nv = 2 + dims;
    long nc = (long)np[0] * np[1] * np[2];
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; ++c) prim2con(dims, g, P + nv * c, U + nv * c);
}

/* function_Limit on all cells, src/3dim/algos.jl:5-12 */
void ornd_k_limit(int dims, const int np[3], double* P, double fl) {
    const int nv = 2 + dims;
    long nc = (long)np[0] * np[1] * np[2];
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; ++c) {
        P[nv * c + 0] = jmax(P[nv * c + 0], fl);
        P[nv * c + 1] = jmax(P[nv * c + 1], fl);
    }
}

/* function_Fluxes for one axis, src/3dim/algos.jl:14-176 (2D: src/2dim/algos.jl:11-168).
 * Face i+1/2 is stored at F[:, i]. Faces are computed for every index in
 * [2, n-4] (0-based) on all axes, as the reference's guards do; the left
 * state is ql_{i+1/2} of cell i, the right state qr of cell i+1. */
void ornd_k_fluxes(int dims, const int np[3], const double* P, double g, double fl, double* F, int d,
                   int rec, int riemann) {
    const int nv = 2 + dims;
    long st[3] = {1, np[0], (long)np[0] * np[1]};
    int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    for (int a = 0; a < dims; ++a) {
        lo[a] = 2;
        hi[a] = np[a] - 3;
    }
    long sd = st[d];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = lo[2]; k < hi[2]; ++k)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int i = lo[0]; i < hi[0]; ++i) {
                long c = CELL(np, i, j, k);
                double PL[5], PR[5];
                for (int v = 0; v < nv; ++v) {
                    const double* q = P + v;
                    double qr, ql;
                    recon(rec, q[nv * (c - 2 * sd)], q[nv * (c - sd)], q[nv * c], q[nv * (c + sd)],
                          q[nv * (c + 2 * sd)], &qr, &ql);
                    PL[v] = ql;
                    recon(rec, q[nv * (c - sd)], q[nv * c], q[nv * (c + sd)], q[nv * (c + 2 * sd)],
                          q[nv * (c + 3 * sd)], &qr, &ql);
                    PR[v] = qr;
                }
                for (int v = 0; v < 2; ++v) {
                    PL[v] = jmax(fl, PL[v]);
                    PR[v] = jmax(fl, PR[v]);
                }
                or_face_flux(dims, d, riemann, g, PL, PR, F + nv * c);
            }
}

/* function_Update, src/3dim/algos.jl:178-200: interior cells [3, n-4] */
void ornd_k_update(int dims, const int np[3], const double* U, double* Ub, double dt, const double dxs[3],
                   const double* Fx, const double* Fy, const double* Fz) {
    const int nv = 2 + dims;
    long st[3] = {1, np[0], (long)np[0] * np[1]};
    int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    for (int a = 0; a < dims; ++a) {
        lo[a] = 3;
        hi[a] = np[a] - 3;
    }
    const double* Fs[3] = {Fx, Fy, Fz};
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = lo[2]; k < hi[2]; ++k)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int i = lo[0]; i < hi[0]; ++i) {
                long c = CELL(np, i, j, k);
                for (int v = 0; v < nv; ++v) {
                    double r = U[nv * c + v];
                    for (int a = 0; a < dims; ++a)
                        r = r - dt / dxs[a] * (Fs[a][nv * c + v] - Fs[a][nv * (c - st[a]) + v]);
                    Ub[nv * c + v] = r;
                }
            }
}

/* function_UtoP on interior cells */
static int64_t k_utop(int dims, const int np[3], const double* U, double* P, double g, int n_iter,
                      double tol) {
    const int nv = 2 + dims;
    int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    for (int a = 0; a < dims; ++a) {
        lo[a] = 3;
        hi[a] = np[a] - 3;
    }
    int64_t fails = 0;
#pragma omp parallel for collapse(2) schedule(dynamic, 1) reduction(+ : fails)
    for (int k = lo[2]; k < hi[2]; ++k)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int i = lo[0]; i < hi[0]; ++i) {
                long c = CELL(np, i, j, k);
                int r = or_con2prim(dims, g, n_iter, tol, U + nv * c, P + nv * c);
                if (r < 0) fails++;
            }
    return fails;
}
void ornd_k_utop(int dims, const int np[3], const double* U, double* P, double g, int n_iter, double tol) {
    (void)k_utop(dims, np, U, P, g, n_iter, tol);
}

ornd_t* ornd_create(int dims, const int n[3], const double* P_aos, double g, double fl, int n_iter,
                    double tol, int rec, int riemann, int rk) {
    ornd_t* s = (ornd_t*)calloc(1, sizeof(ornd_t));
    s->dims = dims;
    s->nv = 2 + dims;
    for (int a = 0; a < 3; ++a) s->n[a] = a < dims ? n[a] + 2 * NG : 1;
    s->ncell = (long)s->n[0] * s->n[1] * s->n[2];
    s->g = g;
    s->floor_ = fl;
    s->n_iter = n_iter;
    s->tol = tol;
    s->recon = rec;
    s->riemann = riemann;
    s->rk = rk;
    s->dx[0] = s->dx[1] = s->dx[2] = 1.0;
    size_t bytes = sizeof(double) * s->nv * s->ncell;
    s->P = (double*)malloc(bytes);
    s->U0 = (double*)malloc(bytes);
    s->U1 = (double*)calloc(1, bytes);
    for (int a = 0; a < dims; ++a) s->F[a] = (double*)calloc(1, bytes);
    memcpy(s->P, P_aos, bytes);
    for (int f = 0; f < 6; ++f) s->bc_kind[f] = OR_BC_OUTFLOW;
    /* PtoU(P.arr, U.arr, eos) at the start of HARM_HLL (src/3dim/algos.jl:259) */
    ornd_k_ptou(dims, s->n, s->P, s->U0, g);
    s->t = 0.0;
    return s;
}

void ornd_set_grid(ornd_t* s, double dx, double dy, double dz) {
    s->dx[0] = dx;
    s->dx[1] = dy;
    s->dx[2] = dz;
}

void ornd_set_boundary(ornd_t* s, int face, int kind, const double* par, int np) {
    s->bc_kind[face] = kind;
    memset(s->bc_par[face], 0, sizeof(s->bc_par[face]));
    for (int i = 0; i < np && i < 16; ++i) s->bc_par[face][i] = par[i];
}

/* Ghost fill at the start of a step. This is the on-device replacement of the
 * user boundary callback `TurnOff` (examples/Jet3D/HARM_jet_breakout.jl:131-158,
 * examples/Jet2D/HARM_jet_breakout.jl:84-99): first the decay of FIXED faces,
 * then faces in the order y-lo, y-hi, z-lo, z-hi, x-lo, x-hi, each spanning the
 * full padded extent of the other axes. OUTFLOW copies the first interior
 * cell into the three ghost layers. NOZZLE holds a fixed inflow state inside
 * a radius (in cells, measured from the given centre in the face plane) and
 * is OUTFLOW outside it. */
static void bc_fill(ornd_t* s, double t) {
    const int nv = s->nv, dims = s->dims;
    const int* np = s->n;
    /* decay (FIXED faces) */
    for (int face = 0; face < 2 * dims; ++face) {
        if (s->bc_kind[face] != OR_BC_FIXED) continue;
        const double* par = s->bc_par[face];
        int var = (int)par[0];
        double t_on = par[1], t_off = par[2], fac = par[3];
        if (!(t > t_on && t < t_off)) continue;
        int a = face / 2, side = face % 2;
        int lo[3] = {0, 0, 0}, hi[3] = {np[0], np[1], np[2]};
        lo[a] = side ? np[a] - NG : 0;
        hi[a] = side ? np[a] : NG;
        for (int k = lo[2]; k < hi[2]; ++k)
            for (int j = lo[1]; j < hi[1]; ++j)
                for (int i = lo[0]; i < hi[0]; ++i) {
                    long c = CELL(np, i, j, k);
                    s->P[nv * c + var] *= fac;
                }
    }
    static const int order[6] = {2, 3, 4, 5, 0, 1};
    for (int oi = 0; oi < 6; ++oi) {
        int face = order[oi];
        int a = face / 2, side = face % 2;
        if (a >= dims) continue;
        int kind = s->bc_kind[face];
        if (kind == OR_BC_FIXED) continue;
        const double* par = s->bc_par[face];
        int src = side ? np[a] - NG - 1 : NG;
        int lo[3] = {0, 0, 0}, hi[3] = {np[0], np[1], np[2]};
        lo[a] = side ? np[a] - NG : 0;
        hi[a] = side ? np[a] : NG;
        int b1 = (a + 1) % 3, b2 = (a + 2) % 3; /* in-plane axes */
        if (b1 > b2) { int tmp = b1; b1 = b2; b2 = tmp; }
        for (int k = lo[2]; k < hi[2]; ++k)
            for (int j = lo[1]; j < hi[1]; ++j)
                for (int i = lo[0]; i < hi[0]; ++i) {
                    int idx[3] = {i, j, k};
                    long c = CELL(np, i, j, k);
                    int inside = 0;
                    if (kind == OR_BC_NOZZLE) {
                        double r2 = 0.0;
                        double y1 = (b1 < dims) ? (idx[b1] - NG + 0.5) - par[1] : 0.0;
                        double y2 = (b2 < dims) ? (idx[b2] - NG + 0.5) - par[2] : 0.0;
                        r2 = y1 * y1 + y2 * y2;
                        inside = r2 < par[0] * par[0];
                    }
                    if (inside) {
                        s->P[nv * c + 0] = par[3];
                        s->P[nv * c + 1] = par[4];
                        for (int m = 0; m < dims; ++m) s->P[nv * c + 2 + m] = par[5 + m];
                    } else {
                        int sidx[3] = {i, j, k};
                        sidx[a] = src;
                        long cs = CELL(np, sidx[0], sidx[1], sidx[2]);
                        for (int v = 0; v < nv; ++v) s->P[nv * c + v] = s->P[nv * cs + v];
                    }
                }
    }
}

/* U_out = a*U0 + b*(Us - dt/dx*dFx - ...) for stages with a != 0 (SSP-RK3) */
static void update_rk(ornd_t* s, const double* U0, const double* Us, double* Uo, double dt, double a,
                      double b) {
    const int nv = s->nv, dims = s->dims;
    const int* np = s->n;
    long st[3] = {1, np[0], (long)np[0] * np[1]};
    int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    for (int ax = 0; ax < dims; ++ax) {
        lo[ax] = 3;
        hi[ax] = np[ax] - 3;
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = lo[2]; k < hi[2]; ++k)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int i = lo[0]; i < hi[0]; ++i) {
                long c = CELL(np, i, j, k);
                for (int v = 0; v < nv; ++v) {
                    double r = Us[nv * c + v];
                    for (int ax = 0; ax < dims; ++ax)
                        r = r - dt / s->dx[ax] * (s->F[ax][nv * c + v] - s->F[ax][nv * (c - st[ax]) + v]);
                    Uo[nv * c + v] = a * U0[nv * c + v] + b * r;
                }
            }
}

static void all_fluxes(ornd_t* s) {
    for (int a = 0; a < s->dims; ++a)
        ornd_k_fluxes(s->dims, s->n, s->P, s->g, s->floor_, s->F[a], a, s->recon, s->riemann);
}

static void c2p_and_limit(ornd_t* s, const double* U) {
    s->c2p_fail += k_utop(s->dims, s->n, U, s->P, s->g, s->n_iter, s->tol);
    ornd_k_limit(s->dims, s->n, s->P, s->floor_);
}

/* The time loop body of HARM_HLL (src/3dim/algos.jl:274-329,
 * src/2dim/algos.jl:256-310): boundary, then RK2 midpoint (reference) or
 * SSP-RK3 (extension). */
void ornd_step(ornd_t* s, double dt, int nsteps) {
    for (int n = 0; n < nsteps; ++n) {
        bc_fill(s, s->t);
        if (s->rk == 3) {
            all_fluxes(s);
            ornd_k_update(s->dims, s->n, s->U0, s->U1, dt, s->dx, s->F[0], s->F[1], s->F[2]);
            c2p_and_limit(s, s->U1);
            all_fluxes(s);
            update_rk(s, s->U0, s->U1, s->U1, dt, 0.75, 0.25);
            c2p_and_limit(s, s->U1);
            all_fluxes(s);
            update_rk(s, s->U0, s->U1, s->U0, dt, 1.0 / 3.0, 2.0 / 3.0);
            c2p_and_limit(s, s->U0);
        } else {
            all_fluxes(s);
            ornd_k_update(s->dims, s->n, s->U0, s->U1, dt / 2, s->dx, s->F[0], s->F[1], s->F[2]);
            c2p_and_limit(s, s->U1);
            all_fluxes(s);
            ornd_k_update(s->dims, s->n, s->U0, s->U0, dt, s->dx, s->F[0], s->F[1], s->F[2]);
            c2p_and_limit(s, s->U0);
        }
        s->t += dt;
    }
}

void ornd_get_prims(const ornd_t* s, double* P) { memcpy(P, s->P, sizeof(double) * s->nv * s->ncell); }
void ornd_get_cons(const ornd_t* s, double* U) { memcpy(U, s->U0, sizeof(double) * s->nv * s->ncell); }
double ornd_time(const ornd_t* s) { return s->t; }
int64_t ornd_c2p_failures(const ornd_t* s) { return s->c2p_fail; }
void ornd_destroy(ornd_t* s) {
    if (!s) return;
    free(s->P); free(s->U0); free(s->U1);
    for (int a = 0; a < 3; ++a) free(s->F[a]);
    free(s);
}
