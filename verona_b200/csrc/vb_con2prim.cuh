// Conservative-to-primitive recovery ("con2prim"), FP64, one cell per thread.
//
// c2p_1d / c2p_2d / c2p_3d restate the reference's three per-dimension
// algorithms in the reference's own evaluation order; c2p_w is the
// guess-driven 1D Newton on W = rho h gamma^2 with a bracketed fallback used
// by the learned-guess path. Every loop is bounded by n_iter (or a fixed cap);
// nothing here spins, traps or asserts -- failures are returned as codes.
#pragma once
#include "vb_ns.h"
#include "vb_physics.cuh"

namespace VB_NS {

VB_HD double vb_nan() { return NAN; }

// 3x3 solve of the 1D Newton (src/1dim/structs.jl:94; StaticArrays `\`):
// adjugate formula with the determinant as a column triple product.
VB_HD void solve3(const double* A, const double* b, double* x) {
#define a(r, c) A[((r)-1) + 3 * ((c)-1)]
    double c1 = a(2, 2) * a(3, 3) - a(3, 2) * a(2, 3);
    double c2 = a(3, 2) * a(1, 3) - a(1, 2) * a(3, 3);
    double c3 = a(1, 2) * a(2, 3) - a(2, 2) * a(1, 3);
    double det = a(1, 1) * c1 + a(2, 1) * c2 + a(3, 1) * c3;
    x[0] = qdiv((a(2, 2) * a(3, 3) - a(2, 3) * a(3, 2)) * b[0] + (a(1, 3) * a(3, 2) - a(1, 2) * a(3, 3)) * b[1] +
                    (a(1, 2) * a(2, 3) - a(1, 3) * a(2, 2)) * b[2],
                det);
    x[1] = qdiv((a(2, 3) * a(3, 1) - a(2, 1) * a(3, 3)) * b[0] + (a(1, 1) * a(3, 3) - a(1, 3) * a(3, 1)) * b[1] +
                    (a(1, 3) * a(2, 1) - a(1, 1) * a(2, 3)) * b[2],
                det);
    x[2] = qdiv((a(2, 1) * a(3, 2) - a(2, 2) * a(3, 1)) * b[0] + (a(1, 2) * a(3, 1) - a(1, 1) * a(3, 2)) * b[1] +
                    (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) * b[2],
                det);
#undef a
}

// 1D UtoP, src/1dim/structs.jl:78-105 (F_ptoU :48-54, Jacobian :32-46).
// The stop rule drops the last delta. Returns the iteration count.
VB_HD int c2p_1d(double g, int n_iter, double tol, const double* U, double* P) {
    double x1 = P[0], x2 = P[1], x3 = P[2];
    int it;
    for (it = 1; it <= n_iter; ++it) {
        double gam = sqrt(sq(x3) + 1.0);
        double w = g * x2 + x1;
        double f[3], J[9], dl[3];
        f[0] = gam * x1;
        f[1] = (g - 1.0) * x2 - sq(gam) * w;
        f[2] = x3 * gam * w;
        double gj = sqrt(1.0 + sq(x3));
        double wj = g * x2 + x1;
        J[0] = gj;
        J[3] = 0.0;
        J[6] = qdiv(x1 * x3, gj);
        J[1] = -sq(gj);
        J[4] = (g - 1.0) - sq(gj) * g;
        J[7] = -2.0 * x3 * wj;
        J[2] = gj * x3;
        J[5] = gj * x3 * g;
        J[8] = (2.0 * sq(x3) + 1.0) / gj * wj;
        f[0] = f[0] - U[0];
        f[1] = f[1] - U[1];
        f[2] = f[2] - U[2];
        solve3(J, f, dl);
        if (qsqrt(sq(dl[0]) + sq(dl[1]) + sq(dl[2])) < tol) break;
        x1 = x1 - dl[0];
        x2 = x2 - dl[1];
        x3 = x3 - dl[2];
    }
    P[0] = x1;
    P[1] = x2;
    P[2] = x3;
    return it;
}

// LU_dec_pivot!, src/2dim/structs.jl:121-208. Returns false on a row-wise
// singular matrix (the reference raises an error there).
VB_HD bool lu_pivot4(double* A, double* t, double* x) {
#define I4(i, j) (((j)-1) * 4 + (i)-1)
    // every loop is unrolled and the pivot row swap is a predicated swap with
    // each candidate row, so all indices are compile-time and A, t, rn stay
    // in registers
    double rn[4];
#pragma unroll
    for (int i = 1; i <= 4; ++i) {
        double am = 0.0;
#pragma unroll
        for (int j = 1; j <= 4; ++j) {
            double tmp = fabs(A[I4(i, j)]);
            if (tmp > am) am = tmp;
        }
        if (am == 0.0) return false;
        rn[i - 1] = 1.0 / am;
    }
#pragma unroll
    for (int k = 1; k <= 4; ++k) {
        int piv = k;
        double pv = fabs(A[I4(k, k)]) * rn[k - 1];
#pragma unroll
        for (int i = k + 1; i <= 4; ++i) {
            double tmp = fabs(A[I4(i, k)]) * rn[i - 1];
            if (tmp > pv) {
                pv = tmp;
                piv = i;
            }
        }
#pragma unroll
        for (int i = k + 1; i <= 4; ++i) {
            if (piv != i) continue;
#pragma unroll
            for (int j = 1; j <= 4; ++j) {
                double tmp = A[I4(k, j)];
                A[I4(k, j)] = A[I4(i, j)];
                A[I4(i, j)] = tmp;
            }
            double tmp = t[k - 1];
            t[k - 1] = t[i - 1];
            t[i - 1] = tmp;
            tmp = rn[k - 1];
            rn[k - 1] = rn[i - 1];
            rn[i - 1] = tmp;
        }
#pragma unroll
        for (int i = k + 1; i <= 4; ++i) {
            A[I4(i, k)] = qdiv(A[I4(i, k)], A[I4(k, k)]);
#pragma unroll
            for (int j = k + 1; j <= 4; ++j) A[I4(i, j)] = fma(-A[I4(i, k)], A[I4(k, j)], A[I4(i, j)]);
        }
    }
#pragma unroll
    for (int i = 1; i <= 4; ++i) {
        x[i - 1] = t[i - 1];
#pragma unroll
        for (int j = 1; j <= i - 1; ++j) x[i - 1] = fma(-A[I4(i, j)], x[j - 1], x[i - 1]);
    }
#pragma unroll
    for (int i = 4; i >= 1; --i) {
#pragma unroll
        for (int j = i + 1; j <= 4; ++j) x[i - 1] = fma(-A[I4(i, j)], x[j - 1], x[i - 1]);
        x[i - 1] = qdiv(x[i - 1], A[I4(i, i)]);
    }
#undef I4
    return true;
}

// 2D function_UtoP, src/2dim/structs.jl:249-330. Returns the iteration count,
// -1 on a singular Jacobian.
VB_HD int c2p_2d(double g, int n_iter, double tol, const double* U, double* P) {
    int it;
    for (it = 1; it <= n_iter; ++it) {
        double gam = sqrt(sq(P[2]) + sq(P[3]) + 1.0);
        double w = g * P[1] + P[0];
        double f[4], J[16], o[4];
        f[0] = gam * P[0] - U[0];
        f[1] = (g - 1.0) * P[1] - sq(gam) * w - U[1];
        f[2] = P[2] * gam * w - U[2];
        f[3] = P[3] * gam * w - U[3];
        J[0] = gam;
        J[4] = 0.0;
        J[8] = qdiv(P[0] * P[2], gam);
        J[12] = qdiv(P[0] * P[3], gam);
        J[1] = -sq(gam);
        J[5] = (g - 1.0) - sq(gam) * g;
        J[9] = -2.0 * P[2] * w;
        J[13] = -2.0 * P[3] * w;
        J[2] = gam * P[2];
        J[6] = gam * P[2] * g;
        J[10] = (2.0 * sq(P[2]) + sq(P[3]) + 1.0) / gam * w;
        J[14] = qdiv(P[2] * P[3], gam) * w;
        J[3] = gam * P[3];
        J[7] = gam * P[3] * g;
        J[11] = qdiv(P[2] * P[3], gam) * w;
        J[15] = (2.0 * sq(P[3]) + sq(P[2]) + 1.0) / gam * w;
        if (!lu_pivot4(J, f, o)) return -1;
        if (qsqrt(sq(o[0]) + sq(o[1]) + sq(o[2]) + sq(o[3])) < tol) break;
        P[0] = P[0] - o[0];
        P[1] = P[1] - o[1];
        P[2] = P[2] - o[2];
        P[3] = P[3] - o[3];
    }
    return it;
}

// LU_dec_5D! / LU_dec_2D!, src/3dim/structs.jl:144-214 (no pivoting)
template <int N> VB_HD void lu_plain(double* A, const double* t, double* x) {
#define IX(i, j) (((j)-1) * N + (i)-1)
    for (int k = 1; k <= N; ++k)
        for (int i = k + 1; i <= N; ++i) {
            A[IX(i, k)] = qdiv(A[IX(i, k)], A[IX(k, k)]);
            for (int j = k + 1; j <= N; ++j) A[IX(i, j)] -= A[IX(i, k)] * A[IX(k, j)];
        }
    for (int i = 1; i <= N; ++i) {
        x[i - 1] = t[i - 1];
        for (int j = 1; j <= i - 1; ++j) x[i - 1] -= A[IX(i, j)] * x[j - 1];
    }
    for (int i = N; i >= 1; --i) {
        for (int j = i + 1; j <= N; ++j) x[i - 1] -= A[IX(i, j)] * x[j - 1];
        x[i - 1] = qdiv(x[i - 1], A[IX(i, i)]);
    }
#undef IX
}

// Final primitive state from a converged W (src/3dim/structs.jl:598-609).
VB_HD void prims_from_W(double g, double D, double Qx, double Qy, double Qz, double S2, double W,
                        double* P) {
    double v2 = qdiv(S2, sq(W));
    double gm = 1.0 / sqrt(1.0 - v2);
    gm = jmin(gm, 50.0);
    double rho = jmax(1e-8, D / gm);
    double UU = jmax(1e-8, (W / sq(gm) - D / gm) / g);
    P[0] = rho;
    P[1] = UU;
    P[2] = qdiv(gm * Qx, W);
    P[3] = qdiv(gm * Qy, W);
    P[4] = qdiv(gm * Qz, W);
}

#ifdef __CUDA_ARCH__
#define VB_NOINLINE __noinline__
#else
#define VB_NOINLINE
#endif

static VB_NOINLINE __host__ __device__ int c2p_3d_tail(double g, int n_iter, double tol, const double* Uc, double* P);

// 3D function_UtoP, src/3dim/structs.jl:258-620: 1DW Newton -> Noble 2D
// Newton with line search -> 5x5 primitive Newton -> bisection. Returns the
// stage that converged (1..4) or -1 (cell set to NaN, as the reference does).
// The 1DW stage, which converges for almost every cell, is inline; the rest
// of the cascade (c2p_3d_tail) is an out-of-line call so that its registers
// do not count against the stencil kernels.
VB_HD int c2p_3d(double g, int n_iter, double tol, const double* Uc, double* P) {
    const double D = Uc[0], Q_t = Uc[1], Q_x = Uc[2], Q_y = Uc[3], Q_z = Uc[4];
    double S2, W, v2;
    {
        S2 = Q_x * Q_x + Q_y * Q_y + Q_z * Q_z;
        double gm = sqrt(sq(P[2]) + sq(P[3]) + sq(P[4]) + 1.0);
        double w_small = P[0] + g * P[1];
        W = w_small * sq(gm);
        const double W_max = 1e30;
        double W_min = qsqrt(S2) * (1.0 + 1e-15);
        for (int guard = 0; guard < 400 && qdiv(S2, sq(W)) >= 1.0 && W < W_max; ++guard) W *= 10.0;
        v2 = jmin(qdiv(S2, sq(W)), 1.0 - 1e-15);
        for (int it = 0; it < n_iter; ++it) {
            if (W < W_min) W = W_min;
            v2 = qdiv(S2, sq(W));
            if (v2 < 0.0)
                v2 = 0.0;
            else if (v2 > 1.0 - 1e-15)
                v2 = 1.0 - 1e-15;
            double k = (g - 1.0) / g;
            double bf = Q_t + W - k * (W * (1.0 - v2) - D * sqrt(1.0 - v2));
            double W3 = W * W * W;
            double bj = 1.0 - ((g - 1.0) / g) * (1.0 - v2) -
                        ((g - 1.0) / g) * (W * qdiv(2.0 * S2, W3) - D * qdiv(S2, W3 * sqrt(1.0 - v2)));
            double dW = qdiv(bf, bj);
            double Wp = W - dW;
            if (Wp < W_min)
                W = 0.5 * (W + W_min);
            else
                W = Wp;
            if (dW < 0) dW = -dW;
            if (sq(dW) < sq(tol)) {
                prims_from_W(g, D, Q_x, Q_y, Q_z, S2, W, P);
                return 1;
            }
        }
    }
    return c2p_3d_tail(g, n_iter, tol, Uc, P);
}

// Stages 2-4 of the 3D cascade (src/3dim/structs.jl:345-619), entered when
// the 1DW Newton did not converge; P still holds the guess.
static VB_NOINLINE __host__ __device__ int c2p_3d_tail(double g, int n_iter, double tol, const double* Uc, double* P) {
    const double D = Uc[0], Q_t = Uc[1], Q_x = Uc[2], Q_y = Uc[3], Q_z = Uc[4];
    const bool conv1 = false;
    bool conv2 = false, conv5 = false, convb = false;
    double S2, W, v2;
    {
        S2 = Q_x * Q_x + Q_y * Q_y + Q_z * Q_z;
        double gm = sqrt(sq(P[2]) + sq(P[3]) + sq(P[4]) + 1.0);
        double w_small = P[0] + g * P[1];
        W = w_small * sq(gm);
        const double W_max = 1e30;
        for (int guard = 0; guard < 400 && S2 / sq(W) >= 1.0 && W < W_max; ++guard) W *= 10.0;
        v2 = jmin(S2 / sq(W), 1.0 - 1e-15);
        for (int it = 0; it < n_iter; ++it) {
            double W_old = W, v2_old = v2;
            double k = (g - 1.0) / g;
            double f[2], J[4], o[2];
            f[0] = v2 - S2 / sq(W);
            f[1] = Q_t + W - k * (W * (1.0 - v2) - D * sqrt(1.0 - v2));
            J[0] = 2.0 * S2 / (W * W * W);
            J[1] = 1.0 - k * (1.0 - v2);
            J[2] = 1.0;
            J[3] = k * (W - D / (2.0 * sqrt(1.0 - v2)));
            lu_plain<2>(J, f, o);
            double dW = o[0], dv2 = o[1];
            double alpha = 1.0;
            bool ok = false;
            for (int ls = 0; ls < 10; ++ls) {
                double s = sqrt(W - alpha * dW);
                double Wc = sq(s);
                double v2c = v2 - alpha * dv2;
                if (Wc <= 0 || Wc > W_max) Wc = W_old;
                if (v2c < 0)
                    v2c = 0.0;
                else if (v2c >= 1)
                    v2c = 1.0 - 1e-15;
                double r1 = v2c - S2 / sq(Wc);
                double r2 = Q_t + Wc - k * (Wc * (1.0 - v2c) - D * sqrt(1.0 - v2c));
                double errc = sq(r1) + sq(r2);
                double r1o = v2 - S2 / sq(W);
                double r2o = Q_t + W - k * (W * (1.0 - v2) - D * sqrt(1.0 - v2));
                double erro = sq(r1o) + sq(r2o);
                if (errc <= erro) {
                    W = Wc;
                    v2 = v2c;
                    ok = true;
                    break;
                } else {
                    alpha *= 0.5;
                }
            }
            if (!ok) {
                W = W_old;
                v2 = v2_old;
            }
            double relW = sqrt(sq(W - W_old)) / jmax(fabs(W_old), sq(tol));
            double relv2 = sqrt(sq(v2 - v2_old)) / jmax(fabs(v2_old), sq(tol));
            if (relW + relv2 < tol) {
                conv2 = true;
                break;
            }
        }
    }
    if (!conv1 && !conv2) {
        for (int it = 0; it < n_iter; ++it) {
            double gam = sqrt(sq(P[2]) + sq(P[3]) + sq(P[4]) + 1.0);
            double w = g * P[1] + P[0];
            double f[5], J[25], o[5];
            f[0] = gam * P[0] - Uc[0];
            f[1] = (g - 1.0) * P[1] - sq(gam) * w - Uc[1];
            f[2] = P[2] * gam * w - Uc[2];
            f[3] = P[3] * gam * w - Uc[3];
            f[4] = P[4] * gam * w - Uc[4];
            J[0] = gam;
            J[5] = 0.0;
            J[10] = P[2] * P[0] / gam;
            J[15] = P[3] * P[0] / gam;
            J[20] = P[4] * P[0] / gam;
            J[1] = -sq(gam);
            J[6] = g * (-sq(gam)) + g - 1.0;
            J[11] = -2.0 * P[2] * w;
            J[16] = -2.0 * P[3] * w;
            J[21] = -2.0 * P[4] * w;
            J[2] = P[2] * gam;
            J[7] = g * P[2] * gam;
            J[12] = sq(P[2]) * w / gam + w * gam;
            J[17] = P[2] * P[3] * w / gam;
            J[22] = P[2] * P[4] * w / gam;
            J[3] = P[3] * gam;
            J[8] = g * P[3] * gam;
            J[13] = P[2] * P[3] * w / gam;
            J[18] = sq(P[3]) * w / gam + w * gam;
            J[23] = P[3] * P[4] * w / gam;
            J[4] = P[4] * gam;
            J[9] = g * P[4] * gam;
            J[14] = P[2] * P[4] * w / gam;
            J[19] = P[3] * P[4] * w / gam;
            J[24] = sq(P[4]) * w / gam + w * gam;
            lu_plain<5>(J, f, o);
            if (sq(o[0]) + sq(o[1]) + sq(o[2]) + sq(o[3]) + sq(o[4]) < sq(tol)) {
                if (isfinite(P[0]) && isfinite(P[1]) && isfinite(P[2]) && isfinite(P[3]) && isfinite(P[4])) {
                    conv5 = true;
                    P[0] = jmax(1e-8, P[0]);
                    P[1] = jmax(1e-8, P[1]);
                    double gm = sqrt(sq(P[2]) + sq(P[3]) + sq(P[4]) + 1.0);
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
    if (!conv1 && !conv2 && !conv5) {
        S2 = Q_x * Q_x + Q_y * Q_y + Q_z * Q_z;
        double k = (g - 1.0) / g;
        double W_min = jmax(1e-15, sqrt(S2));
        double W_max = W_min * 10.0;
#define RES(Wv) (Q_t + (Wv) - k * ((Wv) * (1.0 - S2 / sq(Wv)) - D * sqrt(jmax(0.0, 1.0 - S2 / sq(Wv)))))
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
                if (sq(fm) < sq(1e-6)) {
                    convb = true;
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
    if (conv1 || conv2 || convb) prims_from_W(g, D, Q_x, Q_y, Q_z, S2, W, P);
    if (!conv1 && !conv2 && !conv5 && !convb) {
        for (int v = 0; v < 5; ++v) P[v] = vb_nan();
        return -1;
    }
    return conv1 ? 1 : conv2 ? 2 : conv5 ? 3 : 4;
}

// ---- guess-driven W Newton with a bracketed fallback -------------------------
// Residual of the 1DW scheme (Noble et al. 2006) written in W alone:
// f(W) = Q_t + W - k (W (1 - v^2) - D sqrt(1 - v^2)), v^2 = S^2 / W^2.
// Evaluated from 1/W and 1/sqrt(1 - v^2), one divide and one reciprocal square
// root per call: with a = 1 - v^2, s = sqrt(a) = a / sqrt(a),
//   f  = Q_t + W - k (W a - D s),
//   f' = 1 - k (a + 2 v^2 - D v^2 / (W s))       (d v^2 / dW = -2 v^2 / W),
// k = (Gamma - 1) / Gamma.
struct WRes {
    double f, df;
};
// Reciprocal and reciprocal square root of the W Newton: the hardware
// approximations of sm_100a (rcp.approx.ftz.f64, rsqrt.approx.ftz.f64) refined
// by two Newton-Raphson steps each; a step doubles the correct bits (a 23-bit
// seed ends within an ulp, checked by emulation), and the recovered states
// equal those of the IEEE-divide form to the W tolerance on every cell of the
// exact-answer test of the W Newton:
//   1/x:       e = 1 - x y,              y <- y + y e
//   1/sqrt(a): t = 1/2 - (a/2) y^2,      y <- y + y t
// For positive normal arguments (W, 1 - v^2 > 0 here; a zero or NaN argument
// gives NaN, which the Newton treats as a failed step). The IEEE divide and
// square root sequences carry special-case handling this loop does not need;
// the reference con2prim cascade keeps them.
VB_HD double rcp_nr(double x) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
#else
    return 1.0 / x;
#endif
}
VB_HD double rsqrt_d(double a) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    const double h = 0.5 * a;
    double t = fma(-h * y, y, 0.5);
    y = fma(y, t, y);
    t = fma(-h * y, y, 0.5);
    return fma(y, t, y);
#else
    return 1.0 / sqrt(a);
#endif
}
VB_HD WRes w_residual(double k, double D, double Q_t, double S2, double W) {
    const double iW = rcp_nr(W);
    double v2 = S2 * iW * iW;
    if (v2 > 1.0 - 1e-15) v2 = 1.0 - 1e-15;
    const double a = 1.0 - v2;
    const double rs = rsqrt_d(a);
    WRes r;
    r.f = Q_t + W - k * (W * a - D * (a * rs));
    r.df = 1.0 - k * (a + 2.0 * v2 - D * v2 * iW * rs);
    return r;
}

// The final-state formula of prims_from_W (src/3dim/structs.jl:334-340) from
// 1/W and 1/sqrt(1 - v^2) (the W Newton's refinement, not the reference
// cascade, whose prims_from_W keeps the reference's operation order).
VB_HD void prims_from_W_fast(double g, double D, double Qx, double Qy, double Qz, double S2, double W, double* P) {
    const double iW = rcp_nr(W);
    const double a = 1.0 - S2 * iW * iW;
    const double rs = rsqrt_d(a);
    const double gm = jmin(rs, 50.0);
    const double igm = gm < rs ? 1.0 / 50.0 : a * rs;  // 1 / gm
    P[0] = jmax(1e-8, D * igm);
    P[1] = jmax(1e-8, (W * igm * igm - D * igm) * rcp_nr(g));
    const double f = gm * iW;
    P[2] = Qx * f;
    P[3] = Qy * f;
    P[4] = Qz * f;
}

// Newton on W from a guess, to |dW| <= rtol * W, at most max_newton steps;
// then a safeguarded (bracketed) Newton from the physical bracket
// [sqrt(S^2)(1+1e-15), W_hi]. Writes the primitive state through the
// reference's final-state formula and floors. Returns total iterations, or
// -(iterations) if both failed (cell set to NaN). *used_fallback is set when
// the bracketed phase ran.
VB_HD int c2p_w(double g, const double* Uc, double W0, double rtol, int max_newton, int max_bracket,
                double* P, int* used_fallback) {
    const double D = Uc[0], Q_t = Uc[1];
    const double Qx = Uc[2], Qy = Uc[3], Qz = Uc[4];
    const double S2 = Qx * Qx + Qy * Qy + Qz * Qz;
    const double Wlo0 = qsqrt(S2) * (1.0 + 1e-15);
    const double k = (g - 1.0) / g;
    double W = W0;
    int it = 0;
    *used_fallback = 0;
    if (!(W > Wlo0) || !isfinite(W)) W = fmax(Wlo0 * 1.0000001, D - Q_t);
    for (; it < max_newton; ++it) {
        WRes r = w_residual(k, D, Q_t, S2, W);
        double dW = r.f * rcp_nr(r.df);
        double Wn = W - dW;
        if (!(Wn > Wlo0)) Wn = 0.5 * (W + Wlo0);
        bool done = fabs(Wn - W) <= rtol * fabs(Wn);
        W = Wn;
        if (done && isfinite(W)) {
            prims_from_W_fast(g, D, Qx, Qy, Qz, S2, W, P);
            return it + 1;
        }
    }
    // Bracketed Newton: f(Wlo) <= 0 for a physical state; grow Whi until f > 0.
    *used_fallback = 1;
    double lo = Wlo0, hi = fmax(2.0 * Wlo0, D - Q_t + 1.0);
    WRes rl = w_residual(k, D, Q_t, S2, lo);
    WRes rh = w_residual(k, D, Q_t, S2, hi);
    for (int grow = 0; grow < 200 && rh.f * rl.f > 0.0; ++grow) {
        hi *= 4.0;
        rh = w_residual(k, D, Q_t, S2, hi);
    }
    if (!(rh.f * rl.f <= 0.0)) {
        for (int v = 0; v < 5; ++v) P[v] = vb_nan();
        return -(it + 1);
    }
    W = (W > lo && W < hi) ? W : 0.5 * (lo + hi);
    for (int b = 0; b < max_bracket; ++b, ++it) {
        WRes r = w_residual(k, D, Q_t, S2, W);
        if ((r.f < 0.0) == (rl.f < 0.0)) {
            lo = W;
            rl = r;
        } else {
            hi = W;
        }
        double Wn = W - r.f / r.df;
        if (!(Wn > lo && Wn < hi)) Wn = 0.5 * (lo + hi);
        if (fabs(Wn - W) <= rtol * fabs(Wn) || (hi - lo) <= rtol * hi) {
            prims_from_W_fast(g, D, Qx, Qy, Qz, S2, Wn, P);
            return it + 1;
        }
        W = Wn;
    }
    for (int v = 0; v < 5; ++v) P[v] = vb_nan();
    return -(it + 1);
}

// ---- precision-gated con2prim of the FP32-bulk form ----------------------------
// In the FP32-bulk form the recovered primitives are stored in FP32 and feed
// only the FP32 reconstruction; U and the RK accumulation stay FP64. Where the
// inversion U -> P is well conditioned an FP32 Newton is enough, and FP64 is
// kept for the cells where it is not: high Lorentz factor (1 - v^2 loses
// digits) and cold moving gas (p is then a small difference of kinetic and
// total energy). The FP32 Newton solves for the pressure with a residual free
// of O(D) - O(D) cancellations: with E = D + tau (tau = E - D formed in FP64),
// W = E + p, v^2 = S^2 / W^2, s = sqrt(1 - v^2) and k' = Gamma / (Gamma - 1),
//   f(p) = (tau + p)(1 - v^2) - k' p - D v^2 s / (1 + s)
// (the W residual of the 1DW scheme, src/3dim/structs.jl:273-343, divided by
// -k = -(Gamma - 1) / Gamma, with D (1 - v^2) - D s rewritten as
// -D v^2 s / (1 + s)),
//   f'(p) = (1 - v^2) + (tau + p) 2 v^2 / W - k' + D h'(v^2) 2 v^2 / W,
//   h'(v^2) = s / (1 + s) - v^2 / (2 s (1 + s)^2).
// Gate: p0 > 0, v^2 < 1/2 (Lorentz factor below sqrt 2) and v^2 D < 10 p
// (kinetic over thermal energy below about 10), checked on the guess and
// again on the converged pressure (a W guess a little off can put p0 far
// above a cold gas's pressure); a cell that fails either check, or whose
// Newton does not converge in C2P32_MAX_IT steps, goes to the FP64 W Newton.
// The reciprocals and the reciprocal square root are the sm_100a hardware
// approximations (relative error below 2^-22, as FP32 rounding), four per
// iteration; the Newton stops once a step is below 1e-5 of p, where its
// quadratic convergence leaves an error far below FP32 rounding. Every
// operation is an explicit instruction (inline PTX or a round-to-nearest
// intrinsic), so the result does not depend on the contraction or division
// flags of the translation unit: the fused and the two-kernel learned forms
// agree bit for bit.
constexpr float C2P32_MAX_V2 = 0.5f;
constexpr float C2P32_MAX_KIN = 10.0f;
constexpr float C2P32_RTOL = 1e-5f;
constexpr int C2P32_MAX_IT = 6;

#ifdef __CUDA_ARCH__
VB_HD float f_add(float a, float b) { return __fadd_rn(a, b); }
VB_HD float f_sub(float a, float b) { return __fsub_rn(a, b); }
VB_HD float f_mul(float a, float b) { return __fmul_rn(a, b); }
VB_HD float f_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
VB_HD float f_rcp(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
VB_HD float f_rsqrt(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
#else
VB_HD float f_add(float a, float b) { return a + b; }
VB_HD float f_sub(float a, float b) { return a - b; }
VB_HD float f_mul(float a, float b) { return a * b; }
VB_HD float f_fma(float a, float b, float c) { return fmaf(a, b, c); }
VB_HD float f_rcp(float x) { return 1.0f / x; }
VB_HD float f_rsqrt(float x) { return 1.0f / sqrtf(x); }
#endif

// The conserved state of one cell as the FP32 Newton sees it.
struct C2P32In {
    float D, tau, E, S2, Sx, Sy, Sz;
};

// the gate's conditions at pressure p with v^2 = S^2 / W^2
VB_HD bool c2p32_admits(const C2P32In& in, float v2, float p) {
    return v2 < C2P32_MAX_V2 && f_mul(v2, in.D) < f_mul(C2P32_MAX_KIN, p);
}

// Gate of the FP32 solve from the guess W0 (FP32, the learned guess as both
// learned forms round it): true, with the FP32 inputs and the pressure guess
// p0, when the cell qualifies.
VB_HD bool c2p32_gate(const double* U, float W0, C2P32In& in, float& p0) {
    const double E = -U[1];
    const double S2 = U[2] * U[2] + U[3] * U[3] + U[4] * U[4];
    p0 = (float)((double)W0 - E);
    in.D = (float)U[0];
    in.tau = (float)(E - U[0]);
    in.E = (float)E;
    in.S2 = (float)S2;
    in.Sx = (float)U[2];
    in.Sy = (float)U[3];
    in.Sz = (float)U[4];
    if (!(p0 > 0.0f) || !(W0 > 0.0f) || !(in.D > 0.0f) || !(in.tau > 0.0f)) return false;
    const float iW = f_rcp(W0);
    return c2p32_admits(in, f_mul(f_mul(in.S2, iW), iW), p0);
}

// FP32 Newton on the pressure from p0; returns the iterations on convergence
// (a step below C2P32_RTOL p, and the gate holding at the root), else
// -C2P32_MAX_IT.
VB_HD int c2p_p32(float g, const C2P32In& in, float p0, float& p_out) {
    const float kp = f_mul(g, f_rcp(f_sub(g, 1.0f)));
    float p = p0;
    for (int it = 1; it <= C2P32_MAX_IT; ++it) {
        const float iW = f_rcp(f_add(in.E, p));
        const float v2 = f_mul(f_mul(in.S2, iW), iW);
        const float a = f_sub(1.0f, v2);
        if (!(a > 0.0f)) return -C2P32_MAX_IT;
        const float rs = f_rsqrt(a);          // 1 / s
        const float sr = f_mul(a, rs);        // s
        const float q = f_rcp(f_add(1.0f, sr));
        const float h = f_mul(sr, q);         // s / (1 + s)
        const float tp = f_add(in.tau, p);
        const float Dv2 = f_mul(in.D, v2);
        // f = tp a - k' p - D v^2 h
        const float f = f_sub(f_fma(tp, a, f_mul(-kp, p)), f_mul(Dv2, h));
        const float dv2 = f_mul(-2.0f, f_mul(v2, iW));  // d v^2 / dp
        // h'(v^2) = h - v^2 q^2 / (2 s)
        const float dh = f_sub(h, f_mul(f_mul(f_mul(0.5f, v2), f_mul(q, q)), rs));
        const float df = f_sub(f_sub(f_fma(-tp, dv2, a), kp), f_mul(f_mul(in.D, dh), dv2));
        const float dp = f_mul(f, f_rcp(df));
        float pn = f_sub(p, dp);
        if (!(pn > 0.0f)) pn = f_mul(0.5f, p);
        const bool done = fabsf(f_sub(pn, p)) <= f_mul(C2P32_RTOL, pn);
        p = pn;
        if (done) {
            const float iWn = f_rcp(f_add(in.E, p));
            if (!c2p32_admits(in, f_mul(f_mul(in.S2, iWn), iWn), p)) return -C2P32_MAX_IT;
            p_out = p;
            return it;
        }
    }
    return -C2P32_MAX_IT;
}

// Primitives from the converged FP32 pressure, with the 3D floors of the
// reference's final-state formula (src/3dim/structs.jl:598-609).
VB_HD void prims_from_p32(float g, const C2P32In& in, float p, double* P) {
    const float iW = f_rcp(f_add(in.E, p));
    const float v2 = f_mul(f_mul(in.S2, iW), iW);
    const float a = f_sub(1.0f, v2);
    const float rs = f_rsqrt(a);   // Lorentz factor (below sqrt 2: no cap)
    const float fac = f_mul(iW, rs);  // Lorentz factor / W
    P[0] = (double)fmaxf(1e-8f, f_mul(in.D, f_mul(a, rs)));
    P[1] = (double)fmaxf(1e-8f, f_mul(p, f_rcp(f_sub(g, 1.0f))));
    P[2] = (double)f_mul(in.Sx, fac);
    P[3] = (double)f_mul(in.Sy, fac);
    P[4] = (double)f_mul(in.Sz, fac);
}

// The learned guess's refinement with the precision gate: the FP32 pressure
// Newton where c2p32_gate admits the cell (and it converges), else the FP64 W
// Newton with its bracketed fallback (c2p_w). *fp64 = 1 where the FP64 Newton
// ran. Returns the iterations (negative on failure).
VB_HD int c2p_w_gated(double g, const double* U, float W0f, double rtol, int max_newton, int max_bracket, bool gate,
                      double* P, int* used_fallback, int* fp64) {
    if (gate) {
        C2P32In in;
        float p0;
        if (c2p32_gate(U, W0f, in, p0)) {
            float pp;
            const int r = c2p_p32((float)g, in, p0, pp);
            if (r > 0) {
                prims_from_p32((float)g, in, pp, P);
                *used_fallback = 0;
                *fp64 = 0;
                return r;
            }
        }
    }
    *fp64 = 1;
    return c2p_w(g, U, (double)W0f, rtol, max_newton, max_bracket, P, used_fallback);
}

// The FP32 part of c2p_w_gated alone: true, with the primitives in P and the
// iterations in *iters, when the gate admits the cell and the FP32 Newton
// converges; false when the cell needs the FP64 W Newton.
VB_HD bool c2p_try_fp32(double g, const double* U, float W0f, double* P, int* iters) {
    C2P32In in;
    float p0;
    if (!c2p32_gate(U, W0f, in, p0)) return false;
    float pp;
    const int r = c2p_p32((float)g, in, p0, pp);
    if (r <= 0) return false;
    prims_from_p32((float)g, in, pp, P);
    *iters = r;
    return true;
}

}  // namespace vb
