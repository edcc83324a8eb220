// Host-side check of the W Newton with its bracketed fallback (c2p_w), built
// by nvcc as a host program and run on the CPU by tests/test_index_host.py.
// States P over the learned guess's training ranges (Lorentz factor up to
// 40) go through U = PtoU(P) and back through c2p_w three ways:
//   - from a guess 0.1 % off the true W (Newton only),
//   - from the state-only cold start D + E,
//   - with max_newton = 0, so the bracketed phase alone solves every cell.
// Every recovered state must reproduce U to 1e-9 of its magnitude (the
// comparison through U avoids the cancellation that makes u ill-conditioned
// when p << rho), and the third form must report the fallback on every cell.
// Prints "ok" or the first failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "vb_con2prim.cuh"

using namespace vb;

static unsigned long long rng_state = 0x9E3779B97F4A7C15ull;
static double urand() {  // splitmix64 -> [0, 1)
    unsigned long long z = (rng_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (z >> 11) * (1.0 / 9007199254740992.0);
}

int main() {
    const int n = 20000;
    int bad = 0, fb_seen[3] = {0, 0, 0};
    for (int i = 0; i < n && bad < 5; ++i) {
        const double g = (i & 1) ? 4.0 / 3.0 : 5.0 / 3.0;
        const double rho = std::pow(10.0, -4.0 + 5.0 * urand());
        const double p = rho * std::pow(10.0, -4.0 + 6.0 * urand());
        const double lor = std::pow(10.0, std::log10(40.0) * urand());
        double d[3] = {urand() - 0.5, urand() - 0.5, urand() - 0.5};
        const double nd = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + 1e-300;
        const double um = std::sqrt(lor * lor - 1.0);
        double P[5] = {rho, p / (g - 1.0), um * d[0] / nd, um * d[1] / nd, um * d[2] / nd};
        double U[5];
        prim2con<3>(g, P, U);
        const double W = (P[0] + g * P[1]) * lor * lor;
        const double starts[3] = {W * (1.0 + 1e-3), U[0] - U[1], W * (1.0 + 1e-3)};
        const int max_newton[3] = {8, 8, 0};
        for (int f = 0; f < 3; ++f) {
            double R[5];
            int fb = 0;
            const int it = c2p_w(g, U, starts[f], 1e-12, max_newton[f], 400, R, &fb);
            fb_seen[f] += fb;
            double V[5], scale = 0.0, err = 0.0;
            prim2con<3>(g, R, V);
            for (int v = 0; v < 5; ++v) {
                scale = std::fmax(scale, std::fabs(U[v]));
                err = std::fmax(err, std::fabs(V[v] - U[v]));
            }
            // the 3D floors (rho, u >= 1e-8) change U by design: skip states below them
            const bool floored = rho / lor < 2e-8 || p / (g - 1.0) < 2e-8;
            if (it <= 0 || !(err <= 1e-9 * scale || floored) || (f == 2 && !fb)) {
                std::printf("form %d state %d: it %d fb %d err %.3e scale %.3e rho %.3e p %.3e lorentz %.3f\n", f, i,
                            it, fb, err, scale, rho, p, lor);
                ++bad;
            }
        }
    }
    if (bad) return 1;
    if (fb_seen[2] == 0) {
        std::printf("the bracketed phase never ran\n");
        return 1;
    }
    // the precision-gated refinement of the FP32-bulk learned path
    // (c2p_w_gated): states with Lorentz factor up to 3 and p / rho down to
    // 1e-6, guesses 0.1 % off in W (for cold gas that puts the guessed
    // pressure far above the true one), rounded to FP32. Cells the gate admits are solved in FP32 and must
    // match the exact state to FP32 accuracy (rho and the four-velocity to
    // 1e-6 relative, the internal energy to 2e-5); the rest go to the FP64 W
    // Newton and must reproduce U to 1e-9.
    int n32 = 0, n64 = 0;
    for (int i = 0; i < n && bad < 5; ++i) {
        const double g = (i & 1) ? 4.0 / 3.0 : 5.0 / 3.0;
        const double rho = std::pow(10.0, -4.0 + 5.0 * urand());
        const double p = rho * std::pow(10.0, -6.0 + 8.0 * urand());
        const double lor = std::pow(10.0, std::log10(3.0) * urand());
        double d[3] = {urand() - 0.5, urand() - 0.5, urand() - 0.5};
        const double nd = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + 1e-300;
        const double um = std::sqrt(lor * lor - 1.0);
        double P[5] = {rho, p / (g - 1.0), um * d[0] / nd, um * d[1] / nd, um * d[2] / nd};
        double U[5];
        prim2con<3>(g, P, U);
        const double W = (P[0] + g * P[1]) * lor * lor;
        const float W0 = (float)(W * (1.0 + 1e-3 * (2.0 * urand() - 1.0)));
        double R[5];
        int fb = 0, f64 = -1;
        const int it = c2p_w_gated(g, U, W0, 1e-12, 8, 400, true, R, &fb, &f64);
        const bool floored = rho / lor < 2e-8 || p / (g - 1.0) < 2e-8;
        bool good = it > 0;
        if (good && !f64) {
            ++n32;
            const double er = std::fabs(R[0] - P[0]) / P[0];
            const double eu = std::fabs(R[1] - P[1]) / P[1];
            double ev = 0.0;
            for (int v = 2; v < 5; ++v) ev = std::fmax(ev, std::fabs(R[v] - P[v]));
            good = floored || (er <= 1e-6 && eu <= 2e-5 && ev <= 1e-6 * lor);
        } else if (good) {
            ++n64;
            double V[5], scale = 0.0, err = 0.0;
            prim2con<3>(g, R, V);
            for (int v = 0; v < 5; ++v) {
                scale = std::fmax(scale, std::fabs(U[v]));
                err = std::fmax(err, std::fabs(V[v] - U[v]));
            }
            good = floored || err <= 1e-9 * scale;
        }
        if (!good) {
            std::printf("gated state %d: it %d fp64 %d rho %.3e p %.3e lorentz %.3f -> %.9e %.9e\n", i, it, f64, rho, p,
                        lor, R[0], R[1] * (g - 1.0));
            ++bad;
        }
    }
    if (bad) return 1;
    if (n32 < n / 10 || n64 < n / 10) {
        std::printf("gate split %d FP32 / %d FP64: both paths must run\n", n32, n64);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
