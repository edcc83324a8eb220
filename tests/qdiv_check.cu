// The FP64 zero-dividend forms of vb_physics.cuh (qdiv, qdiv_pos, qsqrt)
// against the IEEE divide and square root, bit for bit, over special and
// ordinary values: signed zeros, subnormals, normals of both signs, the
// infinities and NaN, as dividends and divisors. qdiv must equal a / b for
// every pair except a zero dividend over a subnormal divisor below 2^-1024
// (documented: its reciprocal overflows); qdiv_pos must equal it wherever the
// divisor is positive or +inf; qsqrt must equal sqrt everywhere. NaN results
// compare as NaN (payloads are not part of the contract). Built by nvcc and
// run by tests/test_index_host.py: on the host by default, on the device
// (the same comparisons in a kernel, where the divide is the GPU's IEEE
// sequence and the opaque move is real) with the argument "device".
// Prints "ok" or the first mismatches.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "vb_physics.cuh"

using namespace vb;

static const double kVals[] = {0.0,     -0.0,     1.0,       -1.0,     6.0,      1e-42,     -3.5e-200, 1e300,
                               -1e300,  5e-324,   -5e-324,   2.2e-308, 1e-310,   4.9e-309,  INFINITY,  -INFINITY,
                               NAN,     0.1,      -7.25,     1e-16,    123456.0, 1e154,     -1e-154};
constexpr int kN = sizeof(kVals) / sizeof(kVals[0]);

__host__ __device__ inline bool same(double x, double y) {
    if (x != x || y != y) return (x != x) && (y != y);
    unsigned long long a, b;
    memcpy(&a, &x, 8);
    memcpy(&b, &y, 8);
    return a == b;
}

// a zero dividend over a divisor whose reciprocal overflows
__host__ __device__ inline bool excepted(double a, double b) { return a == 0.0 && b != 0.0 && fabs(b) <= 0x1p-1024; }

// counts mismatches of the three forms over all pairs; records the first few
__host__ __device__ int check_all(const double* v, int n, int* bad_i, int* bad_j, int* bad_k, int max_bad) {
    int bad = 0;
    for (int i = 0; i < n; ++i) {
        const double a = v[i];
        if (!same(qsqrt(a), sqrt(a))) {
            if (bad < max_bad) bad_i[bad] = i, bad_j[bad] = -1, bad_k[bad] = 2;
            ++bad;
        }
        for (int j = 0; j < n; ++j) {
            const double b = v[j];
            const double ref = a / b;
            if (!excepted(a, b) && !same(qdiv(a, b), ref)) {
                if (bad < max_bad) bad_i[bad] = i, bad_j[bad] = j, bad_k[bad] = 0;
                ++bad;
            }
            if ((b > 0.0) && !same(qdiv_pos(a, b), ref)) {
                if (bad < max_bad) bad_i[bad] = i, bad_j[bad] = j, bad_k[bad] = 1;
                ++bad;
            }
        }
    }
    return bad;
}

__global__ void k_check(const double* v, int n, int* out) {
    out[0] = check_all(v, n, out + 1, out + 9, out + 17, 8);
}

int main(int argc, char** argv) {
    const bool device = argc > 1 && strcmp(argv[1], "device") == 0;
    int res[25] = {0};
    if (!device) {
        res[0] = check_all(kVals, kN, res + 1, res + 9, res + 17, 8);
    } else {
        double* dv = nullptr;
        int* dout = nullptr;
        if (cudaMalloc(&dv, sizeof(kVals)) != cudaSuccess || cudaMalloc(&dout, sizeof(res)) != cudaSuccess) {
            std::printf("cudaMalloc failed\n");
            return 1;
        }
        cudaMemcpy(dv, kVals, sizeof(kVals), cudaMemcpyHostToDevice);
        cudaMemset(dout, 0, sizeof(res));
        k_check<<<1, 1>>>(dv, kN, dout);
        if (cudaDeviceSynchronize() != cudaSuccess) {
            std::printf("kernel failed\n");
            return 1;
        }
        cudaMemcpy(res, dout, sizeof(res), cudaMemcpyDeviceToHost);
        cudaFree(dv);
        cudaFree(dout);
    }
    if (res[0]) {
        const char* form[3] = {"qdiv", "qdiv_pos", "qsqrt"};
        for (int k = 0; k < res[0] && k < 8; ++k) {
            const int i = res[1 + k], j = res[9 + k];
            std::printf("%s(%.17g, %.17g) differs\n", form[res[17 + k]], kVals[i], j >= 0 ? kVals[j] : 0.0);
        }
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
