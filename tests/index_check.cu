// Host-side check of the index maps the stage kernels use on the pitched SoA
// layout: the interior cell map (CellMap, multiply-high division) and the
// dense-to-pitched map of the layout-conversion kernels (soa_index), against
// plain loops, for grids with and without row padding. Built by nvcc and run
// on the CPU by tests/test_index_host.py; prints "ok" or the first mismatch.
#include <cstdio>
#include <cstdlib>

#include "vb_stage.cuh"

using namespace vb;

static int check_grid(int N0, int N1, int N2, int pad) {
    const int n0 = N0 + 2 * NG, n1 = N1 + 2 * NG, n2 = N2 + 2 * NG;
    Grid g{};
    g.dims = 3;
    g.nv = 5;
    g.n[0] = n0;
    g.n[1] = n1;
    g.n[2] = n2;
    g.sy = pad ? (n0 + 3) / 4 * 4 : n0;
    g.sz = g.sy * n1;
    g.vs = (g.sz * n2 + 31) / 32 * 32;
    CellMap cm;
    cm.init(N0, N1, g.sy, g.sz, NG);
    long long e = 0;
    for (int k = 0; k < N2; ++k)
        for (int j = 0; j < N1; ++j)
            for (int i = 0; i < N0; ++i, ++e) {
                const long long want = (i + NG) + g.sy * (j + NG) + g.sz * (k + NG);
                const long long got = cm.padded((uint32_t)e);
                if (got != want) {
                    printf("CellMap %d %d %d pad %d: e %lld -> %lld, want %lld\n", N0, N1, N2, pad, e, got, want);
                    return 1;
                }
            }
    long long c = 0;
    for (int k = 0; k < n2; ++k)
        for (int j = 0; j < n1; ++j)
            for (int i = 0; i < n0; ++i, ++c) {
                const long long want = i + g.sy * j + g.sz * k;
                const long long got = soa_index(g, c);
                if (got != want || got >= g.vs) {
                    printf("soa_index %d %d %d pad %d: c %lld -> %lld, want %lld\n", N0, N1, N2, pad, c, got, want);
                    return 1;
                }
            }
    return 0;
}

int main() {
    const int sizes[][3] = {{1, 1, 1}, {2, 3, 5}, {32, 8, 1}, {33, 9, 7}, {64, 16, 69}, {70, 21, 4},
                            {127, 5, 3}, {512, 2, 2}, {30, 30, 30}};
    for (const auto& s : sizes)
        for (int pad = 0; pad < 2; ++pad)
            if (check_grid(s[0], s[1], s[2], pad)) return 1;
    srand(7);
    for (int t = 0; t < 40; ++t) {
        const int N0 = 1 + rand() % 300, N1 = 1 + rand() % 40, N2 = 1 + rand() % 12;
        if (check_grid(N0, N1, N2, 1)) return 1;
    }
    printf("ok\n");
    return 0;
}
