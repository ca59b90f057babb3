// Host-only check of the stage kernel's shared-memory carve-up and pair
// table (compiled by tests/test_layout.py with nvcc; runs on the CPU).
// Prints one line per problem: "bad ..." for any violation, then "ok N".
#include <cstdio>
#include "heom_kernels.cuh"

int main()
{
    long checked = 0, bad = 0;
    for (int n = 1; n <= 16; ++n) {
        // pair table: every element covered exactly once (diagonal padding duplicate allowed)
        int seen[256] = {0};
        const int P = heomk::pairs_of(n);
        for (int p = 0; p < P; ++p) {
            int e1, e2, i, j, d;
            heomk::pair_elements(n, p, &e1, &e2, &i, &j, &d);
            if (e1 < 0 || e1 >= n * n || e2 < 0 || e2 >= n * n) { printf("bad pair range n=%d p=%d\n", n, p); ++bad; }
            seen[e1]++;
            if (e2 != e1) seen[e2]++;
            if (!d && !(i < j && e1 == i * n + j && e2 == j * n + i)) { printf("bad offdiag n=%d p=%d\n", n, p); ++bad; }
        }
        for (int e = 0; e < n * n; ++e)
            if (seen[e] != 1) { printf("bad coverage n=%d e=%d count=%d\n", n, e, seen[e]); ++bad; }
        for (int W = 1; W <= 64; ++W)
            for (int depth = 1; depth <= 40; ++depth) {
                const int LS = depth + 1, NW = (2 * W + 3) & ~3, TWB = (W + 15) & ~15;
                const heomk::PairSmem L = heomk::pair_smem_layout(n, W, NW, TWB, LS);
                const int kmin = 0, h = 3 * W * LS * 16, cplus = h + n * n * 16, hr = cplus + W * LS * 8;
                const int end = hr + n * (n + 1) * 8;
                if (kmin % 16 || h % 16 || cplus % 8 || hr % 8 || end > L.lut) { printf("bad lut n=%d W=%d LS=%d\n", n, W, LS); ++bad; }
                if (L.lut % 16 || L.slot % 16 || L.team % 16 || L.tile_off % 16 || L.nbr_off % 16 ||
                    L.tup_off % 16 || L.pss_off % 16) { printf("bad slot n=%d W=%d\n", n, W); ++bad; }
                if (L.nbr_off - L.tile_off < n * (n + 1) * 16 || L.tup_off - L.nbr_off < NW * 4 ||
                    L.pss_off - L.tup_off < TWB || L.slot - L.pss_off < 16) { printf("bad sizes n=%d W=%d\n", n, W); ++bad; }
                if (NW % 4 || NW < 2 * W || TWB % 16 || TWB < W) { printf("bad pads W=%d\n", W); ++bad; }
                ++checked;
            }
    }
    printf("%s %ld\n", bad ? "FAILED" : "ok", checked);
    return bad ? 1 : 0;
}
