// Host-only check of the stage kernel's shared-memory carve-up and pair
// table (compiled by tests/test_layout.py with nvcc; runs on the CPU).
// Prints one line per problem: "bad ..." for any violation, then "ok N".
#include <cstdio>
#include "heom_kernels.cuh"
#include "pair_tables.inc"

static int swz_h(int r) { return ((r & 1) << 2) | (r & 1) | (((r >> 1) & 1) << 1); }

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
                // khat 3W double2, (sqrt(n), sqrt(n+1)) for n = 0..LS, chat W doubles, pos W int16
                if (3 * W * 16 + (LS + 1) * 16 + W * 8 + W * 2 > L.lut) { printf("bad lut n=%d W=%d LS=%d\n", n, W, LS); ++bad; }
                if (L.lut % 16 || L.slot % 16 || L.team % 16 || L.tile_off % 16 || L.nbr_off % 16 ||
                    L.tup_off % 16 || L.pss_off % 16 || L.xch_off % 16) { printf("bad slot n=%d W=%d\n", n, W); ++bad; }
                if (L.nbr_off - L.tile_off < n * heomk::tile_stride(n) * 16 || L.tup_off - L.nbr_off < NW * 4 ||
                    L.pss_off - L.tup_off < TWB || L.slot - L.pss_off < 16 || L.xch_off < 2 * L.slot ||
                    L.team - L.xch_off < heomk::kXchBytes)
                    { printf("bad sizes n=%d W=%d\n", n, W); ++bad; }
                if (NW % 4 || NW < 2 * W || TWB % 16 || TWB < W) { printf("bad pads W=%d\n", W); ++bad; }
                ++checked;
            }
        // tile positions: inside the row, one per element
        {
            int used[16 * 20] = {0};
            for (int i = 0; i < n; ++i)
                for (int k = 0; k < n; ++k) {
                    const int q = heomk::tile_pos(n, i, k);
                    if (q - i * heomk::tile_stride(n) >= heomk::tile_stride(n) || used[q]++)
                        { printf("bad tile position n=%d (%d,%d)\n", n, i, k); ++bad; }
                }
        }
        // team kernel: conflict-free quarter-warp operand reads (16-byte bank groups: index mod 8)
        // and exchange writes; lanes 8q..8q+7 hold g = 2q, 2q+1 and t = 0..3
        if (n > 8)
            for (int b = 0; b < 2; ++b)
                for (int s = 0; s < 4; ++s)
                    for (int q = 0; q < 4; ++q)
                        for (int which = 0; which < 3; ++which) {
                            int used[8] = {0};
                            for (int g = 2 * q; g <= 2 * q + 1; ++g)
                                for (int t = 0; t < 4; ++t) {
                                    int pos;
                                    if (which == 0) pos = heomk::tile_pos(n, 8 * b + g, 4 * s + t); // A
                                    else if (which == 1) pos = heomk::tile_pos(n, 4 * s + t, 8 * b + g); // B
                                    else pos = (8 * b + g) * heomk::kXchStride + 8 * (s & 1) + 2 * t + (s >> 1); // C: J = s & 1, c0/c1 = s >> 1
                                    if (used[pos % 8]++) { printf("bank conflict n=%d b=%d s=%d q=%d w=%d\n", n, b, s, q, which); ++bad; }
                                }
                        }
    }
    // searched sector tables for N <= 8: coverage, and for N = 8 conflict-free
    // operand and exchange reads of the tensor-pipe kernel
    for (int n = 1; n <= 8; ++n) {
        const int P = heomk::pairs_of(n);
        int seen[64] = {0};
        for (int p = 0; p < P; ++p) {
            const int e1 = kPairE1[n][p], e2 = kPairE2[n][p];
            if (e1 < 0 || e1 >= n * n || e2 < 0 || e2 >= n * n) { printf("bad table range n=%d\n", n); ++bad; continue; }
            const int i1 = e1 / n, j1 = e1 % n, i2 = e2 / n, j2 = e2 % n;
            const bool d1 = i1 == j1, d2 = i2 == j2;
            if (d1 != d2 || (!d1 && !(i1 == j2 && j1 == i2))) { printf("bad pair n=%d p=%d\n", n, p); ++bad; }
            seen[e1]++;
            if (e2 != e1) seen[e2]++;
        }
        for (int e = 0; e < n * n; ++e)
            if (seen[e] != 1) { printf("bad table coverage n=%d e=%d\n", n, e); ++bad; }
        for (int W = 1; W <= 64; ++W) {
            const int NW = (2 * W + 3) & ~3, TWB = (W + 15) & ~15;
            const int sb = heomk::dmma_slot_bytes(P, NW, TWB), wb = heomk::dmma_warp_bytes(P, NW, TWB);
            if (sb % 16 || wb % 16 || sb < P * 32 + NW * 4 + TWB + 16) { printf("bad dmma slot n=%d W=%d\n", n, W); ++bad; }
            if (heomk::dmma_smem_bytes(P, W, NW, TWB, 41) > 227 * 1024) { printf("dmma smem too big n=%d W=%d\n", n, W); ++bad; }
        }
    }
    {
        const int n = 8;
        int sec[64], half[64];
        for (int p = 0; p < 32; ++p) {
            sec[kPairE1[n][p]] = p; half[kPairE1[n][p]] = 0;
            sec[kPairE2[n][p]] = p; half[kPairE2[n][p]] = 1;
        }
        for (int q = 0; q < 4; ++q)
            for (int s = 0; s < 2; ++s)
                for (int which = 0; which < 2; ++which) {
                    int used[8] = {0};
                    for (int rr = 2 * q; rr <= 2 * q + 1; ++rr)
                        for (int t = 0; t < 4; ++t) {
                            const int col = 4 * s + t;
                            if (which == 1 && rr == col) continue;
                            const int e = which == 0 ? rr * n + col : col * n + rr;
                            if (used[(2 * sec[e] + half[e]) % 8]++) { printf("bank conflict operand q=%d s=%d\n", q, s); ++bad; }
                        }
                }
        for (int k = 0; k < 4; ++k)
            for (int which = 0; which < 2; ++which) {
                int used[8] = {0};
                for (int p = 8 * k; p < 8 * k + 8; ++p) {
                    const int e = which == 0 ? kPairE1[n][p] : kPairE2[n][p];
                    if (used[((e % n) ^ swz_h(e / n)) % 8]++) { printf("bank conflict exchange k=%d\n", k); ++bad; }
                }
            }
    }
    printf("%s %ld\n", bad ? "FAILED" : "ok", checked);
    return bad ? 1 : 0;
}
