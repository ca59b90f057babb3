// heom_lockstep.cuh -- sm_100a stage kernel of a lockstep ensemble class.
//
// A lockstep class holds K >= 8 instances of one hierarchy shape (same states,
// baths, Matsubara terms and depth: the realisations of a static-disorder
// ensemble) with the state stored instance-minor: sector p of ADO u of
// instance k at ((u * P + p) * Kp + k) * 32 bytes, Kp = K rounded up to 32.
// Each stage evaluates the same per-element derivative as heom_dmma_stage
// (heom_ode.cl:24-451, the RK4 write fused), in the same operation order, so
// that every instance's results are those of a single-instance solve; what
// changes is the traffic: a sector row of 32 instances is one coalesced
// 1-KB read, and the neighbour indices, coefficients and site bookkeeping of
// an ADO are resolved once for all of its instances.

#pragma once

#include "heom_kernels.cuh"

namespace heomk {

struct LockParams {
    PairParams p;     // in/out/y/acc in the lockstep layout; nbr/tup/pss rows of one instance; hfrag [K][256]
    LaneTab lt;
    CoefTabs ct;
    int K;            // instances
    int Kp;           // instance stride (K rounded up to 32)
    int64_t nodes;    // ADOs of every instance
};

constexpr int kLockWarps = 8;
// one slot of one site at the current ADO: its neighbour rows and coefficients
struct __align__(16) LockSlot {
    int64_t op, om;   // byte offsets of the rows of ADO n + e (plus) and n - e (minus); -1: absent
    double c, sm;     // plus-side coefficient chat * sqrt(n + 1), minus-side scale sqrt(n)
    double2 kap[3];   // the three kappa-hat values of the slot's mode
    int present, pad[3];
};
// one pair sector: its sites and same-term values
struct __align__(16) LockSector {
    int sa, sb, diag, pad; // sites of side 0 and side 1 (element i1, then j1 or, diagonal, i2)
    double2 g1, g2;        // gamma0 of its two elements
};
__host__ __device__ inline int lock_row_bytes(int NW, int TWB) { return ((NW * 4 + 15) & ~15) + ((TWB + 15) & ~15) + 16; }
__host__ inline size_t lockstep_smem_bytes(int P, int W, int NW, int TWB, int LS)
{
    return (size_t)dmma_lut_bytes(W, LS) + 2 * (size_t)P * 32 * 32 /* two tiles */ + 32 * 32 * 32 /* commutators */ +
           (size_t)kLockWarps * 64 * 16 + 32 * sizeof(LockSector) + 32 * sizeof(LockSlot) +
           2 * (size_t)lock_row_bytes(NW, TWB);
}

// 32 bytes at base + off (bytes) when off >= 0, zeros otherwise: the test, the address and the
// load in one asm block
__device__ __forceinline__ void ld256_at(const double2* base, int64_t off, double2& a, double2& b)
{
    asm("{\n .reg .pred q;\n .reg .b64 ad;\n setp.ge.s64 q, %5, 0;\n add.s64 ad, %4, %5;\n"
        " mov.f64 %0, 0d0000000000000000;\n mov.f64 %1, 0d0000000000000000;\n"
        " mov.f64 %2, 0d0000000000000000;\n mov.f64 %3, 0d0000000000000000;\n"
        " @q ld.global.nc.v4.f64 {%0,%1,%2,%3}, [ad];\n}\n"
        : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y)
        : "l"(base), "l"(off));
}
// as ld256_at, and only when skip == 0
__device__ __forceinline__ void ld256_at_unless(const double2* base, int64_t off, unsigned skip, double2& a, double2& b)
{
    asm("{\n .reg .pred q;\n .reg .b64 ad;\n setp.ge.s64 q, %5, 0;\n setp.eq.and.u32 q, %6, 0, q;\n"
        " add.s64 ad, %4, %5;\n"
        " mov.f64 %0, 0d0000000000000000;\n mov.f64 %1, 0d0000000000000000;\n"
        " mov.f64 %2, 0d0000000000000000;\n mov.f64 %3, 0d0000000000000000;\n"
        " @q ld.global.nc.v4.f64 {%0,%1,%2,%3}, [ad];\n}\n"
        : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y)
        : "l"(base), "l"(off), "r"(skip));
}
// 32 bytes through the coherent path, schedulable: the stage kernel stores to the same address only
// values computed from the loaded ones, which orders the load first
__device__ __forceinline__ void ld256_co(const double2* src, double2& a, double2& b)
{
    asm("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];\n" : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(src));
}

// Two CTAs of 8 warps per SM. CTA b keeps the instance block b % (Kp / 32)
// and sweeps the ADOs u = b / (Kp / 32), + gridDim / (Kp / 32), ...; the next
// ADO's tiles and rows are copied (cp.async) while the current one runs.
// Phase A: warp w forms the commutator of instances w, w + 8, w + 16, w + 24
// of the block (real symmetric H: their fragments stay in registers, the A
// operand being -hb exactly); the last warp first resolves every slot of every
// site at this ADO into a table (neighbour rows, coefficients), so that phase
// B's sectors read broadcast entries. Phase B: one warp per sector, a lane per
// instance; every global read of a sector (the neighbour rows of both sides,
// y and acc) is issued, predicated, before its arithmetic.
template <int N, int HK, int SLT>
__global__ void __launch_bounds__(kLockWarps * 32, 2) heom_lockstep_stage(const LockParams lp)
{
    static_assert(N <= 8 && N * SLT <= 32, "lockstep stage handles N <= 8");
    constexpr int P = pairs_of(N);
    constexpr int IPW = 32 / kLockWarps;  // instances per warp in phase A
    constexpr int SB = SLT <= 1 ? 2 : 1; // sides whose neighbour rows are read in one batch
    constexpr int TW = kLockWarps - 1;   // the warp that builds the site table
    const PairParams& p = lp.p;
    extern __shared__ __align__(128) unsigned char smem[];
    const int W = p.W, LS = p.LS, SL = p.SL;
    double2* s_kh = reinterpret_cast<double2*>(smem);
    double2* s_sq = s_kh + 3 * W;
    double* s_ch = reinterpret_cast<double*>(s_sq + LS + 1);
    for (int q = threadIdx.x; q < 3 * W; q += blockDim.x) s_kh[q] = lp.ct.khat[q];
    for (int q = threadIdx.x; q < W; q += blockDim.x) s_ch[q] = lp.ct.chat[q];
    for (int q = threadIdx.x; q <= LS; q += blockDim.x)
        s_sq[q] = make_double2(lp.ct.sq[q], q < LS ? lp.ct.sq[q + 1] : 0.0);
    unsigned char* base = smem + dmma_lut_bytes(W, LS);
    double2* tiles = reinterpret_cast<double2*>(base);      // [2][P][32] sectors (2 double2 each)
    double2* ctile = tiles + 2 * 2 * P * 32;                 // [32][32] commutator values (rows >= P unused)
    double2* xch = ctile + 2 * 32 * 32 + (threadIdx.x >> 5) * 64;
    LockSector* sectors = reinterpret_cast<LockSector*>(ctile + 2 * 32 * 32 + kLockWarps * 64);
    LockSlot* slots = reinterpret_cast<LockSlot*>(sectors + 32);
    unsigned char* rows0 = reinterpret_cast<unsigned char*>(slots + 32);
    const int rowb = lock_row_bytes(p.NW, p.TWB);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kblocks = lp.Kp >> 5;
    const int kb = blockIdx.x % kblocks;
    const int64_t ustep = gridDim.x / kblocks;
    const int64_t Kp = lp.Kp;
    const int64_t PK2 = (int64_t)P * Kp * 2; // double2 elements of one ADO (all instances)

    if (threadIdx.x < P) {
        const int e1 = lp.lt.e1[threadIdx.x], e2 = lp.lt.e2[threadIdx.x];
        const int i1 = e1 / N, j1 = e1 - i1 * N, i2 = e2 / N;
        LockSector sc;
        sc.sa = i1;
        sc.diag = i1 == j1;
        sc.sb = sc.diag ? i2 : j1;
        sc.pad = 0;
        sc.g1 = p.gamma0[e1];
        sc.g2 = p.gamma0[e2];
        sectors[threadIdx.x] = sc;
    }

    // real symmetric H: hb of this warp's instances for the whole sweep
    double hbk[IPW][2];
#pragma unroll
    for (int j = 0; j < IPW; ++j) {
        const int k = kb * 32 + warp + kLockWarps * j;
#pragma unroll
        for (int s = 0; s < 2; ++s)
            hbk[j][s] = (HK != H_GENERIC && k < lp.K) ? __ldg(p.hfrag + (size_t)k * 256 + 32 * s + lane) : 0.0;
    }

    const bool owner = lane < P;
    const int ae1 = owner ? lp.lt.e1[lane] : 0, ae2 = owner ? lp.lt.e2[lane] : 0;
    const int ai1 = ae1 / N, aj1 = ae1 - ai1 * N, ai2 = ae2 / N, aj2 = ae2 - ai2 * N;
    const int fs0 = lp.lt.fs[lane][0], fs1 = lp.lt.fs[lane][1];
    const int ha0 = lp.lt.ha[lane][0], ha1 = lp.lt.ha[lane][1];
    const int r = lane >> 2, t = lane & 3;
    const int xr1 = 8 * ai1 + (aj1 ^ swz(ai1)), xr2 = 8 * ai2 + (aj2 ^ swz(ai2));
    const int xw0 = 8 * r + ((2 * t) ^ swz(r)), xw1 = 8 * r + ((2 * t + 1) ^ swz(r));
    // Phase A offsets (double2, from a tile buffer) of this lane's operands for the warp's first
    // instance; its instance warp + 8 j adds 16 j, since the column swizzle k ^ (p & 3) changes
    // bits 0-1 of k only. An operand outside the N x N block reads an arbitrary finite tile value
    // (sector 0): its partner fragment of H is zero, so it adds only zeros, to rows and columns
    // that are not read.
    // Shared tiles store half h of instance column k at position h ^ ((k >> 2) & 1): a warp's
    // 16-byte accesses to one half of 32 columns then cover all eight 16-byte bank groups.
    const int hw = (warp >> 2) & 1; // (k >> 2) & 1 of the warp's phase A instances
    int oa[2], ob[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int fs = s == 0 ? fs0 : fs1, ha = s == 0 ? ha0 : ha1;
        const int row = fs >= 0 ? (fs * 32 + (warp ^ (fs & 3))) * 2 : 0;
        oa[s] = fs >= 0 ? row + (ha ^ hw) : 0;
        ob[s] = fs >= 0 ? (r == 4 * s + t ? row + (ha ^ hw) : row + (ha ^ 1 ^ hw)) : 0; // diagonal: its own transpose
    }
    const int oc = (lane * 32 + (warp ^ (lane & 3))) * 2; // this lane's commutator row (lanes >= P: unused rows)
    // its two commutator stores: first position (lane >> 2) & 1, whichever half lives there
    const int cpa = (lane >> 2) & 1;
    const int xra = (cpa ^ hw) == 0 ? xr1 : xr2, xrb = (cpa ^ hw) == 0 ? xr2 : xr1;
    const int hk = (lane >> 2) & 1; // phase B: position of half 0 of this lane's instance
    // the slot of site (lane / SLT) that lane of the table warp resolves
    const int tsite = lane / SLT, tq = lane - tsite * SLT;
    const int tsl = (warp == TW && tsite < N && tq < SL) ? __ldg(p.slots + tsite * SL + tq) : -1;
    const int tpos = tsl >= 0 ? lp.ct.pos[tsl] : 0;
    // this thread's 16-byte pieces of a tile copy: sectors pp0, pp0 + 4, ... of instance column pk
    const int pp0 = threadIdx.x >> 6, pk = (threadIdx.x >> 1) & 31, ph = threadIdx.x & 1;
    const int dst0 = (pp0 * 32 + (pk ^ (pp0 & 3))) * 2 + (ph ^ ((pk >> 2) & 1));
    const int64_t src0 = ((int64_t)pp0 * Kp + pk) * 2 + ph + (int64_t)kb * 64;

    // asynchronous copies of ADO u's tiles (this block's 32 instances) and rows into buffer b
    auto prefetch = [&](int64_t u, int b) {
        double2* dst = tiles + b * 2 * P * 32 + dst0;
        const double2* src = p.in + u * PK2 + src0;
        for (int pp = pp0; pp < P; pp += 4, dst += 4 * 64, src += 8 * Kp) cp_async16(dst, src);
        unsigned char* rows = rows0 + b * rowb;
        for (int q = threadIdx.x * 4; q < p.NW; q += blockDim.x * 4)
            cp_async16(reinterpret_cast<int32_t*>(rows) + q, p.nbr + u * p.NW + q);
        unsigned char* tu = rows + ((p.NW * 4 + 15) & ~15);
        for (int q = threadIdx.x * 16; q < p.TWB; q += blockDim.x * 16) cp_async16(tu + q, p.tup + u * p.TWB + q);
        if (threadIdx.x == 0) cp_async16(tu + ((p.TWB + 15) & ~15), p.pss + u);
    };

    const int k = kb * 32 + lane;
    const bool live = k < lp.K;
    const bool read_acc = p.use_acc && !p.acc_init;
    int64_t u = blockIdx.x / kblocks;
    int cur = 0;
    if (u < lp.nodes) prefetch(u, 0);
    for (; u < lp.nodes; u += ustep, cur ^= 1) {
        cp_async_wait_all();
        __syncthreads();
        // the next ADO's copies fly while this one runs (its buffer was last read before the barrier)
        if (u + ustep < lp.nodes) prefetch(u + ustep, cur ^ 1);
        const double2* tile = tiles + cur * 2 * P * 32;
        const unsigned char* rows = rows0 + cur * rowb;
        const unsigned char* tu = rows + ((p.NW * 4 + 15) & ~15);
        const double2 pss = *reinterpret_cast<const double2*>(tu + ((p.TWB + 15) & ~15));

        // ---- the site table of this ADO ----
        if (warp == TW && lane < N * SLT) {
            LockSlot e;
            e.pad[0] = e.pad[1] = e.pad[2] = 0;
            if (tsl >= 0) {
                const int2 pm = reinterpret_cast<const int2*>(rows)[tsl];
                const double2 sqp = s_sq[tu[tsl]];
                e.op = pm.x >= 0 ? pm.x * PK2 * 16 : -1;
                e.om = pm.y >= 0 ? pm.y * PK2 * 16 : -1;
                e.present = 1;
                e.c = s_ch[tpos] * sqp.y;
                e.sm = sqp.x;
                e.kap[0] = s_kh[tpos];
                e.kap[1] = s_kh[W + tpos];
                e.kap[2] = s_kh[2 * W + tpos];
            } else {
                e.op = e.om = -1;
                e.present = 0;
                e.c = e.sm = 0.0;
                e.kap[0] = e.kap[1] = e.kap[2] = make_double2(0.0, 0.0);
            }
            slots[lane] = e;
        }

        // ---- A: commutator of every instance of the block ----
        {
            double gf[HK == H_GENERIC ? IPW : 1][2][4];
            if (HK == H_GENERIC) {
#pragma unroll
                for (int j = 0; j < IPW; ++j) {
                    const int kj = kb * 32 + warp + kLockWarps * j;
                    const double* f = p.hfrag + (size_t)(kj < lp.K ? kj : 0) * 256 + lane;
#pragma unroll
                    for (int s = 0; s < 2; ++s)
#pragma unroll
                        for (int c = 0; c < 4; ++c) gf[HK == H_GENERIC ? j : 0][s][c] = __ldg(f + 32 * (2 * c + s));
                }
            }
#pragma unroll
            for (int j0 = 0; j0 < IPW; j0 += 2) {
                double cr[2][2], ci[2][2]; // the two instances' accumulators
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                    const int j = j0 + jj;
                    double hb_r[2], hb_i[2], ha_r[2], ha_i[2];
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        if (HK == H_GENERIC) {
                            hb_r[s] = gf[HK == H_GENERIC ? j : 0][s][0];
                            hb_i[s] = gf[HK == H_GENERIC ? j : 0][s][1];
                            ha_r[s] = gf[HK == H_GENERIC ? j : 0][s][2];
                            ha_i[s] = gf[HK == H_GENERIC ? j : 0][s][3];
                        } else {
                            hb_r[s] = hbk[j][s];
                            ha_r[s] = -hbk[j][s]; // -H(r, c) = -H(c, r): H is real symmetric
                            hb_i[s] = ha_i[s] = 0.0;
                        }
                    }
                    cr[jj][0] = cr[jj][1] = ci[jj][0] = ci[jj][1] = 0.0;
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        const double2 A = tile[oa[s] + 16 * j], B = tile[ob[s] + 16 * j];
                        dmma(cr[jj][0], cr[jj][1], A.x, hb_r[s]);
                        dmma(ci[jj][0], ci[jj][1], A.y, hb_r[s]);
                        dmma(cr[jj][0], cr[jj][1], ha_r[s], B.x);
                        dmma(ci[jj][0], ci[jj][1], ha_r[s], B.y);
                        if (HK == H_GENERIC) {
                            dmma(cr[jj][0], cr[jj][1], -A.y, hb_i[s]);
                            dmma(ci[jj][0], ci[jj][1], A.x, hb_i[s]);
                            dmma(cr[jj][0], cr[jj][1], -ha_i[s], B.y);
                            dmma(ci[jj][0], ci[jj][1], ha_i[s], B.x);
                        }
                    }
                }
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                    const int j = j0 + jj;
                    xch[xw0] = make_double2(cr[jj][0], ci[jj][0]);
                    xch[xw1] = make_double2(cr[jj][1], ci[jj][1]);
                    __syncwarp();
                    ctile[oc + 16 * j + cpa] = xch[xra];
                    ctile[oc + 16 * j + (cpa ^ 1)] = xch[xrb];
                    __syncwarp();
                }
            }
        }
        __syncthreads();

        // ---- B: per sector, lane = instance ----
        for (int ps = warp; ps < P; ps += kLockWarps) {
            const LockSector sc = sectors[ps];
            const bool diag = sc.diag != 0;
            const int64_t lofs = ((int64_t)ps * Kp + k) * 2; // this lane's sector within an ADO
            const double2* in_l = p.in + lofs;
            const int64_t off = u * PK2 + lofs;
            double2 x1, x2, a1, a2;
            double2 L1, L2, s1, s2;
#pragma unroll
            for (int sd0 = 0; sd0 < 2; sd0 += SB) {
                // neighbour rows of SB sides (absent rows: no load, zeros)
                double2 xp[SB][SLT][2], xm[SB][SLT][2];
#pragma unroll
                for (int b = 0; b < SB; ++b) {
                    const LockSlot* es = slots + ((sd0 + b) == 0 ? sc.sa : sc.sb) * SLT;
#pragma unroll
                    for (int q = 0; q < SLT; ++q) {
                        const longlong2 o = *reinterpret_cast<const longlong2*>(&es[q].op);
                        ld256_at_unless(in_l, o.x, sc.diag, xp[b][q][0], xp[b][q][1]);
                        ld256_at(in_l, o.y, xm[b][q][0], xm[b][q][1]);
                    }
                }
                if (sd0 == 0) {
                    if (p.y) ld256_co(p.y + off, x1, x2); // kernel parameters: uniform branches
                    if (read_acc) ld256_co(p.acc + off, a1, a2);
                    const int col = (ps * 32 + (lane ^ (ps & 3))) * 2;
                    s1 = tile[col + hk];
                    s2 = tile[col + (hk ^ 1)];
                    const double2 c1 = ctile[col + hk], c2 = ctile[col + (hk ^ 1)];
                    L1 = make_double2(-c1.y, c1.x); // i * (w H - H w) / hbar
                    L2 = make_double2(-c2.y, c2.x);
                    cmac(L1, make_double2(pss.x + sc.g1.x, pss.y + sc.g1.y), s1);
                    cmac(L2, make_double2(pss.x + sc.g2.x, pss.y + sc.g2.y), s2);
                }
#pragma unroll
                for (int b = 0; b < SB; ++b) {
                    const int sd = sd0 + b;
                    const LockSlot* es = slots + (sd == 0 ? sc.sa : sc.sb) * SLT;
#pragma unroll
                    for (int q = 0; q < SLT; ++q) {
                        if (!es[q].present) continue; // warp-uniform
                        const double2 cs = *reinterpret_cast<const double2*>(&es[q].c);
                        const double c = diag ? 0.0 : cs.x;
                        const double sm = cs.y;
                        const double2 m1 = make_double2(xm[b][q][0].x * sm, xm[b][q][0].y * sm);
                        const double2 m2 = make_double2(xm[b][q][1].x * sm, xm[b][q][1].y * sm);
                        const double2 t1 = xp[b][q][0], t2 = xp[b][q][1];
                        const double2 kd = es[q].kap[diag ? 2 : 0], k1 = es[q].kap[1];
                        if (sd == 0) {
                            L1.x = fma(-c, t1.y, L1.x);
                            L1.y = fma(c, t1.x, L1.y);
                            L2.x = fma(c, t2.y, L2.x);
                            L2.y = fma(-c, t2.x, L2.y);
                            cmac(L1, kd, m1);
                            if (!diag) cmac(L2, k1, m2);
                        } else {
                            L1.x = fma(c, t1.y, L1.x);
                            L1.y = fma(-c, t1.x, L1.y);
                            L2.x = fma(-c, t2.y, L2.x);
                            L2.y = fma(c, t2.x, L2.y);
                            if (!diag) cmac(L1, k1, m1);
                            cmac(L2, kd, m2);
                        }
                    }
                }
            }
            if (!p.y) {
                x1 = s1;
                x2 = s2;
            }
            double2 o1 = make_double2(p.alpha.x * x1.x - p.alpha.y * x1.y, p.alpha.x * x1.y + p.alpha.y * x1.x);
            double2 o2 = make_double2(p.alpha.x * x2.x - p.alpha.y * x2.y, p.alpha.x * x2.y + p.alpha.y * x2.x);
            cmac(o1, p.beta, L1);
            cmac(o2, p.beta, L2);
            st256_cs_if(live, p.out + off, o1, o2);
            if (p.use_acc) {
                if (!read_acc) {
                    a1 = s1;
                    a2 = s2;
                }
                cmac(a1, p.acc_beta, L1);
                cmac(a2, p.acc_beta, L2);
                st256_if(live, p.acc + off, a1, a2);
            }
        }
    }
    cp_async_wait_all(); // no copy left in flight when the CTA retires
}

} // namespace heomk
