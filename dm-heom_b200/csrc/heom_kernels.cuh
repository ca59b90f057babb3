// heom_kernels.cuh -- sm_100a kernels of the HEOM derivative + RK4 path.
//
// heom_pair_stage evaluates the HEOM time derivative L(w) for every ADO of
// the hierarchy (the reference's heom_ode kernel,
// dm-heom/cl/heom/heom_ode.cl:24-451) and fuses the Runge-Kutta write of the
// stage into the same pass (the NOMA_NUM_ODE_ACCUMULATE /
// NOMA_NUM_ODE_SUBDIAGONAL write modes, heom_ode.cl:416-434, generalised to a
// complex stage coefficient).
//
// Per element (i, j) of ADO u the derivative is
//   L(w)_u(i,j) = i * sum_k [ w_u(i,k) Hs(k,j) - Hs(i,k) w_u(k,j) ]        (:89-114, Hs = H / hbar)
//               + (pf_same_sum[u] + gamma0(i,j)) w_u(i,j)                 (:131-168)
//               + sum over slots e = b*M+m of the baths b of site i:
//                    i cplus(n) w_{u+e}(i,j) + kappa_i(n) w_{u-e}(i,j)      (:183-221, :280-342)
//               + sum over slots e of the baths of site j:
//                   -i cplus(n) w_{u+e}(i,j) + kappa_j(n) w_{u-e}(i,j)      (:223-259, :344-403)
// with n the tuple entry of u for slot e and
//   cplus(n)   = sqrt((n+1) |c_e| / hbar)                                 (:211, :249)
//   kappa_i(n) = sqrt(n hbar / |c_e|) (i c_e / hbar + [m==0] pf_circ[b])  (:301-337)
//   kappa_j(n) = sqrt(n hbar / |c_e|) (-i c_e / hbar + [m==0] pf_circ[b]) (:363-398)
// For a diagonal element the site-i and site-j plus terms cancel exactly and
// the minus terms combine to kappa_i + kappa_j ("kappa_d"); both are folded
// on the host.
//
// HBM layout ("pair layout"): an ADO is P = N(N-1)/2 + ceil(N/2) sectors of
// 32 B.  Sector p < N(N-1)/2 holds the symmetric pair (w(i,j), w(j,i)), i < j;
// the remaining sectors hold pairs of diagonal elements (w(2k,2k),
// w(2k+1,2k+1)) (for odd N the last holds w(N-1,N-1) twice).  The neighbour
// terms only ever read the "cross" of a neighbour -- row b and column b for a
// bath b of the element's sites -- and in this layout a cross is N whole
// sectors; both elements of a sector need the same neighbours.  For N = 8 an
// ADO is exactly 32 sectors (1 KB): one warp per ADO, one sector per lane.
//
// Work mapping: N <= 8 one warp per ADO (heom_dmma_stage), N = 9..16 a team
// of TW = ceil(P/32) warps per ADO (heom_pair_stage); in both the commutator
// runs on the FP64 tensor pipe (m8n8k4) and the lane that owns a sector does
// its bath terms and the stage write.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace heomk {

constexpr int kCtaWarps = 8;

__host__ __device__ constexpr int pairs_of(int n) { return n * (n - 1) / 2 + (n + 1) / 2; }
__host__ __device__ constexpr int team_warps(int n) { return (pairs_of(n) + 31) / 32; }

// element indices (row-major, e = i*N + j) of the two halves of sector p
__host__ __device__ inline void pair_elements(int n, int p, int* e1, int* e2, int* i_out, int* j_out,
                                              int* diag)
{
    const int noff = n * (n - 1) / 2;
    if (p < noff) {
        int i = 0, q = p;
        while (q >= n - 1 - i) {
            q -= n - 1 - i;
            ++i;
        }
        const int j = i + 1 + q;
        *e1 = i * n + j;
        *e2 = j * n + i;
        *i_out = i;
        *j_out = j;
        *diag = 0;
    } else {
        const int k = p - noff;
        const int a = 2 * k;
        const int b = (2 * k + 1 < n) ? 2 * k + 1 : a;
        *e1 = a * n + a;
        *e2 = b * n + b;
        *i_out = a;
        *j_out = b;
        *diag = 1;
    }
}

struct PairParams {
    const double2* __restrict__ in;  // [nodes][2P] (sector p = double2 pair 2p, 2p+1)
    const double2* y;                // AXPY against y instead of in (may alias out)
    double2* out;
    double2* acc;                    // accumulate mode
    double2 alpha;                   // out = alpha * x + beta * L
    double2 beta;
    double2 acc_beta;                // acc = (acc_init ? in : acc) + acc_beta * L
    int acc_init;
    int use_acc;
    const int32_t* __restrict__ nbr; // [nodes][NW]: (plus, minus) of every slot, padded to NW (multiple of 4)
    const uint8_t* __restrict__ tup; // [nodes][TWB] tuple bytes, padded to TWB (multiple of 16)
    const double2* __restrict__ pss; // [nodes]
    const double* __restrict__ hfrag;  // [n_inst][frag_doubles(N)] MMA operand fragments of H / hbar
    const int32_t* __restrict__ inst;  // [nodes] instance of each ADO; NULL when the handle holds one instance
    const double2* __restrict__ gamma0;// [N*N]
    const int16_t* __restrict__ slots; // [N][SL], -1 padded
    int64_t nodes;
    int W, NW, TWB, LS, SL;
};

enum HKind : int { H_REAL_SYM = 0, H_GENERIC = 1 };

// MMA operand fragments of H / hbar, per instance: N <= 8 one 8 x 8 block and
// two k-slices, N = 9..16 a zero-padded 16 x 16 grid of 2 x 2 blocks and four
// k-slices.  Layout [kind][block b][k-slice s][lane], lane l = 4g + t:
// kind 0/1 = Re/Im of hb = H(4s+t, 8b+g) (B operand of w H for block column b),
// kind 2/3 = Re/Im of ha = -H(8b+g, 4s+t) (A operand of -H w for block row b).
__host__ __device__ constexpr int frag_blocks(int n) { return n <= 8 ? 1 : 2; }
__host__ __device__ constexpr int frag_slices(int n) { return n <= 8 ? 2 : 4; }
__host__ __device__ constexpr int frag_doubles(int n) { return 4 * frag_blocks(n) * frag_slices(n) * 32; }
__host__ __device__ constexpr int frag_index(int n, int kind, int b, int s, int lane)
{
    return ((kind * frag_blocks(n) + b) * frag_slices(n) + s) * 32 + lane;
}

// Team kernel (N = 9..16): the staged ADO is row-major with row stride
// TS = 4 (mod 8) double2 and the columns of rows with bit 1 set swapped in
// pairs (k ^ 2), so that the quarter-warp reads of both MMA operands,
// A = w(8I+g, 4s+t) and B = w(4s+t, 8J+g), hit eight distinct 16-byte bank groups.
__host__ __device__ constexpr int tile_stride(int n) { return (n + 3) / 8 * 8 + 4; }
__host__ __device__ constexpr int tile_pos(int n, int i, int k) { return i * tile_stride(n) + (k ^ (i & 2)); }
// exchange tile of the commutator: 16 rows of 17 double2 (conflict-free C writes)
constexpr int kXchStride = 17;
constexpr int kXchBytes = 16 * kXchStride * 16;

// shared look-up tables of both stage kernels: khat 3*W double2, (sqrt(n),
// sqrt(n+1)) LS+1 double2, chat W doubles, pos W int16 (the last read by the
// team kernel only)
__host__ __device__ inline int dmma_lut_bytes(int W, int LS)
{
    return ((3 * W * 16 + (LS + 1) * 16 + W * 8 + W * 2) + 15) & ~15;
}

// dynamic shared memory carve-up (bytes); everything 16-B aligned
struct PairSmem {
    int lut;     // coefficient tables (dmma_lut_bytes)
    int team;    // per team: 2 slots + the exchange tile
    int slot;    // per slot: tile + nbr + tup + pss
    int tile_off, nbr_off, tup_off, pss_off, xch_off;
};

__host__ __device__ inline PairSmem pair_smem_layout(int n, int W, int NW, int TWB, int LS)
{
    PairSmem s;
    s.lut = dmma_lut_bytes(W, LS);
    const int tile = n * tile_stride(n) * 16;
    s.tile_off = 0;
    s.nbr_off = tile;
    s.tup_off = s.nbr_off + ((NW * 4 + 15) & ~15);
    s.pss_off = s.tup_off + ((TWB + 15) & ~15);
    s.slot = s.pss_off + 16;
    s.xch_off = 2 * s.slot;
    s.team = s.xch_off + kXchBytes;
    return s;
}

__host__ inline size_t pair_smem_bytes(int n, int W, int NW, int TWB, int LS)
{
    const PairSmem s = pair_smem_layout(n, W, NW, TWB, LS);
    const int teams = kCtaWarps / team_warps(n);
    return (size_t)s.lut + (size_t)teams * s.team;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int TW>
__device__ __forceinline__ void team_sync(int team)
{
    if (TW == 1) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;\n" ::"r"(team + 1), "r"(TW * 32) : "memory");
    }
}

__device__ __forceinline__ void cmac(double2& acc, const double2 a, const double2 b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

__device__ __forceinline__ double2 ldg2(const double2* p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// N <= 8: one warp per ADO, commutator on the FP64 tensor pipe.
//
// The tile is zero-padded to 8 x 8.  For k-slice s in {0, 1} lane l = 4r + t
// needs the MMA operands A = w(r, 4s+t) (for w H) and B = w(4s+t, r) (for
// H w): the two halves of one pair sector, read from the staged tile.  Eight
// m8n8k4 MMAs (real H; sixteen for complex H) give C = w H - H w at
// (r, 2t), (r, 2t+1); the result goes through a swizzled row-major tile to the
// lane that owns the sector.  The sector order (pair_tables.inc) makes both
// the operand reads and the exchange reads free of bank conflicts.
//
// Pipeline: per warp two slots, each filled by 1-D TMA bulk copies (tile,
// neighbour row, tuple row, pf_same_sum) that complete on the slot's
// mbarrier; the copies of ADO k+1 fly while ADO k is computed.  Every wait is
// bounded; on expiry the kernel sets *p.err and the warp stops.
// ---------------------------------------------------------------------------

struct LaneTab {
    signed char e1[32], e2[32]; // owned sector: element indices (row-major)
    signed char fs[32][2];      // operand sector of k-slice s (-1: zero padding)
    signed char ha[32][2];      // half of that sector holding A = w(r, 4s+t)
};

// Factored bath coefficients: cplus(n) = chat * sqrt(n+1), kappa(n) = khat * sqrt(n)
// (heom_ode.cl:211,249 and :321,383).  Per-slot constants are stored at
// position pos(slot) = m * B + b (slot = b*M + m) so that the lanes of a warp,
// which read the same m for different baths, hit different banks.
struct CoefTabs {
    const double* chat;   // [W] at pos(slot)
    const double2* khat;  // [3][W] at pos(slot): kappa_i, kappa_j, kappa_i + kappa_j (n = 1)
    const double* sq;     // [D+2]: sqrt(n)
    const int16_t* pos;   // [W] slot -> position
};

struct DmmaParams {
    PairParams p;
    LaneTab lt;
    CoefTabs ct;
    int* err;
};

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void ld256(const double2* src, double2& a, double2& b)
{
    asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];\n"
                 : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y)
                 : "l"(src));
}

__device__ __forceinline__ void ld256_cg(const double2* src, double2& a, double2& b)
{
    asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];\n"
                 : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y)
                 : "l"(src));
}

// 32-byte stores when ok, without a branch (streaming / default cache policy)
__device__ __forceinline__ void st256_cs_if(bool ok, double2* dst, double2 a, double2 b)
{
    asm volatile("{\n .reg .pred q;\n setp.ne.u32 q, %5, 0;\n @q st.global.cs.v4.f64 [%0], {%1,%2,%3,%4};\n}\n" ::"l"(dst),
                 "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y), "r"((unsigned)ok)
                 : "memory");
}
__device__ __forceinline__ void st256_if(bool ok, double2* dst, double2 a, double2 b)
{
    asm volatile("{\n .reg .pred q;\n setp.ne.u32 q, %5, 0;\n @q st.global.v4.f64 [%0], {%1,%2,%3,%4};\n}\n" ::"l"(dst),
                 "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y), "r"((unsigned)ok)
                 : "memory");
}

__device__ __forceinline__ void st256_cs(double2* dst, double2 a, double2 b)
{
    asm volatile("st.global.cs.v4.f64 [%0], {%1,%2,%3,%4};\n" ::"l"(dst), "d"(a.x), "d"(a.y), "d"(b.x),
                 "d"(b.y)
                 : "memory");
}

__device__ __forceinline__ void st256(double2* dst, double2 a, double2 b)
{
    asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};\n" ::"l"(dst), "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y)
                 : "memory");
}

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// bounded wait for the phase `parity` of an mbarrier; false on expiry
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity)
{
    const unsigned a = smem_addr(bar);
    for (int it = 0; it < (1 << 24); ++it) {
        unsigned done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ int swz(int r) { return ((r & 1) << 2) | (r & 1) | (((r >> 1) & 1) << 1); }

// bytes of one pipeline slot and of a warp's shared area for the DMMA kernel
__host__ __device__ inline int dmma_slot_bytes(int P, int NW, int TWB)
{
    return P * 32 + ((NW * 4 + 15) & ~15) + ((TWB + 15) & ~15) + 16;
}
__host__ __device__ inline int dmma_warp_bytes(int P, int NW, int TWB)
{
    return 2 * dmma_slot_bytes(P, NW, TWB) + 64 * 16 /* exchange tile */ + 16 /* 2 mbarriers */;
}
__host__ inline size_t dmma_smem_bytes(int P, int W, int NW, int TWB, int LS)
{
    return (size_t)dmma_lut_bytes(W, LS) + (size_t)kCtaWarps * dmma_warp_bytes(P, NW, TWB);
}

// MI: the handle holds several instances (p.inst set); each ADO's instance
// selects its H fragments, reloaded whenever the instance changes.
// ADJ: apply the adjoint operator L^H instead of L.  The caller passes the
// tables of -H^H (fragments), conj(pf_same_sum) and conj(gamma0); in the bath
// terms the roles of the neighbours swap: the plus neighbour enters with
// conj(khat) sqrt(n+1), the minus neighbour with -/+ i chat sqrt(n).
template <int N, int HK, int SLT, bool MI, bool ADJ>
__global__ void __launch_bounds__(kCtaWarps * 32, 2) heom_dmma_stage(const DmmaParams dp)
{
    static_assert(N <= 8, "DMMA stage handles N <= 8");
    constexpr int P = pairs_of(N);
    const PairParams& p = dp.p;
    extern __shared__ __align__(128) unsigned char smem[];
    const int W = p.W, LS = p.LS, SL = p.SL;

    double2* s_kh = reinterpret_cast<double2*>(smem);            // 3 * W
    double2* s_sq = s_kh + 3 * W;                                 // LS + 1: (sqrt(n), sqrt(n+1))
    double* s_ch = reinterpret_cast<double*>(s_sq + LS + 1);      // W
    for (int q = threadIdx.x; q < 3 * W; q += blockDim.x) s_kh[q] = dp.ct.khat[q];
    for (int q = threadIdx.x; q < W; q += blockDim.x) s_ch[q] = dp.ct.chat[q];
    for (int q = threadIdx.x; q <= LS; q += blockDim.x)
        s_sq[q] = make_double2(dp.ct.sq[q], q < LS ? dp.ct.sq[q + 1] : 0.0);
    const int lut = dmma_lut_bytes(W, LS);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int slot_b = dmma_slot_bytes(P, p.NW, p.TWB);
    unsigned char* wbase = smem + lut + warp * dmma_warp_bytes(P, p.NW, p.TWB);
    double2* xch = reinterpret_cast<double2*>(wbase + 2 * slot_b);      // 8 x 8 swizzled
    uint64_t* bars = reinterpret_cast<uint64_t*>(wbase + 2 * slot_b + 64 * 16);
    const int tile_b = P * 32;
    const int nbr_off = tile_b;
    const int tup_off = nbr_off + ((p.NW * 4 + 15) & ~15);
    const int pss_off = tup_off + ((p.TWB + 15) & ~15);
    const unsigned tx_bytes = (unsigned)(tile_b + p.NW * 4 + p.TWB + 16);

    // lane tables
    const bool owner = lane < P;
    const int e1 = owner ? dp.lt.e1[lane] : 0, e2 = owner ? dp.lt.e2[lane] : 0;
    const int i1 = e1 / N, j1 = e1 - i1 * N, i2 = e2 / N, j2 = e2 - i2 * N;
    const int diag = (i1 == j1);
    const int si = i1, sj = j1; // sites of the element pair (diagonal: the two diagonal sites are i1 and i2)
    const int fs0 = dp.lt.fs[lane][0], fs1 = dp.lt.fs[lane][1];
    const int ha0 = dp.lt.ha[lane][0], ha1 = dp.lt.ha[lane][1];
    const int r = lane >> 2, t = lane & 3;
    const int xr1 = 8 * i1 + (j1 ^ swz(i1)), xr2 = 8 * i2 + (j2 ^ swz(i2));
    const int xw0 = 8 * r + ((2 * t) ^ swz(r)), xw1 = 8 * r + ((2 * t + 1) ^ swz(r));

    // operand fragments of H / hbar for k-slice s (zero outside the N x N block):
    //   hb = H(4s+t, r) (B operand of w H), ha = -H(r, 4s+t) (A operand of -H w);
    // packed per instance as [re hb s0, s1 | im hb | re ha | im ha][lane]
    double hb_r[2], hb_i[2], ha_r[2], ha_i[2];
    auto load_frag = [&](int ci, double* br, double* bi, double* ar, double* ai) {
        const double* f = dp.p.hfrag + (size_t)ci * 256 + lane;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            br[s] = __ldg(f + 32 * s);
            ar[s] = __ldg(f + 32 * (4 + s));
            if (HK == H_GENERIC) {
                bi[s] = __ldg(f + 32 * (2 + s));
                ai[s] = __ldg(f + 32 * (6 + s));
            } else {
                bi[s] = ai[s] = 0.0;
            }
        }
    };
    const double2 g1 = owner ? p.gamma0[e1] : make_double2(0.0, 0.0);
    const double2 g2 = owner ? p.gamma0[e2] : make_double2(0.0, 0.0);
    int sli[SLT], slj[SLT], pi[SLT], pj[SLT];
#pragma unroll
    for (int q = 0; q < SLT; ++q) {
        // diagonal sectors: element 1 = (i1,i1) uses the slots of site i1, element 2 = (i2,i2) those of i2
        const int a = si, b = diag ? i2 : sj;
        sli[q] = (owner && q < SL) ? p.slots[a * SL + q] : -1;
        slj[q] = (owner && q < SL) ? p.slots[b * SL + q] : -1;
        pi[q] = sli[q] >= 0 ? dp.ct.pos[sli[q]] : 0;
        pj[q] = slj[q] >= 0 ? dp.ct.pos[slj[q]] : 0;
    }
    const double2* kap_i1 = s_kh + (diag ? 2 : 0) * W;
    const double2* kap_j1 = s_kh + 1 * W;
    const double2* kap_i2 = s_kh + 1 * W;
    const double2* kap_j2 = s_kh + (diag ? 2 : 0) * W;

    if (lane == 0) {
        mbar_init(&bars[0]);
        mbar_init(&bars[1]);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    const int64_t nodes = p.nodes;
    const int64_t stride = (int64_t)gridDim.x * kCtaWarps;
    int64_t u = (int64_t)blockIdx.x * kCtaWarps + warp;
    unsigned ph0 = 0u, ph1 = 0u; // mbarrier phase parity of slot 0 / slot 1
    // instance of the current ADO (warp-uniform); its fragments are in hb_* / ha_*
    int ci = (MI && u < nodes) ? __ldg(p.inst + u) : 0;
    // the next ADO's instance, read one iteration ahead of its use so that the
    // instance compare never waits on the load
    int ni_ahead = (MI && u + stride < nodes) ? __ldg(p.inst + u + stride) : ci;
    load_frag(ci, hb_r, hb_i, ha_r, ha_i);

    auto issue = [&](int64_t v, int sl) {
        unsigned char* slot = wbase + sl * slot_b;
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect(&bars[sl], tx_bytes);
        bulk_g2s(slot, p.in + v * (2 * P), tile_b, &bars[sl]);
        bulk_g2s(slot + nbr_off, p.nbr + v * p.NW, p.NW * 4, &bars[sl]);
        bulk_g2s(slot + tup_off, p.tup + v * p.TWB, p.TWB, &bars[sl]);
        bulk_g2s(slot + pss_off, p.pss + v, 16, &bars[sl]);
    };
    if (u < nodes && lane == 0) issue(u, 0);
    int cur = 0;
    bool failed = false;
    for (; u < nodes; u += stride) {
        const int64_t un = u + stride;
        if (un < nodes && lane == 0) issue(un, cur ^ 1);
        // the next ADO's instance and, when it differs, its fragments (used from the next iteration)
        int ni = ci;
        double nb_r[2], nb_i[2], na_r[2], na_i[2];
        if (MI && un < nodes) {
            ni = ni_ahead;
            if (ni != ci) load_frag(ni, nb_r, nb_i, na_r, na_i);
            ni_ahead = un + stride < nodes ? __ldg(p.inst + un + stride) : ni;
        }
        if (!mbar_wait(&bars[cur], cur ? ph1 : ph0)) {
            failed = true;
            break;
        }
        if (cur) ph1 ^= 1u; else ph0 ^= 1u;
        const unsigned char* slot = wbase + cur * slot_b;
        const double2* tile = reinterpret_cast<const double2*>(slot);
        const int32_t* nb = reinterpret_cast<const int32_t*>(slot + nbr_off);
        const unsigned char* tu = slot + tup_off;
        const double2 pss = *reinterpret_cast<const double2*>(slot + pss_off);

        // ---- commutator on the tensor pipe ----
        double cr0 = 0.0, cr1 = 0.0, ci0 = 0.0, ci1 = 0.0;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int fs = s == 0 ? fs0 : fs1;
            const int ha = s == 0 ? ha0 : ha1;
            double2 A = make_double2(0.0, 0.0), B = A;
            if (fs >= 0) {
                A = tile[2 * fs + ha];
                B = (r == 4 * s + t) ? A : tile[2 * fs + (ha ^ 1)];
            }
            dmma(cr0, cr1, A.x, hb_r[s]); // Re(w) Re(H)
            dmma(ci0, ci1, A.y, hb_r[s]); // Im(w) Re(H)
            dmma(cr0, cr1, ha_r[s], B.x); // -Re(H) Re(w)
            dmma(ci0, ci1, ha_r[s], B.y); // -Re(H) Im(w)
            if (HK == H_GENERIC) {
                dmma(cr0, cr1, -A.y, hb_i[s]); // -Im(w) Im(H)
                dmma(ci0, ci1, A.x, hb_i[s]);  //  Re(w) Im(H)
                dmma(cr0, cr1, -ha_i[s], B.y); // +Im(H) Im(w)
                dmma(ci0, ci1, ha_i[s], B.x);  // -Im(H) Re(w)
            }
        }
        xch[xw0] = make_double2(cr0, ci0);
        xch[xw1] = make_double2(cr1, ci1);
        __syncwarp();

        if (owner) {
            const double2 c1 = xch[xr1], c2 = xch[xr2];
            // read the halves in a staggered order (conflict-free quarter warps)
            const int h0 = (lane >> 2) & 1;
            const double2 sa = tile[2 * lane + h0], sb = tile[2 * lane + (h0 ^ 1)];
            const double2 s1 = h0 ? sb : sa, s2 = h0 ? sa : sb;
            double2 L1 = make_double2(-c1.y, c1.x); // i * (w H - H w) / hbar
            double2 L2 = make_double2(-c2.y, c2.x);
            cmac(L1, make_double2(pss.x + g1.x, pss.y + g1.y), s1);
            cmac(L2, make_double2(pss.x + g2.x, pss.y + g2.y), s2);

            // one slot per site: both sides' neighbour rows in one batch (one round trip per ADO)
            constexpr int SB = SLT == 1 ? 2 : 1;
#pragma unroll
            for (int sd0 = 0; sd0 < 2; sd0 += SB) {
                double2 xp[SB][SLT][2], xm[SB][SLT][2];
                int nn[SB][SLT];
#pragma unroll
                for (int bb = 0; bb < SB; ++bb) {
                    const int sd = sd0 + bb;
#pragma unroll
                    for (int q = 0; q < SLT; ++q) {
                        const int sl = sd == 0 ? sli[q] : slj[q];
                        // diagonal elements: the plus terms of L cancel (the minus terms of L^H)
                        const int2 pm = sl >= 0 ? reinterpret_cast<const int2*>(nb)[sl] : make_int2(-1, -1);
                        const int32_t vp = (ADJ || !diag) ? pm.x : -1;
                        const int32_t vm = (!ADJ || !diag) ? pm.y : -1;
                        nn[bb][q] = sl >= 0 ? tu[sl] : 0;
                        xp[bb][q][0] = xp[bb][q][1] = xm[bb][q][0] = xm[bb][q][1] = make_double2(0.0, 0.0);
                        if (vp >= 0) ld256(p.in + (int64_t)vp * (2 * P) + 2 * lane, xp[bb][q][0], xp[bb][q][1]);
                        if (vm >= 0) ld256(p.in + (int64_t)vm * (2 * P) + 2 * lane, xm[bb][q][0], xm[bb][q][1]);
                    }
                }
#pragma unroll
                for (int bb = 0; bb < SB; ++bb) {
                    const int sd = sd0 + bb;
#pragma unroll
                    for (int q = 0; q < SLT; ++q) {
                        const int sl = sd == 0 ? sli[q] : slj[q];
                        if (sl < 0) continue;
                        const int ps = sd == 0 ? pi[q] : pj[q];
                        const double2 sqp = s_sq[nn[bb][q]];
                        const double sq_lo = sqp.x, sq_hi = sqp.y;
                        // L:   i-coefficient term on the plus neighbour (chat sqrt(n+1)),
                        //      complex term on the minus neighbour (khat sqrt(n))
                        // L^H: i-coefficient term on the minus neighbour (-chat sqrt(n)),
                        //      complex term on the plus neighbour (conj(khat) sqrt(n+1))
                        const double c = diag ? 0.0 : (ADJ ? -s_ch[ps] * sq_lo : s_ch[ps] * sq_hi);
                        const double sk = ADJ ? sq_hi : sq_lo;
                        const double2 t1 = ADJ ? xm[bb][q][0] : xp[bb][q][0], t2 = ADJ ? xm[bb][q][1] : xp[bb][q][1];
                        const double2 k1 = ADJ ? xp[bb][q][0] : xm[bb][q][0], k2 = ADJ ? xp[bb][q][1] : xm[bb][q][1];
                        // the complex-coefficient neighbour scales as sqrt(n) (sqrt(n+1) for L^H); fold it in
                        const double2 m1 = make_double2(k1.x * sk, k1.y * sk);
                        const double2 m2 = make_double2(k2.x * sk, k2.y * sk);
                        auto kap = [&](const double2* tab) {
                            const double2 v = tab[ps];
                            return ADJ ? make_double2(v.x, -v.y) : v;
                        };
                        if (sd == 0) {
                            L1.x = fma(-c, t1.y, L1.x);
                            L1.y = fma(c, t1.x, L1.y);
                            L2.x = fma(c, t2.y, L2.x);
                            L2.y = fma(-c, t2.x, L2.y);
                            cmac(L1, kap(kap_i1), m1);
                            if (!diag) cmac(L2, kap(kap_i2), m2);
                        } else {
                            L1.x = fma(c, t1.y, L1.x);
                            L1.y = fma(-c, t1.x, L1.y);
                            L2.x = fma(-c, t2.y, L2.x);
                            L2.y = fma(c, t2.x, L2.y);
                            if (!diag) cmac(L1, kap(kap_j1), m1);
                            cmac(L2, kap(kap_j2), m2);
                        }
                    }
                }
            }

            const int64_t off = u * (2 * P) + 2 * lane;
            double2 x1 = s1, x2 = s2;
            if (p.y) ld256_cg(p.y + off, x1, x2);
            double2 o1 = make_double2(p.alpha.x * x1.x - p.alpha.y * x1.y, p.alpha.x * x1.y + p.alpha.y * x1.x);
            double2 o2 = make_double2(p.alpha.x * x2.x - p.alpha.y * x2.y, p.alpha.x * x2.y + p.alpha.y * x2.x);
            cmac(o1, p.beta, L1);
            cmac(o2, p.beta, L2);
            st256_cs(p.out + off, o1, o2);
            if (p.use_acc) {
                double2 a1 = s1, a2 = s2;
                if (!p.acc_init) ld256_cg(p.acc + off, a1, a2);
                cmac(a1, p.acc_beta, L1);
                cmac(a2, p.acc_beta, L2);
                st256(p.acc + off, a1, a2);
            }
        }
        __syncwarp();
        cur ^= 1;
        if (MI && ni != ci) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                hb_r[s] = nb_r[s];
                hb_i[s] = nb_i[s];
                ha_r[s] = na_r[s];
                ha_i[s] = na_i[s];
            }
            ci = ni;
        }
    }
    if (failed) {
        if (lane == 0) atomicExch(dp.err, 1);
        // let copies still in flight land before the warp leaves (bounded)
        mbar_wait(&bars[cur ^ 1], cur ? ph0 : ph1);
    }
}

// ---------------------------------------------------------------------------
// Lockstep ensembles (N <= 8): K instances that share the hierarchy graph and
// the bath tables and differ in H only (the realisations of a static-disorder
// ensemble of one depth) are stored instance-minor: sector p of ADO u of
// instance k at sector index (u * P + p) * Kp + k (Kp = K rounded up to 32),
// so that the 32 instances of a block sit side by side in every row.
//
// Work item = (ADO u, block of 32 instances), swept grid-stride by a CTA of
// eight warps:
//   A  the block's 32 tiles arrive by 16-byte cp.async in a shared tile
//      [p][32] whose columns are swizzled (k ^ (p & 3)), which keeps the
//      conflict-free operand reads of the pair order; warp w computes the
//      commutator of instances w, w+8, w+16, w+24 on the tensor pipe (the
//      operand mapping and exchange of heom_dmma_stage) and writes the two
//      commutator values of every sector into a second shared tile;
//   B  warp w takes sectors w, w+8, ...; lane k is instance k of the block.
//      Neighbour indices, tuple entries and bath coefficients are the same
//      for every lane (warp-uniform), and each neighbour read is one
//      contiguous 1-KB row (32 instances x 32 B) of the neighbour ADO, where
//      heom_dmma_stage gathers 32-B sectors of eight different neighbours.
// The derivative is the same element by element as heom_dmma_stage's (the
// same bath-term order; the commutator from the same MMA sequence).
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// N = 9..16: a team of TW = ceil(P / 32) warps per ADO, thread p of the team
// owns sector p.  Teams loop over ADOs (grid-stride) with a two-slot
// pipeline: while ADO k is computed, its successor's tile (scattered into the
// row-major tile_pos layout), neighbour row, tuple row and pf_same_sum arrive
// by cp.async.
//
// Commutator on the FP64 tensor pipe: the tile is zero-padded to 16 x 16 and
// cut into 2 x 2 blocks of 8 x 8; block (I, J) of C = w H - H w takes
// ceil(N/4) k-slices of m8n8k4 MMAs (A = w(8I+g, 4s+t) against the H
// fragment hb(J, s); ha(I, s) against B = w(4s+t, 8J+g)).  Warp wt of the
// team computes blocks [4 wt / TW, 4 (wt+1) / TW) and writes them to the
// team's exchange tile; after a team barrier every owner reads the two
// elements of its sector.  (Cutting the work finer, into the real and
// imaginary parts of each block, balances the warps of a three-warp team but
// doubles the operand reads and measured slower.)  The bath terms follow the
// same formulas as the DMMA kernel, one 32-byte sector load per neighbour.
// ---------------------------------------------------------------------------

// issue the asynchronous copies of ADO u into a team slot
template <int N>
__device__ __forceinline__ void prefetch_ado(unsigned char* slot, const PairParams& p, const PairSmem& L,
                                             int64_t u, int lt, int tt, int e1, int e2, bool active)
{
    double2* tile = reinterpret_cast<double2*>(slot + L.tile_off);
    if (active) {
        const double2* src = p.in + u * (2 * pairs_of(N));
        const int i1 = e1 / N, j1 = e1 - i1 * N, i2 = e2 / N, j2 = e2 - i2 * N;
        cp_async16(tile + tile_pos(N, i1, j1), src + 2 * lt);
        cp_async16(tile + tile_pos(N, i2, j2), src + 2 * lt + 1);
    }
    int32_t* nb = reinterpret_cast<int32_t*>(slot + L.nbr_off);
    for (int q = lt * 4; q < p.NW; q += tt * 4) cp_async16(nb + q, p.nbr + u * p.NW + q);
    unsigned char* tu = slot + L.tup_off;
    for (int q = lt * 16; q < p.TWB; q += tt * 16) cp_async16(tu + q, p.tup + u * p.TWB + q);
    if (lt == 0) cp_async16(slot + L.pss_off, p.pss + u);
}

// ADJ: the adjoint operator L^H (see heom_dmma_stage).  The bath
// coefficients are the factored tables of heom_dmma_stage (CoefTabs).
// (three CTAs per SM where at most two slots per state keep the register
// demand low enough; two otherwise)
template <int N, int HK, int SLT, bool ADJ>
__global__ void __launch_bounds__(kCtaWarps * 32, SLT <= 2 ? 3 : 2) heom_pair_stage(const DmmaParams dp)
{
    static_assert(N > 8 && N <= 16, "team kernel handles N = 9..16");
    constexpr int P = pairs_of(N);
    constexpr int TW = team_warps(N);
    constexpr int TT = 32 * TW;
    constexpr int TEAMS = kCtaWarps / TW;
    constexpr int KS = (N + 3) / 4; // k-slices of the padded commutator
    constexpr int FD = frag_doubles(N);
    extern __shared__ __align__(128) unsigned char smem[];
    const PairParams& p = dp.p;
    const PairSmem L = pair_smem_layout(N, p.W, p.NW, p.TWB, p.LS);
    const int W = p.W, LS = p.LS, SL = p.SL;

    double2* s_kh = reinterpret_cast<double2*>(smem);      // 3 * W
    double2* s_sq = s_kh + 3 * W;                           // LS + 1: (sqrt(n), sqrt(n+1))
    double* s_ch = reinterpret_cast<double*>(s_sq + LS + 1); // W
    int16_t* s_pos = reinterpret_cast<int16_t*>(s_ch + W);   // W
    for (int q = threadIdx.x; q < 3 * W; q += blockDim.x) s_kh[q] = dp.ct.khat[q];
    for (int q = threadIdx.x; q < W; q += blockDim.x) s_ch[q] = dp.ct.chat[q];
    for (int q = threadIdx.x; q <= LS; q += blockDim.x)
        s_sq[q] = make_double2(dp.ct.sq[q], q < LS ? dp.ct.sq[q + 1] : 0.0);
    for (int q = threadIdx.x; q < W; q += blockDim.x) s_pos[q] = dp.ct.pos[q];

    const int team = threadIdx.x / TT;
    const int lt = threadIdx.x - team * TT;
    const bool active = team < TEAMS && lt < P;
    unsigned char* team_base = smem + L.lut + team * L.team;
    double2* xch = reinterpret_cast<double2*>(team_base + L.xch_off);
    const int wt = lt >> 5, lane = lt & 31, g = lane >> 2, t4 = lane & 3;
    const int blk0 = wt * 4 / TW, blk1 = (wt + 1) * 4 / TW; // commutator blocks of this warp

    int e1 = 0, e2 = 0, i = 0, j = 0, diag = 0;
    if (active) pair_elements(N, lt, &e1, &e2, &i, &j, &diag);

    const double2 g1 = active ? p.gamma0[e1] : make_double2(0.0, 0.0);
    const double2 g2 = active ? p.gamma0[e2] : make_double2(0.0, 0.0);
    int sli[SLT], slj[SLT];
#pragma unroll
    for (int q = 0; q < SLT; ++q) {
        sli[q] = (active && q < SL) ? p.slots[i * SL + q] : -1;
        slj[q] = (active && q < SL) ? p.slots[j * SL + q] : -1;
    }
    // coefficient tables seen by the two elements of this sector
    const double2* kap_i1 = s_kh + (diag ? 2 : 0) * W; // element 1, slots of site i
    const double2* kap_j1 = s_kh + 1 * W;              // element 1, slots of site j (off-diagonal)
    const double2* kap_i2 = s_kh + 1 * W;              // element 2 = (j,i), slots of site i (its j side)
    const double2* kap_j2 = s_kh + (diag ? 2 : 0) * W; // element 2, slots of site j

    __syncthreads();
    if (team >= TEAMS) return;

    const int64_t nodes = p.nodes;
    const int64_t stride = (int64_t)gridDim.x * TEAMS;
    int64_t u = (int64_t)blockIdx.x * TEAMS + team;
    int cur = 0;
    if (u < nodes) prefetch_ado<N>(team_base, p, L, u, lt, TT, e1, e2, active);
    cp_async_wait_all();
    team_sync<TW>(team);
    int ci = (p.inst && u < nodes) ? __ldg(p.inst + u) : 0; // instance of the current ADO

    for (; u < nodes; u += stride) {
        unsigned char* slot = team_base + cur * L.slot;
        const int64_t un = u + stride;
        int ni = ci;
        if (un < nodes) {
            prefetch_ado<N>(team_base + (cur ^ 1) * L.slot, p, L, un, lt, TT, e1, e2, active);
            if (p.inst) ni = __ldg(p.inst + un);
        }
        const double2* t = reinterpret_cast<const double2*>(slot + L.tile_off);

        // ---- commutator w H - H w / hbar on the tensor pipe, into the exchange tile ----
        const double* fr = p.hfrag + (size_t)ci * FD;
#pragma unroll
        for (int blk = 0; blk < 4; ++blk) {
            if (blk < blk0 || blk >= blk1) continue;
            const int I = blk >> 1, J = blk & 1;
            double cr0 = 0.0, cr1 = 0.0, ci0 = 0.0, ci1 = 0.0;
#pragma unroll
            for (int s = 0; s < KS; ++s) {
                const int ra = 8 * I + g, ka = 4 * s + t4; // A = w(ra, ka), B = w(ka, cb)
                const int cb = 8 * J + g;
                const double2 z = make_double2(0.0, 0.0);
                const double2 A = (ra < N && ka < N) ? t[tile_pos(N, ra, ka)] : z;
                const double2 B = (ka < N && cb < N) ? t[tile_pos(N, ka, cb)] : z;
                const double hbr = __ldg(fr + frag_index(N, 0, J, s, lane));
                const double har = __ldg(fr + frag_index(N, 2, I, s, lane));
                dmma(cr0, cr1, A.x, hbr); // Re(w) Re(H)
                dmma(ci0, ci1, A.y, hbr); // Im(w) Re(H)
                dmma(cr0, cr1, har, B.x); // -Re(H) Re(w)
                dmma(ci0, ci1, har, B.y); // -Re(H) Im(w)
                if (HK == H_GENERIC) {
                    const double hbi = __ldg(fr + frag_index(N, 1, J, s, lane));
                    const double hai = __ldg(fr + frag_index(N, 3, I, s, lane));
                    dmma(cr0, cr1, -A.y, hbi); // -Im(w) Im(H)
                    dmma(ci0, ci1, A.x, hbi);  //  Re(w) Im(H)
                    dmma(cr0, cr1, -hai, B.y); // +Im(H) Im(w)
                    dmma(ci0, ci1, hai, B.x);  // -Im(H) Re(w)
                }
            }
            double2* xr = xch + (8 * I + g) * kXchStride + 8 * J + 2 * t4;
            xr[0] = make_double2(cr0, ci0);
            xr[1] = make_double2(cr1, ci1);
        }

        // the bath terms first: they need only the staged tile and the
        // neighbours, so a warp that finished its commutator blocks goes on
        // while the others complete theirs; the exchange tile is read after
        // the team barrier
        const int i1 = e1 / N, j1 = e1 - i1 * N, i2 = e2 / N, j2 = e2 - i2 * N;
        double2 L1 = make_double2(0.0, 0.0), L2 = L1, s1 = L1, s2 = L1;
        if (active) {
            const int32_t* nb = reinterpret_cast<const int32_t*>(slot + L.nbr_off);
            const unsigned char* tu = slot + L.tup_off;
            const double2 pss = *reinterpret_cast<const double2*>(slot + L.pss_off);
            s1 = t[tile_pos(N, i1, j1)];
            s2 = t[tile_pos(N, i2, j2)];

            // ---- same term ----
            cmac(L1, make_double2(pss.x + g1.x, pss.y + g1.y), s1);
            cmac(L2, make_double2(pss.x + g2.x, pss.y + g2.y), s2);

            // ---- neighbours: per side all loads first, then the updates ----
            // side 0 = slots of site i, side 1 = slots of site j
            // one slot per state: both sides' neighbour rows in one batch
            constexpr int SB = SLT == 1 ? 2 : 1;
#pragma unroll
            for (int sd0 = 0; sd0 < 2; sd0 += SB) {
                double2 xp[SB][SLT][2], xm[SB][SLT][2];
                int nn[SB][SLT];
#pragma unroll
                for (int bb = 0; bb < SB; ++bb) {
                    const int sd = sd0 + bb;
#pragma unroll
                    for (int q = 0; q < SLT; ++q) {
                        const int sl = sd == 0 ? sli[q] : slj[q];
                        const int2 pm = sl >= 0 ? reinterpret_cast<const int2*>(nb)[sl] : make_int2(-1, -1);
                        const int32_t vp = (ADJ || !diag) ? pm.x : -1;
                        const int32_t vm = (!ADJ || !diag) ? pm.y : -1;
                        nn[bb][q] = sl >= 0 ? tu[sl] : 0;
                        xp[bb][q][0] = xp[bb][q][1] = xm[bb][q][0] = xm[bb][q][1] = make_double2(0.0, 0.0);
                        if (vp >= 0) ld256(p.in + (int64_t)vp * (2 * P) + 2 * lt, xp[bb][q][0], xp[bb][q][1]);
                        if (vm >= 0) ld256(p.in + (int64_t)vm * (2 * P) + 2 * lt, xm[bb][q][0], xm[bb][q][1]);
                    }
                }
#pragma unroll
                for (int bb = 0; bb < SB; ++bb) {
                    const int sd = sd0 + bb;
#pragma unroll
                    for (int q = 0; q < SLT; ++q) {
                        const int sl = sd == 0 ? sli[q] : slj[q];
                        if (sl < 0) continue;
                        const int ps = s_pos[sl];
                        const double2 sqp = s_sq[nn[bb][q]];
                        const double sq_lo = sqp.x, sq_hi = sqp.y;
                        // L: i chat sqrt(n+1) on the plus neighbour, khat sqrt(n) on the minus one;
                        // L^H: -i chat sqrt(n) on the minus neighbour, conj(khat) sqrt(n+1) on the plus one
                        const double c = diag ? 0.0 : (ADJ ? -s_ch[ps] * sq_lo : s_ch[ps] * sq_hi);
                        const double sk = ADJ ? sq_hi : sq_lo;
                        const double2 t1 = ADJ ? xm[bb][q][0] : xp[bb][q][0], t2 = ADJ ? xm[bb][q][1] : xp[bb][q][1];
                        const double2 k1 = ADJ ? xp[bb][q][0] : xm[bb][q][0], k2 = ADJ ? xp[bb][q][1] : xm[bb][q][1];
                        const double2 m1 = make_double2(k1.x * sk, k1.y * sk);
                        const double2 m2 = make_double2(k2.x * sk, k2.y * sk);
                        auto kap = [&](const double2* tab) {
                            const double2 v = tab[ps];
                            return ADJ ? make_double2(v.x, -v.y) : v;
                        };
                        if (sd == 0) {
                            // site i: element 1 (i,j) i-side (+i c, kappa_i); element 2 (j,i) j-side (-i c, kappa_j)
                            L1.x = fma(-c, t1.y, L1.x);
                            L1.y = fma(c, t1.x, L1.y);
                            L2.x = fma(c, t2.y, L2.x);
                            L2.y = fma(-c, t2.x, L2.y);
                            cmac(L1, kap(kap_i1), m1);
                            if (!diag) cmac(L2, kap(kap_i2), m2);
                        } else {
                            // site j: element 1 j-side (-i c, kappa_j); element 2 i-side (+i c, kappa_i)
                            L1.x = fma(c, t1.y, L1.x);
                            L1.y = fma(-c, t1.x, L1.y);
                            L2.x = fma(-c, t2.y, L2.x);
                            L2.y = fma(c, t2.x, L2.y);
                            if (!diag) cmac(L1, kap(kap_j1), m1);
                            cmac(L2, kap(kap_j2), m2);
                        }
                    }
                }
            }

        }
        team_sync<TW>(team);

        if (active) {
            // ---- commutator: i * (w H - H w) / hbar from the exchange tile ----
            const double2 c1 = xch[i1 * kXchStride + j1], c2 = xch[i2 * kXchStride + j2];
            L1.x -= c1.y;
            L1.y += c1.x;
            L2.x -= c2.y;
            L2.y += c2.x;

            // ---- stage write ----
            const int64_t off = u * (2 * P) + 2 * lt;
            double2 x1 = s1, x2 = s2;
            if (p.y) ld256_cg(p.y + off, x1, x2);
            double2 r1 = make_double2(p.alpha.x * x1.x - p.alpha.y * x1.y, p.alpha.x * x1.y + p.alpha.y * x1.x);
            double2 r2 = make_double2(p.alpha.x * x2.x - p.alpha.y * x2.y, p.alpha.x * x2.y + p.alpha.y * x2.x);
            cmac(r1, p.beta, L1);
            cmac(r2, p.beta, L2);
            st256_cs(p.out + off, r1, r2);
            if (p.use_acc) {
                double2 a1 = s1, a2 = s2;
                if (!p.acc_init) ld256_cg(p.acc + off, a1, a2);
                cmac(a1, p.acc_beta, L1);
                cmac(a2, p.acc_beta, L2);
                st256(p.acc + off, a1, a2);
            }
        }
        cp_async_wait_all();
        team_sync<TW>(team);
        cur ^= 1;
        ci = ni;
    }
}

// out = y + h * sum_l c_l k_l over doubles, terms with c_l == 0 skipped, in
// the operation order of rk_weighted_add.cl:78-95 (no contraction).
struct WaddParams {
    double* out;
    const double* y;
    const double* k[7];
    double c[7];
    int n;
    double h;
    int64_t len;
};

__global__ void heom_weighted_add(const WaddParams p)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < p.len; e += stride) {
        double acc = 0.0;
        for (int l = 0; l < p.n; ++l)
            if (p.c[l] != 0.0) acc = __dadd_rn(acc, __dmul_rn(p.c[l], p.k[l][e]));
        acc = __dmul_rn(acc, p.h);
        acc = __dadd_rn(acc, p.y[e]);
        p.out[e] = acc;
    }
}

// Reference layout (row-major tiles in uid order) <-> pair layout in the
// internal ADO order, over the reference ADOs [r0, r0 + count) whose tiles
// are (or go) back to back in `ref`.  pe[2p], pe[2p+1] = element indices of
// the halves of sector p (equal for the padding half).  One thread per
// (ADO, sector): the pair side is written / read as whole 32-byte sectors.
__global__ void heom_to_pairs(double2* __restrict__ dst, const double2* __restrict__ ref,
                              const int64_t* __restrict__ int_of_ref, const int16_t* __restrict__ pe,
                              int64_t r0, int64_t count, int n, int P)
{
    const int64_t total = count * P;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += stride) {
        const int64_t r = q / P;
        const int pr = (int)(q - r * P);
        const int64_t u = int_of_ref[r0 + r];
        const double2* src = ref + r * n * n;
        dst[(u * P + pr) * 2] = src[pe[2 * pr]];
        dst[(u * P + pr) * 2 + 1] = src[pe[2 * pr + 1]];
    }
}

__global__ void heom_from_pairs(double2* __restrict__ ref, const double2* __restrict__ src,
                                const int64_t* __restrict__ int_of_ref, const int16_t* __restrict__ pe,
                                int64_t r0, int64_t count, int n, int P)
{
    const int64_t total = count * P;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += stride) {
        const int64_t r = q / P;
        const int pr = (int)(q - r * P);
        const int64_t u = int_of_ref[r0 + r];
        double2* dst = ref + r * n * n;
        const int e1 = pe[2 * pr], e2 = pe[2 * pr + 1];
        dst[e1] = src[(u * P + pr) * 2];
        if (e2 != e1) dst[e2] = src[(u * P + pr) * 2 + 1];
    }
}

// Copy the top matrix of every instance (block k: internal ADO tops[k], pair
// layout) into row `row` of a row-major log [rows][n_inst][n*n].
// sector index of sector p of internal ADO u: the per-instance layout (kp = 0)
// or the lockstep layout of instance k (stride kp)
__device__ __forceinline__ int64_t sector_index(int64_t u, int p, int P, int64_t kp, int64_t k)
{
    return kp ? (u * P + p) * kp + k : u * P + p;
}

// block b: the instance k0 + b of a lockstep handle (kp > 0), ignored otherwise
__global__ void heom_record_top(double2* __restrict__ log, const double2* __restrict__ y,
                                const int16_t* __restrict__ pe, const int64_t* __restrict__ tops, int n, int P,
                                int64_t row, int64_t kp, int64_t k0)
{
    const int k = blockIdx.x;
    const int64_t u = tops[k];
    double2* dst = log + (row * gridDim.x + k) * n * n;
    for (int pr = threadIdx.x; pr < P; pr += blockDim.x) {
        const int e1 = pe[2 * pr], e2 = pe[2 * pr + 1];
        const int64_t sx = sector_index(u, pr, P, kp, k0 + k);
        dst[e1] = y[sx * 2];
        if (e2 != e1) dst[e2] = y[sx * 2 + 1];
    }
}

// heom_record_top into row *base + j (a device offset, for captured graphs)
__global__ void heom_record_top_at(double2* __restrict__ log, const double2* __restrict__ y,
                                   const int16_t* __restrict__ pe, const int64_t* __restrict__ tops, int n, int P,
                                   const int64_t* __restrict__ base, int64_t j)
{
    const int k = blockIdx.x;
    const int64_t u = tops[k];
    double2* dst = log + ((*base + j) * gridDim.x + k) * n * n;
    for (int pr = threadIdx.x; pr < P; pr += blockDim.x) {
        const int e1 = pe[2 * pr], e2 = pe[2 * pr + 1];
        dst[e1] = y[(u * P + pr) * 2];
        if (e2 != e1) dst[e2] = y[(u * P + pr) * 2 + 1];
    }
}

// Write row-major top matrices top[k] ([n_inst][n*n]) into the pair layout
// of each instance's top ADO (block k).
__global__ void heom_write_top(double2* __restrict__ y, const double2* __restrict__ top,
                               const int16_t* __restrict__ pe, const int64_t* __restrict__ tops, int n, int P,
                               int64_t kp, int64_t k0)
{
    const int k = blockIdx.x;
    const int64_t u = tops[k];
    const double2* src = top + (int64_t)k * n * n;
    for (int pr = threadIdx.x; pr < P; pr += blockDim.x) {
        const int64_t sx = sector_index(u, pr, P, kp, k0 + k);
        y[sx * 2] = src[pe[2 * pr]];
        y[sx * 2 + 1] = src[pe[2 * pr + 1]];
    }
}

// ---------------------------------------------------------------------------
// Adjoint gradients.  For one RK4 stage factor F_k = I + beta_k h L of the
// product form, dJ/dtheta gains Re(beta_k h <a, dL/dtheta w>), with a the
// adjoint after the later factors and w the stage input (<x, y> = x^H y).
//   H:      <a, dL/dH_ab w> = (i/hbar) Z(a,b),
//           Z = sum_u (w_u^T conj(a_u) - conj(a_u) w_u^T)          (all a, b at once)
//   lambda, gamma (shared by all baths): L is linear in its coefficient
//           tables, so dL/dtheta is L with H = 0 and the tables replaced by
//           their derivatives (dpss, dgamma0, dchat, dkhat).
// One warp per ADO; lanes own sectors (pair layout).  The blocks are split
// among the instances of the handle (each block sweeps one instance's ADOs),
// and every block adds weight * (its sum) to its own row of `partial`
// (deterministic; summed per instance on the host at the end).
// ---------------------------------------------------------------------------
struct GradParams {
    const double2* __restrict__ a;     // adjoint (pair layout, internal order)
    const double2* __restrict__ w;     // forward stage input
    const int32_t* __restrict__ nbr;   // [nodes][NW] (plus, minus) of every slot
    const uint8_t* __restrict__ tup;   // [nodes][TWB]
    const int16_t* __restrict__ pe;    // [2P] element indices of the sector halves
    const int16_t* __restrict__ slots; // [N][SL] slot ids of each state, -1 padded
    const double* __restrict__ dpss;   // [nodes] d pf_same_sum / d gamma (real)
    const double2* __restrict__ dg0;   // [2][N*N] d gamma0 / d(lambda, gamma)
    const double* __restrict__ dchat;  // [2][W] d chat
    const double2* __restrict__ dkhat; // [2][3][W] d khat (side i, side j, diagonal)
    const double* __restrict__ sq;     // [LS+1] sqrt(n)
    double2 weight;                    // beta_k h
    double2* partial;                  // [gridDim.x][N*N + 2]
    const int64_t* inst_base;          // [instances + 1] first ADO of every instance
    int blocks_per_inst;               // blocks [k*bpi, (k+1)*bpi) sweep instance k only
    int N, P, W, NW, TWB, SL;
    int want_h;                        // accumulate Z (the H gradient)
    int want_bath;                     // accumulate <a, L_theta' w> (the lambda and gamma gradients)
};

__host__ __device__ inline int grad_warp_bytes(int n) { return 2 * n * (n + 1) * 16; }
__host__ inline size_t grad_smem_bytes(int n)
{
    return (size_t)kCtaWarps * grad_warp_bytes(n) + (size_t)kCtaWarps * (n * n + 2) * 16;
}

__global__ void __launch_bounds__(kCtaWarps * 32) heom_adjoint_grad(const GradParams g)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int N = g.N, P = g.P, W = g.W, SL = g.SL, NN = N * N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double2* At = reinterpret_cast<double2*>(smem + warp * grad_warp_bytes(N)); // [N][N+1]
    double2* Wt = At + N * (N + 1);
    double2* red = reinterpret_cast<double2*>(smem + kCtaWarps * grad_warp_bytes(N)); // [warps][NN+2]
    // Z on the FP64 tensor pipe: blocks (I, J) of 8 x 8 of the zero-padded Z (one block for
    // N <= 8, 2 x 2 for N <= 16), accumulated over the warp's ADOs in the MMA fragments:
    // lane 4g + t holds Z(8I+g, 8J+2t) and Z(8I+g, 8J+2t+1), real and imaginary parts
    const int gq = lane >> 2, t4 = lane & 3;
    const int nblk = N <= 8 ? 1 : 4, ks = (N + 3) / 4;
    double zr[4][2], zi[4][2];
#pragma unroll
    for (int b = 0; b < 4; ++b) zr[b][0] = zr[b][1] = zi[b][0] = zi[b][1] = 0.0;
    double2 dl = make_double2(0.0, 0.0), dgm = dl;
    auto el = [&](const double2* T, int r, int c) {
        return (r < N && c < N) ? T[r * (N + 1) + c] : make_double2(0.0, 0.0);
    };

    const int inst = blockIdx.x / g.blocks_per_inst, jb = blockIdx.x - inst * g.blocks_per_inst;
    const int64_t stride = (int64_t)g.blocks_per_inst * kCtaWarps, end = g.inst_base[inst + 1];
    for (int64_t u = g.inst_base[inst] + (int64_t)jb * kCtaWarps + warp; u < end; u += stride) {
        const int32_t* nb = g.nbr + u * g.NW;
        const uint8_t* tu = g.tup + u * g.TWB;
        const double dps = g.dpss[u];
        for (int p = lane; p < P; p += 32) {
            const int e1 = g.pe[2 * p], e2 = g.pe[2 * p + 1];
            const int i1 = e1 / N, j1 = e1 - i1 * N, i2 = e2 / N, j2 = e2 - i2 * N;
            double2 a1, a2, w1, w2;
            ld256(g.a + (u * P + p) * 2, a1, a2);
            ld256(g.w + (u * P + p) * 2, w1, w2);
            At[i1 * (N + 1) + j1] = a1;
            At[i2 * (N + 1) + j2] = a2;
            Wt[i1 * (N + 1) + j1] = w1;
            Wt[i2 * (N + 1) + j2] = w2;
            const bool diag = i1 == j1;
            const bool twin = e2 == e1; // padding half of an odd diagonal pair
            if (!g.want_bath) continue;
            // derivative of the operator applied to w, for theta = lambda (0), gamma (1)
            double2 D1[2], D2[2];
            for (int th = 0; th < 2; ++th) {
                const double2 s1 = g.dg0[th * NN + e1], s2 = g.dg0[th * NN + e2];
                const double sp = th == 1 ? dps : 0.0;
                D1[th] = make_double2((sp + s1.x) * w1.x - s1.y * w1.y, (sp + s1.x) * w1.y + s1.y * w1.x);
                D2[th] = make_double2((sp + s2.x) * w2.x - s2.y * w2.y, (sp + s2.x) * w2.y + s2.y * w2.x);
            }
            // bath terms: side 0 = slots of site i1, side 1 = slots of site j1
            // (diagonal pairs: element 1 takes the slots of i1, element 2 those of i2)
            for (int sd = 0; sd < 2; ++sd) {
                const int site = sd == 0 ? i1 : (diag ? i2 : j1);
                for (int q = 0; q < SL; ++q) {
                    const int sl = g.slots[site * SL + q];
                    if (sl < 0) continue;
                    const int n = tu[sl];
                    const int2 pm = reinterpret_cast<const int2*>(nb)[sl];
                    const int32_t vp = diag ? -1 : pm.x;
                    const int32_t vm = pm.y;
                    double2 p1 = make_double2(0.0, 0.0), p2 = p1, m1 = p1, m2 = p1;
                    if (vp >= 0) ld256(g.w + ((int64_t)vp * P + p) * 2, p1, p2);
                    if (vm >= 0) ld256(g.w + ((int64_t)vm * P + p) * 2, m1, m2);
                    const double shi = g.sq[n + 1], slo = g.sq[n];
                    for (int th = 0; th < 2; ++th) {
                        const double c = g.dchat[th * W + sl] * shi;
                        const double2* kh = g.dkhat + th * 3 * W;
                        if (diag) {
                            // element (site, site): kappa_i + kappa_j only
                            const double2 k = kh[2 * W + sl];
                            double2& D = sd == 0 ? D1[th] : D2[th];
                            cmac(D, make_double2(k.x * slo, k.y * slo), sd == 0 ? m1 : m2);
                        } else if (sd == 0) {
                            // site i: element 1 (i,j) i-side, element 2 (j,i) j-side
                            D1[th].x -= c * p1.y; D1[th].y += c * p1.x;
                            D2[th].x += c * p2.y; D2[th].y -= c * p2.x;
                            const double2 ki = kh[sl], kj = kh[W + sl];
                            cmac(D1[th], make_double2(ki.x * slo, ki.y * slo), m1);
                            cmac(D2[th], make_double2(kj.x * slo, kj.y * slo), m2);
                        } else {
                            D1[th].x += c * p1.y; D1[th].y -= c * p1.x;
                            D2[th].x -= c * p2.y; D2[th].y += c * p2.x;
                            const double2 ki = kh[sl], kj = kh[W + sl];
                            cmac(D1[th], make_double2(kj.x * slo, kj.y * slo), m1);
                            cmac(D2[th], make_double2(ki.x * slo, ki.y * slo), m2);
                        }
                    }
                }
            }
            // <a, D>: conj(a) * D over the sector's elements (a padding half counts once)
            double2* acc[2] = {&dl, &dgm};
            for (int th = 0; th < 2; ++th) {
                acc[th]->x += a1.x * D1[th].x + a1.y * D1[th].y;
                acc[th]->y += a1.x * D1[th].y - a1.y * D1[th].x;
                if (!twin) {
                    acc[th]->x += a2.x * D2[th].x + a2.y * D2[th].y;
                    acc[th]->y += a2.x * D2[th].y - a2.y * D2[th].x;
                }
            }
        }
        __syncwarp();
        // Z(k,l) = sum_i w(i,k) conj(a(i,l)) - sum_j conj(a(k,j)) w(l,j):
        //   Re Z = Wr^T Ar + Wi^T Ai - Ar Wr^T - Ai Wi^T, Im Z = Wi^T Ar - Wr^T Ai - Ar Wi^T + Ai Wr^T
        if (g.want_h) {
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                if (b >= nblk) continue;
                const int I = b >> 1, J = b & 1;
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    if (s >= ks) continue;
                    const int k0 = 4 * s + t4;
                    const double2 wT = el(Wt, k0, 8 * I + gq); // A operand of W^T A: W(4s+t, 8I+g)
                    const double2 aB = el(At, k0, 8 * J + gq); // B operand of W^T A: A(4s+t, 8J+g)
                    const double2 aA = el(At, 8 * I + gq, k0); // A operand of A W^T: A(8I+g, 4s+t)
                    const double2 wB = el(Wt, 8 * J + gq, k0); // B operand of A W^T: W(8J+g, 4s+t)
                    dmma(zr[b][0], zr[b][1], wT.x, aB.x);
                    dmma(zr[b][0], zr[b][1], wT.y, aB.y);
                    dmma(zr[b][0], zr[b][1], -aA.x, wB.x);
                    dmma(zr[b][0], zr[b][1], -aA.y, wB.y);
                    dmma(zi[b][0], zi[b][1], wT.y, aB.x);
                    dmma(zi[b][0], zi[b][1], -wT.x, aB.y);
                    dmma(zi[b][0], zi[b][1], -aA.x, wB.y);
                    dmma(zi[b][0], zi[b][1], aA.y, wB.x);
                }
            }
        }
        __syncwarp();
    }
    // block sum in a fixed order, then weight * sum into this block's row
    double2* mine = red + warp * (NN + 2);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        if (b >= nblk) continue;
        const int r = 8 * (b >> 1) + gq;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int c = 8 * (b & 1) + 2 * t4 + e;
            if (r < N && c < N) mine[r * N + c] = make_double2(zr[b][e], zi[b][e]);
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        dl.x += __shfl_down_sync(0xffffffffu, dl.x, off);
        dl.y += __shfl_down_sync(0xffffffffu, dl.y, off);
        dgm.x += __shfl_down_sync(0xffffffffu, dgm.x, off);
        dgm.y += __shfl_down_sync(0xffffffffu, dgm.y, off);
    }
    if (lane == 0) {
        mine[NN] = dl;
        mine[NN + 1] = dgm;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NN + 2; q += blockDim.x) {
        double2 s = make_double2(0.0, 0.0);
        for (int v = 0; v < kCtaWarps; ++v) {
            s.x += red[v * (NN + 2) + q].x;
            s.y += red[v * (NN + 2) + q].y;
        }
        double2& out = g.partial[(int64_t)blockIdx.x * (NN + 2) + q];
        out.x += g.weight.x * s.x - g.weight.y * s.y;
        out.y += g.weight.x * s.y + g.weight.y * s.x;
    }
}

// y[top of instance k] += w * O_k (O_k row-major n x n complex, obs =
// [instances][n*n]), pair layout; block k.  w = weights[*base + j] (a device
// offset, so one captured graph serves every segment).
__global__ void heom_add_top(double2* __restrict__ y, const double2* __restrict__ obs_all,
                             const int16_t* __restrict__ pe, const int64_t* __restrict__ tops, int n, int P,
                             const double* __restrict__ weights, const int64_t* __restrict__ base, int64_t j)
{
    const double weight = weights[*base + j];
    if (weight == 0.0) return;
    const int64_t top = tops[blockIdx.x];
    const double2* obs = obs_all + (int64_t)blockIdx.x * n * n;
    for (int pr = threadIdx.x; pr < P; pr += blockDim.x) {
        const int e1 = pe[2 * pr], e2 = pe[2 * pr + 1];
        double2& h1 = y[(top * P + pr) * 2];
        double2& h2 = y[(top * P + pr) * 2 + 1];
        h1.x += weight * obs[e1].x;
        h1.y += weight * obs[e1].y;
        if (e2 != e1) {
            h2.x += weight * obs[e2].x;
            h2.y += weight * obs[e2].y;
        } else {
            h2 = h1; // padding half mirrors its element
        }
    }
}

// ---------------------------------------------------------------------------
// Time-dependent Hamiltonian (the e_field pre-evaluate action of the
// reference, e_field.hpp:63-85): H(t) = H - E(t) D- - conj(E(t)) D+ with
// E(t) = sum over the pulses of e0 exp(-(t - tc)^2 / (2 w^2)) exp(i (phi + omega t)).
// One block builds the operand tables of H(t) for `nt` times t0 + c_s dt of
// every instance: stage times c = (0, 1/2, 1) of an RK4 step when `time` is
// given (t0 = *time, then *time += dt), or the single time t0 of an explicit
// evaluation.
// ---------------------------------------------------------------------------
struct Pulse {
    double e0, tc, w, omega, phi;
};
struct FieldParams {
    const double2* h0;     // [K][N*N] H / hbar of every instance
    const double2* dplus;  // [N*N] D+ / hbar
    const double2* dminus; // [N*N] D- / hbar
    Pulse pulse[2];        // pump, probe
    double* time;          // step mode: device time of the propagation state (advanced by dt)
    double t0, dt;         // explicit mode: the evaluation time t0 (time == nullptr)
    double2* hs_t;         // [nt][K][N*N]
    double* frag_t;        // [nt][K][frag_doubles(N)]
    int K, N, nt;
};

__device__ inline double2 field_at(const FieldParams& f, double t)
{
    double er = 0.0, ei = 0.0;
    for (int q = 0; q < 2; ++q) {
        const Pulse& pl = f.pulse[q];
        const double d = t - pl.tc;
        const double env = pl.e0 * exp(-d * d / (2.0 * pl.w * pl.w));
        double sn, cs;
        sincos(pl.phi + pl.omega * t, &sn, &cs);
        er += env * cs;
        ei += env * sn;
    }
    return make_double2(er, ei);
}

__global__ void heom_field_tables(const FieldParams f)
{
    const int N = f.N, NN = N * N;
    const double t0 = f.time ? *f.time : f.t0;
    const double cst[3] = {0.0, 0.5, 1.0};
    for (int s = 0; s < f.nt; ++s) {
        const double2 E = field_at(f, t0 + cst[s] * f.dt);
        for (int k = 0; k < f.K; ++k) {
            double2* hs = f.hs_t + ((size_t)s * f.K + k) * NN;
            for (int q = threadIdx.x; q < NN; q += blockDim.x) {
                const double2 h = f.h0[(size_t)k * NN + q], dm = f.dminus[q], dp = f.dplus[q];
                // H - E D- - conj(E) D+
                const double re = h.x - (E.x * dm.x - E.y * dm.y) - (E.x * dp.x + E.y * dp.y);
                const double im = h.y - (E.x * dm.y + E.y * dm.x) - (E.x * dp.y - E.y * dp.x);
                hs[q] = make_double2(re, im);
            }
            __syncthreads();
            {
                const int fd = frag_doubles(N), nb = frag_blocks(N), ns = frag_slices(N);
                for (int q = threadIdx.x; q < fd; q += blockDim.x) {
                    // operand fragments as in the host tables ([kind][block][k-slice][lane], frag_index)
                    const int l = q & 31, part = q >> 5, sl = part % ns, b = (part / ns) % nb, kind = part / (ns * nb);
                    const int r = 8 * b + (l >> 2), c = 4 * sl + (l & 3);
                    double v = 0.0;
                    if (r < N && c < N) {
                        const double2 hcr = hs[c * N + r], hrc = hs[r * N + c];
                        v = kind == 0 ? hcr.x : kind == 1 ? hcr.y : kind == 2 ? -hrc.x : -hrc.y;
                    }
                    f.frag_t[((size_t)s * f.K + k) * fd + q] = v;
                }
            }
            __syncthreads();
        }
    }
    if (f.time && threadIdx.x == 0) *f.time = t0 + f.dt;
}

// ---------------------------------------------------------------------------
// Hierarchy arithmetic (hierarchy_arithmetic_{add,subtract,scale,dot_product,
// mmult_left,mmult_right}.cl) on whole state buffers in the pair layout, in
// the reference's operation order (complex products as a.x*b.x - a.y*b.y,
// sums in k order, no contraction).  out may alias a or b.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b)
{
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

// op 0: a + b, 1: a - b, 2: a * conj(b), 3: f * a
__global__ void heom_hier_elementwise(double2* out, const double2* a, const double2* b, double2 f, int64_t len, int op)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += stride) {
        const double2 x = a[e];
        double2 r;
        if (op == 0) {
            const double2 y = b[e];
            r = make_double2(__dadd_rn(x.x, y.x), __dadd_rn(x.y, y.y));
        } else if (op == 1) {
            const double2 y = b[e];
            r = make_double2(__dsub_rn(x.x, y.x), __dsub_rn(x.y, y.y));
        } else if (op == 2) {
            const double2 y = b[e];
            r = cmul_rn(x, make_double2(y.x, -y.y));
        } else {
            r = cmul_rn(f, x);
        }
        out[e] = r;
    }
}

// every ADO: out_u = M a_u (left) or a_u M (right); one warp per ADO, the
// tile staged in shared memory ([warp][N*N] double2)
__global__ void heom_hier_mmult(double2* out, const double2* a, const double2* __restrict__ m,
                                const int16_t* __restrict__ pe, int64_t nodes, int n, int P, int left)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, NN = n * n;
    double2* t = reinterpret_cast<double2*>(smem) + warp * 2 * NN;
    double2* r = t + NN;
    const int64_t stride = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t u = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; u < nodes; u += stride) {
        for (int pr = lane; pr < P; pr += 32) {
            t[pe[2 * pr]] = a[(u * P + pr) * 2];
            t[pe[2 * pr + 1]] = a[(u * P + pr) * 2 + 1];
        }
        __syncwarp();
        for (int q = lane; q < NN; q += 32) {
            const int i = q / n, j = q - i * n;
            double2 v = make_double2(0.0, 0.0);
            for (int k = 0; k < n; ++k) {
                const double2 p = left ? cmul_rn(m[i * n + k], t[k * n + j]) : cmul_rn(t[i * n + k], m[k * n + j]);
                v = make_double2(__dadd_rn(v.x, p.x), __dadd_rn(v.y, p.y));
            }
            r[q] = v;
        }
        __syncwarp();
        for (int pr = lane; pr < P; pr += 32) {
            out[(u * P + pr) * 2] = r[pe[2 * pr]];
            out[(u * P + pr) * 2 + 1] = r[pe[2 * pr + 1]];
        }
        __syncwarp();
    }
}

// Frobenius norm squared of every ADO, sum |sigma(i,j)|^2 (hierarchy_norm.cl:15-45),
// written at the ADO's reference index.  One warp per ADO; a padding half of
// an odd diagonal pair counts once.
__global__ void heom_hierarchy_norm(double* __restrict__ norms, const double2* __restrict__ y,
                                    const int64_t* __restrict__ ref_of_int, const int16_t* __restrict__ pe,
                                    int64_t nodes, int P)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t u = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < nodes; u += stride) {
        double acc = 0.0;
        for (int pr = lane; pr < P; pr += 32) {
            const double2 a = y[(u * P + pr) * 2], b = y[(u * P + pr) * 2 + 1];
            acc += a.x * a.x + a.y * a.y;
            if (pe[2 * pr + 1] != pe[2 * pr]) acc += b.x * b.x + b.y * b.y;
        }
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if (lane == 0) norms[ref_of_int[u]] = acc;
    }
}

// Sets *flag when any element is not finite.
__global__ void heom_check_finite(const double* __restrict__ y, int64_t len, int* flag)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int bad = 0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += stride)
        bad |= !isfinite(y[e]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(flag, 1);
}

} // namespace heomk
