// heom_kernels.cuh -- sm_100a kernels of the HEOM derivative + RK4 path.
//
// One launch of heom_stage evaluates the HEOM time derivative L(w) for every
// ADO of the hierarchy (the reference's heom_ode kernel,
// dm-heom/cl/heom/heom_ode.cl:24-451) and fuses the Runge-Kutta write of the
// stage into the same pass (the reference's NOMA_NUM_ODE_ACCUMULATE /
// NOMA_NUM_ODE_SUBDIAGONAL modes, heom_ode.cl:416-434, generalised to a
// complex stage coefficient).
//
// Per element (i, j) of ADO u the derivative is
//   L(w)_u(i,j) = i * sum_k [ w_u(i,k) Hs(k,j) - Hs(i,k) w_u(k,j) ]        (:89-114, Hs = H / hbar)
//               + (pf_same_sum[u] + gamma0(i,j)) w_u(i,j)                 (:131-168)
//               + sum over baths b of site i, Matsubara terms m:
//                    i cplus(n) w_{u+e}(i,j) + kappa_i(n) w_{u-e}(i,j)      (:183-221, :280-342)
//               + sum over baths b of site j, Matsubara terms m:
//                   -i cplus(n) w_{u+e}(i,j) + kappa_j(n) w_{u-e}(i,j)      (:223-259, :344-403)
// where n is the tuple entry of u for slot e = b*M+m,
//   cplus(n)   = sqrt((n+1) |c_e| / hbar)                                 (:211, :249)
//   kappa_i(n) = sqrt(n hbar / |c_e|) (i c_e / hbar + [m==0] pf_circ[b])  (:301-337)
//   kappa_j(n) = sqrt(n hbar / |c_e|) (-i c_e / hbar + [m==0] pf_circ[b]) (:363-398)
// For i == j the site-i and site-j plus terms cancel exactly and the minus
// terms combine to kappa_i + kappa_j; both are folded on the host.
//
// Layout in HBM (state buffers): ADO-major, each ADO an N x N row-major tile of
// double2 (re, im); ADOs in the handle's internal order.  Per-ADO tables:
// nbr[u][0..W) = plus neighbours, nbr[u][W..2W) = minus neighbours (internal
// index, -1 when absent, masked, or gated off as in the reference), tup[u][W]
// tuple entries, pss[u] = pf_same_sum.
//
// Mapping: one thread per matrix element, G = 256 / N^2 ADOs per CTA
// iteration, persistent grid-stride loop over ADO groups.  The group's tiles
// are staged in shared memory for the commutator; neighbour elements are read
// with read-only loads (L2 keeps the neighbours of nearby ADOs resident).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace heomk {

enum Epi : int {
    EPI_PURE = 0,      // out = L(w)
    EPI_AXPY_SELF = 1, // out = w + beta L(w)
    EPI_AXPY_Y = 2,    // out = y + beta L(w)   (out may alias y)
    EPI_ACC = 3,       // out = L(w); acc = (acc_init ? w : acc) + beta L(w)
};

struct StageParams {
    const double2* __restrict__ in;
    const double2* y;
    double2* out;
    double2* acc;
    double2 beta;
    int acc_init;
    const int32_t* __restrict__ nbr;   // [nodes][2W]
    const uint8_t* __restrict__ tup;   // [nodes][W]
    const double2* __restrict__ pss;   // [nodes]
    const double* __restrict__ cplus;  // [W][LS]
    const double2* __restrict__ kmin;  // [3][W][LS]: kappa_i, kappa_j, kappa_i + kappa_j
    const double2* __restrict__ hs;    // [N*N]
    const double2* __restrict__ gamma0;// [N*N]
    const int16_t* __restrict__ slots; // [N][SL], -1 padded
    int64_t nodes;
    int W;
    int LS;
    int SL;
};

constexpr int kThreads = 256;

// dynamic shared memory of heom_stage for G ADOs per iteration
inline size_t stage_smem_bytes(int G, int W, int LS)
{
    return (size_t)G * 16 + (size_t)3 * W * LS * 16 + (size_t)W * LS * 8 + (size_t)G * 2 * W * 4 +
           (size_t)G * W * 4;
}

__device__ __forceinline__ double2 ld_ro(const double2* p) { return __ldg(p); }

__device__ __forceinline__ void cmac(double2& acc, const double2 a, const double2 b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

template <int N, bool REAL_H, int EPI>
__global__ void __launch_bounds__(kThreads, 2) heom_stage(const StageParams p)
{
    constexpr int NN = N * N;
    constexpr int G = kThreads / NN;
    __shared__ double2 tile[G * NN];
    extern __shared__ __align__(16) unsigned char dyn[];
    // dynamic shared memory (stage_smem_bytes): pss, LUTs, nbr rows, tuple rows
    const int W = p.W;
    const int LS = p.LS;
    double2* s_pss = reinterpret_cast<double2*>(dyn);                 // G
    double2* s_kmin = s_pss + G;                                      // 3 * W * LS
    double* s_cplus = reinterpret_cast<double*>(s_kmin + 3 * W * LS); // W * LS
    int32_t* s_nbr = reinterpret_cast<int32_t*>(s_cplus + W * LS);    // G * 2W
    int32_t* s_tup = s_nbr + G * 2 * W;                               // G * W

    const int t = threadIdx.x;
    for (int q = t; q < 3 * W * LS; q += kThreads) s_kmin[q] = p.kmin[q];
    for (int q = t; q < W * LS; q += kThreads) s_cplus[q] = p.cplus[q];

    const int g = t / NN;
    const int e = t - g * NN;
    const bool lane_ok = g < G;
    const int i = e / N;
    const int j = e - i * N;

    // Hamiltonian row i and column j (scaled by 1/hbar) kept in registers
    double2 hrow[N], hcol[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        hrow[k] = lane_ok ? p.hs[i * N + k] : make_double2(0.0, 0.0);
        hcol[k] = lane_ok ? p.hs[k * N + j] : make_double2(0.0, 0.0);
    }
    const double2 g0 = lane_ok ? p.gamma0[e] : make_double2(0.0, 0.0);
    const int SL = p.SL;
    const int16_t* slot_i = p.slots + i * SL;
    const int16_t* slot_j = p.slots + j * SL;
    const double2* kap_i = s_kmin + (i == j ? 2 : 0) * W * LS;
    const double2* kap_j = s_kmin + 1 * W * LS;

    const int64_t nodes = p.nodes;
    const int64_t stride = (int64_t)gridDim.x * G;
    for (int64_t base = (int64_t)blockIdx.x * G; base < nodes; base += stride) {
        const int64_t u = base + g;
        const bool ok = lane_ok && u < nodes;
        __syncthreads(); // previous iteration finished with the shared buffers
        double2 s = make_double2(0.0, 0.0);
        if (ok) s = ld_ro(p.in + u * NN + e);
        if (lane_ok) tile[g * NN + e] = s;
        for (int q = t; q < G * 2 * W; q += kThreads) {
            const int gg = q / (2 * W);
            const int64_t uu = base + gg;
            s_nbr[q] = uu < nodes ? __ldg(p.nbr + uu * 2 * W + (q - gg * 2 * W)) : -1;
        }
        for (int q = t; q < G * W; q += kThreads) {
            const int gg = q / W;
            const int64_t uu = base + gg;
            s_tup[q] = uu < nodes ? (int32_t)__ldg(p.tup + uu * W + (q - gg * W)) : 0;
        }
        if (t < G) s_pss[t] = (base + t < nodes) ? ld_ro(p.pss + base + t) : make_double2(0.0, 0.0);
        __syncthreads();
        if (!ok) continue;

        // ---- commutator: i * (w Hs - Hs w) ----
        const double2* w = tile + g * NN;
        double cr = 0.0, ci = 0.0;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const double2 a = w[i * N + k];
            const double2 b = w[k * N + j];
            if (REAL_H) {
                cr = fma(a.x, hcol[k].x, cr);
                cr = fma(-hrow[k].x, b.x, cr);
                ci = fma(a.y, hcol[k].x, ci);
                ci = fma(-hrow[k].x, b.y, ci);
            } else {
                cr = fma(a.x, hcol[k].x, cr);
                cr = fma(-a.y, hcol[k].y, cr);
                ci = fma(a.x, hcol[k].y, ci);
                ci = fma(a.y, hcol[k].x, ci);
                cr = fma(-hrow[k].x, b.x, cr);
                cr = fma(hrow[k].y, b.y, cr);
                ci = fma(-hrow[k].x, b.y, ci);
                ci = fma(-hrow[k].y, b.x, ci);
            }
        }
        double2 L = make_double2(-ci, cr);

        // ---- same term ----
        const double2 pss = s_pss[g];
        const double2 gam = make_double2(pss.x + g0.x, pss.y + g0.y);
        cmac(L, gam, s);

        // ---- plus / minus neighbours ----
        const int32_t* nb = s_nbr + g * 2 * W;
        const int32_t* tu = s_tup + g * W;
        for (int q = 0; q < SL; ++q) {
            const int sl = slot_i[q];
            if (sl < 0) break;
            const int n = tu[sl];
            if (i != j) {
                const int32_t v = nb[sl];
                if (v >= 0) {
                    const double c = s_cplus[sl * LS + n];
                    const double2 x = ld_ro(p.in + (int64_t)v * NN + e);
                    L.x = fma(-c, x.y, L.x);
                    L.y = fma(c, x.x, L.y);
                }
            }
            const int32_t v = nb[W + sl];
            if (v >= 0) {
                const double2 x = ld_ro(p.in + (int64_t)v * NN + e);
                cmac(L, kap_i[sl * LS + n], x);
            }
        }
        if (i != j) {
            for (int q = 0; q < SL; ++q) {
                const int sl = slot_j[q];
                if (sl < 0) break;
                const int n = tu[sl];
                const int32_t vp = nb[sl];
                if (vp >= 0) {
                    const double c = s_cplus[sl * LS + n];
                    const double2 x = ld_ro(p.in + (int64_t)vp * NN + e);
                    L.x = fma(c, x.y, L.x);
                    L.y = fma(-c, x.x, L.y);
                }
                const int32_t vm = nb[W + sl];
                if (vm >= 0) {
                    const double2 x = ld_ro(p.in + (int64_t)vm * NN + e);
                    cmac(L, kap_j[sl * LS + n], x);
                }
            }
        }

        // ---- stage write ----
        const int64_t off = u * NN + e;
        if (EPI == EPI_PURE) {
            __stcs(p.out + off, L);
        } else if (EPI == EPI_AXPY_SELF || EPI == EPI_AXPY_Y) {
            double2 r = (EPI == EPI_AXPY_SELF) ? s : p.y[off];
            cmac(r, p.beta, L);
            __stcs(p.out + off, r);
        } else { // EPI_ACC
            __stcs(p.out + off, L);
            double2 a = p.acc_init ? s : p.acc[off];
            cmac(a, p.beta, L);
            p.acc[off] = a;
        }
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

// dst[int] = src[ref] for whole N x N tiles (to_internal) or the reverse.
__global__ void heom_permute_tiles(double2* __restrict__ dst, const double2* __restrict__ src,
                                   const int64_t* __restrict__ ref_of_int, int64_t nodes, int nn,
                                   int to_internal)
{
    const int64_t total = nodes * nn;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += stride) {
        const int64_t u = q / nn;
        const int64_t e = q - u * nn;
        const int64_t r = ref_of_int[u];
        if (to_internal)
            dst[q] = src[r * nn + e];
        else
            dst[r * nn + e] = src[q];
    }
}

// Copy the top matrix (internal index top_int) into log row `row`.
__global__ void heom_record_top(double2* __restrict__ log, const double2* __restrict__ y,
                                int64_t top_int, int nn, int64_t row)
{
    for (int e = threadIdx.x; e < nn; e += blockDim.x) log[row * nn + e] = y[top_int * nn + e];
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
