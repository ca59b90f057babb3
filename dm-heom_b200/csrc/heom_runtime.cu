// heom_runtime.cu -- implementation of the C ABI in include/heom_b200.h.
//
// Owns the device copies of the hierarchy tables (the role of heom::ode,
// dm-heom/src/heom/ode.cpp:35-95), the propagation state (the y_n buffers of
// population_dynamics_solver, dm-heom/include/heom/population_dynamics_solver.hpp:90-91)
// and the RK4 stepping that the reference delegates to the noma/num stepper
// (population_dynamics_solver.hpp:242).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "heom_b200.h"
#include "heom_kernels.cuh"
#include "heom_lockstep.cuh"
#include "host/heom_host.hpp"

namespace {
#include "pair_tables.inc"
}

using heomk::PairParams;

namespace {

constexpr double kHbar = 1.05457148e-34; // dm-heom/cl/heom/common.cl:46
constexpr int kMaxStates = 16;
constexpr int kMaxWidth = 255;

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                        \
    do {                                                                                      \
        cudaError_t err_ = (expr);                                                            \
        if (err_ != cudaSuccess)                                                              \
            return fail(HEOM_E_CUDA, "%s failed: %s", #expr, cudaGetErrorString(err_));        \
    } while (0)

// Factors of the RK4 stability polynomial 1 + z + z^2/2 + z^3/6 + z^4/24 =
// prod_k (1 - z / r_k); the stage coefficient is -1/r_k (times the step size).
// Roots r = -1.7294442310677054566 +/- 0.8889743761218658272 i and
//           -0.2705557689322945434 +/- 2.5047759043624344897 i
// (computed at 50 digits; the four -1/r_k sum to 1).
constexpr double kProdBeta[4][2] = {
    {0.4573733434972976, 0.23510048799854266},
    {0.4573733434972976, -0.23510048799854266},
    {0.04262665650270243, -0.3946329531721134},
    {0.04262665650270243, 0.3946329531721134},
};

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() { reset(); }
    void reset()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    int alloc(size_t count)
    {
        reset();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(HEOM_E_NOMEM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T),
                        cudaGetErrorString(e));
        }
        n = count;
        return 0;
    }
};

typedef void (*dmma_fn_t)(const heomk::DmmaParams);
typedef dmma_fn_t stage_fn_t;

template <int N, int HK, bool ADJ>
stage_fn_t pick_slt(int slt)
{
    switch (slt) {
    case 1: return heomk::heom_pair_stage<N, HK, 1, ADJ>;
    case 2: return heomk::heom_pair_stage<N, HK, 2, ADJ>;
    case 4: return heomk::heom_pair_stage<N, HK, 4, ADJ>;
    default: return heomk::heom_pair_stage<N, HK, 8, ADJ>;
    }
}

template <int N>
stage_fn_t pick_n(int hk, int slt, bool adj)
{
    if (adj)
        return hk == heomk::H_REAL_SYM ? pick_slt<N, heomk::H_REAL_SYM, true>(slt)
                                       : pick_slt<N, heomk::H_GENERIC, true>(slt);
    return hk == heomk::H_REAL_SYM ? pick_slt<N, heomk::H_REAL_SYM, false>(slt)
                                   : pick_slt<N, heomk::H_GENERIC, false>(slt);
}

// team kernel (tensor-pipe commutator, a team of warps per ADO): N = 9..16
stage_fn_t pick_stage(int n, int hk, int slt, bool adj)
{
    switch (n) {
#define HEOM_CASE(K) \
    case K: return pick_n<K>(hk, slt, adj);
        HEOM_CASE(9) HEOM_CASE(10) HEOM_CASE(11) HEOM_CASE(12)
        HEOM_CASE(13) HEOM_CASE(14) HEOM_CASE(15) HEOM_CASE(16)
#undef HEOM_CASE
    default: return nullptr;
    }
}

template <int N, int HK, bool MI, bool ADJ>
dmma_fn_t pick_dslt(int slt)
{
    switch (slt) {
    case 1: return heomk::heom_dmma_stage<N, HK, 1, MI, ADJ>;
    case 2: return heomk::heom_dmma_stage<N, HK, 2, MI, ADJ>;
    case 4: return heomk::heom_dmma_stage<N, HK, 4, MI, ADJ>;
    default: return heomk::heom_dmma_stage<N, HK, 8, MI, ADJ>;
    }
}

// variants: one instance, several instances (batch), adjoint of one instance
template <int N, int HK>
dmma_fn_t pick_dmode(int slt, bool multi, bool adj)
{
    if (adj) return multi ? pick_dslt<N, HK, true, true>(slt) : pick_dslt<N, HK, false, true>(slt);
    return multi ? pick_dslt<N, HK, true, false>(slt) : pick_dslt<N, HK, false, false>(slt);
}

template <int N>
dmma_fn_t pick_dn(int hk, int slt, bool multi, bool adj)
{
    return hk == heomk::H_REAL_SYM ? pick_dmode<N, heomk::H_REAL_SYM>(slt, multi, adj)
                                   : pick_dmode<N, heomk::H_GENERIC>(slt, multi, adj);
}

// tensor-pipe kernel: N = 1..8
dmma_fn_t pick_dmma(int n, int hk, int slt, bool multi, bool adj)
{
    switch (n) {
#define HEOM_CASE(K) \
    case K: return pick_dn<K>(hk, slt, multi, adj);
        HEOM_CASE(1) HEOM_CASE(2) HEOM_CASE(3) HEOM_CASE(4) HEOM_CASE(5) HEOM_CASE(6)
        HEOM_CASE(7) HEOM_CASE(8)
#undef HEOM_CASE
    default: return nullptr;
    }
}

typedef void (*lock_fn_t)(const heomk::LockParams);

template <int N, int HK>
lock_fn_t pick_lslt(int slt)
{
    return slt <= 1   ? heomk::heom_lockstep_stage<N, HK, 1>
           : slt <= 2 ? heomk::heom_lockstep_stage<N, HK, 2>
                      : heomk::heom_lockstep_stage<N, HK, 4>;
}

// lockstep ensemble kernel: N = 1..8, at most four slots per state
lock_fn_t pick_lock(int n, int hk, int slt)
{
    if (slt > 4) return nullptr;
    switch (n) {
#define HEOM_CASE(K) \
    case K: return hk == heomk::H_REAL_SYM ? pick_lslt<K, heomk::H_REAL_SYM>(slt) : pick_lslt<K, heomk::H_GENERIC>(slt);
        HEOM_CASE(1) HEOM_CASE(2) HEOM_CASE(3) HEOM_CASE(4) HEOM_CASE(5) HEOM_CASE(6)
        HEOM_CASE(7) HEOM_CASE(8)
#undef HEOM_CASE
    default: return nullptr;
    }
}

// tables that replace the handle's own in one stage launch: those of the
// adjoint operator L^H (adjoint = true: conj(pf_same_sum), conj(gamma0), -H^H),
// or those of a time-dependent H(t) (adjoint = false, handle's pss and gamma0)
struct AdjTabs {
    const double2* pss;    // conj(pf_same_sum)
    const double2* gamma0; // conj(gamma0)
    const double* hfrag;   // fragments of -H^H
    bool adjoint = true;
    // optional bath-coefficient tables (flow tracking: a zero table switches a term off)
    const double* chat = nullptr;
    const double2* khat = nullptr;
};

// stage write modes (runtime parameters of the one stage kernel)
enum Epi : int {
    EPI_PURE = 0,      // out = L(w)
    EPI_AXPY_SELF = 1, // out = w + beta L(w)
    EPI_AXPY_Y = 2,    // out = y + beta L(w)   (out may alias y)
    EPI_ACC = 3,       // out = L(w); acc = (acc_init ? w : acc) + beta L(w)
    EPI_AXPY_ACC = 4,  // out = (y ? y : w) + beta L(w); acc = (acc_init ? w : acc) + acc_beta L(w)
};

// number of tuples over d coordinates with sum <= r
int64_t simplex_count(int d, int r, const std::vector<std::vector<int64_t>>& binom)
{
    if (r < 0) return 0;
    return binom[r + d][d];
}

} // namespace

namespace heomhost {
int set_error(int code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}
} // namespace heomhost

struct heom_buffer {
    heom_handle* owner = nullptr;
    DevBuf<double2> data;
    bool borrowed = false;
};

struct heom_handle {
    heom_options opt{};
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;

    // sizes shared by every instance of the handle
    int N = 0, M = 0, B = 0, BPS = 0, W = 0, D = 0; // D = largest depth
    int64_t nodes = 0;                              // ADOs of all instances
    int64_t n_active = 0;                           // ADOs the stage kernels sweep (internal [0, n_active))
    bool compact = false;                           // masked ADOs moved behind the active ones and not swept
    int LS = 0, SL = 0, SLT = 2;
    int P = 0;          // 32-byte sectors per ADO (pair layout)
    int NW = 0, TWB = 0; // padded widths of the neighbour and tuple rows
    int hkind = heomk::H_REAL_SYM;

    // instances: ADOs [inst_base[k], inst_base[k+1]) in both the reference
    // and the internal order belong to instance k
    int n_inst = 1;
    std::vector<int64_t> inst_base;
    std::vector<int32_t> inst_depth, inst_fnp; // depth and first_non_plus_id per instance

    // host copies in reference layout, instances back to back (plus / minus
    // hold indices into the concatenation)
    std::vector<int32_t> coupling, tuples, plus, minus;
    std::vector<double> ham, pss, pf_same, pf_circ, cbk, cbk_sqrt;
    std::vector<uint8_t> mask;
    std::vector<int64_t> int_of_ref, ref_of_int;
    std::vector<int64_t> top_int; // internal index of each instance's top ADO

    // device tables
    DevBuf<int32_t> d_nbr;
    DevBuf<uint8_t> d_tup;
    DevBuf<double2> d_pss, d_hs, d_gamma0;
    DevBuf<double> d_hfrag;          // per-instance MMA fragments of H / hbar
    DevBuf<int32_t> d_inst;          // instance of each internal ADO (n_inst > 1)
    DevBuf<int64_t> d_top;
    DevBuf<int16_t> d_slots;
    DevBuf<double> d_chat, d_sq;     // factored bath coefficients (both stage kernels)
    DevBuf<double2> d_khat;
    DevBuf<int16_t> d_pos;
    DevBuf<int64_t> d_int_of_ref, d_ref_of_int;
    DevBuf<int16_t> d_pair;          // [P][2] element indices of the sector halves
    std::vector<int16_t> pair_tab;   // host copy
    heomk::LaneTab lane_tab{};       // DMMA kernel lane tables (N <= 8)
    DevBuf<int> d_err;               // set by a stage kernel whose pipeline wait expired

    // propagation state + stage buffers
    heom_buffer y;
    DevBuf<double2> work[5];
    DevBuf<double2> xfer;   // reference-layout staging buffer for host transfers (xfer_ados ADOs)
    int64_t xfer_ados = 0;
    DevBuf<double2> toplog;
    DevBuf<double2> topbuf; // row-major top matrices of all instances
    DevBuf<int> d_flag;

    // launch accounting and shape
    int64_t launches = 0;
    int per_sm[2][2] = {{0, 0}, {0, 0}}; // resident stage CTAs per SM, per [adjoint][H kind]
    int grid_override = 0;   // stage grid chosen by an autotuner (0: one full wave)
    size_t stage_smem = 0;

    // time-dependent H (heom_set_field): H(t) = H - E(t) D- - conj(E(t)) D+
    bool field_on = false;
    heomk::Pulse pulses[2] = {};
    DevBuf<double2> d_dplus, d_dminus;     // D+ / hbar, D- / hbar
    DevBuf<double2> field_hs;              // [3][K][N*N]
    DevBuf<double> field_frag;             // [3][K][frag_doubles(N)]
    DevBuf<double> d_time;                 // time of the propagation state (device, advanced by field steps)
    double time = 0.0;                     // host mirror

    // host pre-evaluate actions (ode::add_pre_evaluate_action), run before every heom_solve
    std::vector<std::pair<heom_pre_evaluate_fn, void*>> actions;

    // flow tracking (heom_set_flow_buffers): acc_coeff x the plus / minus terms of every heom_solve
    heom_buffer* flow_above = nullptr;
    heom_buffer* flow_below = nullptr;
    DevBuf<double2> flow_scratch;
    // buffers created on this handle and not yet destroyed (orphaned by heom_destroy)
    std::vector<heom_buffer*> live_buffers;
    DevBuf<double> d_zero;                 // zeros, as long as the longest table they replace

    // cached graph of one RK4 step
    cudaGraphExec_t step_graph = nullptr;
    double graph_dt = 0.0;

    // lockstep layout (instances of one hierarchy graph, ensembles only): sector
    // p of internal ADO u of instance k at sector index (u * P + p) * kp + k
    int64_t kp = 0;          // instance stride (instances rounded up to 32); 0: the per-instance layout
    int64_t inst_nodes = 0;  // ADOs of every instance (lockstep)

    size_t state_elems() const { return (size_t)(kp ? inst_nodes * kp : nodes) * 2 * P; } // double2 per state
    size_t ref_elems() const { return (size_t)nodes * N * N; }   // double2 per reference-layout state
};

namespace {

int build_neighbours(heom_handle* h)
{
    // internal neighbour table with the reference's gating folded in:
    //   plus read only when uid < first_non_plus_id (heom_ode.cl:183) and mask[plus] != 0 (:199)
    //   minus read only when tuple > 0 (:293) and mask[minus] != 0 (:297)
    const int W = h->W, NW = h->NW, TWB = h->TWB;
    std::vector<int32_t> nbr((size_t)h->nodes * NW, -1);
    std::vector<uint8_t> tup((size_t)h->nodes * TWB, 0);
    std::vector<double2> pss(h->nodes);
    std::vector<int32_t> inst(h->n_inst > 1 ? h->nodes : 0);
    for (int k = 0; k < h->n_inst; ++k) {
        const int64_t base = h->inst_base[k];
        for (int64_t r = base; r < h->inst_base[k + 1]; ++r) {
            const int64_t u = h->int_of_ref[r];
            const bool has_plus = r - base < h->inst_fnp[k];
            for (int m = 0; m < W; ++m) {
                const int32_t t = h->tuples[r * W + m];
                tup[u * TWB + m] = (uint8_t)t;
                int32_t pv = -1, mv = -1;
                const int32_t pr = h->plus[r * W + m];
                if (has_plus && pr >= 0 && h->mask[pr]) pv = (int32_t)h->int_of_ref[pr];
                const int32_t mr = h->minus[r * W + m];
                if (t > 0 && mr >= 0 && h->mask[mr]) mv = (int32_t)h->int_of_ref[mr];
                nbr[u * NW + 2 * m] = pv;
                nbr[u * NW + 2 * m + 1] = mv;
            }
            pss[u] = make_double2(h->pss[2 * r], h->pss[2 * r + 1]);
            if (h->n_inst > 1) inst[u] = k;
        }
    }
    if (!h->d_nbr.p) {
        if (int rc = h->d_nbr.alloc(nbr.size())) return rc;
        if (int rc = h->d_tup.alloc(tup.size())) return rc;
        if (int rc = h->d_pss.alloc(pss.size())) return rc;
        if (h->n_inst > 1)
            if (int rc = h->d_inst.alloc(inst.size())) return rc;
    }
    CUDA_TRY(cudaMemcpy(h->d_nbr.p, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->d_tup.p, tup.data(), tup.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->d_pss.p, pss.data(), pss.size() * 16, cudaMemcpyHostToDevice));
    if (h->n_inst > 1) CUDA_TRY(cudaMemcpy(h->d_inst.p, inst.data(), inst.size() * 4, cudaMemcpyHostToDevice));
    return 0;
}

// device-side forms of one instance's H (interleaved re/im, J): H / hbar
// row-major (hs) and the MMA operand fragments (frag, heomk::frag_index: lane l = 4g + t, block b, k-slice s,
// row r = 8b + g, column c = 4s + t; hb = H(c, r), ha = -H(r, c); zero outside N x N)
void h_tables(const double* hk, int N, double2* hs, double* frag)
{
    for (int q = 0; q < N * N; ++q) hs[q] = make_double2(hk[2 * q] / kHbar, hk[2 * q + 1] / kHbar);
    for (int b = 0; b < heomk::frag_blocks(N); ++b)
        for (int sl = 0; sl < heomk::frag_slices(N); ++sl)
            for (int l = 0; l < 32; ++l) {
                const int r = 8 * b + (l >> 2), c = 4 * sl + (l & 3);
                if (r >= N || c >= N) continue;
                const double2 hcr = hs[c * N + r], hrc = hs[r * N + c];
                frag[heomk::frag_index(N, 0, b, sl, l)] = hcr.x;
                frag[heomk::frag_index(N, 1, b, sl, l)] = hcr.y;
                frag[heomk::frag_index(N, 2, b, sl, l)] = -hrc.x;
                frag[heomk::frag_index(N, 3, b, sl, l)] = -hrc.y;
            }
}

bool real_symmetric(const double* hk, int N)
{
    for (int q = 0; q < N * N; ++q)
        if (hk[2 * q + 1] != 0.0) return false;
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < i; ++j)
            if (hk[2 * (i * N + j)] != hk[2 * (j * N + i)]) return false;
    return true;
}

// same term (heom_ode.cl:138-168): for i != j subtract pf_same of every bath
// coupled to site i and to site j (linear in pf_same)
std::vector<double2> gamma0_table(const heom_handle* h, const std::vector<double>& pf_same)
{
    const int N = h->N;
    std::vector<double2> g0(N * N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            double gr = 0.0, gi = 0.0;
            if (i != j)
                for (int b = 0; b < h->BPS; ++b) {
                    const int bi = h->coupling[i * h->BPS + b];
                    if (bi >= 0) { gr -= pf_same[2 * bi]; gi -= pf_same[2 * bi + 1]; }
                    const int bj = h->coupling[j * h->BPS + b];
                    if (bj >= 0) { gr -= pf_same[2 * bj]; gi -= pf_same[2 * bj + 1]; }
                }
            g0[i * N + j] = make_double2(gr, gi);
        }
    return g0;
}

int upload_hamiltonian(heom_handle* h)
{
    const int N = h->N, K = h->n_inst;
    std::vector<double2> hs((size_t)K * N * N);
    const size_t fd = heomk::frag_doubles(N);
    std::vector<double> frag((size_t)K * fd, 0.0);
    bool real_sym = true;
    for (int k = 0; k < K; ++k) {
        const double* hk = h->ham.data() + (size_t)k * 2 * N * N;
        h_tables(hk, N, hs.data() + (size_t)k * N * N, frag.data() + (size_t)k * fd);
        real_sym = real_sym && real_symmetric(hk, N);
    }
    // real symmetric H (every instance) takes the cheaper kernel variants; a
    // time-dependent H(t) is complex
    h->hkind = real_sym && !h->field_on ? heomk::H_REAL_SYM : heomk::H_GENERIC;
    const std::vector<double2> g0 = gamma0_table(h, h->pf_same);
    if (!h->d_hs.p) {
        if (int rc = h->d_hs.alloc(hs.size())) return rc;
        if (int rc = h->d_hfrag.alloc(frag.size())) return rc;
        if (int rc = h->d_gamma0.alloc(N * N)) return rc;
    }
    CUDA_TRY(cudaMemcpy(h->d_hs.p, hs.data(), hs.size() * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->d_hfrag.p, frag.data(), frag.size() * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->d_gamma0.p, g0.data(), g0.size() * 16, cudaMemcpyHostToDevice));
    // the kernel variant may change: rebuild the cached step graph
    if (h->step_graph) {
        cudaGraphExecDestroy(h->step_graph);
        h->step_graph = nullptr;
    }
    return 0;
}

int upload_coefficients(heom_handle* h)
{
    const int W = h->W, LS = h->LS, M = h->M;
    // slots of each state: b * M + m for every bath b coupled to the state
    std::vector<int16_t> slots((size_t)h->N * h->SL, (int16_t)-1);
    for (int s = 0; s < h->N; ++s) {
        int q = 0;
        for (int b = 0; b < h->BPS; ++b) {
            const int bs = h->coupling[s * h->BPS + b];
            if (bs < 0) continue;
            for (int m = 0; m < M; ++m) slots[s * h->SL + q++] = (int16_t)(bs * M + m);
        }
    }
    // factored form: cplus(n) = chat sqrt(n+1), kappa(n) = khat sqrt(n), stored at pos(slot) = m*B + b
    {
        std::vector<double> chat(W, 0.0), sq(LS + 1, 0.0);
        std::vector<double2> khat((size_t)3 * W, make_double2(0.0, 0.0));
        std::vector<int16_t> pos(W, 0);
        for (int sl = 0; sl < W; ++sl) {
            const int b = sl / M, m = sl - b * M;
            const int ps = m * h->B + b;
            pos[sl] = (int16_t)ps;
            const double cr = h->cbk[2 * sl], ci = h->cbk[2 * sl + 1];
            const double qr = m == 0 ? h->pf_circ[2 * b] : 0.0;
            const double qi = m == 0 ? h->pf_circ[2 * b + 1] : 0.0;
            const double habs = std::hypot(cr, ci);
            chat[ps] = std::sqrt(habs / kHbar);
            const double sc = std::sqrt(kHbar / habs);
            khat[0 * W + ps] = make_double2(sc * (-ci / kHbar + qr), sc * (cr / kHbar + qi));
            khat[1 * W + ps] = make_double2(sc * (ci / kHbar + qr), sc * (-cr / kHbar + qi));
            khat[2 * W + ps] = make_double2(2.0 * sc * qr, 2.0 * sc * qi);
        }
        for (int n = 0; n <= LS; ++n) sq[n] = std::sqrt((double)n);
        if (int rc = h->d_chat.alloc(W)) return rc;
        if (int rc = h->d_khat.alloc(3 * W)) return rc;
        if (int rc = h->d_sq.alloc(LS + 1)) return rc;
        if (int rc = h->d_pos.alloc(W)) return rc;
        CUDA_TRY(cudaMemcpy(h->d_chat.p, chat.data(), W * 8, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(h->d_khat.p, khat.data(), 3 * W * 16, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(h->d_sq.p, sq.data(), (LS + 1) * 8, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(h->d_pos.p, pos.data(), W * 2, cudaMemcpyHostToDevice));
    }
    if (int rc = h->d_slots.alloc(slots.size())) return rc;
    CUDA_TRY(cudaMemcpy(h->d_slots.p, slots.data(), slots.size() * 2, cudaMemcpyHostToDevice));
    return 0;
}

PairParams base_params(const heom_handle* h)
{
    PairParams p{};
    p.nbr = h->d_nbr.p;
    p.tup = h->d_tup.p;
    p.pss = h->d_pss.p;
    p.hfrag = h->d_hfrag.p;
    p.inst = h->n_inst > 1 ? h->d_inst.p : nullptr;
    p.gamma0 = h->d_gamma0.p;
    p.slots = h->d_slots.p;
    p.nodes = h->n_active;
    p.W = h->W;
    p.NW = h->NW;
    p.TWB = h->TWB;
    p.LS = h->LS;
    p.SL = h->SL;
    return p;
}

// The dynamic shared-memory limit is an attribute of the kernel function,
// shared by every handle that launches it (with its own sizes): it only grows.
std::mutex g_smem_mu;
std::vector<std::pair<int, std::pair<const void*, size_t>>> g_smem_allowed; // (device, (function, bytes))

int allow_dynamic_smem(const void* fn, size_t smem)
{
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_smem_mu);
    for (auto& e : g_smem_allowed)
        if (e.first == dev && e.second.first == fn) {
            if (e.second.second >= smem) return 0;
            CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            e.second.second = smem;
            return 0;
        }
    CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    g_smem_allowed.push_back({dev, {fn, smem}});
    return 0;
}

int cta_threads(int n) { return (heomk::kCtaWarps / heomk::team_warps(n)) * heomk::team_warps(n) * 32; }
int cta_teams(int n) { return heomk::kCtaWarps / heomk::team_warps(n); }

// resolve the launch shape of the stage kernel (outside of any stream capture)
int resolve_stage(heom_handle* h, const void** fn_out, int* blocks_out = nullptr, bool adj = false)
{
    const void* fn = nullptr;
    size_t smem = 0;
    int threads = 0;
    if (h->kp) {
        if (adj) return fail(HEOM_E_UNSUPPORTED, "the lockstep layout has no adjoint stage");
        fn = (const void*)pick_lock(h->N, h->hkind, h->SL); // its own slot count: 1, 2 or 4 slots per site
        smem = heomk::lockstep_smem_bytes(h->P, h->W, h->NW, h->TWB, h->LS);
        threads = heomk::kLockWarps * 32;
    } else if (h->N <= 8) {
        fn = (const void*)pick_dmma(h->N, h->hkind, h->SL == 1 ? 1 : h->SLT, h->n_inst > 1, adj); // one slot: exact
        smem = heomk::dmma_smem_bytes(h->P, h->W, h->NW, h->TWB, h->LS);
        threads = heomk::kCtaWarps * 32;
    } else {
        fn = (const void*)pick_stage(h->N, h->hkind, h->SL == 1 ? 1 : h->SLT, adj); // one slot: exact
        smem = heomk::pair_smem_bytes(h->N, h->W, h->NW, h->TWB, h->LS);
        threads = cta_threads(h->N);
    }
    if (!fn) return fail(HEOM_E_UNSUPPORTED, "states = %d not supported", h->N);
    int& per_sm = h->per_sm[adj ? 1 : 0][h->hkind];
    if (per_sm == 0) {
        if (smem > 227 * 1024) return fail(HEOM_E_UNSUPPORTED, "stage kernel needs %zu B of shared memory", smem);
        if (int rc = allow_dynamic_smem(fn, smem)) return rc;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
        if (per_sm < 1) return fail(HEOM_E_UNSUPPORTED, "stage kernel cannot be resident");
    }
    const int teams = h->N <= 8 ? heomk::kCtaWarps : cta_teams(h->N);
    const int64_t groups = h->kp ? h->inst_nodes * (h->kp / 32)
                                 : std::max<int64_t>(1, (h->n_active + teams - 1) / teams);
    const int64_t want = h->grid_override > 0 ? h->grid_override : (int64_t)per_sm * h->sm_count;
    int64_t blocks = std::max<int64_t>(1, std::min<int64_t>(groups, want));
    if (h->kp) { // every CTA keeps one instance block: a multiple of the block count
        const int64_t kb = h->kp / 32;
        blocks = std::max<int64_t>(kb, blocks / kb * kb);
    }
    if (blocks_out) *blocks_out = (int)blocks;
    h->stage_smem = smem;
    *fn_out = fn;
    return 0;
}

int launch_stage(heom_handle* h, int epi, const double2* in, const double2* y, double2* out,
                 double2* acc, double2 beta, int acc_init, const AdjTabs* adj = nullptr,
                 double2 acc_beta = make_double2(0.0, 0.0))
{
    const void* fn = nullptr;
    int blocks = 0;
    if (int rc = resolve_stage(h, &fn, &blocks, adj && adj->adjoint)) return rc;
    PairParams p = base_params(h);
    if (adj) {
        p.pss = adj->pss;
        p.gamma0 = adj->gamma0;
        p.hfrag = adj->hfrag;
    }
    p.in = in;
    p.out = out;
    switch (epi) {
    case EPI_PURE:
        p.alpha = make_double2(0.0, 0.0);
        p.beta = make_double2(1.0, 0.0);
        break;
    case EPI_AXPY_SELF:
        p.alpha = make_double2(1.0, 0.0);
        p.beta = beta;
        break;
    case EPI_AXPY_Y:
        p.y = y;
        p.alpha = make_double2(1.0, 0.0);
        p.beta = beta;
        break;
    case EPI_AXPY_ACC:
        p.y = y;
        p.alpha = make_double2(1.0, 0.0);
        p.beta = beta;
        p.acc = acc;
        p.use_acc = 1;
        p.acc_beta = acc_beta;
        p.acc_init = acc_init;
        break;
    default: // EPI_ACC
        p.alpha = make_double2(0.0, 0.0);
        p.beta = make_double2(1.0, 0.0);
        p.acc = acc;
        p.use_acc = 1;
        p.acc_beta = beta;
        p.acc_init = acc_init;
        break;
    }
    heomk::DmmaParams dp;
    dp.p = p;
    dp.lt = h->lane_tab;
    dp.ct.chat = adj && adj->chat ? adj->chat : h->d_chat.p;
    dp.ct.khat = adj && adj->khat ? adj->khat : h->d_khat.p;
    dp.ct.sq = h->d_sq.p;
    dp.ct.pos = h->d_pos.p;
    dp.err = h->d_err.p;
    if (h->kp) {
        // lockstep: every instance uses instance 0's rows of the shared tables
        heomk::LockParams lp;
        lp.p = dp.p;
        lp.p.nodes = h->inst_nodes;
        lp.p.inst = nullptr;
        lp.lt = dp.lt;
        lp.ct = dp.ct;
        lp.K = h->n_inst;
        lp.Kp = (int)h->kp;
        lp.nodes = h->inst_nodes;
        ((lock_fn_t)fn)<<<blocks, heomk::kLockWarps * 32, h->stage_smem, h->stream>>>(lp);
        h->launches++;
        CUDA_TRY(cudaGetLastError());
        return 0;
    }
    ((dmma_fn_t)fn)<<<blocks, h->N <= 8 ? heomk::kCtaWarps * 32 : cta_threads(h->N), h->stage_smem, h->stream>>>(dp);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_wadd(heom_handle* h, int n, double step, double2* out, const double2* y,
                const double* c, const double2* const* k)
{
    heomk::WaddParams p{};
    p.out = reinterpret_cast<double*>(out);
    p.y = reinterpret_cast<const double*>(y);
    p.n = n;
    p.h = step;
    p.len = (int64_t)h->state_elems() * 2;
    for (int l = 0; l < 7; ++l) {
        p.c[l] = l < n ? c[l] : 0.0;
        p.k[l] = l < n ? reinterpret_cast<const double*>(k[l]) : p.y;
    }
    const int blocks = std::max(1, std::min<int>((int)((p.len + 255) / 256), h->sm_count * 8));
    heomk::heom_weighted_add<<<blocks, 256, 0, h->stream>>>(p);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    return 0;
}

// heom_ode.cl:436-441: flow_from_above += acc_coeff * plus term, flow_from_below
// += acc_coeff * minus term of the evaluation of `in`; each term alone is L
// with H, the same term and the other term's coefficients zeroed (no launch
// when no flow buffer is set)
int launch_flows(heom_handle* h, const double2* in, double acc_coeff)
{
    if (!h->flow_above && !h->flow_below) return 0;
    const double2* z2 = reinterpret_cast<const double2*>(h->d_zero.p);
    const double* z1 = h->d_zero.p;
    for (int part = 0; part < 2; ++part) {
        heom_buffer* dst = part == 0 ? h->flow_above : h->flow_below;
        if (!dst) continue;
        AdjTabs t;
        t.pss = z2;
        t.gamma0 = z2;
        t.hfrag = z1;
        t.adjoint = false;
        if (part == 0) {
            t.khat = z2;
        } else {
            t.chat = z1;
        }
        if (int rc = launch_stage(h, EPI_ACC, in, nullptr, h->flow_scratch.p, dst->data.p,
                                  make_double2(acc_coeff, 0.0), 0, &t))
            return rc;
    }
    return 0;
}

int ensure_work(heom_handle* h, int count)
{
    for (int q = 0; q < count; ++q)
        if (!h->work[q].p) {
            if (int rc = h->work[q].alloc(h->state_elems())) return rc;
            CUDA_TRY(cudaMemset(h->work[q].p, 0, h->state_elems() * sizeof(double2)));
        }
    return 0;
}

heomk::FieldParams field_params(heom_handle* h, int nt)
{
    heomk::FieldParams f{};
    f.h0 = h->d_hs.p;
    f.dplus = h->d_dplus.p;
    f.dminus = h->d_dminus.p;
    f.pulse[0] = h->pulses[0];
    f.pulse[1] = h->pulses[1];
    f.hs_t = h->field_hs.p;
    f.frag_t = h->field_frag.p;
    f.K = h->n_inst;
    f.N = h->N;
    f.nt = nt;
    return f;
}

// the tables of H at field time slot s (built by heom_field_tables)
AdjTabs field_tabs(const heom_handle* h, int s)
{
    AdjTabs t;
    t.pss = h->d_pss.p;
    t.gamma0 = h->d_gamma0.p;
    t.hfrag = h->field_frag.p + (size_t)s * h->n_inst * heomk::frag_doubles(h->N);
    t.adjoint = false;
    return t;
}

// one classical RK4 step with a time-dependent H: the tables of H(t),
// H(t + dt/2), H(t + dt) from the device time, then four fused stages
//   s1 = y + dt/2 L(t) y            acc = y + dt/6 L(t) y
//   s2 = y + dt/2 L(t+dt/2) s1      acc += dt/3 L(t+dt/2) s1
//   s1 = y + dt L(t+dt/2) s2        acc += dt/3 L(t+dt/2) s2
//   y  = acc + dt/6 L(t+dt) s1
int enqueue_field_step(heom_handle* h, double dt)
{
    heomk::FieldParams f = field_params(h, 3);
    f.time = h->d_time.p;
    f.dt = dt;
    heomk::heom_field_tables<<<1, 256, 0, h->stream>>>(f);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    double2* y = h->y.data.p;
    double2* s1 = h->work[0].p;
    double2* s2 = h->work[1].p;
    double2* acc = h->work[2].p;
    const AdjTabs t0 = field_tabs(h, 0), th = field_tabs(h, 1), t1 = field_tabs(h, 2);
    auto c = [](double v) { return make_double2(v, 0.0); };
    if (int rc = launch_stage(h, EPI_AXPY_ACC, y, nullptr, s1, acc, c(dt / 2), 1, &t0, c(dt / 6))) return rc;
    if (int rc = launch_stage(h, EPI_AXPY_ACC, s1, y, s2, acc, c(dt / 2), 0, &th, c(dt / 3))) return rc;
    if (int rc = launch_stage(h, EPI_AXPY_ACC, s2, y, s1, acc, c(dt), 0, &th, c(dt / 3))) return rc;
    return launch_stage(h, EPI_AXPY_Y, s1, acc, y, nullptr, c(dt / 6), 0, &t1);
}

// one RK4 step with flow tracking (population_dynamics_solver.hpp:236-263 with
// track_flows): the flow buffers are zeroed, then the classical RK4 of four
// pure evaluations and rk_weighted_add (the reference's structure) runs with
// every evaluation of stage input s_i adding dt b_i x its plus and minus
// terms, b = (1/6, 1/3, 1/3, 1/6): after the step the buffers hold the
// step's flows from the layer above and from the layer below
int enqueue_flow_step(heom_handle* h, double dt)
{
    for (heom_buffer* b : {h->flow_above, h->flow_below})
        if (b) CUDA_TRY(cudaMemsetAsync(b->data.p, 0, h->state_elems() * sizeof(double2), h->stream));
    double2* y = h->y.data.p;
    const double2 zero = make_double2(0.0, 0.0);
    double2* k1 = h->work[0].p;
    double2* k2 = h->work[1].p;
    double2* k3 = h->work[2].p;
    double2* k4 = h->work[3].p;
    double2* st = h->work[4].p;
    const double2* ks[4] = {k1, k2, k3, k4};
    const double a2[1] = {0.5}, a3[2] = {0.0, 0.5}, a4[3] = {0.0, 0.0, 1.0};
    const double bb[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
    if (int rc = launch_stage(h, EPI_PURE, y, nullptr, k1, nullptr, zero, 0)) return rc;
    if (int rc = launch_flows(h, y, dt * bb[0])) return rc;
    if (int rc = launch_wadd(h, 1, dt, st, y, a2, ks)) return rc;
    if (int rc = launch_stage(h, EPI_PURE, st, nullptr, k2, nullptr, zero, 0)) return rc;
    if (int rc = launch_flows(h, st, dt * bb[1])) return rc;
    if (int rc = launch_wadd(h, 2, dt, st, y, a3, ks)) return rc;
    if (int rc = launch_stage(h, EPI_PURE, st, nullptr, k3, nullptr, zero, 0)) return rc;
    if (int rc = launch_flows(h, st, dt * bb[2])) return rc;
    if (int rc = launch_wadd(h, 3, dt, st, y, a4, ks)) return rc;
    if (int rc = launch_stage(h, EPI_PURE, st, nullptr, k4, nullptr, zero, 0)) return rc;
    if (int rc = launch_flows(h, st, dt * bb[3])) return rc;
    return launch_wadd(h, 4, dt, y, y, bb, ks);
}

// enqueue one RK4 step of y_n (in place) on the handle's stream
int enqueue_step(heom_handle* h, double dt)
{
    double2* y = h->y.data.p;
    const double2 zero = make_double2(0.0, 0.0);
    if (h->field_on) return enqueue_field_step(h, dt);
    if (h->flow_above || h->flow_below) return enqueue_flow_step(h, dt);
    switch (h->opt.rk4_scheme) {
    case HEOM_RK4_PRODUCT: {
        double2* a = h->work[0].p;
        double2* b = h->work[1].p;
        const double2* ins[4] = {y, a, b, a};
        double2* outs[4] = {a, b, a, y};
        for (int k = 0; k < 4; ++k) {
            const double2 beta = make_double2(dt * kProdBeta[k][0], dt * kProdBeta[k][1]);
            if (int rc = launch_stage(h, EPI_AXPY_SELF, ins[k], nullptr, outs[k], nullptr, beta, 0))
                return rc;
        }
        return 0;
    }
    case HEOM_RK4_HORNER: {
        double2* a = h->work[0].p;
        double2* b = h->work[1].p;
        const double c[4] = {dt / 4.0, dt / 3.0, dt / 2.0, dt};
        if (int rc = launch_stage(h, EPI_AXPY_SELF, y, nullptr, a, nullptr, make_double2(c[0], 0.0), 0)) return rc;
        if (int rc = launch_stage(h, EPI_AXPY_Y, a, y, b, nullptr, make_double2(c[1], 0.0), 0)) return rc;
        if (int rc = launch_stage(h, EPI_AXPY_Y, b, y, a, nullptr, make_double2(c[2], 0.0), 0)) return rc;
        if (int rc = launch_stage(h, EPI_AXPY_Y, a, y, y, nullptr, make_double2(c[3], 0.0), 0)) return rc;
        return 0;
    }
    default: { // HEOM_RK4_REFERENCE
        double2* k1 = h->work[0].p;
        double2* k2 = h->work[1].p;
        double2* k3 = h->work[2].p;
        double2* k4 = h->work[3].p;
        double2* st = h->work[4].p;
        const double2* ks[4] = {k1, k2, k3, k4};
        const double a2[1] = {0.5}, a3[2] = {0.0, 0.5}, a4[3] = {0.0, 0.0, 1.0};
        const double bb[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
        if (int rc = launch_stage(h, EPI_PURE, y, nullptr, k1, nullptr, zero, 0)) return rc;
        if (int rc = launch_wadd(h, 1, dt, st, y, a2, ks)) return rc;
        if (int rc = launch_stage(h, EPI_PURE, st, nullptr, k2, nullptr, zero, 0)) return rc;
        if (int rc = launch_wadd(h, 2, dt, st, y, a3, ks)) return rc;
        if (int rc = launch_stage(h, EPI_PURE, st, nullptr, k3, nullptr, zero, 0)) return rc;
        if (int rc = launch_wadd(h, 3, dt, st, y, a4, ks)) return rc;
        if (int rc = launch_stage(h, EPI_PURE, st, nullptr, k4, nullptr, zero, 0)) return rc;
        return launch_wadd(h, 4, dt, y, y, bb, ks);
    }
    }
}

int prepare_scheme(heom_handle* h)
{
    if (h->field_on) return ensure_work(h, 3);
    if (h->flow_above || h->flow_below) return ensure_work(h, 5);
    switch (h->opt.rk4_scheme) {
    case HEOM_RK4_PRODUCT:
    case HEOM_RK4_HORNER: return ensure_work(h, 2);
    case HEOM_RK4_REFERENCE: return ensure_work(h, 5);
    default: return fail(HEOM_E_ARG, "unknown rk4 scheme %d", h->opt.rk4_scheme);
    }
}

int launches_per_step(const heom_handle* h)
{
    if (h->field_on) return 5;
    if (h->flow_above || h->flow_below) return 8 + 4 * ((h->flow_above ? 1 : 0) + (h->flow_below ? 1 : 0));
    return h->opt.rk4_scheme == HEOM_RK4_REFERENCE ? 8 : 4;
}

int run_steps(heom_handle* h, double dt, int64_t steps)
{
    if (steps <= 0) return 0;
    if (!h->actions.empty())
        return fail(HEOM_E_UNSUPPORTED, "host pre-evaluate actions run with heom_solve only; the stepping calls take "
                                        "a device-side time dependence (heom_set_field)");
    if (int rc = prepare_scheme(h)) return rc;
    h->time += (double)steps * dt; // host mirror of the state's time (the device copy moves with field steps)
    if (!h->opt.use_graphs) {
        for (int64_t s = 0; s < steps; ++s)
            if (int rc = enqueue_step(h, dt)) return rc;
        return 0;
    }
    if (h->step_graph && h->graph_dt != dt) {
        cudaGraphExecDestroy(h->step_graph);
        h->step_graph = nullptr;
    }
    if (!h->step_graph) {
        // make sure launch shapes are resolved outside of capture
        const void* fn = nullptr;
        if (int rc = resolve_stage(h, &fn)) return rc;
        cudaGraph_t graph = nullptr;
        const int64_t saved = h->launches;
        CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(h, dt);
        cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
        h->launches = saved;
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return fail(HEOM_E_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&h->step_graph, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return fail(HEOM_E_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce));
        h->graph_dt = dt;
    }
    for (int64_t s = 0; s < steps; ++s) {
        CUDA_TRY(cudaGraphLaunch(h->step_graph, h->stream));
        h->launches += launches_per_step(h);
    }
    return 0;
}

int check_desc(const heom_instance_desc* d)
{
    if (!d) return fail(HEOM_E_ARG, "desc is NULL");
    if (d->states < 1 || d->states > kMaxStates)
        return fail(HEOM_E_UNSUPPORTED, "states = %d outside 1..%d", d->states, kMaxStates);
    if (d->matsubaras < 1 || d->baths < 1 || d->baths_per_state < 1)
        return fail(HEOM_E_ARG, "matsubaras, baths and baths_per_state must be >= 1");
    if (d->ado_width != d->baths * d->matsubaras)
        return fail(HEOM_E_TABLE, "ado_width %d != baths * matsubaras", d->ado_width);
    if (d->ado_width > kMaxWidth) return fail(HEOM_E_UNSUPPORTED, "ado_width %d too large", d->ado_width);
    if (d->ado_depth < 1 || d->ado_depth > 250) return fail(HEOM_E_UNSUPPORTED, "ado_depth %d", d->ado_depth);
    if (d->matrices < 1 || d->matrices > INT32_MAX) return fail(HEOM_E_ARG, "matrices = %lld", (long long)d->matrices);
    if (d->first_non_plus_id < 0 || d->first_non_plus_id > d->matrices)
        return fail(HEOM_E_TABLE, "first_non_plus_id out of range");
    if (!d->baths_coupling || !d->hamiltonian || !d->ado_tuples || !d->ado_plus || !d->ado_minus ||
        !d->pf_same_sum || !d->pf_same || !d->pf_circ || !d->cbk || !d->cbk_sqrt)
        return fail(HEOM_E_ARG, "a table pointer is NULL");
    for (int q = 0; q < d->states * d->baths_per_state; ++q)
        if (d->baths_coupling[q] >= d->baths) return fail(HEOM_E_TABLE, "baths_coupling value out of range");
    const int64_t n = d->matrices * d->ado_width;
    for (int64_t q = 0; q < n; ++q) {
        const int32_t t = d->ado_tuples[q], p = d->ado_plus[q], m = d->ado_minus[q];
        if (t < 0 || t > d->ado_depth) return fail(HEOM_E_TABLE, "ado_tuples[%lld] = %d out of range", (long long)q, t);
        if (!(p == HEOM_INVALID_UID || (p >= 0 && p < d->matrices)))
            return fail(HEOM_E_TABLE, "ado_plus[%lld] = %d out of range", (long long)q, p);
        if (!(m == HEOM_INVALID_UID || (m >= 0 && m < d->matrices)))
            return fail(HEOM_E_TABLE, "ado_minus[%lld] = %d out of range", (long long)q, m);
        if (t > 0 && m == HEOM_INVALID_UID)
            return fail(HEOM_E_TABLE, "ado_minus[%lld] missing for a non-zero tuple entry", (long long)q);
    }
    return 0;
}

// instances of one handle share states, baths, their coupling and bath
// tables; depth, hierarchy tables and Hamiltonian may differ
int check_same_class(const heom_instance_desc* a, const heom_instance_desc* b)
{
    if (a->states != b->states || a->matsubaras != b->matsubaras || a->baths != b->baths ||
        a->baths_per_state != b->baths_per_state || a->ado_width != b->ado_width)
        return fail(HEOM_E_ARG, "sizes differ");
    auto same = [](const void* x, const void* y, size_t bytes) { return std::memcmp(x, y, bytes) == 0; };
    if (!same(a->baths_coupling, b->baths_coupling, sizeof(int32_t) * a->states * a->baths_per_state))
        return fail(HEOM_E_ARG, "baths_coupling differs");
    if (!same(a->pf_same, b->pf_same, sizeof(double) * 2 * a->baths) ||
        !same(a->pf_circ, b->pf_circ, sizeof(double) * 2 * a->baths) ||
        !same(a->cbk, b->cbk, sizeof(double) * 2 * a->baths * a->matsubaras) ||
        !same(a->cbk_sqrt, b->cbk_sqrt, sizeof(double) * a->baths * a->matsubaras))
        return fail(HEOM_E_ARG, "bath tables differ");
    return 0;
}

// sector tables of the pair layout: the searched order for N <= 8
// (pair_tables.inc), the canonical order of heomk::pair_elements above
int build_pair_tables(heom_handle* h)
{
    const int N = h->N, P = h->P;
    h->pair_tab.assign(2 * P, 0);
    for (int p = 0; p < P; ++p) {
        int e1, e2, i, j, d;
        if (N <= 8) {
            e1 = kPairE1[N][p];
            e2 = kPairE2[N][p];
        } else {
            heomk::pair_elements(N, p, &e1, &e2, &i, &j, &d);
        }
        h->pair_tab[2 * p] = (int16_t)e1;
        h->pair_tab[2 * p + 1] = (int16_t)e2;
    }
    if (N <= 8) {
        heomk::LaneTab& lt = h->lane_tab;
        for (int l = 0; l < 32; ++l) {
            lt.e1[l] = (signed char)(l < P ? h->pair_tab[2 * l] : 0);
            lt.e2[l] = (signed char)(l < P ? h->pair_tab[2 * l + 1] : 0);
            const int r = l >> 2, t = l & 3;
            for (int s = 0; s < 2; ++s) {
                const int k = 4 * s + t;
                lt.fs[l][s] = -1;
                lt.ha[l][s] = 0;
                if (r >= N || k >= N) continue;
                const int e = r * N + k;
                for (int p = 0; p < P; ++p) {
                    if (h->pair_tab[2 * p] == e) { lt.fs[l][s] = (signed char)p; lt.ha[l][s] = 0; break; }
                    if (h->pair_tab[2 * p + 1] == e) { lt.fs[l][s] = (signed char)p; lt.ha[l][s] = 1; break; }
                }
                if (lt.fs[l][s] < 0) return fail(HEOM_E_UNSUPPORTED, "pair table misses element %d", e);
            }
        }
    }
    if (int rc = h->d_pair.alloc(2 * P)) return rc;
    CUDA_TRY(cudaMemcpy(h->d_pair.p, h->pair_tab.data(), 2 * P * sizeof(int16_t), cudaMemcpyHostToDevice));
    return 0;
}

// internal order, per instance: lexicographic rank of the tuple when the
// instance's tuples form the complete hierarchy, else the reference order
void build_order(heom_handle* h)
{
    const int W = h->W;
    h->int_of_ref.assign(h->nodes, 0);
    h->ref_of_int.assign(h->nodes, 0);
    h->top_int.assign(h->n_inst, 0);
    std::vector<std::vector<int64_t>> binom(W + h->D + 2, std::vector<int64_t>(W + 2, 0));
    for (int a = 0; a < W + h->D + 2; ++a) {
        binom[a][0] = 1;
        for (int b = 1; b <= std::min(a, W + 1); ++b)
            binom[a][b] = binom[a - 1][b - 1] + (b <= a - 1 ? binom[a - 1][b] : 0);
    }
    for (int k = 0; k < h->n_inst; ++k) {
        const int D = h->inst_depth[k];
        const int64_t base = h->inst_base[k], nodes = h->inst_base[k + 1] - base;
        bool lex = h->opt.ado_order == HEOM_ORDER_LEX && binom[W + D][W] == nodes;
        std::vector<char> seen(lex ? nodes : 0, 0);
        for (int64_t r = 0; lex && r < nodes; ++r) {
            int64_t rank = 0;
            int prefix = 0;
            for (int m = 0; m < W; ++m) {
                const int t = h->tuples[(base + r) * W + m];
                for (int x = 0; x < t; ++x) rank += simplex_count(W - 1 - m, D - prefix - x, binom);
                prefix += t;
            }
            if (prefix > D || rank < 0 || rank >= nodes || seen[rank]) {
                lex = false;
                break;
            }
            seen[rank] = 1;
            h->int_of_ref[base + r] = base + rank;
        }
        if (!lex)
            for (int64_t r = 0; r < nodes; ++r) h->int_of_ref[base + r] = base + r;
        h->top_int[k] = h->int_of_ref[base];
    }
    h->n_active = h->nodes;
    if (h->compact) {
        // active ADOs first, masked ones behind, each group in the order above
        std::vector<int64_t> by_int(h->nodes);
        for (int64_t r = 0; r < h->nodes; ++r) by_int[h->int_of_ref[r]] = r;
        int64_t a = 0;
        for (int64_t q = 0; q < h->nodes; ++q)
            if (h->mask[by_int[q]]) ++a;
        h->n_active = a;
        int64_t ia = 0, im = a;
        for (int64_t q = 0; q < h->nodes; ++q) {
            const int64_t r = by_int[q];
            h->int_of_ref[r] = h->mask[r] ? ia++ : im++;
        }
        for (int k = 0; k < h->n_inst; ++k) h->top_int[k] = h->int_of_ref[h->inst_base[k]];
    }
    for (int64_t r = 0; r < h->nodes; ++r) h->ref_of_int[h->int_of_ref[r]] = r;
}


int conv_blocks(const heom_handle* h, int64_t count)
{
    const int64_t total = count * h->P;
    return (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)h->sm_count * 16));
}

// host reference-layout state (all instances) -> pair layout, in chunks of xfer_ados ADOs
int to_internal(heom_handle* h, double2* dst, const double* host)
{
    const int64_t nn = (int64_t)h->N * h->N;
    for (int64_t r0 = 0; r0 < h->nodes; r0 += h->xfer_ados) {
        const int64_t count = std::min<int64_t>(h->xfer_ados, h->nodes - r0);
        CUDA_TRY(cudaMemcpyAsync(h->xfer.p, host + r0 * nn * 2, count * nn * sizeof(double2),
                                 cudaMemcpyHostToDevice, h->stream));
        heomk::heom_to_pairs<<<conv_blocks(h, count), 256, 0, h->stream>>>(dst, h->xfer.p, h->d_int_of_ref.p,
                                                                             h->d_pair.p, r0, count, h->N, h->P);
        h->launches++;
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int from_internal(heom_handle* h, double* host, const double2* src)
{
    const int64_t nn = (int64_t)h->N * h->N;
    for (int64_t r0 = 0; r0 < h->nodes; r0 += h->xfer_ados) {
        const int64_t count = std::min<int64_t>(h->xfer_ados, h->nodes - r0);
        heomk::heom_from_pairs<<<conv_blocks(h, count), 256, 0, h->stream>>>(h->xfer.p, src, h->d_int_of_ref.p,
                                                                               h->d_pair.p, r0, count, h->N, h->P);
        h->launches++;
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(host + r0 * nn * 2, h->xfer.p, count * nn * sizeof(double2),
                                 cudaMemcpyDeviceToHost, h->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

// rebuild the internal order (and everything indexed by it) after a change of
// the mask or of the compaction mode; the propagation state keeps its values
// Switch a freshly created batch handle whose instances share one hierarchy
// graph (one depth) and have no mask to the lockstep layout: sector p of
// internal ADO u of instance k at sector index (u * P + p) * kp + k, kp =
// instances rounded up to 32.  Only the ensemble builds such handles; the
// entry points that read or write the state in another layout refuse them.
int make_lockstep(heom_handle* h)
{
    if (h->N > 8 || h->n_inst < 2 || h->SL > 4 || h->compact || h->field_on)
        return fail(HEOM_E_UNSUPPORTED, "lockstep layout: needs 2+ instances of at most 8 states");
    const int64_t n0 = h->inst_base[1] - h->inst_base[0];
    for (int k = 0; k < h->n_inst; ++k)
        if (h->inst_base[k + 1] - h->inst_base[k] != n0 || h->inst_depth[k] != h->inst_depth[0])
            return fail(HEOM_E_UNSUPPORTED, "lockstep layout: instances of different depths");
    for (uint8_t m : h->mask)
        if (!m) return fail(HEOM_E_UNSUPPORTED, "lockstep layout: masked hierarchies are not supported");
    // the instance-minor state first: if it cannot be had, the handle stays the batch handle it was
    const int64_t kp = (h->n_inst + 31) / 32 * 32;
    const size_t elems = (size_t)n0 * kp * 2 * h->P;
    double2* ny = nullptr;
    if (cudaMalloc(&ny, elems * sizeof(double2)) != cudaSuccess)
        return fail(HEOM_E_NOMEM, "lockstep layout: cudaMalloc of %zu bytes failed", elems * sizeof(double2));
    const std::vector<int64_t> tops(h->n_inst, h->top_int[0] - h->inst_base[0]);
    if (cudaMemset(ny, 0, elems * sizeof(double2)) != cudaSuccess ||
        cudaMemcpy(h->d_top.p, tops.data(), tops.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(ny);
        return fail(HEOM_E_CUDA, "lockstep layout: %s", cudaGetErrorString(cudaGetLastError()));
    }
    h->y.data.reset();
    h->y.data.p = ny;
    h->y.data.n = elems;
    h->inst_nodes = n0;
    h->kp = kp;
    for (auto& w : h->work) w.reset();
    for (auto& a : h->per_sm) a[0] = a[1] = 0;
    h->stage_smem = 0;
    if (h->step_graph) {
        cudaGraphExecDestroy(h->step_graph);
        h->step_graph = nullptr;
    }
    return 0;
}

int lockstep_refuses(const heom_handle* h, const char* what)
{
    return fail(HEOM_E_UNSUPPORTED, "%s: not available on a lockstep ensemble class (instance-minor state)", what);
}

int reorder(heom_handle* h)
{
    std::vector<double> ref((size_t)h->nodes * h->N * h->N * 2);
    if (int rc = from_internal(h, ref.data(), h->y.data.p)) return rc;
    build_order(h);
    CUDA_TRY(cudaMemcpy(h->d_int_of_ref.p, h->int_of_ref.data(), h->nodes * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->d_ref_of_int.p, h->ref_of_int.data(), h->nodes * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->d_top.p, h->top_int.data(), h->n_inst * 8, cudaMemcpyHostToDevice));
    if (int rc = build_neighbours(h)) return rc;
    for (auto& w : h->work)
        if (w.p) CUDA_TRY(cudaMemset(w.p, 0, h->state_elems() * sizeof(double2)));
    if (h->step_graph) {
        cudaGraphExecDestroy(h->step_graph);
        h->step_graph = nullptr;
    }
    return to_internal(h, h->y.data.p, ref.data());
}

// ---------------------------------------------------------------------------
// Static scratch for heom_rk4_steps_noalloc: three state-sized buffers (the
// caller's state converted to the pair layout, and the two stage buffers of
// the product-form RK4 step).  The array is part of this module, so every GPU
// that loads the library holds it until the process exits.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocBufferBytes = size_t(16) << 20; // per buffer
constexpr int kNoAllocBuffers = 3;
constexpr int kNoAllocMaxDevices = 128;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};

} // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBuffers * kNoAllocBufferBytes];

namespace {

// Device address of the static scratch on `device`, which the caller has made
// current.  Resolved once per device: in host code the array's name is only a
// host-side stand-in, so kernels are always given this address.
int noalloc_scratch(int device, unsigned char** out)
{
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(HEOM_E_ARG, "device ordinal %d out of range", device);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(HEOM_E_CUDA, "cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
        g_noalloc_addr[device] = ptr;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[device]);
    return 0;
}

// a stage kernel whose bounded pipeline wait expired leaves a flag behind
int check_kernel_error(heom_handle* h)
{
    int err = 0;
    CUDA_TRY(cudaMemcpy(&err, h->d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        cudaMemset(h->d_err.p, 0, sizeof(int));
        return fail(HEOM_E_CUDA, "stage kernel pipeline wait expired (results of this call are invalid)");
    }
    return 0;
}

int hier_check(const heom_handle* h, const heom_buffer* a, const heom_buffer* b, const heom_buffer* out)
{
    if (h && h->kp) return lockstep_refuses(h, "hierarchy arithmetic");
    if (!h || !a || !out || a->owner != h || out->owner != h || (b && b->owner != h))
        return fail(HEOM_E_ARG, "buffers must belong to the handle");
    return 0;
}

int hier_elementwise(heom_handle* h, const heom_buffer* a, const heom_buffer* b, heom_buffer* out, double2 f, int op)
{
    if (int rc = hier_check(h, a, b, out)) return rc;
    if (op != 3 && !b) return fail(HEOM_E_ARG, "NULL buffer");
    CUDA_TRY(cudaSetDevice(h->device));
    const int64_t len = (int64_t)h->state_elems();
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((len + 255) / 256, (int64_t)h->sm_count * 8));
    heomk::heom_hier_elementwise<<<blocks, 256, 0, h->stream>>>(out->data.p, a->data.p, b ? b->data.p : a->data.p, f,
                                                                len, op);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int hier_mmult(heom_handle* h, const heom_buffer* a, const double* m, heom_buffer* out, int left)
{
    if (int rc = hier_check(h, a, nullptr, out)) return rc;
    if (!m) return fail(HEOM_E_ARG, "NULL matrix");
    CUDA_TRY(cudaSetDevice(h->device));
    const int NN = h->N * h->N;
    DevBuf<double2> dm;
    if (int rc = dm.alloc(NN)) return rc;
    CUDA_TRY(cudaMemcpyAsync(dm.p, m, NN * 16, cudaMemcpyHostToDevice, h->stream));
    const size_t smem = (size_t)8 * 2 * NN * 16;
    if (int rc = allow_dynamic_smem((const void*)heomk::heom_hier_mmult, smem)) return rc;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((h->nodes + 7) / 8, (int64_t)h->sm_count * 8));
    heomk::heom_hier_mmult<<<blocks, 256, smem, h->stream>>>(out->data.p, a->data.p, dm.p, h->d_pair.p, h->nodes, h->N,
                                                             h->P, left);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

} // namespace

extern "C" {

const char* heom_last_error(void) { return g_last_error.c_str(); }

void heom_default_options(heom_options* opt)
{
    if (!opt) return;
    opt->device = 0;
    opt->ado_order = HEOM_ORDER_LEX;
    opt->rk4_scheme = HEOM_RK4_PRODUCT;
    opt->use_graphs = 1;
}

int heom_create(const heom_instance_desc* d, const heom_options* opt, heom_handle** out)
{
    return heom_create_batch(d, 1, opt, out);
}

int heom_create_batch(const heom_instance_desc* descs, int32_t count, const heom_options* opt, heom_handle** out)
{
    if (!out) return fail(HEOM_E_ARG, "out is NULL");
    *out = nullptr;
    if (!descs || count < 1) return fail(HEOM_E_ARG, "descs is NULL or count < 1");
    for (int k = 0; k < count; ++k) {
        if (int rc = check_desc(&descs[k])) {
            if (count > 1) g_last_error = "instance " + std::to_string(k) + ": " + g_last_error;
            return rc;
        }
        if (int rc = check_same_class(&descs[0], &descs[k]))
            return fail(rc, "instance %d does not share states, baths and Matsubara terms with instance 0: %s", k,
                        g_last_error.c_str());
    }
    const heom_instance_desc* d = &descs[0];
    std::unique_ptr<heom_handle> h(new heom_handle());
    heom_default_options(&h->opt);
    if (opt) h->opt = *opt;
    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (h->opt.device < 0 || h->opt.device >= ndev)
        return fail(HEOM_E_CUDA, "device %d not available (%d devices)", h->opt.device, ndev);
    h->device = h->opt.device;
    CUDA_TRY(cudaSetDevice(h->device));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, h->device));
    if (prop.major < 10)
        return fail(HEOM_E_CUDA, "device %d is sm_%d%d; this build targets sm_100a", h->device, prop.major, prop.minor);
    h->sm_count = prop.multiProcessorCount;
    CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));

    h->N = d->states;
    h->M = d->matsubaras;
    h->B = d->baths;
    h->BPS = d->baths_per_state;
    h->W = d->ado_width;
    h->n_inst = count;
    h->inst_base.assign(count + 1, 0);
    h->D = 0;
    for (int k = 0; k < count; ++k) {
        h->inst_base[k + 1] = h->inst_base[k] + descs[k].matrices;
        h->inst_depth.push_back(descs[k].ado_depth);
        h->inst_fnp.push_back(descs[k].first_non_plus_id);
        h->D = std::max(h->D, descs[k].ado_depth);
    }
    h->nodes = h->inst_base[count];
    if (h->nodes > INT32_MAX) return fail(HEOM_E_UNSUPPORTED, "%lld ADOs in one handle (at most 2^31 - 1)",
                                          (long long)h->nodes);
    h->LS = h->D + 1;
    h->SL = h->BPS * h->M;
    if (h->SL > 8) return fail(HEOM_E_UNSUPPORTED, "baths_per_state * matsubaras = %d > 8", h->SL);
    h->SLT = h->SL <= 2 ? 2 : h->SL <= 4 ? 4 : 8;
    h->P = heomk::pairs_of(h->N);
    h->NW = (2 * h->W + 3) & ~3;
    h->TWB = (h->W + 15) & ~15;
    const int W = h->W;
    h->coupling.assign(d->baths_coupling, d->baths_coupling + h->N * h->BPS);
    h->pf_same.assign(d->pf_same, d->pf_same + 2 * h->B);
    h->pf_circ.assign(d->pf_circ, d->pf_circ + 2 * h->B);
    h->cbk.assign(d->cbk, d->cbk + 2 * h->B * h->M);
    h->cbk_sqrt.assign(d->cbk_sqrt, d->cbk_sqrt + h->B * h->M);
    h->tuples.resize((size_t)h->nodes * W);
    h->plus.resize((size_t)h->nodes * W);
    h->minus.resize((size_t)h->nodes * W);
    h->pss.resize((size_t)h->nodes * 2);
    h->ham.resize((size_t)count * 2 * h->N * h->N);
    for (int k = 0; k < count; ++k) {
        const heom_instance_desc* e = &descs[k];
        const int64_t base = h->inst_base[k], nw = e->matrices * W;
        std::copy(e->ado_tuples, e->ado_tuples + nw, h->tuples.begin() + base * W);
        for (int64_t q = 0; q < nw; ++q) {
            h->plus[base * W + q] = e->ado_plus[q] == HEOM_INVALID_UID ? -1 : (int32_t)(base + e->ado_plus[q]);
            h->minus[base * W + q] = e->ado_minus[q] == HEOM_INVALID_UID ? -1 : (int32_t)(base + e->ado_minus[q]);
        }
        std::copy(e->pf_same_sum, e->pf_same_sum + 2 * e->matrices, h->pss.begin() + 2 * base);
        std::copy(e->hamiltonian, e->hamiltonian + 2 * h->N * h->N, h->ham.begin() + (size_t)k * 2 * h->N * h->N);
    }
    h->mask.assign(h->nodes, 1);
    for (int q = 0; q < h->B * h->M; ++q)
        if (!(std::hypot(h->cbk[2 * q], h->cbk[2 * q + 1]) > 0.0))
            return fail(HEOM_E_TABLE, "cbk[%d] is zero or not finite", q);

    if (int rc = build_pair_tables(h.get())) return rc;
    build_order(h.get());
    if (int rc = h->d_int_of_ref.alloc(h->nodes)) return rc;
    CUDA_TRY(cudaMemcpy(h->d_int_of_ref.p, h->int_of_ref.data(), h->nodes * 8, cudaMemcpyHostToDevice));
    if (int rc = h->d_ref_of_int.alloc(h->nodes)) return rc;
    CUDA_TRY(cudaMemcpy(h->d_ref_of_int.p, h->ref_of_int.data(), h->nodes * 8, cudaMemcpyHostToDevice));
    if (int rc = h->d_top.alloc(count)) return rc;
    CUDA_TRY(cudaMemcpy(h->d_top.p, h->top_int.data(), count * 8, cudaMemcpyHostToDevice));
    if (int rc = build_neighbours(h.get())) return rc;
    if (int rc = upload_coefficients(h.get())) return rc;
    if (int rc = upload_hamiltonian(h.get())) return rc;
    h->y.owner = h.get();
    h->y.borrowed = true;
    if (int rc = h->y.data.alloc(h->state_elems())) return rc;
    CUDA_TRY(cudaMemset(h->y.data.p, 0, h->state_elems() * sizeof(double2)));
    // host transfers go through a staging buffer of at most 64 MiB
    const int64_t nn = (int64_t)h->N * h->N;
    h->xfer_ados = std::max<int64_t>(1, std::min<int64_t>(h->nodes, (int64_t(64) << 20) / (nn * 16)));
    if (int rc = h->xfer.alloc((size_t)h->xfer_ados * nn)) return rc;
    if (int rc = h->topbuf.alloc((size_t)count * nn)) return rc;
    if (int rc = h->d_flag.alloc(1)) return rc;
    if (int rc = h->d_err.alloc(1)) return rc;
    CUDA_TRY(cudaMemset(h->d_err.p, 0, sizeof(int)));
    *out = h.release();
    return 0;
}

int heom_destroy(heom_handle* h)
{
    if (!h) return 0;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
    // buffers that outlive their handle keep no device memory and no owner;
    // heom_buffer_destroy then only frees the struct
    for (heom_buffer* b : h->live_buffers) {
        b->data.reset();
        b->owner = nullptr;
    }
    cudaStream_t s = h->stream;
    delete h;
    if (s) cudaStreamDestroy(s);
    return 0;
}

int heom_set_hamiltonian(heom_handle* h, const double* ham)
{
    if (!h || !ham) return fail(HEOM_E_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->ham.assign(ham, ham + (size_t)h->n_inst * 2 * h->N * h->N);
    return upload_hamiltonian(h);
}

int heom_set_instance_hamiltonian(heom_handle* h, int32_t inst, const double* ham)
{
    if (!h || !ham) return fail(HEOM_E_ARG, "NULL argument");
    if (inst < 0 || inst >= h->n_inst) return fail(HEOM_E_ARG, "instance %d out of range", inst);
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    const size_t nn2 = (size_t)2 * h->N * h->N;
    std::copy(ham, ham + nn2, h->ham.begin() + inst * nn2);
    return upload_hamiltonian(h);
}

int heom_set_mask(heom_handle* h, const uint8_t* mask)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_set_mask");
    if (!h || !mask) return fail(HEOM_E_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int64_t q = 0; q < h->nodes; ++q)
        if (mask[q] > 2) return fail(HEOM_E_ARG, "mask[%lld] = %d is not a mask value", (long long)q, mask[q]);
    h->mask.assign(mask, mask + h->nodes);
    if (h->compact) {
        h->compact = false;
        return reorder(h);
    }
    return build_neighbours(h);
}

int heom_set_mask_compact(heom_handle* h, const uint8_t* mask)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_set_mask_compact");
    if (!h || !mask) return fail(HEOM_E_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int64_t q = 0; q < h->nodes; ++q)
        if (mask[q] > 2) return fail(HEOM_E_ARG, "mask[%lld] = %d is not a mask value", (long long)q, mask[q]);
    for (int k = 0; k < h->n_inst; ++k)
        if (!mask[h->inst_base[k]]) return fail(HEOM_E_ARG, "instance %d: the top ADO is masked", k);
    h->mask.assign(mask, mask + h->nodes);
    h->compact = true;
    return reorder(h);
}

int64_t heom_active_matrices(const heom_handle* h) { return h ? h->n_active : 0; }

int heom_set_field(heom_handle* h, const double* dipole_plus, const double* dipole_minus, const heom_pulse* pump,
                   const heom_pulse* probe)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_set_field");
    if (!h || !dipole_plus || !dipole_minus || !pump || !probe) return fail(HEOM_E_ARG, "NULL argument");
    const heom_pulse* pl[2] = {pump, probe};
    for (int q = 0; q < 2; ++q)
        if (!(pl[q]->time_width > 0.0) || !std::isfinite(pl[q]->efield) || !std::isfinite(pl[q]->time_center) ||
            !std::isfinite(pl[q]->frequency) || !std::isfinite(pl[q]->phase))
            return fail(HEOM_E_ARG, "pulse %d: width must be > 0 and every value finite", q);
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    const int N = h->N, K = h->n_inst;
    std::vector<double2> dp(N * N), dm(N * N);
    for (int q = 0; q < N * N; ++q) {
        dp[q] = make_double2(dipole_plus[2 * q] / kHbar, dipole_plus[2 * q + 1] / kHbar);
        dm[q] = make_double2(dipole_minus[2 * q] / kHbar, dipole_minus[2 * q + 1] / kHbar);
    }
    for (int q = 0; q < 2; ++q)
        h->pulses[q] = heomk::Pulse{pl[q]->efield, pl[q]->time_center, pl[q]->time_width, pl[q]->frequency,
                                    pl[q]->phase};
    if (!h->d_dplus.p) {
        if (int rc = h->d_dplus.alloc(N * N)) return rc;
        if (int rc = h->d_dminus.alloc(N * N)) return rc;
        if (int rc = h->field_hs.alloc((size_t)3 * K * N * N)) return rc;
        if (int rc = h->field_frag.alloc((size_t)3 * K * heomk::frag_doubles(N))) return rc;
        if (int rc = h->d_time.alloc(1)) return rc;
    }
    CUDA_TRY(cudaMemcpy(h->d_dplus.p, dp.data(), N * N * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->d_dminus.p, dm.data(), N * N * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->d_time.p, &h->time, 8, cudaMemcpyHostToDevice));
    h->field_on = true;
    return upload_hamiltonian(h); // complex kernel variant; drops the step graph
}

int heom_clear_field(heom_handle* h)
{
    if (!h) return fail(HEOM_E_ARG, "NULL handle");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->field_on = false;
    return upload_hamiltonian(h);
}

int heom_set_time(heom_handle* h, double time)
{
    if (!h || !std::isfinite(time)) return fail(HEOM_E_ARG, "bad argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->time = time;
    if (h->d_time.p) CUDA_TRY(cudaMemcpy(h->d_time.p, &h->time, 8, cudaMemcpyHostToDevice));
    return 0;
}

double heom_time(const heom_handle* h) { return h ? h->time : 0.0; }

int heom_hierarchy_add(heom_handle* h, const heom_buffer* a, const heom_buffer* b, heom_buffer* out)
{
    return hier_elementwise(h, a, b, out, make_double2(0.0, 0.0), 0);
}
int heom_hierarchy_subtract(heom_handle* h, const heom_buffer* a, const heom_buffer* b, heom_buffer* out)
{
    return hier_elementwise(h, a, b, out, make_double2(0.0, 0.0), 1);
}
int heom_hierarchy_dot_product(heom_handle* h, const heom_buffer* a, const heom_buffer* b, heom_buffer* out)
{
    return hier_elementwise(h, a, b, out, make_double2(0.0, 0.0), 2);
}
int heom_hierarchy_scale(heom_handle* h, const heom_buffer* a, double re, double im, heom_buffer* out)
{
    return hier_elementwise(h, a, nullptr, out, make_double2(re, im), 3);
}
int heom_hierarchy_mmult_left(heom_handle* h, const heom_buffer* a, const double* m, heom_buffer* out)
{
    return hier_mmult(h, a, m, out, 1);
}
int heom_hierarchy_mmult_right(heom_handle* h, const heom_buffer* a, const double* m, heom_buffer* out)
{
    return hier_mmult(h, a, m, out, 0);
}

int heom_add_pre_evaluate_action(heom_handle* h, heom_pre_evaluate_fn fn, void* user)
{
    if (!h || !fn) return fail(HEOM_E_ARG, "NULL argument");
    h->actions.push_back({fn, user});
    return 0;
}

int heom_clear_pre_evaluate_actions(heom_handle* h)
{
    if (!h) return fail(HEOM_E_ARG, "NULL handle");
    h->actions.clear();
    return 0;
}

int heom_get_mask(const heom_handle* h, uint8_t* mask)
{
    if (!h || !mask) return fail(HEOM_E_ARG, "NULL argument");
    std::copy(h->mask.begin(), h->mask.end(), mask);
    return 0;
}

int heom_buffer_hierarchy_norm(heom_handle* h, const heom_buffer* b, double* norms)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_buffer_hierarchy_norm");
    if (!h || !b || b->owner != h || !norms) return fail(HEOM_E_ARG, "bad argument");
    CUDA_TRY(cudaSetDevice(h->device));
    DevBuf<double> d_norm;
    if (int rc = d_norm.alloc(h->nodes)) return rc;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((h->nodes + 7) / 8, (int64_t)h->sm_count * 8));
    heomk::heom_hierarchy_norm<<<blocks, 256, 0, h->stream>>>(d_norm.p, b->data.p, h->d_ref_of_int.p, h->d_pair.p,
                                                              h->nodes, h->P);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(norms, d_norm.p, h->nodes * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int heom_hierarchy_norm(heom_handle* h, double threshold, double* norms)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_hierarchy_norm");
    if (!h) return fail(HEOM_E_ARG, "NULL handle");
    CUDA_TRY(cudaSetDevice(h->device));
    DevBuf<double> d_norm;
    if (int rc = d_norm.alloc(h->nodes)) return rc;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((h->nodes + 7) / 8, (int64_t)h->sm_count * 8));
    heomk::heom_hierarchy_norm<<<blocks, 256, 0, h->stream>>>(d_norm.p, h->y.data.p, h->d_ref_of_int.p, h->d_pair.p,
                                                              h->nodes, h->P);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    std::vector<double> nv(h->nodes);
    CUDA_TRY(cudaMemcpyAsync(nv.data(), d_norm.p, h->nodes * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (norms) std::copy(nv.begin(), nv.end(), norms);
    if (threshold < 0.0) return 0;
    // deactivate unprotected ADOs at or below the threshold (hierarchy_norm.cl:42-44)
    std::vector<uint8_t> mask = h->mask;
    bool changed = false;
    for (int64_t r = 0; r < h->nodes; ++r)
        if (nv[r] - threshold <= 0.0 && mask[r] != 2 && mask[r] != 0) {
            mask[r] = 0;
            changed = true;
        }
    if (!changed) return 0;
    return h->compact ? heom_set_mask_compact(h, mask.data()) : heom_set_mask(h, mask.data());
}

size_t heom_buffer_size_byte(const heom_handle* h) { return h ? h->state_elems() * sizeof(double2) : 0; }

int heom_buffer_create(heom_handle* h, heom_buffer** out)
{
    if (!h || !out) return fail(HEOM_E_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(h->device));
    std::unique_ptr<heom_buffer> b(new heom_buffer());
    b->owner = h;
    if (int rc = b->data.alloc(h->state_elems())) return rc;
    CUDA_TRY(cudaMemset(b->data.p, 0, h->state_elems() * sizeof(double2)));
    h->live_buffers.push_back(b.get());
    *out = b.release();
    return 0;
}

int heom_buffer_destroy(heom_buffer* b)
{
    if (!b) return 0;
    if (b->borrowed) return fail(HEOM_E_ARG, "cannot destroy a borrowed buffer view");
    if (heom_handle* h = b->owner) {
        cudaSetDevice(h->device);
        if (h->flow_above == b || h->flow_below == b) {
            if (h->flow_above == b) h->flow_above = nullptr;
            if (h->flow_below == b) h->flow_below = nullptr;
            if (h->step_graph) {
                cudaGraphExecDestroy(h->step_graph);
                h->step_graph = nullptr;
            }
        }
        auto& v = h->live_buffers;
        v.erase(std::remove(v.begin(), v.end(), b), v.end());
    }
    delete b;
    return 0;
}

int heom_buffer_write(heom_handle* h, heom_buffer* b, const double* host)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_buffer_write");
    if (!h || !b || !host || b->owner != h) return fail(HEOM_E_ARG, "bad argument");
    CUDA_TRY(cudaSetDevice(h->device));
    return to_internal(h, b->data.p, host);
}

int heom_buffer_read(heom_handle* h, const heom_buffer* b, double* host)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_buffer_read");
    if (!h || !b || !host || b->owner != h) return fail(HEOM_E_ARG, "bad argument");
    CUDA_TRY(cudaSetDevice(h->device));
    return from_internal(h, host, b->data.p);
}

int heom_solve(heom_handle* h, double time, double step_size, const heom_buffer* in, heom_buffer* out,
               double out_coeff, heom_buffer* acc, double acc_coeff, int acc_init, int mode)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_solve");
    if (!h || !in || in->owner != h) return fail(HEOM_E_ARG, "bad input buffer");
    CUDA_TRY(cudaSetDevice(h->device));
    int rc = 0;
    // host pre-evaluate actions in registration order (ode.cpp:17-22)
    for (auto& a : h->actions)
        if (int arc = a.first(a.second, h, time, step_size, in, out))
            return fail(arc < 0 ? arc : HEOM_E_ARG, "pre-evaluate action returned %d", arc);
    // device field (ode.cpp:99, e_field.hpp:69): H at time + step_size
    AdjTabs ft;
    const AdjTabs* tabs = nullptr;
    if (h->field_on) {
        heomk::FieldParams f = field_params(h, 1);
        f.t0 = time + step_size;
        heomk::heom_field_tables<<<1, 256, 0, h->stream>>>(f);
        h->launches++;
        CUDA_TRY(cudaGetLastError());
        ft = field_tabs(h, 0);
        tabs = &ft;
    }
    switch (mode) {
    case HEOM_SOLVE_PURE:
        if (!out || out->owner != h || out == in) return fail(HEOM_E_ARG, "bad output buffer");
        rc = launch_stage(h, EPI_PURE, in->data.p, nullptr, out->data.p, nullptr,
                          make_double2(0.0, 0.0), 0, tabs);
        break;
    case HEOM_SOLVE_ACCUMULATE:
        if (!out || out->owner != h || out == in || !acc || acc->owner != h || acc == in || acc == out)
            return fail(HEOM_E_ARG, "bad output/accumulation buffer");
        rc = launch_stage(h, EPI_ACC, in->data.p, nullptr, out->data.p, acc->data.p,
                          make_double2(acc_coeff, 0.0), acc_init ? 1 : 0, tabs);
        break;
    case HEOM_SOLVE_SUBDIAGONAL:
        if (!acc || acc->owner != h || acc == in) return fail(HEOM_E_ARG, "bad accumulation buffer");
        rc = launch_stage(h, EPI_AXPY_SELF, in->data.p, nullptr, acc->data.p, nullptr,
                          make_double2(out_coeff, 0.0), 0, tabs);
        break;
    default: return fail(HEOM_E_ARG, "unknown solve mode %d", mode);
    }
    if (rc) return rc;
    if (int frc = launch_flows(h, in->data.p, acc_coeff)) return frc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return check_kernel_error(h);
}

int heom_set_flow_buffers(heom_handle* h, heom_buffer* flow_from_above, heom_buffer* flow_from_below)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_set_flow_buffers");
    if (!h) return fail(HEOM_E_ARG, "NULL handle");
    if ((flow_from_above && flow_from_above->owner != h) || (flow_from_below && flow_from_below->owner != h))
        return fail(HEOM_E_ARG, "flow buffers must belong to the handle");
    if (flow_from_above && flow_from_above == flow_from_below)
        return fail(HEOM_E_ARG, "the two flow buffers must differ");
    CUDA_TRY(cudaSetDevice(h->device));
    if ((flow_from_above || flow_from_below) && !h->d_zero.p) {
        const size_t K = h->n_inst, N = h->N;
        size_t len = std::max<size_t>({K * heomk::frag_doubles((int)N), K * N * (N + 1), 2 * K * N * N, (size_t)6 * h->W * h->LS,
                                       (size_t)6 * h->W, (size_t)2 * h->nodes});
        if (int rc = h->d_zero.alloc(len)) return rc;
        CUDA_TRY(cudaMemset(h->d_zero.p, 0, len * 8));
        if (int rc = h->flow_scratch.alloc(h->state_elems())) return rc;
    }
    h->flow_above = flow_from_above;
    h->flow_below = flow_from_below;
    if (h->step_graph) { // the captured step does not track (or stops tracking) the flows
        cudaGraphExecDestroy(h->step_graph);
        h->step_graph = nullptr;
    }
    return 0;
}

int heom_weighted_add(heom_handle* h, int n, double step, heom_buffer* out, const heom_buffer* y,
                      const double* coeffs, const heom_buffer* const* k)
{
    if (!h || !out || !y || n < 0 || n > 7 || (n > 0 && (!coeffs || !k)))
        return fail(HEOM_E_ARG, "bad argument");
    const double2* kp[7];
    for (int l = 0; l < n; ++l) {
        if (!k[l] || k[l]->owner != h) return fail(HEOM_E_ARG, "bad k buffer");
        kp[l] = k[l]->data.p;
    }
    CUDA_TRY(cudaSetDevice(h->device));
    if (int rc = launch_wadd(h, n, step, out->data.p, y->data.p, coeffs, kp)) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int heom_set_state(heom_handle* h, const double* host)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_set_state");
    if (!h || !host) return fail(HEOM_E_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(h->device));
    return to_internal(h, h->y.data.p, host);
}

int heom_get_state(heom_handle* h, double* host)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_get_state");
    if (!h || !host) return fail(HEOM_E_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(h->device));
    return from_internal(h, host, h->y.data.p);
}

int heom_set_top(heom_handle* h, const double* top)
{
    if (!h || !top) return fail(HEOM_E_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(h->device));
    const size_t nn = (size_t)h->N * h->N * h->n_inst;
    CUDA_TRY(cudaMemcpyAsync(h->topbuf.p, top, nn * 16, cudaMemcpyHostToDevice, h->stream));
    heomk::heom_write_top<<<h->n_inst, 128, 0, h->stream>>>(h->y.data.p, h->topbuf.p, h->d_pair.p, h->d_top.p, h->N,
                                                            h->P, h->kp, 0);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int heom_get_top(heom_handle* h, double* top)
{
    if (!h || !top) return fail(HEOM_E_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(h->device));
    const size_t nn = (size_t)h->N * h->N * h->n_inst;
    heomk::heom_record_top<<<h->n_inst, 128, 0, h->stream>>>(h->topbuf.p, h->y.data.p, h->d_pair.p, h->d_top.p, h->N,
                                                             h->P, 0, h->kp, 0);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(top, h->topbuf.p, nn * 16, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int heom_set_instance_top(heom_handle* h, int32_t inst, const double* top)
{
    if (!h || !top) return fail(HEOM_E_ARG, "NULL argument");
    if (inst < 0 || inst >= h->n_inst) return fail(HEOM_E_ARG, "instance %d out of range", inst);
    CUDA_TRY(cudaSetDevice(h->device));
    const size_t nn = (size_t)h->N * h->N;
    CUDA_TRY(cudaMemcpyAsync(h->topbuf.p, top, nn * 16, cudaMemcpyHostToDevice, h->stream));
    heomk::heom_write_top<<<1, 128, 0, h->stream>>>(h->y.data.p, h->topbuf.p, h->d_pair.p, h->d_top.p + inst, h->N,
                                                    h->P, h->kp, inst);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int heom_get_instance_top(heom_handle* h, int32_t inst, double* top)
{
    if (!h || !top) return fail(HEOM_E_ARG, "NULL argument");
    if (inst < 0 || inst >= h->n_inst) return fail(HEOM_E_ARG, "instance %d out of range", inst);
    CUDA_TRY(cudaSetDevice(h->device));
    const size_t nn = (size_t)h->N * h->N;
    heomk::heom_record_top<<<1, 128, 0, h->stream>>>(h->topbuf.p, h->y.data.p, h->d_pair.p, h->d_top.p + inst, h->N,
                                                     h->P, 0, h->kp, inst);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(top, h->topbuf.p, nn * 16, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int heom_state_buffer(heom_handle* h, heom_buffer** view)
{
    if (!h || !view) return fail(HEOM_E_ARG, "NULL argument");
    *view = &h->y;
    return 0;
}

int heom_rk4_steps_async(heom_handle* h, double dt, int64_t steps)
{
    if (!h || steps < 0 || !(dt > 0.0)) return fail(HEOM_E_ARG, "bad argument");
    CUDA_TRY(cudaSetDevice(h->device));
    return run_steps(h, dt, steps);
}

int heom_synchronize(heom_handle* h)
{
    if (!h) return fail(HEOM_E_ARG, "NULL handle");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return check_kernel_error(h);
}

int heom_rk4_steps(heom_handle* h, double dt, int64_t steps)
{
    if (int rc = heom_rk4_steps_async(h, dt, steps)) return rc;
    return heom_synchronize(h);
}

int heom_propagate(heom_handle* h, double dt, int64_t steps, int64_t observe_every, double* host_tops)
{
    if (!h || !host_tops || steps < 0 || observe_every <= 0 || steps % observe_every != 0 || !(dt > 0.0))
        return fail(HEOM_E_ARG, "bad argument (steps must be a multiple of observe_every)");
    CUDA_TRY(cudaSetDevice(h->device));
    const int64_t rows = steps / observe_every + 1;
    const int64_t nn = (int64_t)h->N * h->N * h->n_inst;
    if ((int64_t)h->toplog.n < rows * nn)
        if (int rc = h->toplog.alloc(rows * nn)) return rc;
    heomk::heom_record_top<<<h->n_inst, 128, 0, h->stream>>>(h->toplog.p, h->y.data.p, h->d_pair.p, h->d_top.p, h->N,
                                                             h->P, 0, h->kp, 0);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    for (int64_t r = 1; r < rows; ++r) {
        if (int rc = run_steps(h, dt, observe_every)) return rc;
        heomk::heom_record_top<<<h->n_inst, 128, 0, h->stream>>>(h->toplog.p, h->y.data.p, h->d_pair.p, h->d_top.p,
                                                                 h->N, h->P, r, h->kp, 0);
        h->launches++;
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaMemcpyAsync(host_tops, h->toplog.p, rows * nn * 16, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    // failure detection: a non-finite state is reported instead of returned silently
    CUDA_TRY(cudaMemsetAsync(h->d_flag.p, 0, sizeof(int), h->stream));
    heomk::heom_check_finite<<<h->sm_count * 4, 256, 0, h->stream>>>(
        reinterpret_cast<const double*>(h->y.data.p), (int64_t)h->state_elems() * 2, h->d_flag.p);
    h->launches++;
    int flag = 0;
    CUDA_TRY(cudaMemcpyAsync(&flag, h->d_flag.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (int rc = check_kernel_error(h)) return rc;
    if (flag) return fail(HEOM_E_NONFINITE, "non-finite value in the hierarchy state after propagation");
    return 0;
}

int heom_rk4_steps_noalloc(heom_handle* h, double* d_state, double dt, int64_t steps)
{
    if (h && h->kp) return lockstep_refuses(h, "heom_rk4_steps_noalloc");
    if (!h || !d_state || steps < 0 || !(dt > 0.0)) return fail(HEOM_E_ARG, "bad argument");
    if (reinterpret_cast<uintptr_t>(d_state) % 16 != 0) return fail(HEOM_E_ARG, "d_state must be 16-byte aligned");
    // the static scratch holds the three buffers of the time-independent
    // product form and nothing else: refuse handle state that step cannot honour
    if (!h->actions.empty())
        return fail(HEOM_E_UNSUPPORTED, "host pre-evaluate actions run with heom_solve only; the stepping calls take "
                                        "a device-side time dependence (heom_set_field)");
    if (h->field_on)
        return fail(HEOM_E_UNSUPPORTED, "heom_rk4_steps_noalloc: a time-dependent field needs the classical RK4 "
                                        "buffers (use heom_rk4_steps)");
    if (h->flow_above || h->flow_below)
        return fail(HEOM_E_UNSUPPORTED, "heom_rk4_steps_noalloc: flow tracking needs buffers the static scratch "
                                        "does not hold (use heom_rk4_steps)");
    const size_t need = h->state_elems() * sizeof(double2);
    if (need > kNoAllocBufferBytes)
        return fail(HEOM_E_UNSUPPORTED,
                    "heom_rk4_steps_noalloc: this hierarchy needs %zu bytes per state buffer; the static scratch "
                    "holds %zu bytes per buffer (use heom_rk4_steps)",
                    need, kNoAllocBufferBytes);
    CUDA_TRY(cudaSetDevice(h->device));
    unsigned char* base = nullptr;
    if (int rc = noalloc_scratch(h->device, &base)) return rc;
    double2* y = reinterpret_cast<double2*>(base);
    double2* a = reinterpret_cast<double2*>(base + kNoAllocBufferBytes);
    double2* b = reinterpret_cast<double2*>(base + 2 * kNoAllocBufferBytes);
    // every element of y, a and b is written before it is read in this call, so
    // what an earlier call left in the array needs no clearing
    const int cblocks = conv_blocks(h, h->nodes);
    heomk::heom_to_pairs<<<cblocks, 256, 0, h->stream>>>(y, reinterpret_cast<const double2*>(d_state),
                                                          h->d_int_of_ref.p, h->d_pair.p, 0, h->nodes, h->N, h->P);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    const double2* ins[4] = {y, a, b, a};
    double2* outs[4] = {a, b, a, y};
    for (int64_t s = 0; s < steps; ++s)
        for (int k = 0; k < 4; ++k) {
            const double2 beta = make_double2(dt * kProdBeta[k][0], dt * kProdBeta[k][1]);
            if (int rc = launch_stage(h, EPI_AXPY_SELF, ins[k], nullptr, outs[k], nullptr, beta, 0)) return rc;
        }
    heomk::heom_from_pairs<<<cblocks, 256, 0, h->stream>>>(reinterpret_cast<double2*>(d_state), y,
                                                            h->d_int_of_ref.p, h->d_pair.p, 0, h->nodes, h->N, h->P);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return check_kernel_error(h);
}

void* heom_stream(heom_handle* h) { return h ? (void*)h->stream : nullptr; }
int64_t heom_matrices(const heom_handle* h) { return h ? h->nodes : 0; }
int32_t heom_states(const heom_handle* h) { return h ? h->N : 0; }
int64_t heom_kernel_launches(const heom_handle* h) { return h ? h->launches : 0; }
int32_t heom_instances(const heom_handle* h) { return h ? h->n_inst : 0; }
int64_t heom_instance_matrices(const heom_handle* h, int32_t inst)
{
    return (h && inst >= 0 && inst < h->n_inst) ? h->inst_base[inst + 1] - h->inst_base[inst] : 0;
}
int64_t heom_instance_offset(const heom_handle* h, int32_t inst)
{
    return (h && inst >= 0 && inst < h->n_inst) ? h->inst_base[inst] : -1;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Ensembles: classes of batch handles stepped together.  One RK4 step is one
// CUDA graph: a fork on the ensemble's stream, every class's stage launches on
// the class's own stream (concurrent branches), a join.  The stage grid of
// every class is chosen by timing candidate shapes (ens_autotune).
// ---------------------------------------------------------------------------

struct heom_ensemble {
    heom_options opt{};
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<heom_handle*> cls;
    std::vector<int32_t> cls_of, idx_of; // per instance
    std::vector<int64_t> top_off;        // per instance, doubles into a row of tops
    int64_t row_len = 0;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t step_graph = nullptr;
    double graph_dt = 0.0;
    bool tuned = false;
    bool serial = false; // classes one after another in the step graph (else side by side)
    double tuned_us = 0.0;

    ~heom_ensemble()
    {
        if (stream) cudaStreamSynchronize(stream);
        if (step_graph) cudaGraphExecDestroy(step_graph);
        for (heom_handle* c : cls) heom_destroy(c);
        if (fork) cudaEventDestroy(fork);
        for (cudaEvent_t ev : join) cudaEventDestroy(ev);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// group instances into classes that can share a batch handle (first-fit, in order)
void group_classes(const heom_instance_desc* descs, int32_t count, std::vector<std::vector<int32_t>>& groups)
{
    groups.clear();
    for (int32_t k = 0; k < count; ++k) {
        bool placed = false;
        for (auto& g : groups)
            if (check_same_class(&descs[g[0]], &descs[k]) == 0) {
                g.push_back(k);
                placed = true;
                break;
            }
        if (!placed) groups.push_back({k});
    }
    g_last_error.clear();
}

// the ensemble's classes: every class of group_classes, split for N <= 8 into
// its instances of one depth that are at least kLockstepMin many (a lockstep
// class each) and the rest (one batch handle of mixed depths)
constexpr size_t kLockstepMin = 8;
struct ClassPlan {
    std::vector<int32_t> members;
    bool lockstep = false;
};

std::vector<ClassPlan> plan_classes(const heom_instance_desc* descs, int32_t count, bool lockstep)
{
    std::vector<std::vector<int32_t>> groups;
    group_classes(descs, count, groups);
    std::vector<ClassPlan> plan;
    for (auto& g : groups) {
        if (!lockstep || descs[g[0]].states > 8) {
            plan.push_back({g, false});
            continue;
        }
        std::vector<std::pair<int64_t, std::vector<int32_t>>> by_size;
        for (int32_t k : g) {
            bool placed = false;
            for (auto& b : by_size)
                if (b.first == descs[k].matrices && descs[b.second[0]].ado_depth == descs[k].ado_depth) {
                    b.second.push_back(k);
                    placed = true;
                    break;
                }
            if (!placed) by_size.push_back({descs[k].matrices, {k}});
        }
        std::vector<int32_t> rest;
        for (auto& b : by_size) {
            if (b.second.size() >= kLockstepMin) plan.push_back({b.second, true});
            else rest.insert(rest.end(), b.second.begin(), b.second.end());
        }
        if (!rest.empty()) {
            std::sort(rest.begin(), rest.end());
            plan.push_back({rest, false});
        }
    }
    return plan;
}

// device bytes of one batch handle of these instances
size_t class_footprint(const heom_instance_desc* descs, const std::vector<int32_t>& members, int scheme, bool lockstep)
{
    const heom_instance_desc& d = descs[members[0]];
    int64_t nodes = 0;
    for (int32_t k : members) nodes += descs[k].matrices;
    const int P = heomk::pairs_of(d.states);
    const int W = d.ado_width;
    size_t state = (size_t)nodes * P * 32;
    if (lockstep) // a lockstep class pads to 32 instances
        state = state / members.size() * ((members.size() + 31) / 32 * 32);
    const int buffers = 1 + (scheme == HEOM_RK4_REFERENCE ? 5 : 2);
    const size_t per_ado = (size_t)((2 * W + 3) & ~3) * 4 + ((W + 15) & ~15) + 16 + 8 + (members.size() > 1 ? 4 : 0);
    const size_t nn16 = (size_t)d.states * d.states * 16;
    const size_t xfer = std::min<size_t>((size_t)nodes * nn16, (size_t(64) << 20) + nn16);
    return state * buffers + per_ado * nodes + xfer + members.size() * (nn16 * 3 + 2048);
}

int ens_enqueue_step(heom_ensemble* e, double dt)
{
    CUDA_TRY(cudaEventRecord(e->fork, e->stream));
    cudaEvent_t prev = e->fork;
    for (size_t c = 0; c < e->cls.size(); ++c) {
        heom_handle* h = e->cls[c];
        CUDA_TRY(cudaStreamWaitEvent(h->stream, e->serial ? prev : e->fork, 0));
        if (int rc = enqueue_step(h, dt)) return rc;
        CUDA_TRY(cudaEventRecord(e->join[c], h->stream));
        if (e->serial) prev = e->join[c];
        else CUDA_TRY(cudaStreamWaitEvent(e->stream, e->join[c], 0));
    }
    if (e->serial) CUDA_TRY(cudaStreamWaitEvent(e->stream, prev, 0));
    return 0;
}

void ens_drop_graph(heom_ensemble* e)
{
    if (e->step_graph) {
        cudaGraphExecDestroy(e->step_graph);
        e->step_graph = nullptr;
    }
}

// one stage of every class (stage buffers only) as a graph, for timing
int ens_probe_graph(heom_ensemble* e, cudaGraphExec_t* out)
{
    std::vector<int64_t> saved;
    for (heom_handle* h : e->cls) saved.push_back(h->launches);
    cudaGraph_t graph = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    cudaError_t ce = cudaEventRecord(e->fork, e->stream);
    cudaEvent_t prev = e->fork;
    for (size_t c = 0; c < e->cls.size() && !rc && ce == cudaSuccess; ++c) {
        heom_handle* h = e->cls[c];
        ce = cudaStreamWaitEvent(h->stream, e->serial ? prev : e->fork, 0);
        if (ce == cudaSuccess)
            rc = launch_stage(h, EPI_AXPY_SELF, h->work[0].p, nullptr, h->work[1].p, nullptr,
                              make_double2(1e-30, 0.0), 0);
        if (!rc && ce == cudaSuccess) ce = cudaEventRecord(e->join[c], h->stream);
        if (e->serial) prev = e->join[c];
        else if (!rc && ce == cudaSuccess) ce = cudaStreamWaitEvent(e->stream, e->join[c], 0);
    }
    if (e->serial && !rc && ce == cudaSuccess) ce = cudaStreamWaitEvent(e->stream, prev, 0);
    cudaError_t ce2 = cudaStreamEndCapture(e->stream, &graph);
    for (size_t c = 0; c < e->cls.size(); ++c) e->cls[c]->launches = saved[c];
    if (rc || ce != cudaSuccess || ce2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (rc) return rc;
        return fail(HEOM_E_CUDA, "probe capture failed: %s",
                    cudaGetErrorString(ce != cudaSuccess ? ce : ce2));
    }
    ce = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return fail(HEOM_E_CUDA, "probe instantiate failed: %s", cudaGetErrorString(ce));
    return 0;
}

std::mutex g_tune_mu;
struct TuneEntry {
    std::string sig;
    std::vector<int> blocks;
    bool serial;
    double us;
};
std::vector<TuneEntry> g_tune_cache;

std::string ens_signature(const heom_ensemble* e)
{
    std::string sig;
    for (const heom_handle* h : e->cls) {
        char buf[160];
        snprintf(buf, sizeof buf, "%d:%d:%d:%d:%lld:%d:%d|", h->sm_count, h->N, h->W, h->LS, (long long)h->nodes,
                 h->hkind, h->SLT);
        sig += buf;
    }
    return sig;
}

int ens_autotune(heom_ensemble* e, double* best_us)
{
    const size_t C = e->cls.size();
    std::vector<int> full(C), groups(C);
    std::vector<double> work(C);
    double total = 0.0;
    for (size_t c = 0; c < C; ++c) {
        heom_handle* h = e->cls[c];
        if (int rc = prepare_scheme(h)) return rc;
        h->grid_override = 0;
        const void* fn = nullptr;
        int blocks = 0;
        if (int rc = resolve_stage(h, &fn, &blocks)) return rc;
        full[c] = h->per_sm[0][h->hkind] * h->sm_count;
        groups[c] = blocks;
        // a stage costs about one warp pass per ADO (N <= 8) or per team member
        // (N > 8), whatever the sectors an ADO fills
        work[c] = (double)h->n_active * (h->N <= 8 ? 1 : heomk::team_warps(h->N));
        total += work[c];
    }
    const std::string sig = ens_signature(e);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        for (auto& entry : g_tune_cache)
            if (entry.sig == sig) {
                for (size_t c = 0; c < C; ++c) e->cls[c]->grid_override = entry.blocks[c];
                e->serial = entry.serial;
                e->tuned_us = entry.us;
                e->tuned = true;
                ens_drop_graph(e);
                if (best_us) *best_us = e->tuned_us;
                return 0;
            }
    }
    // candidates: every class a full wave; shares of one wave in proportion to
    // the class's bytes (classes run side by side), scaled by 1/2, 1, 2
    std::vector<std::vector<int>> cand;
    cand.push_back(full);
    std::vector<int> half(C);
    for (size_t c = 0; c < C; ++c) half[c] = std::max(1, full[c] / 2);
    cand.push_back(half);
    for (double f : {0.5, 1.0, 2.0}) {
        std::vector<int> v(C);
        for (size_t c = 0; c < C; ++c) v[c] = std::max(1, (int)std::ceil(f * full[c] * work[c] / total));
        cand.push_back(v);
    }
    // identical launch shapes (after the cap at one block per ADO group) are timed once
    for (auto& v : cand)
        for (size_t c = 0; c < C; ++c) v[c] = std::min(v[c], std::max(groups[c], 1));
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    // every shape side by side; with more than one class also the full waves one class after another
    // (a class of large instances fills the device alone; side by side they share L2)
    std::vector<std::pair<std::vector<int>, bool>> shapes;
    for (auto& v : cand) shapes.push_back({v, false});
    if (C > 1) {
        std::vector<int> fullc = full;
        for (size_t c = 0; c < C; ++c) fullc[c] = std::min(fullc[c], std::max(groups[c], 1));
        shapes.push_back({fullc, true});
    }

    cudaEvent_t t0 = nullptr, t1 = nullptr;
    CUDA_TRY(cudaEventCreate(&t0));
    CUDA_TRY(cudaEventCreate(&t1));
    double best = 1e300;
    size_t pick = 0;
    int rc = 0;
    for (size_t q = 0; q < shapes.size() && !rc; ++q) {
        for (size_t c = 0; c < C; ++c) e->cls[c]->grid_override = shapes[q].first[c];
        e->serial = shapes[q].second;
        cudaGraphExec_t g = nullptr;
        if ((rc = ens_probe_graph(e, &g))) break;
        const int warm = 2, reps = 5;
        cudaError_t ce = cudaSuccess;
        for (int r = 0; r < warm && ce == cudaSuccess; ++r) ce = cudaGraphLaunch(g, e->stream);
        if (ce == cudaSuccess) ce = cudaEventRecord(t0, e->stream);
        for (int r = 0; r < reps && ce == cudaSuccess; ++r) ce = cudaGraphLaunch(g, e->stream);
        if (ce == cudaSuccess) ce = cudaEventRecord(t1, e->stream);
        if (ce == cudaSuccess) ce = cudaEventSynchronize(t1);
        float ms = 0.0f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, t0, t1);
        cudaGraphExecDestroy(g);
        if (ce != cudaSuccess) {
            rc = fail(HEOM_E_CUDA, "autotune timing failed: %s", cudaGetErrorString(ce));
            break;
        }
        for (heom_handle* h : e->cls) h->launches += warm + reps;
        const double us = 1e3 * ms / reps;
        if (us < best) {
            best = us;
            pick = q;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return rc;
    for (heom_handle* h : e->cls)
        if (int rc2 = check_kernel_error(h)) return rc2;
    for (size_t c = 0; c < C; ++c) e->cls[c]->grid_override = shapes[pick].first[c];
    e->serial = shapes[pick].second;
    e->tuned = true;
    e->tuned_us = best;
    ens_drop_graph(e);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache.push_back({sig, shapes[pick].first, shapes[pick].second, best});
    }
    if (best_us) *best_us = best;
    return 0;
}

int ens_run_steps(heom_ensemble* e, double dt, int64_t steps)
{
    if (steps <= 0) return 0;
    if (!e->tuned)
        if (int rc = ens_autotune(e, nullptr)) return rc;
    for (heom_handle* h : e->cls) {
        if (int rc = prepare_scheme(h)) return rc;
        const void* fn = nullptr;
        if (int rc = resolve_stage(h, &fn)) return rc;
        if (h->stage_smem == 0) return fail(HEOM_E_CUDA, "stage kernel shape unresolved");
    }
    if (!e->opt.use_graphs) {
        for (int64_t s = 0; s < steps; ++s)
            if (int rc = ens_enqueue_step(e, dt)) return rc;
        return 0;
    }
    if (e->step_graph && e->graph_dt != dt) ens_drop_graph(e);
    if (!e->step_graph) {
        std::vector<int64_t> saved;
        for (heom_handle* h : e->cls) saved.push_back(h->launches);
        cudaGraph_t graph = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        int rc = ens_enqueue_step(e, dt);
        cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
        for (size_t c = 0; c < e->cls.size(); ++c) e->cls[c]->launches = saved[c];
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return fail(HEOM_E_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&e->step_graph, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return fail(HEOM_E_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce));
        e->graph_dt = dt;
    }
    for (int64_t s = 0; s < steps; ++s) {
        CUDA_TRY(cudaGraphLaunch(e->step_graph, e->stream));
        for (heom_handle* h : e->cls) h->launches += launches_per_step(h);
    }
    return 0;
}

int ens_check(heom_ensemble* e, int32_t inst, heom_handle** h, int32_t* idx)
{
    if (!e) return fail(HEOM_E_ARG, "NULL ensemble");
    if (inst < 0 || inst >= (int32_t)e->cls_of.size()) return fail(HEOM_E_ARG, "instance %d out of range", inst);
    *h = e->cls[e->cls_of[inst]];
    *idx = e->idx_of[inst];
    return 0;
}

} // namespace

extern "C" {

int heom_ensemble_footprint(const heom_instance_desc* descs, int32_t count, const heom_options* opt, size_t* bytes)
{
    if (!descs || count < 1 || !bytes) return fail(HEOM_E_ARG, "bad argument");
    for (int32_t k = 0; k < count; ++k)
        if (int rc = check_desc(&descs[k])) return fail(rc, "instance %d: %s", k, g_last_error.c_str());
    heom_options o;
    heom_default_options(&o);
    if (opt) o = *opt;
    size_t total = 0;
    for (auto& c : plan_classes(descs, count, o.rk4_scheme == HEOM_RK4_PRODUCT || o.rk4_scheme == HEOM_RK4_HORNER))
        total += class_footprint(descs, c.members, o.rk4_scheme, c.lockstep);
    *bytes = total;
    return 0;
}

int heom_ensemble_create(const heom_instance_desc* descs, int32_t count, const heom_options* opt, heom_ensemble** out)
{
    if (!out) return fail(HEOM_E_ARG, "out is NULL");
    *out = nullptr;
    size_t need = 0;
    if (int rc = heom_ensemble_footprint(descs, count, opt, &need)) return rc;
    std::unique_ptr<heom_ensemble> e(new heom_ensemble());
    heom_default_options(&e->opt);
    if (opt) e->opt = *opt;
    e->device = e->opt.device;
    CUDA_TRY(cudaSetDevice(e->device));
    size_t free_b = 0, total_b = 0;
    CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    if (need > free_b)
        return fail(HEOM_E_NOMEM, "ensemble needs %.3f GB of device memory, %.3f GB are free", need / 1e9,
                    free_b / 1e9);
    CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
    const std::vector<ClassPlan> plan =
        plan_classes(descs, count, e->opt.rk4_scheme == HEOM_RK4_PRODUCT || e->opt.rk4_scheme == HEOM_RK4_HORNER);
    e->cls_of.assign(count, 0);
    e->idx_of.assign(count, 0);
    for (size_t c = 0; c < plan.size(); ++c) {
        const std::vector<int32_t>& g = plan[c].members;
        std::vector<heom_instance_desc> members;
        for (size_t i = 0; i < g.size(); ++i) {
            members.push_back(descs[g[i]]);
            e->cls_of[g[i]] = (int32_t)c;
            e->idx_of[g[i]] = (int32_t)i;
        }
        heom_handle* h = nullptr;
        if (int rc = heom_create_batch(members.data(), (int32_t)members.size(), &e->opt, &h))
            return fail(rc, "class %zu: %s", c, g_last_error.c_str());
        // instances of one hierarchy graph: the lockstep layout when its kernel applies
        if (plan[c].lockstep && make_lockstep(h) != 0) g_last_error.clear();
        e->cls.push_back(h);
        cudaEvent_t ev = nullptr;
        CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        e->join.push_back(ev);
    }
    e->top_off.assign(count, 0);
    for (int32_t k = 0; k < count; ++k) {
        e->top_off[k] = e->row_len;
        e->row_len += (int64_t)2 * descs[k].states * descs[k].states;
    }
    *out = e.release();
    return 0;
}

int heom_ensemble_destroy(heom_ensemble* e)
{
    if (!e) return 0;
    cudaSetDevice(e->device);
    delete e;
    return 0;
}

int32_t heom_ensemble_instances(const heom_ensemble* e) { return e ? (int32_t)e->cls_of.size() : 0; }
int32_t heom_ensemble_classes(const heom_ensemble* e) { return e ? (int32_t)e->cls.size() : 0; }

int heom_ensemble_locate(const heom_ensemble* e, int32_t inst, int32_t* cls, int32_t* index)
{
    if (!e || inst < 0 || inst >= (int32_t)e->cls_of.size()) return fail(HEOM_E_ARG, "instance out of range");
    if (cls) *cls = e->cls_of[inst];
    if (index) *index = e->idx_of[inst];
    return 0;
}

heom_handle* heom_ensemble_class(heom_ensemble* e, int32_t cls)
{
    return (e && cls >= 0 && cls < (int32_t)e->cls.size()) ? e->cls[cls] : nullptr;
}

int heom_ensemble_set_hamiltonian(heom_ensemble* e, int32_t inst, const double* ham)
{
    heom_handle* h = nullptr;
    int32_t idx = 0;
    if (int rc = ens_check(e, inst, &h, &idx)) return rc;
    CUDA_TRY(cudaSetDevice(e->device));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    const int old_kind = h->hkind;
    if (int rc = heom_set_instance_hamiltonian(h, idx, ham)) return rc;
    ens_drop_graph(e);
    if (h->hkind != old_kind) e->tuned = false; // another kernel variant: shapes are re-timed
    return 0;
}

int heom_ensemble_clear(heom_ensemble* e)
{
    if (!e) return fail(HEOM_E_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(e->device));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (heom_handle* h : e->cls) {
        CUDA_TRY(cudaMemsetAsync(h->y.data.p, 0, h->state_elems() * sizeof(double2), h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    return 0;
}

int heom_ensemble_set_top(heom_ensemble* e, int32_t inst, const double* top)
{
    heom_handle* h = nullptr;
    int32_t idx = 0;
    if (int rc = ens_check(e, inst, &h, &idx)) return rc;
    CUDA_TRY(cudaSetDevice(e->device));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return heom_set_instance_top(h, idx, top);
}

int heom_ensemble_get_top(heom_ensemble* e, int32_t inst, double* top)
{
    heom_handle* h = nullptr;
    int32_t idx = 0;
    if (int rc = ens_check(e, inst, &h, &idx)) return rc;
    CUDA_TRY(cudaSetDevice(e->device));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return heom_get_instance_top(h, idx, top);
}

int heom_ensemble_autotune(heom_ensemble* e, double* best_stage_us)
{
    if (!e) return fail(HEOM_E_ARG, "NULL ensemble");
    CUDA_TRY(cudaSetDevice(e->device));
    return ens_autotune(e, best_stage_us);
}

int heom_ensemble_rk4_steps(heom_ensemble* e, double dt, int64_t steps)
{
    if (!e || steps < 0 || !(dt > 0.0)) return fail(HEOM_E_ARG, "bad argument");
    CUDA_TRY(cudaSetDevice(e->device));
    if (int rc = ens_run_steps(e, dt, steps)) return rc;
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (heom_handle* h : e->cls)
        if (int rc = check_kernel_error(h)) return rc;
    return 0;
}

int heom_ensemble_propagate(heom_ensemble* e, double dt, int64_t steps, int64_t observe_every, double* host_tops)
{
    if (!e || !host_tops || steps < 0 || observe_every <= 0 || steps % observe_every != 0 || !(dt > 0.0))
        return fail(HEOM_E_ARG, "bad argument (steps must be a multiple of observe_every)");
    CUDA_TRY(cudaSetDevice(e->device));
    const int64_t rows = steps / observe_every + 1;
    for (heom_handle* h : e->cls) {
        const int64_t nn = (int64_t)h->N * h->N * h->n_inst;
        if ((int64_t)h->toplog.n < rows * nn)
            if (int rc = h->toplog.alloc(rows * nn)) return rc;
        CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    auto record = [&](int64_t row) -> int {
        for (heom_handle* h : e->cls) {
            heomk::heom_record_top<<<h->n_inst, 128, 0, e->stream>>>(h->toplog.p, h->y.data.p, h->d_pair.p,
                                                                     h->d_top.p, h->N, h->P, row, h->kp, 0);
            h->launches++;
            CUDA_TRY(cudaGetLastError());
        }
        return 0;
    };
    if (int rc = record(0)) return rc;
    for (int64_t r = 1; r < rows; ++r) {
        if (int rc = ens_run_steps(e, dt, observe_every)) return rc;
        if (int rc = record(r)) return rc;
    }
    // gather every class's log, then scatter into instance order
    std::vector<std::vector<double>> logs(e->cls.size());
    for (size_t c = 0; c < e->cls.size(); ++c) {
        heom_handle* h = e->cls[c];
        logs[c].resize((size_t)rows * h->n_inst * h->N * h->N * 2);
        CUDA_TRY(cudaMemcpyAsync(logs[c].data(), h->toplog.p, logs[c].size() * 8, cudaMemcpyDeviceToHost, e->stream));
    }
    // failure detection: a non-finite state is reported instead of returned silently
    for (heom_handle* h : e->cls) {
        CUDA_TRY(cudaMemsetAsync(h->d_flag.p, 0, sizeof(int), e->stream));
        heomk::heom_check_finite<<<h->sm_count * 4, 256, 0, e->stream>>>(
            reinterpret_cast<const double*>(h->y.data.p), (int64_t)h->state_elems() * 2, h->d_flag.p);
        h->launches++;
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (int32_t k = 0; k < (int32_t)e->cls_of.size(); ++k) {
        const heom_handle* h = e->cls[e->cls_of[k]];
        const int64_t nn2 = (int64_t)h->N * h->N * 2;
        for (int64_t r = 0; r < rows; ++r)
            std::memcpy(host_tops + r * e->row_len + e->top_off[k],
                        logs[e->cls_of[k]].data() + (r * h->n_inst + e->idx_of[k]) * nn2, nn2 * 8);
    }
    for (heom_handle* h : e->cls) {
        if (int rc = check_kernel_error(h)) return rc;
        int flag = 0;
        CUDA_TRY(cudaMemcpy(&flag, h->d_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (flag) return fail(HEOM_E_NONFINITE, "non-finite value in the hierarchy state after propagation");
    }
    return 0;
}

int64_t heom_ensemble_top_row_len(const heom_ensemble* e) { return e ? e->row_len : 0; }
int64_t heom_ensemble_top_offset(const heom_ensemble* e, int32_t inst)
{
    return (e && inst >= 0 && inst < (int32_t)e->top_off.size()) ? e->top_off[inst] : -1;
}

int64_t heom_ensemble_kernel_launches(const heom_ensemble* e)
{
    int64_t n = 0;
    if (e)
        for (const heom_handle* h : e->cls) n += h->launches;
    return n;
}

void* heom_ensemble_stream(heom_ensemble* e) { return e ? (void*)e->stream : nullptr; }

} // extern "C"

// ---------------------------------------------------------------------------
// Adjoint gradients of J = sum_n w_n Re(sum_ij conj(O_ij) rho_n(i,j)) over an
// RK4 propagation (the product form: y_{n+1} = F_3 F_2 F_1 F_0 y_n with
// F_k = I + beta_k dt L).  The adjoint g_n = dJ/dy_n obeys
// g_n = w_n O_top + F_0^H F_1^H F_2^H F_3^H g_{n+1}, F_k^H = I + conj(beta_k) dt L^H,
// and every factor adds Re(beta_k dt <a_k, dL/dtheta w_k>) to dJ/dtheta (a_k
// the adjoint after F_k^H's successors, w_k the forward stage input).
// Checkpoints every S = ceil(sqrt(steps)) steps; each segment's stage inputs
// are recomputed (same kernels, bit-identical) before its backward sweep.
// When those ceil(steps/S) + 4S + 3 states exceed the memory limit, the sweep
// reverses the steps by recursive checkpointing in the slots that fit
// (lean_reverse): same kernels, same backward order, bit-identical results.
// ---------------------------------------------------------------------------

struct heom_adjoint {
    heom_handle* h = nullptr;
    AdjTabs tabs{};
    DevBuf<double2> pss_adj, g0_adj;
    DevBuf<double> hfrag_adj;
    DevBuf<double> dpss;       // [nodes] d pf_same_sum / d gamma (internal order)
    DevBuf<double2> dg0;       // [2][N*N]
    DevBuf<double> dchat;      // [2][W]
    DevBuf<double2> dkhat;     // [2][3][W]
    DevBuf<double2> obs;       // [K][N*N]
    DevBuf<double2> partial;   // [grid][N*N + 2]
    DevBuf<int64_t> inst_base; // [K + 1]
    int grid = 0, bpi = 0;     // blocks of the gradient kernel, per instance
    size_t grad_smem = 0;
    DevBuf<double2> cps, seg, scratch, ga, gb, toplog;
    int64_t cap_cps = 0, cap_seg = 0, cap_rows = 0;
    int64_t mem_limit = 0;     // bytes for the sweep's states (0: free device memory)
    int64_t rec_slots = 0;     // recursive-checkpointing slots of the last sweep (0: sqrt layout)
    int want_h = 1, want_bath = 1; // gradients the sweep accumulates (from the output pointers)
    DevBuf<double> d_w;        // loss weights [steps + 1]
    DevBuf<int64_t> d_base;    // step offset of the segment being run (read by the captured kernels)
    int64_t cap_w = 0;
    // captured graphs per segment length: [0] forward with tops, [1] stage-input recompute, [2] backward
    struct Graphs {
        int64_t len = 0;
        cudaGraphExec_t g[3] = {nullptr, nullptr, nullptr};
    };
    std::vector<Graphs> graphs;
    double graph_dt = 0.0;
    void drop_graphs()
    {
        for (auto& e : graphs)
            for (auto& x : e.g)
                if (x) cudaGraphExecDestroy(x);
        graphs.clear();
    }
    ~heom_adjoint()
    {
        drop_graphs();
        if (h) heom_destroy(h);
    }
};

namespace {

// L^H tables of every instance and the derivative tables (shared bath tables)
int adj_tables(heom_adjoint* A, const heomhost::system_params& sp)
{
    heom_handle* h = A->h;
    const int N = h->N, W = h->W, M = h->M, K = h->n_inst;
    // L^H: conj(pf_same_sum), conj(gamma0), -H^H
    std::vector<double2> pss(h->nodes);
    for (int64_t r = 0; r < h->nodes; ++r)
        pss[h->int_of_ref[r]] = make_double2(h->pss[2 * r], -h->pss[2 * r + 1]);
    std::vector<double2> g0 = gamma0_table(h, h->pf_same);
    for (auto& v : g0) v.y = -v.y;
    std::vector<double2> hs((size_t)N * N);
    const size_t fd = heomk::frag_doubles(N);
    std::vector<double> frag((size_t)K * fd, 0.0), hadj(2 * N * N);
    for (int k = 0; k < K; ++k) {
        const double* hk = h->ham.data() + (size_t)k * 2 * N * N;
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) {
                hadj[2 * (i * N + j)] = -hk[2 * (j * N + i)];
                hadj[2 * (i * N + j) + 1] = hk[2 * (j * N + i) + 1];
            }
        h_tables(hadj.data(), N, hs.data(), frag.data() + (size_t)k * fd);
    }
    if (int rc = A->pss_adj.alloc(pss.size())) return rc;
    if (int rc = A->g0_adj.alloc(g0.size())) return rc;
    if (int rc = A->hfrag_adj.alloc(frag.size())) return rc;
    CUDA_TRY(cudaMemcpy(A->pss_adj.p, pss.data(), pss.size() * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(A->g0_adj.p, g0.data(), g0.size() * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(A->hfrag_adj.p, frag.data(), frag.size() * 8, cudaMemcpyHostToDevice));
    A->tabs = AdjTabs{A->pss_adj.p, A->g0_adj.p, A->hfrag_adj.p};

    // derivative tables for theta = lambda (0), gamma (1)
    heomhost::bath_derivs bd = heomhost::bath_derivatives(sp);
    std::vector<double> dchat(2 * W, 0.0), dpss(h->nodes, 0.0);
    std::vector<double2> dkhat(2 * 3 * W, make_double2(0.0, 0.0)), dg0(2 * N * N);
    for (int th = 0; th < 2; ++th) {
        for (int sl = 0; sl < W; ++sl) {
            const int b = sl / M, m = sl - b * M;
            const double cr = h->cbk[2 * sl], ci = h->cbk[2 * sl + 1];
            const double dcr = bd.cbk[th][2 * sl], dci = bd.cbk[th][2 * sl + 1];
            const double qr = m == 0 ? h->pf_circ[2 * b] : 0.0, qi = m == 0 ? h->pf_circ[2 * b + 1] : 0.0;
            const double dqr = m == 0 ? bd.pf_circ[th][2 * b] : 0.0, dqi = m == 0 ? bd.pf_circ[th][2 * b + 1] : 0.0;
            const double a = std::hypot(cr, ci), da = (cr * dcr + ci * dci) / a;
            const double chat = std::sqrt(a / kHbar);
            dchat[th * W + sl] = da / (2.0 * kHbar * chat);
            const double sc = std::sqrt(kHbar / a), dsc = -0.5 * sc * da / a;
            dkhat[th * 3 * W + sl] = make_double2(dsc * (-ci / kHbar + qr) + sc * (-dci / kHbar + dqr),
                                                  dsc * (cr / kHbar + qi) + sc * (dcr / kHbar + dqi));
            dkhat[th * 3 * W + W + sl] = make_double2(dsc * (ci / kHbar + qr) + sc * (dci / kHbar + dqr),
                                                      dsc * (-cr / kHbar + qi) + sc * (-dcr / kHbar + dqi));
            dkhat[th * 3 * W + 2 * W + sl] = make_double2(2.0 * (dsc * qr + sc * dqr), 2.0 * (dsc * qi + sc * dqi));
        }
        const std::vector<double2> g = gamma0_table(h, bd.pf_same[th]);
        std::copy(g.begin(), g.end(), dg0.begin() + th * N * N);
    }
    for (int64_t r = 0; r < h->nodes; ++r) {
        double v = 0.0;
        for (int b = 0; b < h->B; ++b) v -= h->tuples[r * W + b * M];
        dpss[h->int_of_ref[r]] = v;
    }
    if (int rc = A->dchat.alloc(dchat.size())) return rc;
    if (int rc = A->dkhat.alloc(dkhat.size())) return rc;
    if (int rc = A->dg0.alloc(dg0.size())) return rc;
    if (int rc = A->dpss.alloc(dpss.size())) return rc;
    CUDA_TRY(cudaMemcpy(A->dchat.p, dchat.data(), dchat.size() * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(A->dkhat.p, dkhat.data(), dkhat.size() * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(A->dg0.p, dg0.data(), dg0.size() * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(A->dpss.p, dpss.data(), dpss.size() * 8, cudaMemcpyHostToDevice));
    return 0;
}

int adj_grad(heom_adjoint* A, const double2* a, const double2* w, double2 weight)
{
    heom_handle* h = A->h;
    heomk::GradParams g{};
    g.a = a;
    g.w = w;
    g.nbr = h->d_nbr.p;
    g.tup = h->d_tup.p;
    g.pe = h->d_pair.p;
    g.slots = h->d_slots.p;
    g.dpss = A->dpss.p;
    g.dg0 = A->dg0.p;
    g.dchat = A->dchat.p;
    g.dkhat = A->dkhat.p;
    g.sq = h->d_sq.p;
    g.weight = weight;
    g.partial = A->partial.p;
    g.inst_base = A->inst_base.p;
    g.blocks_per_inst = A->bpi;
    g.N = h->N;
    g.P = h->P;
    g.W = h->W;
    g.NW = h->NW;
    g.TWB = h->TWB;
    g.SL = h->SL;
    g.want_h = A->want_h;
    g.want_bath = A->want_bath;
    heomk::heom_adjoint_grad<<<A->grid, heomk::kCtaWarps * 32, A->grad_smem, h->stream>>>(g);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    return 0;
}

// y += weights[*base + j] O at every instance's top
int adj_add_top(heom_adjoint* A, double2* y, int64_t j)
{
    heom_handle* h = A->h;
    heomk::heom_add_top<<<h->n_inst, 128, 0, h->stream>>>(y, A->obs.p, h->d_pair.p, h->d_top.p, h->N, h->P,
                                                          A->d_w.p, A->d_base.p, j);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    return 0;
}

// One segment of `len` steps from y (the forward sweep): every step one RK4
// step and the tops recorded into rows *base + j + 1.
int adj_seg_forward(heom_adjoint* A, double dt, int64_t len)
{
    heom_handle* h = A->h;
    for (int64_t j = 0; j < len; ++j) {
        if (int rc = enqueue_step(h, dt)) return rc;
        heomk::heom_record_top_at<<<h->n_inst, 128, 0, h->stream>>>(A->toplog.p, h->y.data.p, h->d_pair.p,
                                                                    h->d_top.p, h->N, h->P, A->d_base.p, j + 1);
        h->launches++;
        CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

// stage inputs w_k of every step of a segment, from seg[0] (its checkpoint)
int adj_seg_recompute(heom_adjoint* A, double dt, int64_t len)
{
    heom_handle* h = A->h;
    const size_t st = h->state_elems();
    for (int64_t j = 0; j < len; ++j)
        for (int k = 0; k < 4; ++k) {
            const double2* in = A->seg.p + (4 * j + k) * st;
            double2* o = k < 3 ? A->seg.p + (4 * j + k + 1) * st
                               : (j + 1 < len ? A->seg.p + 4 * (j + 1) * st : A->scratch.p);
            const double2 beta = make_double2(dt * kProdBeta[k][0], dt * kProdBeta[k][1]);
            if (int rc = launch_stage(h, EPI_AXPY_SELF, in, nullptr, o, nullptr, beta, 0)) return rc;
        }
    return 0;
}

// backward through a segment: four factors per step (gradient contributions,
// then F_k^H), then the step's loss weight; the adjoint ends in ga (4 swaps a step)
int adj_seg_backward(heom_adjoint* A, double dt, int64_t len)
{
    heom_handle* h = A->h;
    const size_t st = h->state_elems();
    double2* gcur = A->ga.p;
    double2* gnxt = A->gb.p;
    for (int64_t j = len - 1; j >= 0; --j) {
        for (int k = 3; k >= 0; --k) {
            const double2 beta = make_double2(dt * kProdBeta[k][0], dt * kProdBeta[k][1]);
            if (int rc = adj_grad(A, gcur, A->seg.p + (4 * j + k) * st, beta)) return rc;
            const double2 cbeta = make_double2(beta.x, -beta.y);
            if (int rc = launch_stage(h, EPI_AXPY_SELF, gcur, nullptr, gnxt, nullptr, cbeta, 0, &A->tabs)) return rc;
            std::swap(gcur, gnxt);
        }
        if (int rc = adj_add_top(A, gcur, j)) return rc;
    }
    return 0;
}

// run part `which` (0 forward, 1 recompute, 2 backward) of a segment, through
// a graph captured once per segment length when the handle uses graphs
int adj_run(heom_adjoint* A, int which, double dt, int64_t len)
{
    heom_handle* h = A->h;
    auto direct = [&]() -> int {
        return which == 0 ? adj_seg_forward(A, dt, len) : which == 1 ? adj_seg_recompute(A, dt, len)
                                                                       : adj_seg_backward(A, dt, len);
    };
    if (!h->opt.use_graphs) return direct();
    if (A->graph_dt != dt) {
        A->drop_graphs();
        A->graph_dt = dt;
    }
    heom_adjoint::Graphs* e = nullptr;
    for (auto& x : A->graphs)
        if (x.len == len) e = &x;
    if (!e) {
        A->graphs.push_back(heom_adjoint::Graphs());
        e = &A->graphs.back();
        e->len = len;
    }
    if (!e->g[which]) {
        const int64_t saved = h->launches;
        cudaGraph_t graph = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = direct();
        cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
        h->launches = saved;
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return fail(HEOM_E_CUDA, "adjoint graph capture failed: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&e->g[which], graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return fail(HEOM_E_CUDA, "adjoint graph instantiate failed: %s", cudaGetErrorString(ce));
    }
    CUDA_TRY(cudaGraphLaunch(e->g[which], h->stream));
    h->launches += which == 0 ? len * (launches_per_step(h) + 1) : which == 1 ? 4 * len : 9 * len;
    return 0;
}

// Splits of the recursive reversal.  To reverse l steps from a stored state
// with s free slots: advance m steps, store, reverse the last l - m steps with
// s - 1 slots, then the first m with s.  The forward steps this costs obey
// cost(l, s) = min_m [m + cost(l - m, s - 1) + cost(m, s)], cost(1, s) = 0,
// cost(l, 0) = l (l - 1) / 2 (every state recomputed from the stored one);
// solved exactly while s * l^2 stays small, else by the binomial rule (with
// r the least integer with C(s + r, s) >= l: m = l - C(s - 1 + r, s - 1)).
struct RevPlan {
    int64_t T = 0, S = 0;
    bool exact = false;
    std::vector<int32_t> best; // [s][l] optimal m (exact plan)

    void build(int64_t steps, int64_t slots)
    {
        T = steps;
        S = slots;
        exact = (double)S * T * T <= 1e8;
        if (!exact) return;
        std::vector<int64_t> prev(T + 1), cur(T + 1);
        best.assign((size_t)(S + 1) * (T + 1), 1);
        for (int64_t l = 1; l <= T; ++l) prev[l] = l * (l - 1) / 2;
        for (int64_t sl = 1; sl <= S; ++sl) {
            cur[1] = 0;
            for (int64_t l = 2; l <= T; ++l) {
                int64_t bc = INT64_MAX, bm = 1;
                for (int64_t m = 1; m < l; ++m) {
                    const int64_t c = m + prev[l - m] + cur[m];
                    if (c < bc) { bc = c; bm = m; }
                }
                cur[l] = bc;
                best[(size_t)sl * (T + 1) + l] = (int32_t)bm;
            }
            std::swap(prev, cur);
        }
    }
    int64_t split(int64_t l, int64_t s) const
    {
        if (exact) return best[(size_t)s * (T + 1) + l];
        auto binom = [](int64_t n, int64_t k) { // C(n, k), saturating
            long double v = 1.0L;
            for (int64_t q = 1; q <= k; ++q) v = v * (n - k + q) / q;
            return v > 9e18L ? INT64_MAX : (int64_t)(v + 0.5L);
        };
        int64_t r = 0;
        while (binom(s + r, s) < l) ++r;
        return std::max<int64_t>(1, std::min<int64_t>(l - 1, l - binom(s - 1 + r, s - 1)));
    }
};

// recursive reversal: device-side step offsets come from `bases` (bases[j] = j)
struct LeanRun {
    heom_adjoint* A;
    double dt;
    const RevPlan* plan;
    const int64_t* bases;
    size_t st;

    int set_base(int64_t j)
    {
        CUDA_TRY(cudaMemcpyAsync(A->d_base.p, bases + j, 8, cudaMemcpyHostToDevice, A->h->stream));
        return 0;
    }
    // y <- slot, then `len` steps from step a with their tops recorded
    int advance(int64_t sl, int64_t a, int64_t len)
    {
        heom_handle* h = A->h;
        CUDA_TRY(cudaMemcpyAsync(h->y.data.p, A->cps.p + sl * st, st * 16, cudaMemcpyDeviceToDevice, h->stream));
        if (len == 0) return 0;
        if (int rc = set_base(a)) return rc;
        return adj_seg_forward(A, dt, len);
    }
    // backward through step j from its state src: stage inputs, the top of
    // state j + 1 (row j + 1), then the four adjoint factors and the weight of step j
    int step_back(const double2* src, int64_t j)
    {
        heom_handle* h = A->h;
        CUDA_TRY(cudaMemcpyAsync(A->seg.p, src, st * 16, cudaMemcpyDeviceToDevice, h->stream));
        if (int rc = set_base(j)) return rc;
        if (int rc = adj_seg_recompute(A, dt, 1)) return rc;
        heomk::heom_record_top_at<<<h->n_inst, 128, 0, h->stream>>>(A->toplog.p, A->scratch.p, h->d_pair.p,
                                                                    h->d_top.p, h->N, h->P, A->d_base.p, 1);
        h->launches++;
        CUDA_TRY(cudaGetLastError());
        return adj_seg_backward(A, dt, 1);
    }
    // reverse steps [a, b) with state a in slot sl and `free` slots above it unused
    int reverse(int64_t a, int64_t b, int64_t sl, int64_t free)
    {
        const int64_t l = b - a;
        if (l == 1) return step_back(A->cps.p + sl * st, a);
        if (free == 0) {
            for (int64_t j = b - 1; j > a; --j) {
                if (int rc = advance(sl, a, j - a)) return rc;
                if (int rc = step_back(A->h->y.data.p, j)) return rc;
            }
            return step_back(A->cps.p + sl * st, a);
        }
        const int64_t m = a + plan->split(l, free);
        if (int rc = advance(sl, a, m - a)) return rc;
        CUDA_TRY(cudaMemcpyAsync(A->cps.p + (sl + 1) * st, A->h->y.data.p, st * 16, cudaMemcpyDeviceToDevice,
                                 A->h->stream));
        if (int rc = reverse(m, b, sl + 1, free - 1)) return rc;
        return reverse(a, m, sl, free);
    }
};

} // namespace

extern "C" {

int heom_adjoint_create(const heom_system_desc* sys, const heom_options* opt, heom_adjoint** out)
{
    return heom_adjoint_create_batch(sys, 1, opt, out);
}

int heom_adjoint_create_batch(const heom_system_desc* systems, int32_t count, const heom_options* opt,
                              heom_adjoint** out)
{
    if (!systems || !out || count < 1) return fail(HEOM_E_ARG, "NULL argument or count < 1");
    *out = nullptr;
    std::unique_ptr<heom_adjoint> A(new heom_adjoint());
    std::vector<heomhost::system_params> sp(count);
    std::vector<heomhost::instance> inst(count);
    try {
        for (int k = 0; k < count; ++k) {
            sp[k] = heomhost::system_from_desc(systems[k]);
            inst[k] = heomhost::make_instance(sp[k]);
        }
    } catch (const heomhost::config_error& e) {
        return fail(HEOM_E_CONFIG, "%s", e.what());
    } catch (const std::exception& e) {
        return fail(HEOM_E_ARG, "%s", e.what());
    }
    heom_options o;
    heom_default_options(&o);
    if (opt) o = *opt;
    o.rk4_scheme = HEOM_RK4_PRODUCT; // the backward sweep differentiates the product form
    std::vector<heom_instance_desc> d(count);
    for (int k = 0; k < count; ++k) d[k] = inst[k].desc();
    if (int rc = heom_create_batch(d.data(), count, &o, &A->h)) return rc;
    heom_handle* h = A->h;
    CUDA_TRY(cudaSetDevice(h->device));
    if (int rc = adj_tables(A.get(), sp[0])) return rc;
    if (int rc = A->obs.alloc((size_t)count * h->N * h->N)) return rc;
    // gradient kernel: every instance gets the same number of blocks, about two waves in all
    int64_t max_nodes = 1;
    for (int k = 0; k < count; ++k) max_nodes = std::max(max_nodes, h->inst_base[k + 1] - h->inst_base[k]);
    A->bpi = (int)std::max<int64_t>(1, std::min<int64_t>((max_nodes + heomk::kCtaWarps - 1) / heomk::kCtaWarps,
                                                        (2 * (int64_t)h->sm_count + count - 1) / count));
    A->grid = A->bpi * count;
    if (int rc = A->partial.alloc((size_t)A->grid * (h->N * h->N + 2))) return rc;
    if (int rc = A->inst_base.alloc(count + 1)) return rc;
    CUDA_TRY(cudaMemcpy(A->inst_base.p, h->inst_base.data(), (count + 1) * 8, cudaMemcpyHostToDevice));
    A->grad_smem = heomk::grad_smem_bytes(h->N);
    if (int rc = allow_dynamic_smem((const void*)heomk::heom_adjoint_grad, A->grad_smem)) return rc;
    *out = A.release();
    return 0;
}

int heom_adjoint_destroy(heom_adjoint* A)
{
    if (!A) return 0;
    cudaSetDevice(A->h ? A->h->device : 0);
    delete A;
    return 0;
}

heom_handle* heom_adjoint_handle(heom_adjoint* A) { return A ? A->h : nullptr; }
int32_t heom_adjoint_instances(const heom_adjoint* A) { return A && A->h ? A->h->n_inst : 0; }

int heom_adjoint_gradient(heom_adjoint* A, const double* rho0, const double* observable, const double* weights,
                          double dt, int64_t steps, double* loss, double* grad_h, double* grad_lambda,
                          double* grad_gamma, double* grad_rho0)
{
    if (!A || !rho0 || !observable || !weights || steps < 1 || !(dt > 0.0))
        return fail(HEOM_E_ARG, "bad argument");
    heom_handle* h = A->h;
    CUDA_TRY(cudaSetDevice(h->device));
    const int N = h->N, NN = N * N, K = h->n_inst;
    const size_t st = h->state_elems();
    int64_t S = std::max<int64_t>(1, (int64_t)std::ceil(std::sqrt((double)steps)));
    int64_t ncp = (steps + S - 1) / S;
    // device memory: the sqrt layout (checkpoints, stage inputs of one segment)
    // or, when it does not fit, recursive checkpointing in the slots that do;
    // plus the adjoint ping-pong and one scratch state. The forward handle's
    // stage buffers are allocated first, so that free memory counts them, and
    // without a limit a slack stays free for the sweep's small buffers (top
    // log, weights, graphs) and the allocator's granularity.
    if (int rc = prepare_scheme(h)) return rc;
    int64_t slots = 0;
    {
        size_t free_b = 0, total_b = 0;
        CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        const double sb = (double)st * 16.0;
        const double held = (double)(A->cap_cps + A->cap_seg + (A->ga.p ? 3 : 0)) * sb;
        const double slack = std::max(512.0 * 1024 * 1024, 0.02 * (double)total_b);
        const double budget =
            A->mem_limit > 0 ? (double)A->mem_limit : std::max(0.0, (double)free_b - slack) + held;
        if ((double)(ncp + 4 * S + 3) * sb > budget) {
            slots = std::min<int64_t>((int64_t)(budget / sb) - 7, steps);
            if (slots < 1)
                return fail(HEOM_E_NOMEM, "adjoint needs at least 8 states of %.3f GB; %.3f GB available",
                            sb / 1e9, budget / 1e9);
            S = 1;
            ncp = slots;
        }
    }
    A->rec_slots = slots;
    // the gradients to accumulate (NULL outputs are skipped); the captured graphs hold them
    const int want_h = grad_h ? 1 : 0, want_bath = (grad_lambda || grad_gamma) ? 1 : 0;
    if (want_h != A->want_h || want_bath != A->want_bath) {
        A->drop_graphs();
        A->want_h = want_h;
        A->want_bath = want_bath;
    }
    // the captured graphs hold buffer addresses: any reallocation drops them
    const bool shrink = slots > 0 && (A->cap_cps > ncp || A->cap_seg > 4);
    if (shrink || ncp > A->cap_cps || 4 * S > A->cap_seg || steps + 1 > A->cap_rows || steps + 1 > A->cap_w)
        A->drop_graphs();
    if (shrink) { // release the sqrt layout before the recursive one takes its place
        A->cps.reset();
        A->seg.reset();
        A->cap_cps = A->cap_seg = 0;
    }
    if (ncp > A->cap_cps) {
        if (int rc = A->cps.alloc(ncp * st)) return rc;
        A->cap_cps = ncp;
    }
    if (4 * S > A->cap_seg) {
        if (int rc = A->seg.alloc(4 * S * st)) return rc;
        A->cap_seg = 4 * S;
    }
    if (!A->ga.p) {
        if (int rc = A->ga.alloc(st)) return rc;
        if (int rc = A->gb.alloc(st)) return rc;
        if (int rc = A->scratch.alloc(st)) return rc;
    }
    if (steps + 1 > A->cap_rows) {
        if (int rc = A->toplog.alloc((steps + 1) * NN * K)) return rc;
        A->cap_rows = steps + 1;
    }
    if (steps + 1 > A->cap_w) {
        if (int rc = A->d_w.alloc(steps + 1)) return rc;
        A->cap_w = steps + 1;
    }
    if (!A->d_base.p)
        if (int rc = A->d_base.alloc(1)) return rc;
    if (int rc = prepare_scheme(h)) return rc;
    {
        // resolve both stage kernels' launch shapes outside of any capture
        const void* fn = nullptr;
        if (int rc = resolve_stage(h, &fn)) return rc;
        if (int rc = resolve_stage(h, &fn, nullptr, true)) return rc;
    }
    CUDA_TRY(cudaMemcpy(A->obs.p, observable, (size_t)K * NN * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(A->d_w.p, weights, (steps + 1) * 8, cudaMemcpyHostToDevice));
    std::vector<int64_t> starts(ncp + 1);
    for (int64_t s2 = 0; s2 <= ncp; ++s2) starts[s2] = s2 * S;
    auto set_base = [&](int64_t s2) -> int {
        CUDA_TRY(cudaMemcpyAsync(A->d_base.p, &starts[s2], 8, cudaMemcpyHostToDevice, h->stream));
        return 0;
    };

    // ---- forward: checkpoints and the observed tops ----
    CUDA_TRY(cudaMemsetAsync(h->y.data.p, 0, st * 16, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->topbuf.p, rho0, (size_t)K * NN * 16, cudaMemcpyHostToDevice, h->stream));
    heomk::heom_write_top<<<K, 128, 0, h->stream>>>(h->y.data.p, h->topbuf.p, h->d_pair.p, h->d_top.p, N, h->P, 0, 0);
    h->launches++;
    heomk::heom_record_top<<<K, 128, 0, h->stream>>>(A->toplog.p, h->y.data.p, h->d_pair.p, h->d_top.p, N, h->P, 0, 0,
                                                     0);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    std::vector<int64_t> bases;
    if (slots > 0) {
        // recursive checkpointing: the tops are recorded as the steps are
        // (re)computed; the adjoint starts with the last step's weight
        RevPlan plan;
        plan.build(steps, slots - 1);
        bases.resize(steps + 1);
        for (int64_t j = 0; j <= steps; ++j) bases[j] = j;
        CUDA_TRY(cudaMemcpyAsync(A->cps.p, h->y.data.p, st * 16, cudaMemcpyDeviceToDevice, h->stream));
        CUDA_TRY(cudaMemsetAsync(A->partial.p, 0, (size_t)A->grid * (NN + 2) * 16, h->stream));
        CUDA_TRY(cudaMemsetAsync(A->ga.p, 0, st * 16, h->stream));
        LeanRun run{A, dt, &plan, bases.data(), st};
        if (int rc = run.set_base(steps)) return rc;
        if (int rc = adj_add_top(A, A->ga.p, 0)) return rc;
        if (int rc = run.reverse(0, steps, 0, slots - 1)) return rc;
    }
    for (int64_t sgm = 0; sgm < (slots > 0 ? 0 : ncp); ++sgm) {
        const int64_t len = std::min(S, steps - sgm * S);
        CUDA_TRY(cudaMemcpyAsync(A->cps.p + sgm * st, h->y.data.p, st * 16, cudaMemcpyDeviceToDevice, h->stream));
        if (int rc = set_base(sgm)) return rc;
        if (int rc = adj_run(A, 0, dt, len)) return rc;
    }
    std::vector<double> tops((steps + 1) * NN * K * 2);
    CUDA_TRY(cudaMemcpyAsync(tops.data(), A->toplog.p, tops.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (int rc = check_kernel_error(h)) return rc;
    for (int k = 0; k < K; ++k) {
        long double J = 0.0L;
        const double* o = observable + (size_t)k * NN * 2;
        for (int64_t n = 0; n <= steps; ++n) {
            const double* tp = tops.data() + ((size_t)n * K + k) * NN * 2;
            long double v = 0.0L;
            for (int q = 0; q < NN; ++q) v += (long double)o[2 * q] * tp[2 * q] + (long double)o[2 * q + 1] * tp[2 * q + 1];
            J += (long double)weights[n] * v;
        }
        if (loss) loss[k] = (double)J;
    }

    // ---- backward (sqrt layout; the recursive sweep has run above) ----
    double2* gcur = A->ga.p;
    if (slots == 0) {
        CUDA_TRY(cudaMemsetAsync(A->partial.p, 0, (size_t)A->grid * (NN + 2) * 16, h->stream));
        CUDA_TRY(cudaMemsetAsync(gcur, 0, st * 16, h->stream));
        if (int rc = set_base(ncp)) return rc; // starts[ncp] = ncp * S >= steps
        if (int rc = adj_add_top(A, gcur, steps - ncp * S)) return rc;
    }
    for (int64_t sgm = (slots > 0 ? -1 : ncp - 1); sgm >= 0; --sgm) {
        const int64_t len = std::min(S, steps - sgm * S);
        CUDA_TRY(cudaMemcpyAsync(A->seg.p, A->cps.p + sgm * st, st * 16, cudaMemcpyDeviceToDevice, h->stream));
        if (int rc = set_base(sgm)) return rc;
        if (int rc = adj_run(A, 1, dt, len)) return rc;
        if (int rc = adj_run(A, 2, dt, len)) return rc;
    }
    std::vector<double> part((size_t)A->grid * (NN + 2) * 2);
    CUDA_TRY(cudaMemcpyAsync(part.data(), A->partial.p, part.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    std::vector<double> g0top((size_t)K * NN * 2);
    heomk::heom_record_top<<<K, 128, 0, h->stream>>>(h->topbuf.p, gcur, h->d_pair.p, h->d_top.p, N, h->P, 0, 0, 0);
    h->launches++;
    CUDA_TRY(cudaMemcpyAsync(g0top.data(), h->topbuf.p, g0top.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (int rc = check_kernel_error(h)) return rc;
    // config units: H and lambda per cm^-1, gamma = 1/invnu per fs^-1
    const long double c = heomhost::invcm_to_joule;
    for (int k = 0; k < K; ++k) {
        std::vector<long double> sum((NN + 2) * 2, 0.0L);
        for (int b = k * A->bpi; b < (k + 1) * A->bpi; ++b)
            for (size_t q = 0; q < sum.size(); ++q) sum[q] += part[(size_t)b * (NN + 2) * 2 + q];
        if (grad_h)
            for (int q = 0; q < NN; ++q) {
                grad_h[((size_t)k * NN + q) * 2] = (double)(-sum[2 * q + 1] / kHbar * c); // Re(i Z / hbar)
                grad_h[((size_t)k * NN + q) * 2 + 1] = (double)(-sum[2 * q] / kHbar * c); // Re(i i Z / hbar)
            }
        if (grad_lambda) grad_lambda[k] = (double)(sum[2 * NN] * c);
        if (grad_gamma) grad_gamma[k] = (double)(sum[2 * NN + 2] * 1e15L);
    }
    if (grad_rho0) std::copy(g0top.begin(), g0top.end(), grad_rho0);
    return 0;
}

int64_t heom_adjoint_kernel_launches(const heom_adjoint* A) { return A && A->h ? A->h->launches : 0; }

int heom_adjoint_set_memory_limit(heom_adjoint* A, int64_t bytes)
{
    if (!A || bytes < 0) return fail(HEOM_E_ARG, "bad argument");
    A->mem_limit = bytes;
    return 0;
}

int64_t heom_adjoint_recursive_slots(const heom_adjoint* A) { return A ? A->rec_slots : -1; }

} // extern "C"

// ---------------------------------------------------------------------------
// Adjoint gradients of an ensemble of systems of any sizes: the systems are
// grouped into classes that share states, baths and bath parameters (what a
// batch adjoint needs); within a class, instances are packed, smallest first,
// into groups whose sqrt(steps) checkpoint layout fits in the memory budget,
// and every group is swept by one batch adjoint.  An instance whose layout
// alone does not fit is swept alone; its adjoint falls back to recursive
// checkpointing in the memory there is.  Groups run one after another, each
// adjoint created for its sweep and destroyed after it, so the device holds
// one group's states at a time.
// ---------------------------------------------------------------------------
namespace {

struct ens_system {
    heom_system_desc d{};
    std::vector<double> ham, lam, inv, om;
    std::vector<int32_t> coup;
    int64_t nodes = 0; // hierarchy ADOs
    int32_t P = 0;     // sectors per ADO
};

bool same_adjoint_class(const heom_system_desc& a, const heom_system_desc& b)
{
    if (a.sites != b.sites || a.baths != b.baths || a.baths_max_per_site != b.baths_max_per_site ||
        a.matsubaras != b.matsubaras || a.temperature != b.temperature)
        return false;
    auto eq = [](const void* x, const void* y, size_t n) { return std::memcmp(x, y, n) == 0; };
    return eq(a.baths_coupling, b.baths_coupling, sizeof(int32_t) * a.sites * a.baths_max_per_site) &&
           eq(a.lambda, b.lambda, sizeof(double) * a.baths) && eq(a.invnu, b.invnu, sizeof(double) * a.baths) &&
           eq(a.omega, b.omega, sizeof(double) * a.baths);
}

} // namespace

struct heom_ensemble_adjoint {
    std::vector<ens_system> sys;
    heom_options opt{};
    int64_t mem_limit = 0;
    std::vector<std::vector<int32_t>> groups; // of the last gradient call
    std::vector<int64_t> group_slots;         // recursive-checkpointing slots per group (0: sqrt layout)
    std::vector<int32_t> group_of;            // per instance
    std::vector<int64_t> mat_off;             // per instance: offset of its states^2 matrix (complex elements)
    int64_t launches = 0;
};

extern "C" {

int heom_ensemble_adjoint_create(const heom_system_desc* systems, int32_t count, const heom_options* opt,
                                 heom_ensemble_adjoint** out)
{
    if (!systems || !out || count < 1) return fail(HEOM_E_ARG, "NULL argument or count < 1");
    *out = nullptr;
    std::unique_ptr<heom_ensemble_adjoint> e(new heom_ensemble_adjoint());
    heom_default_options(&e->opt);
    if (opt) e->opt = *opt;
    e->sys.resize(count);
    e->mat_off.resize(count + 1, 0);
    for (int k = 0; k < count; ++k) {
        const heom_system_desc& d = systems[k];
        if (d.sites < 1 || d.sites > kMaxStates || d.baths < 1 || d.baths_max_per_site < 1 || d.matsubaras < 1 ||
            d.ado_depth < 0 || !d.hamiltonian || !d.baths_coupling || !d.lambda || !d.invnu || !d.omega)
            return fail(HEOM_E_ARG, "system %d: bad descriptor", k);
        ens_system& x = e->sys[k];
        x.ham.assign(d.hamiltonian, d.hamiltonian + 2 * d.sites * d.sites);
        x.lam.assign(d.lambda, d.lambda + d.baths);
        x.inv.assign(d.invnu, d.invnu + d.baths);
        x.om.assign(d.omega, d.omega + d.baths);
        x.coup.assign(d.baths_coupling, d.baths_coupling + d.sites * d.baths_max_per_site);
        x.d = d;
        x.d.hamiltonian = x.ham.data();
        x.d.lambda = x.lam.data();
        x.d.invnu = x.inv.data();
        x.d.omega = x.om.data();
        x.d.baths_coupling = x.coup.data();
        // ADOs = C(W + D, D), W = baths x matsubaras
        const int64_t W = (int64_t)d.baths * d.matsubaras;
        long double c = 1.0L;
        for (int64_t i = 1; i <= d.ado_depth; ++i) c = c * (long double)(W + i) / (long double)i;
        x.nodes = (int64_t)std::llround((double)c);
        x.P = heomk::pairs_of(d.sites);
        e->mat_off[k + 1] = e->mat_off[k] + (int64_t)d.sites * d.sites;
    }
    *out = e.release();
    return 0;
}

int heom_ensemble_adjoint_destroy(heom_ensemble_adjoint* e)
{
    delete e;
    return 0;
}

int heom_ensemble_adjoint_set_memory_limit(heom_ensemble_adjoint* e, int64_t bytes)
{
    if (!e || bytes < 0) return fail(HEOM_E_ARG, "bad argument");
    e->mem_limit = bytes;
    return 0;
}

int heom_ensemble_adjoint_gradient(heom_ensemble_adjoint* e, const double* rho0, const double* observable,
                                   const double* weights, double dt, int64_t steps, double* loss, double* grad_h,
                                   double* grad_lambda, double* grad_gamma, double* grad_rho0)
{
    if (!e || !rho0 || !observable || !weights || steps < 1 || !(dt > 0.0)) return fail(HEOM_E_ARG, "bad argument");
    CUDA_TRY(cudaSetDevice(e->opt.device));
    const int count = (int)e->sys.size();
    // memory budget of one group's states: the limit, or 85 % of the free memory
    int64_t budget = e->mem_limit;
    if (budget <= 0) {
        size_t free_b = 0, total_b = 0;
        CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        budget = (int64_t)(0.85 * (double)free_b);
    }
    const int64_t S = std::max<int64_t>(1, (int64_t)std::ceil(std::sqrt((double)steps)));
    const int64_t ncp = (steps + S - 1) / S;
    // sqrt layout of a batch adjoint: checkpoints, the stage inputs of one
    // segment, the adjoint ping-pong and a scratch state, plus the forward
    // handle's state and its two product-form stage buffers
    const int64_t states_needed = ncp + 4 * S + 3 + 3;
    auto bytes_of = [&](int k) { return e->sys[k].nodes * (int64_t)e->sys[k].P * 32; };
    // classes (first fit on the descriptor), then groups per class
    std::vector<std::vector<int32_t>> classes;
    for (int k = 0; k < count; ++k) {
        bool placed = false;
        for (auto& c : classes)
            if (same_adjoint_class(e->sys[c[0]].d, e->sys[k].d)) {
                c.push_back(k);
                placed = true;
                break;
            }
        if (!placed) classes.push_back({k});
    }
    e->groups.clear();
    for (auto& c : classes) {
        std::vector<int32_t> m = c;
        std::stable_sort(m.begin(), m.end(), [&](int a, int b) { return e->sys[a].nodes < e->sys[b].nodes; });
        std::vector<int32_t> g;
        int64_t held = 0;
        for (int k : m) {
            if (!g.empty() && states_needed * (held + bytes_of(k)) > budget) {
                e->groups.push_back(g);
                g.clear();
                held = 0;
            }
            g.push_back(k);
            held += bytes_of(k);
        }
        if (!g.empty()) e->groups.push_back(g);
    }
    e->group_of.assign(count, -1);
    e->group_slots.assign(e->groups.size(), 0);
    for (size_t gi = 0; gi < e->groups.size(); ++gi) {
        const std::vector<int32_t>& g = e->groups[gi];
        const int K = (int)g.size();
        const int N = e->sys[g[0]].d.sites, NN = N * N;
        std::vector<heom_system_desc> d(K);
        for (int q = 0; q < K; ++q) d[q] = e->sys[g[q]].d;
        heom_adjoint* A = nullptr;
        if (int rc = heom_adjoint_create_batch(d.data(), K, &e->opt, &A)) return rc;
        std::unique_ptr<heom_adjoint, int (*)(heom_adjoint*)> hold(A, heom_adjoint_destroy);
        if (e->mem_limit > 0) heom_adjoint_set_memory_limit(A, e->mem_limit);
        // gather the group's per-instance arrays
        std::vector<double> r0(2 * (size_t)K * NN), ob(2 * (size_t)K * NN), gl(K), gg(K), ls(K);
        std::vector<double> gh(grad_h ? 2 * (size_t)K * NN : 0), gr(grad_rho0 ? 2 * (size_t)K * NN : 0);
        for (int q = 0; q < K; ++q) {
            const size_t src = 2 * (size_t)e->mat_off[g[q]];
            std::copy(rho0 + src, rho0 + src + 2 * NN, r0.begin() + 2 * (size_t)q * NN);
            std::copy(observable + src, observable + src + 2 * NN, ob.begin() + 2 * (size_t)q * NN);
        }
        const int64_t before = heom_adjoint_kernel_launches(A);
        if (int rc = heom_adjoint_gradient(A, r0.data(), ob.data(), weights, dt, steps, ls.data(),
                                           grad_h ? gh.data() : nullptr, grad_lambda ? gl.data() : nullptr,
                                           grad_gamma ? gg.data() : nullptr, grad_rho0 ? gr.data() : nullptr))
            return rc;
        e->launches += heom_adjoint_kernel_launches(A) - before;
        e->group_slots[gi] = heom_adjoint_recursive_slots(A);
        for (int q = 0; q < K; ++q) {
            const int k = g[q];
            const size_t dst = 2 * (size_t)e->mat_off[k];
            e->group_of[k] = (int32_t)gi;
            if (loss) loss[k] = ls[q];
            if (grad_lambda) grad_lambda[k] = gl[q];
            if (grad_gamma) grad_gamma[k] = gg[q];
            if (grad_h) std::copy(gh.begin() + 2 * (size_t)q * NN, gh.begin() + 2 * (size_t)(q + 1) * NN, grad_h + dst);
            if (grad_rho0)
                std::copy(gr.begin() + 2 * (size_t)q * NN, gr.begin() + 2 * (size_t)(q + 1) * NN, grad_rho0 + dst);
        }
    }
    return 0;
}

int32_t heom_ensemble_adjoint_groups(const heom_ensemble_adjoint* e) { return e ? (int32_t)e->groups.size() : 0; }

int heom_ensemble_adjoint_group_of(const heom_ensemble_adjoint* e, int32_t inst, int32_t* group,
                                   int64_t* recursive_slots)
{
    if (!e || inst < 0 || inst >= (int32_t)e->sys.size()) return fail(HEOM_E_ARG, "bad argument");
    if (e->group_of.empty()) return fail(HEOM_E_ARG, "no gradient has been computed yet");
    const int32_t g = e->group_of[inst];
    if (group) *group = g;
    if (recursive_slots) *recursive_slots = g >= 0 ? e->group_slots[g] : 0;
    return 0;
}

int64_t heom_ensemble_adjoint_offset(const heom_ensemble_adjoint* e, int32_t inst)
{
    if (!e || inst < 0 || inst > (int32_t)e->sys.size()) return -1;
    return e->mat_off[inst];
}

int64_t heom_ensemble_adjoint_kernel_launches(const heom_ensemble_adjoint* e) { return e ? e->launches : 0; }

} // extern "C"
