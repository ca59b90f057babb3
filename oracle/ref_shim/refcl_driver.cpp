/* Host driver for the reference's own OpenCL kernels compiled as C++: runs
 * the NDRange global {1, nodes}, local {1, 1} of
 * dm-heom/src/app_population_dynamics.cpp:63-67 as an OpenMP loop, one
 * work-item (= one ADO) per iteration.  TEST INFRASTRUCTURE ONLY. */
#include <cstdint>
#include <cstring>
#include <stdexcept>

#include "refcl_prelude.h"

thread_local std::size_t refcl_gid = 0;
std::size_t refcl_nodes = 0;
int refcl_num_states = 0;
int refcl_num_matsubaras = 0;
int refcl_baths_max_per_state = 0;
int refcl_ado_width = 0;
int refcl_baths_coupling_storage[1024];

typedef unsigned char mask_t;
/* Declarations of the kernels as the TUs define them (real_t = double,
 * bool_t = int, mask_t = unsigned char). */
#define REFCL_ODE_ARGS                                                                     \
    const double step_size, double* __restrict sigma_out, const double out_coeff,        \
        double* __restrict sigma_acc, const double acc_coeff, const int acc_init,         \
        const double* __restrict sigma_in, const double* __restrict hamiltonian,         \
        const int* __restrict ado_tuples, const int* __restrict ado_plus,                \
        const int* __restrict ado_minus, const double* __restrict pf_same_sum,           \
        const double* __restrict pf_same, const double* __restrict pf_circ,              \
        const double* __restrict cbk, const double* __restrict cbk_sqrt,                 \
        const int first_non_plus_id, mask_t* __restrict mask,                            \
        double* __restrict flow_from_above, double* __restrict flow_from_below
void refcl_heom_ode_pure(REFCL_ODE_ARGS);
void refcl_heom_ode_acc(REFCL_ODE_ARGS);
void refcl_heom_ode_subdiag(REFCL_ODE_ARGS);
void refcl_heom_ode_noplus(REFCL_ODE_ARGS);
void refcl_heom_ode_nominus(REFCL_ODE_ARGS);
void refcl_rk_weighted_add(const int n, const double h, double* __restrict out,
                           const double* __restrict y_n, double c1, const double* __restrict k1,
                           double c2, const double* __restrict k2, double c3,
                           const double* __restrict k3, double c4, const double* __restrict k4,
                           double c5, const double* __restrict k5, double c6,
                           const double* __restrict k6, double c7, const double* __restrict k7);

extern "C" {

/* mode: 0 = pure evaluation, 1 = NOMA_NUM_ODE_ACCUMULATE, 2 = NOMA_NUM_ODE_SUBDIAGONAL,
 * 3 = pure evaluation with HEOM_ODE_DISABLE_PLUS, 4 = pure evaluation with HEOM_ODE_DISABLE_MINUS */
int refcl_heom_ode(int mode, int states, int matsubaras, int baths_per_state, int ado_width,
                   int64_t nodes, int first_non_plus_id, const int* coupling,
                   double step_size, double* out, double out_coeff, double* acc,
                   double acc_coeff, int acc_init, const double* in, const double* hamiltonian,
                   const int* tuples, const int* plus, const int* minus,
                   const double* pf_same_sum, const double* pf_same, const double* pf_circ,
                   const double* cbk, const double* cbk_sqrt, unsigned char* mask, int threads)
{
    if (states * baths_per_state > 1024) return -1;
    refcl_nodes = (std::size_t)nodes;
    refcl_num_states = states;
    refcl_num_matsubaras = matsubaras;
    refcl_baths_max_per_state = baths_per_state;
    refcl_ado_width = ado_width;
    std::memcpy(refcl_baths_coupling_storage, coupling, sizeof(int) * states * baths_per_state);
    typedef void (*fn_t)(REFCL_ODE_ARGS);
    fn_t fn = mode == 0 ? refcl_heom_ode_pure : mode == 1 ? refcl_heom_ode_acc : mode == 2 ? refcl_heom_ode_subdiag
            : mode == 3 ? refcl_heom_ode_noplus : refcl_heom_ode_nominus;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t u = 0; u < nodes; ++u) {
        refcl_gid = (std::size_t)u;
        fn(step_size, out, out_coeff, acc, acc_coeff, acc_init, in, hamiltonian, tuples, plus,
           minus, pf_same_sum, pf_same, pf_circ, cbk, cbk_sqrt, first_non_plus_id, mask,
           nullptr, nullptr);
    }
    return 0;
}

/* rk_weighted_add over nodes ADOs of states x states complex elements */
int refcl_rk_weighted_add(int states, int64_t nodes, int n, double h, double* out,
                          const double* y, const double* c, const double* const* k, int threads)
{
    if (n < 0 || n > 7) return -1;
    refcl_nodes = (std::size_t)nodes;
    refcl_num_states = states;
    double cc[7] = {0, 0, 0, 0, 0, 0, 0};
    const double* kk[7] = {y, y, y, y, y, y, y};
    for (int l = 0; l < n; ++l) { cc[l] = c[l]; kk[l] = k[l]; }
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t u = 0; u < nodes; ++u) {
        refcl_gid = (std::size_t)u;
        refcl_rk_weighted_add(n, h, out, y, cc[0], kk[0], cc[1], kk[1], cc[2], kk[2], cc[3],
                              kk[3], cc[4], kk[4], cc[5], kk[5], cc[6], kk[6]);
    }
    return 0;
}

}
