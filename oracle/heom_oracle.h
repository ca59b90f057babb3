/*
 * heom_oracle.h -- CPU oracle for the HEOM derivative + RK4 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; it is used by tests/, by the smoke check and by the
 * cpu_baseline / reference arm of bench.py, always as the checker or as the
 * timed CPU baseline, never as the thing that is shipped.
 *
 * It is a plain-C restatement of the reference (noma/dm-heom) algorithm:
 *   - integer partitions        dm-heom/src/heom/integer_partition.cpp:20-106
 *   - hierarchy graph (uids)    dm-heom/src/heom/hierarchy_graph.cpp:30-181
 *   - bath precompute           dm-heom/src/heom/instance.cpp:155-273
 *   - heom_ode derivative       dm-heom/cl/heom/heom_ode.cl:24-451
 *   - rk_weighted_add           dm-heom/cl/heom/rk_weighted_add.cl:19-106
 *   - classical RK4 driver      (the noma/num stepper is an un-vendored
 *                                submodule; the tableau a={1/2,1/2,1},
 *                                b={1/6,1/3,1/3,1/6} is restated, stage
 *                                inputs are formed with rk_weighted_add
 *                                semantics)
 *
 * Pinning: the derivative and weighted-add restatements are compared
 * bit-for-bit with the reference's own OpenCL kernel sources compiled as C++
 * (oracle/_ref, built by oracle/Makefile), and the partition order with the
 * reference's integer_partition.cpp compiled as is.  The host-side graph and
 * precompute depend on Boost in the reference and are restated here.
 *
 * Layouts are the reference's (instance.hpp:202-214): every ADO is an N x N
 * complex matrix stored row-major with interleaved (re, im) doubles, ADOs in
 * uid order; tuples/plus/minus are int32 [nodes x width].
 */
#ifndef HEOM_ORACLE_H
#define HEOM_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HO_HBAR 1.05457148e-34 /* common.cl:46, constants.hpp:22 */
#define HO_KB 1.380650239684840458953781387048428305608616777679979316e-23 /* constants.hpp:23 */
#define HO_INVCM_TO_JOULE 1.986456217327470903861498336971100097137908380913187891e-23 /* constants.hpp:24 */
#define HO_INVALID_UID (-2) /* hierarchy_graph.cpp:24 */

typedef struct ho_graph {
    int32_t width;
    int32_t depth;
    int64_t nodes;
    int32_t first_non_plus;
    int32_t* tuples; /* [nodes * width] */
    int32_t* plus;   /* [nodes * width], HO_INVALID_UID where absent */
    int32_t* minus;  /* [nodes * width], HO_INVALID_UID where absent */
    int64_t* nodes_per_depth; /* [depth + 1] */
} ho_graph;

typedef struct ho_system {
    int32_t states;          /* N (identity sites->states mode) */
    int32_t baths;           /* B */
    int32_t matsubaras;      /* M, including the k = 0 Drude term */
    int32_t baths_per_state; /* columns of the coupling matrix */
    const int32_t* coupling; /* [states * baths_per_state], < 0 = none */
    double temperature;      /* K */
    const double* lambda;    /* [B] J */
    const double* invnu;     /* [B] s */
    const double* omega;     /* [B] rad/s */
} ho_system;

typedef struct ho_problem {
    int32_t states;
    int32_t matsubaras;
    int32_t baths_per_state;
    int32_t ado_width;
    int64_t nodes;
    int32_t first_non_plus;
    const int32_t* coupling;    /* [states * baths_per_state] */
    const double* hamiltonian;  /* [N*N*2] J */
    const int32_t* tuples;
    const int32_t* plus;
    const int32_t* minus;
    const double* pf_same_sum;  /* [nodes*2] */
    const double* pf_same;      /* [B*2] */
    const double* pf_circ;      /* [B*2] */
    const double* cbk;          /* [B*M*2] */
    const double* cbk_sqrt;     /* [B*M] */
    const uint8_t* mask;        /* [nodes] */
} ho_problem;

/* ---- combinatorics / graph ---- */
int64_t ho_binomial(int64_t n, int64_t k);
/* Partitions of n into at most s parts, in the reference's generation
 * order, each written as s entries (parts then zero padding).  Returns the
 * count, or -1 when cap rows are not enough. */
int64_t ho_integer_partitions(int32_t n, int32_t s, int32_t* out, int64_t cap);
int ho_graph_build(int32_t width, int32_t depth, ho_graph* g);
void ho_graph_free(ho_graph* g);

/* ---- bath precompute (instance.cpp:155-273) ---- */
void ho_precompute_baths(const ho_system* sys, const ho_graph* g,
                         double* pf_same_sum, double* pf_same, double* pf_circ,
                         double* cbk, double* cbk_sqrt);
/* Pade tables restated from the mathematics: [N-1/N] Pade approximant of
 * coth(x/2)/2 - 1/x; row (n-1), 10 x 10 layout as constants.cpp:13-75. */
extern const long double ho_eta_pade[100];
extern const long double ho_xi_pade[100];

/* ---- derivative and stepping ---- */
/* heom_ode.cl pure evaluation (no ACCUMULATE/SUBDIAGONAL): out = L(in). */
void ho_derivative(const ho_problem* p, const double* in, double* out, int threads);
/* Same arithmetic in long double (for FP64 error statements). */
void ho_derivative_ld(const ho_problem* p, const long double* in, long double* out, int threads);
/* rk_weighted_add.cl: out = y + h * sum_l c_l k_l, terms with c_l == 0 skipped. */
void ho_rk_weighted_add(int64_t len, int n, double h, double* out, const double* y,
                        const double* c, const double* const* k, int threads);
/* One classical RK4 step y -> y_out (y_out may not alias y).  work must hold
 * 5 state buffers. */
void ho_rk4_step(const ho_problem* p, double h, const double* y, double* y_out,
                 double* work, int threads);
void ho_rk4_step_ld(const ho_problem* p, long double h, const long double* y,
                    long double* y_out, long double* work, int threads);
/* steps RK4 steps; after every observe_every steps (and at t = 0) writes the
 * N diagonal populations Re rho_ii into pops (row per observation).  y is
 * updated in place.  Returns the number of observation rows written. */
int64_t ho_propagate(const ho_problem* p, double h, int64_t steps, int64_t observe_every,
                     double* y, double* pops, int threads);
int64_t ho_propagate_ld(const ho_problem* p, double h, int64_t steps, int64_t observe_every,
                        double* y, double* pops, int threads);

#ifdef __cplusplus
}
#endif
#endif
