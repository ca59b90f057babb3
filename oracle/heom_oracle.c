/*
 * heom_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see heom_oracle.h).
 *
 * Plain C restatement of the reference's HEOM derivative + RK4 path.  Each
 * function cites the reference lines it follows.  Compiled with
 * -ffp-contract=off so that every product is rounded as in the reference's
 * own kernel sources compiled for the host (oracle/_ref).
 */
#include "heom_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "pade_tables.inc"

#define HO_MAX_PADE 10

/* ------------------------------------------------------------------------ */
/* combinatorics                                                             */
/* ------------------------------------------------------------------------ */

int64_t ho_binomial(int64_t n, int64_t k)
{
    if (k < 0 || n < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    int64_t r = 1;
    for (int64_t i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

/*
 * Partitions of n into at most s parts.  The reference generates them with
 * the Zoghbi-Stojmenovic ZS2 scheme (integer_partition.cpp:41-106), which
 * visits partitions (written as non-increasing part sequences) in ascending
 * lexicographic order: 1+1+..+1, 2+1+..+1, 2+2+1.., ..., n.  The same order is
 * produced here by a recursive ascending enumeration of the first part.
 */
typedef struct part_ctx {
    int32_t s;
    int32_t* out;
    int64_t cap;
    int64_t count;
    int32_t cur[64];
    int32_t len;
} part_ctx;

static void part_rec(part_ctx* c, int32_t remaining, int32_t max_part)
{
    if (remaining == 0) {
        if (c->len <= c->s) {
            if (c->count < c->cap) {
                int32_t* row = c->out + c->count * c->s;
                for (int32_t p = 0; p < c->s; ++p) row[p] = p < c->len ? c->cur[p] : 0;
            }
            c->count++;
        }
        return;
    }
    if (c->len >= c->s) return; /* more parts than allowed */
    int32_t top = remaining < max_part ? remaining : max_part;
    for (int32_t p = 1; p <= top; ++p) {
        c->cur[c->len++] = p;
        part_rec(c, remaining - p, p);
        c->len--;
    }
}

int64_t ho_integer_partitions(int32_t n, int32_t s, int32_t* out, int64_t cap)
{
    part_ctx c;
    memset(&c, 0, sizeof c);
    c.s = s;
    c.out = out;
    c.cap = cap;
    if (n <= 0 || n > 63) return -1;
    part_rec(&c, n, n);
    return c.count <= cap ? c.count : -1;
}

/* number of tuples over d coordinates with sum <= r */
static int64_t simplex_count(int32_t d, int32_t r)
{
    if (r < 0) return 0;
    return ho_binomial((int64_t)r + d, d);
}

/* rank of a tuple in ascending lexicographic order of all tuples of the graph
 * (a bijection onto 0..nodes-1 used as the tuple -> uid map) */
static int64_t lex_rank(const int32_t* t, int32_t w, int32_t depth)
{
    int64_t rank = 0;
    int32_t prefix = 0;
    for (int32_t k = 0; k < w; ++k) {
        for (int32_t x = 0; x < t[k]; ++x) rank += simplex_count(w - 1 - k, depth - prefix - x);
        prefix += t[k];
    }
    return rank;
}

/* next lexicographic permutation (ascending), same visiting order as
 * std::next_permutation; returns 0 after the last permutation */
static int next_perm(int32_t* a, int32_t n)
{
    int32_t i = n - 2;
    while (i >= 0 && a[i] >= a[i + 1]) --i;
    if (i < 0) return 0;
    int32_t j = n - 1;
    while (a[j] <= a[i]) --j;
    int32_t tmp = a[i]; a[i] = a[j]; a[j] = tmp;
    for (int32_t l = i + 1, r = n - 1; l < r; ++l, --r) {
        tmp = a[l]; a[l] = a[r]; a[r] = tmp;
    }
    return 1;
}

static int cmp_i32(const void* a, const void* b)
{
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

/* hierarchy_graph.cpp:30-181: layers top to bottom; in each layer the integer
 * partitions of the layer depth in generation order, each sorted ascending
 * and expanded through all its lexicographic permutations. */
int ho_graph_build(int32_t width, int32_t depth, ho_graph* g)
{
    memset(g, 0, sizeof *g);
    if (width <= 0 || depth <= 0 || width > 64) return -1;
    g->width = width;
    g->depth = depth;
    g->nodes = ho_binomial((int64_t)width + depth, width);
    g->first_non_plus = (int32_t)ho_binomial((int64_t)width + depth - 1, width);
    const int64_t nodes = g->nodes;
    g->tuples = (int32_t*)malloc(sizeof(int32_t) * nodes * width);
    g->plus = (int32_t*)malloc(sizeof(int32_t) * nodes * width);
    g->minus = (int32_t*)malloc(sizeof(int32_t) * nodes * width);
    g->nodes_per_depth = (int64_t*)calloc((size_t)depth + 1, sizeof(int64_t));
    int64_t* uid_of_rank = (int64_t*)malloc(sizeof(int64_t) * nodes);
    if (!g->tuples || !g->plus || !g->minus || !g->nodes_per_depth || !uid_of_rank) return -2;

    int64_t uid = 0;
    int32_t tuple[64];
    for (int32_t d = 0; d <= depth; ++d) {
        int64_t np;
        int32_t* parts;
        if (d == 0) {
            np = 1;
            parts = (int32_t*)calloc((size_t)width, sizeof(int32_t));
        } else {
            int64_t cap = ho_binomial((int64_t)d + width - 1, width - 1) + 1; /* >= partitions */
            parts = (int32_t*)malloc(sizeof(int32_t) * cap * width);
            np = ho_integer_partitions(d, width, parts, cap);
            if (np < 0) return -3;
        }
        for (int64_t p = 0; p < np; ++p) {
            memcpy(tuple, parts + p * width, sizeof(int32_t) * width);
            qsort(tuple, (size_t)width, sizeof(int32_t), cmp_i32);
            do {
                if (uid >= nodes) return -4;
                memcpy(g->tuples + uid * width, tuple, sizeof(int32_t) * width);
                uid_of_rank[lex_rank(tuple, width, depth)] = uid;
                g->nodes_per_depth[d]++;
                uid++;
            } while (next_perm(tuple, width));
        }
        free(parts);
    }
    if (uid != nodes) return -5;

    for (int64_t u = 0; u < nodes; ++u) {
        const int32_t* t = g->tuples + u * width;
        int32_t sum = 0;
        for (int32_t j = 0; j < width; ++j) sum += t[j];
        memcpy(tuple, t, sizeof(int32_t) * width);
        for (int32_t j = 0; j < width; ++j) {
            int32_t plus = HO_INVALID_UID, minus = HO_INVALID_UID;
            if (sum < depth) {
                tuple[j] += 1;
                plus = (int32_t)uid_of_rank[lex_rank(tuple, width, depth)];
                tuple[j] -= 1;
            }
            if (tuple[j] > 0) {
                tuple[j] -= 1;
                minus = (int32_t)uid_of_rank[lex_rank(tuple, width, depth)];
                tuple[j] += 1;
            }
            g->plus[u * width + j] = plus;
            g->minus[u * width + j] = minus;
        }
    }
    free(uid_of_rank);
    return 0;
}

void ho_graph_free(ho_graph* g)
{
    free(g->tuples);
    free(g->plus);
    free(g->minus);
    free(g->nodes_per_depth);
    memset(g, 0, sizeof *g);
}

/* ------------------------------------------------------------------------ */
/* bath precompute: instance.cpp:155-273                                     */
/* ------------------------------------------------------------------------ */

void ho_precompute_baths(const ho_system* sys, const ho_graph* g,
                         double* pf_same_sum, double* pf_same, double* pf_circ,
                         double* cbk_out, double* cbk_sqrt)
{
    const double hbar = HO_HBAR;
    const double beta = 1.0 / (HO_KB * sys->temperature);
    const int32_t M = sys->matsubaras;
    const int32_t row = (M - 1) * HO_MAX_PADE;

    for (int32_t b = 0; b < sys->baths; ++b) {
        double _Complex lambda_b = CMPLX(sys->lambda[b], 0.0);
        double _Complex nu_b = CMPLX(1.0 / sys->invnu[b], sys->omega[b]);
        double _Complex pfc = nu_b * lambda_b / hbar;                              /* :176 */
        double _Complex aux = 2.0 * lambda_b / (beta * hbar * hbar * nu_b);          /* :177 */
        pf_circ[2 * b] = creal(pfc);
        pf_circ[2 * b + 1] = cimag(pfc);
        for (int32_t k = 0; k < M; ++k) {
            double _Complex cbk, nubk;
            if (k == 0) {                                                            /* :183-199 */
                double _Complex auxsum = 0.0;
                for (int32_t j = 0; j < M; ++j) {
                    double eta = (double)ho_eta_pade[row + j];
                    double xi = (double)ho_xi_pade[row + j];
                    auxsum += (2.0 * eta * nu_b * nu_b) / (xi * xi / (beta * beta * hbar * hbar) - nu_b * nu_b);
                }
                cbk = 2.0 * lambda_b / (beta * hbar) * (1.0 - auxsum);
                nubk = nu_b;
            } else {                                                                 /* :204-208 */
                double eta = (double)ho_eta_pade[row + k];
                double xi = (double)ho_xi_pade[row + k];
                cbk = 4.0 * lambda_b * nu_b / (beta * beta * hbar * hbar) * (eta * xi) / (xi * xi / (beta * beta * hbar * hbar) - nu_b * nu_b);
                nubk = xi / (beta * hbar);
            }
            cbk_out[2 * (b * M + k)] = creal(cbk);                                   /* :216 */
            cbk_out[2 * (b * M + k) + 1] = cimag(cbk);
            cbk_sqrt[b * M + k] = sqrt(cabs(cbk));                                   /* :217 */
            aux -= cbk / (hbar * nubk);                                              /* :218 */
        }
        pf_same[2 * b] = creal(aux);                                                 /* :220 */
        pf_same[2 * b + 1] = cimag(aux);
    }

    /* :227-262, long double accumulation */
    const int32_t W = g->width;
    for (int64_t id = 0; id < g->nodes; ++id) {
        long double zr = 0.0L, zi = 0.0L;
        for (int32_t b = 0; b < sys->baths; ++b) {
            double nu_r = 1.0 / sys->invnu[b];
            double nu_i = sys->omega[b];
            for (int32_t k = 0; k < M; ++k) {
                long double nr, ni;
                if (k == 0) {
                    nr = (long double)nu_r;
                    ni = (long double)nu_i;
                } else {
                    nr = ho_xi_pade[row + k] / (long double)(beta * hbar);
                    ni = 0.0L;
                }
                int32_t m = b * M + k;
                zr -= nr * (long double)g->tuples[id * W + m];
                zi -= ni * (long double)g->tuples[id * W + m];
            }
        }
        pf_same_sum[2 * id] = (double)zr;
        pf_same_sum[2 * id + 1] = (double)zi;
    }
}

/* ------------------------------------------------------------------------ */
/* derivative: heom_ode.cl:24-451 (pure evaluation)                          */
/* ------------------------------------------------------------------------ */

#define HO_REAL double
#define HO_SQRT sqrt
#define HO_HYPOT hypot
#define HO_FN(name) name
#include "heom_oracle_kernel.inc"
#undef HO_REAL
#undef HO_SQRT
#undef HO_HYPOT
#undef HO_FN

#define HO_REAL long double
#define HO_SQRT sqrtl
#define HO_HYPOT hypotl
#define HO_FN(name) name##_ld
#include "heom_oracle_kernel.inc"
#undef HO_REAL
#undef HO_SQRT
#undef HO_HYPOT
#undef HO_FN

void ho_derivative(const ho_problem* p, const double* in, double* out, int threads)
{
    ho_derivative_impl(p, in, out, threads);
}

void ho_derivative_ld(const ho_problem* p, const long double* in, long double* out, int threads)
{
    ho_derivative_impl_ld(p, in, out, threads);
}

/* rk_weighted_add.cl:78-95 */
void ho_rk_weighted_add(int64_t len, int n, double h, double* out, const double* y,
                        const double* c, const double* const* k, int threads)
{
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t e = 0; e < len; ++e) {
        double acc = 0.0;
        for (int l = 0; l < n; ++l)
            if (c[l] != 0.0) acc += c[l] * k[l][e];
        acc *= h;
        acc += y[e];
        out[e] = acc;
    }
}

void ho_rk4_step(const ho_problem* p, double h, const double* y, double* y_out,
                 double* work, int threads)
{
    ho_rk4_step_impl(p, h, y, y_out, work, threads);
}

void ho_rk4_step_ld(const ho_problem* p, long double h, const long double* y,
                    long double* y_out, long double* work, int threads)
{
    ho_rk4_step_impl_ld(p, h, y, y_out, work, threads);
}

int64_t ho_propagate(const ho_problem* p, double h, int64_t steps, int64_t observe_every,
                     double* y, double* pops, int threads)
{
    const int64_t len = p->nodes * p->states * p->states * 2;
    double* work = (double*)malloc(sizeof(double) * len * 6);
    if (!work) return -1;
    double* a = y;
    double* b = work + 5 * len;
    const int32_t N = p->states;
    int64_t rows = 0;
    if (observe_every > 0) {
        for (int32_t i = 0; i < N; ++i) pops[i] = a[(N + 1) * 2 * i];
        rows = 1;
    }
    for (int64_t s = 0; s < steps; ++s) {
        ho_rk4_step_impl(p, h, a, b, work, threads);
        double* t = a; a = b; b = t;
        if (observe_every > 0 && (s + 1) % observe_every == 0) {
            for (int32_t i = 0; i < N; ++i) pops[rows * N + i] = a[(N + 1) * 2 * i];
            rows++;
        }
    }
    if (a != y) memcpy(y, a, sizeof(double) * len);
    free(work);
    return rows;
}

int64_t ho_propagate_ld(const ho_problem* p, double h, int64_t steps, int64_t observe_every,
                        double* y, double* pops, int threads)
{
    const int64_t len = p->nodes * p->states * p->states * 2;
    long double* work = (long double*)malloc(sizeof(long double) * len * 7);
    if (!work) return -1;
    long double* a = work + 5 * len;
    long double* b = work + 6 * len;
    for (int64_t e = 0; e < len; ++e) a[e] = (long double)y[e];
    const int32_t N = p->states;
    int64_t rows = 0;
    if (observe_every > 0) {
        for (int32_t i = 0; i < N; ++i) pops[i] = (double)a[(N + 1) * 2 * i];
        rows = 1;
    }
    for (int64_t s = 0; s < steps; ++s) {
        ho_rk4_step_impl_ld(p, (long double)h, a, b, work, threads);
        long double* t = a; a = b; b = t;
        if (observe_every > 0 && (s + 1) % observe_every == 0) {
            for (int32_t i = 0; i < N; ++i) pops[rows * N + i] = (double)a[(N + 1) * 2 * i];
            rows++;
        }
    }
    for (int64_t e = 0; e < len; ++e) y[e] = (double)a[e];
    free(work);
    return rows;
}
