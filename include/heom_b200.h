/*
 * heom_b200.h -- C ABI of the B200 HEOM propagator.
 *
 * Drop-in boundary for the reference's OpenCL derivative + RK4 path
 * (noma/dm-heom).  The entry points replace, one for one:
 *
 *   heom_create / heom_destroy       heom::ode ctor + ode::initialise(), which
 *                                    uploads H, tuples, plus, minus, pf_* and
 *                                    cbk tables (dm-heom/src/heom/ode.cpp:23-95)
 *   heom_set_hamiltonian             ode::update_hamiltonian (ode.cpp:198-204) /
 *                                    solver_base::update_hamiltonian
 *                                    (solver_base.hpp:272-277)
 *   heom_set_mask                    ode::set_hierarchy_mask (ode.cpp:206-211) /
 *                                    solver_base::update_hierarchy_mask
 *                                    (solver_base.hpp:289-296)
 *   heom_buffer_create / _destroy    ocl_helper::create_buffer of a hierarchy
 *                                    buffer (population_dynamics_solver.hpp:140-141)
 *   heom_buffer_write / _read        enqueueWriteBuffer / enqueueReadBuffer of a
 *                                    hierarchy buffer (population_dynamics_solver.hpp:162-166,
 *                                    solver_base.hpp:199-222)
 *   heom_solve                       the four ode::solve overloads (ode.cpp:97-195):
 *                                    one heom_ode kernel launch in the write modes
 *                                    pure / NOMA_NUM_ODE_ACCUMULATE /
 *                                    NOMA_NUM_ODE_SUBDIAGONAL (heom_ode.cl:416-434)
 *   heom_weighted_add                rk_weighted_add kernel (rk_weighted_add.cl:19-106)
 *   heom_set_state / heom_get_state  population_dynamics_solver::reset (:159-172) /
 *                                    solver_base::update_instance (:225-228)
 *   heom_set_top / heom_get_top      solver_base::update_hierarchy_top (:279-286) /
 *                                    solver_base::hierarchy_top (:219-222)
 *   heom_rk4_steps                   population_dynamics_solver::step_forward
 *                                    (:233-265) driving the absent noma/num RK4
 *                                    stepper (rk_rk4)
 *   heom_propagate                   the observe loop of
 *                                    app_population_dynamics.cpp:88-106 with the top
 *                                    matrix recorded on the device at every observation
 *
 * Conventions
 *   - Every call returns 0 on success or a negative HEOM_E_* code;
 *     heom_last_error() gives a message for the calling thread's last failure.
 *   - Host arrays use the reference layouts (dm-heom/include/heom/instance.hpp:202-214):
 *     a hierarchy state is [matrices][states][states] complex doubles stored as
 *     interleaved (re, im), ADOs in the reference's uid order; tuples, plus and
 *     minus are int32 [matrices][ado_width]; hierarchy_graph::invalid_uid (-2)
 *     marks absent neighbours.
 *   - Device hierarchy buffers (heom_buffer) are opaque: they hold the state in
 *     the library's own HBM layout (ADOs reordered for neighbour locality).
 *   - A handle owns one CUDA stream; calls on one handle are not thread-safe.
 *     All calls are blocking with respect to the host (like the reference's
 *     CL_TRUE transfers) except where documented.
 *   - Only the CUDA path exists: there is no CPU fallback.  Without a usable
 *     sm_100 device heom_create fails with HEOM_E_CUDA.
 */
#ifndef HEOM_B200_H
#define HEOM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HEOM_OK 0
#define HEOM_E_ARG (-1)       /* invalid argument (null pointer, size, range) */
#define HEOM_E_CUDA (-2)      /* CUDA runtime error or no usable device */
#define HEOM_E_NOMEM (-3)     /* device or host allocation failed */
#define HEOM_E_TABLE (-4)     /* inconsistent hierarchy tables rejected at admission */
#define HEOM_E_UNSUPPORTED (-5) /* size or mode outside what this build supports */
#define HEOM_E_NONFINITE (-6) /* a non-finite value was detected in the state */
#define HEOM_E_CONFIG (-7)    /* configuration file error */

#define HEOM_INVALID_UID (-2)

/* Hierarchy instance in the reference's host layouts: the arguments 7-17 of
 * the heom_ode kernel (heom_ode.cl:24-45) plus the compile-time defines the
 * reference generates (solver_base.hpp:179-195). */
typedef struct heom_instance_desc {
    int32_t states;            /* NUM_STATES */
    int32_t matsubaras;        /* NUM_MATSUBARAS */
    int32_t baths;             /* number of baths (rows of pf_same / pf_circ) */
    int32_t baths_per_state;   /* BATHS_MAX_PER_STATE */
    int32_t ado_width;         /* ADO_WIDTH = baths * matsubaras */
    int32_t ado_depth;         /* hierarchy depth */
    int64_t matrices;          /* NUM_MATRICES (hierarchy nodes) */
    int32_t first_non_plus_id; /* first uid of the last layer */
    const int32_t* baths_coupling; /* [states * baths_per_state], < 0 = none */
    const double* hamiltonian;     /* [states*states*2] J */
    const int32_t* ado_tuples;     /* [matrices * ado_width] */
    const int32_t* ado_plus;       /* [matrices * ado_width] */
    const int32_t* ado_minus;      /* [matrices * ado_width] */
    const double* pf_same_sum;     /* [matrices * 2] */
    const double* pf_same;         /* [baths * 2] */
    const double* pf_circ;         /* [baths * 2] */
    const double* cbk;             /* [baths * matsubaras * 2] */
    const double* cbk_sqrt;        /* [baths * matsubaras] */
} heom_instance_desc;

/* Order of ADOs in device memory. */
#define HEOM_ORDER_LEX 0       /* lexicographic order of the ADO tuples (default) */
#define HEOM_ORDER_REFERENCE 1 /* the reference's uid order */

/* RK4 evaluation schemes for heom_rk4_steps / heom_propagate.  All are the
 * classical 4-stage RK4 (a = 1/2, 1/2, 1; b = 1/6, 1/3, 1/3, 1/6) for the
 * linear, time-independent HEOM operator L; they differ in the order of
 * floating-point operations and in HBM traffic per step:
 *   REFERENCE: four pure derivative evaluations + rk_weighted_add, as the
 *              reference runs them (23 state passes per step)
 *   HORNER:    y + hL(y + h/2 L(y + h/3 L(y + h/4 L y)))       (11 passes)
 *   PRODUCT:   prod_k (I - hL/r_k) y over the four complex roots r_k of
 *              1 + z + z^2/2 + z^3/6 + z^4/24                     (8 passes) */
#define HEOM_RK4_REFERENCE 0
#define HEOM_RK4_HORNER 1
#define HEOM_RK4_PRODUCT 2

typedef struct heom_options {
    int32_t device;      /* CUDA device ordinal */
    int32_t ado_order;   /* HEOM_ORDER_* */
    int32_t rk4_scheme;  /* HEOM_RK4_* */
    int32_t use_graphs;  /* capture the per-step launch sequence in a CUDA graph */
} heom_options;

/* heom_solve write modes (heom_ode.cl:416-434). */
#define HEOM_SOLVE_PURE 0        /* out = L(in) */
#define HEOM_SOLVE_ACCUMULATE 1  /* out = L(in); acc = (acc_init ? in : acc) + acc_coeff L(in) */
#define HEOM_SOLVE_SUBDIAGONAL 2 /* acc = in + out_coeff L(in) */

typedef struct heom_handle heom_handle;
typedef struct heom_buffer heom_buffer;

const char* heom_last_error(void);
void heom_default_options(heom_options* opt);

int heom_create(const heom_instance_desc* desc, const heom_options* opt, heom_handle** out);
int heom_destroy(heom_handle* h);

int heom_set_hamiltonian(heom_handle* h, const double* hamiltonian);
int heom_set_mask(heom_handle* h, const uint8_t* mask);
/* The mask with compaction (no counterpart in the reference): masked ADOs are
 * moved behind the active ones in device memory and no stage kernel sweeps
 * them, so a filtered hierarchy costs only its active ADOs.  The active ADOs
 * (and so every observed top) evolve exactly as with heom_set_mask (bit for
 * bit): the reference computes masked ADOs but never reads them.  Masked
 * entries of the state keep the values they had.  The top ADO of every
 * instance must be active.  heom_set_mask returns to the uncompacted mode. */
int heom_set_mask_compact(heom_handle* h, const uint8_t* mask);
/* Host pre-evaluate actions (ode::add_pre_evaluate_action, ode.hpp:57-59,
 * ode.cpp:17-22): fn(user, h, time, step_size, in, out) runs before every
 * heom_solve, in registration order, and may change the handle (say
 * heom_set_hamiltonian); a non-zero return aborts the solve with that code.
 * The stepping calls refuse to run while host actions are registered (their
 * stages never return to the host); heom_set_field is the device-side
 * time dependence they take. */
typedef int (*heom_pre_evaluate_fn)(void* user, heom_handle* h, double time, double step_size,
                                    const heom_buffer* in, heom_buffer* out);
int heom_add_pre_evaluate_action(heom_handle* h, heom_pre_evaluate_fn fn, void* user);
int heom_clear_pre_evaluate_actions(heom_handle* h);

/* Hierarchy arithmetic (hierarchy_arithmetic_*.cl) on whole buffers of the
 * handle, in the reference's operation order; out may alias an input.
 * dot_product writes the element products a * conj(b) (as the reference's
 * kernel); m is a states*states complex matrix in host memory. */
int heom_hierarchy_add(heom_handle* h, const heom_buffer* a, const heom_buffer* b, heom_buffer* out);
int heom_hierarchy_subtract(heom_handle* h, const heom_buffer* a, const heom_buffer* b, heom_buffer* out);
int heom_hierarchy_dot_product(heom_handle* h, const heom_buffer* a, const heom_buffer* b, heom_buffer* out);
int heom_hierarchy_scale(heom_handle* h, const heom_buffer* a, double re, double im, heom_buffer* out);
int heom_hierarchy_mmult_left(heom_handle* h, const heom_buffer* a, const double* m, heom_buffer* out);
int heom_hierarchy_mmult_right(heom_handle* h, const heom_buffer* a, const double* m, heom_buffer* out);

/* Time-dependent Hamiltonian: the e_field pre-evaluate action of the
 * reference (ode::add_pre_evaluate_action, ode.hpp:57-59; e_field.hpp:63-85).
 * While a field is set, every derivative evaluation at time t uses
 *     H(t) = H - E(t) D- - conj(E(t)) D+,
 *     E(t) = sum over the pump and the probe pulse of
 *            efield exp(-(t - time_center)^2 / (2 time_width^2)) exp(i (phase + frequency t)),
 * built on the device before each evaluation (heom_solve: at time + step_size,
 * as the reference's action; the stepping calls: at t, t + dt/2, t + dt of
 * every step, which is then the classical RK4 whatever the handle's scheme).
 * SI units: times in s, frequency in rad/s, the dipole matrices
 * (states*states complex, interleaved) in J per unit field.  The propagation
 * state carries its time (heom_set_time; advanced by every step). */
typedef struct heom_pulse {
    double efield;
    double time_center;
    double time_width;
    double frequency;
    double phase;
} heom_pulse;
int heom_set_field(heom_handle* h, const double* dipole_plus, const double* dipole_minus, const heom_pulse* pump,
                   const heom_pulse* probe);
int heom_clear_field(heom_handle* h);
int heom_set_time(heom_handle* h, double time);
double heom_time(const heom_handle* h);
/* ADOs the stage kernels sweep (heom_matrices without compaction). */
int64_t heom_active_matrices(const heom_handle* h);
/* The current mask (reference uid order, all instances). */
int heom_get_mask(const heom_handle* h, uint8_t* mask);
/* solver_base::update_hierarchy_norm + hierarchy_norm (solver_base.hpp:225-228,
 * 270-273; hierarchy_norm.cl:15-45): norms[u] = sum_ij |sigma_u(i,j)|^2 of the
 * propagation state, in uid order (norms may be NULL).  With threshold >= 0
 * every ADO at or below it whose mask entry is not protected (2) is switched
 * off, as the reference kernel does to its filter (the compaction mode of the
 * handle is kept); threshold < 0 leaves the mask alone. */
int heom_hierarchy_norm(heom_handle* h, double threshold, double* norms);

int heom_buffer_create(heom_handle* h, heom_buffer** out);
/* Buffers may outlive their handle: heom_destroy frees their device memory
 * and detaches them (every later call but heom_buffer_destroy then fails with
 * HEOM_E_ARG); heom_buffer_destroy frees what is left. */
int heom_buffer_destroy(heom_buffer* b);
int heom_buffer_write(heom_handle* h, heom_buffer* b, const double* host_state);
int heom_buffer_read(heom_handle* h, const heom_buffer* b, double* host_state);
size_t heom_buffer_size_byte(const heom_handle* h);

/* One derivative evaluation with the reference's solve() semantics.  time and
 * step_size go to the pre-evaluate actions and place the field of
 * heom_set_field (H at time + step_size, as the reference's e_field action).
 * out or acc may be NULL where the mode does not write them. */
int heom_solve(heom_handle* h, double time, double step_size, const heom_buffer* in,
               heom_buffer* out, double out_coeff, heom_buffer* acc, double acc_coeff,
               int acc_init, int mode);
/* ode::set_flow_buffers (ode.cpp:213-219): while set, every heom_solve adds
 * acc_coeff times the plus term of the derivative to flow_from_above and
 * acc_coeff times the minus term to flow_from_below (heom_ode.cl:436-441,
 * element by element, reference layout in the buffers).  NULL buffers switch
 * tracking off.  (The reference kernel tests NOMA_NUM_ODE_TRACK_FLOWS while its
 * solver defines HEOM_ODE_TRACK_FLOWS; this build tracks whenever the buffers
 * are set.)  While set, heom_rk4_steps and heom_propagate step as the
 * reference's population_dynamics_solver::step_forward does with
 * solver.track_flows (population_dynamics_solver.hpp:236-263): every step
 * zeroes the buffers, then runs the classical RK4 of four pure evaluations and
 * rk_weighted_add (the HEOM_RK4_REFERENCE structure, whatever the handle's
 * scheme), evaluation i adding dt b_i times its terms (b = 1/6, 1/3, 1/3,
 * 1/6); after a call the buffers hold the last step's flows. */
int heom_set_flow_buffers(heom_handle* h, heom_buffer* flow_from_above, heom_buffer* flow_from_below);
/* The hierarchy norm (sum |sigma_ij|^2 per ADO, uid order) of a buffer, as
 * population_dynamics_solver::update_flow_norm takes it of the flow buffers
 * (population_dynamics_solver.hpp:195-200, hierarchy_norm.cl:15-45). */
int heom_buffer_hierarchy_norm(heom_handle* h, const heom_buffer* b, double* norms);
/* out = y + step_size * sum_l coeffs[l] * k[l] (0 <= n <= 7), terms with a zero
 * coefficient skipped, in rk_weighted_add's operation order. */
int heom_weighted_add(heom_handle* h, int n, double step_size, heom_buffer* out,
                      const heom_buffer* y, const double* coeffs, const heom_buffer* const* k);

/* The handle's own propagation state y_n. */
int heom_set_state(heom_handle* h, const double* host_state);
int heom_get_state(heom_handle* h, double* host_state);
int heom_set_top(heom_handle* h, const double* host_top);
int heom_get_top(heom_handle* h, double* host_top);
int heom_state_buffer(heom_handle* h, heom_buffer** view); /* borrowed view of y_n */

/* Advance y_n by steps RK4 steps of size dt. */
int heom_rk4_steps(heom_handle* h, double dt, int64_t steps);
/* Advance y_n by steps RK4 steps, recording the top matrix (states*states
 * complex, interleaved) at t = 0 and after every observe_every steps into
 * host_tops (rows = steps / observe_every + 1).  steps must be a multiple of
 * observe_every.  Tops are gathered on the device and copied back once. */
int heom_propagate(heom_handle* h, double dt, int64_t steps, int64_t observe_every,
                   double* host_tops);
/* Non-blocking variant of heom_rk4_steps: enqueues the work on the handle's
 * stream and returns; heom_synchronize waits for it. */
int heom_rk4_steps_async(heom_handle* h, double dt, int64_t steps);
int heom_synchronize(heom_handle* h);
/* Advance a hierarchy state that the caller keeps in its own device memory by
 * `steps` RK4 steps of size dt, without allocating anything.  No counterpart
 * in the reference.  It is for callers that cannot call cudaMalloc while they
 * step: code living inside another runtime's device-memory arena, or a
 * latency-critical loop that must not take cudaMalloc's implicit device
 * synchronisation.
 *   d_state: device pointer, 16-byte aligned, to matrices * states * states
 *            complex doubles in the reference layout (uid order, row-major,
 *            interleaved re/im); read and overwritten with the result.
 * The handle's tables are used (create the handle beforehand); the stages use
 * the product-form RK4 whatever the handle's scheme.  Handles with a
 * time-dependent field (heom_set_field), flow buffers or host pre-evaluate
 * actions are refused with HEOM_E_UNSUPPORTED: that work needs buffers the
 * static scratch does not hold.  The call runs on the handle's own stream,
 * which does not wait for other streams: finish every write to d_state (for
 * example, synchronise the stream that wrote it) before the call.  Scratch comes from a
 * static device array of 3 x 16 MiB built into the library and held on every
 * GPU that loads it until exit; hierarchies whose state needs more than
 * 16 MiB in the library's layout are rejected with HEOM_E_UNSUPPORTED.  The
 * first call on a device resolves the array's device address: make that first
 * call before any stream capture.  All calls share the array, so calls that
 * overlap on the GPU (other threads, other handles on the same device) race.
 * Blocking: returns once the result is in d_state. */
int heom_rk4_steps_noalloc(heom_handle* h, double* d_state, double dt, int64_t steps);
/* The handle's CUDA stream (a cudaStream_t), for event timing by callers. */
void* heom_stream(heom_handle* h);

/* Instance facts. */
int64_t heom_matrices(const heom_handle* h);
int32_t heom_states(const heom_handle* h);
/* Number of kernel launches this handle has issued (for launch accounting). */
int64_t heom_kernel_launches(const heom_handle* h);

/* ------------------------------------------------------------------------
 * Batches: several hierarchy instances in one handle.  No counterpart in the
 * reference, which propagates one instance per process.
 * ------------------------------------------------------------------------ */

/* Instances that share states, matsubaras, baths, baths_per_state,
 * baths_coupling and the bath tables (pf_same, pf_circ, cbk, cbk_sqrt) but may
 * differ in depth, hierarchy tables, mask and Hamiltonian (the realisations
 * of a static-disorder ensemble, say) are propagated together: every RK4
 * stage is one kernel launch over the ADOs of all instances.  On such a
 * handle every per-handle host array holds the instances back to back in
 * instance order:
 *   states (heom_set_state, heom_get_state, heom_buffer_*):  sum of matrices x states^2 complex
 *   tops (heom_set_top, heom_get_top):                       count x states^2 complex
 *   tops (heom_propagate):                                   rows x count x states^2 complex
 *   Hamiltonians (heom_set_hamiltonian):                     count x states^2 complex
 *   mask (heom_set_mask):                                    sum of matrices
 * heom_matrices gives the total number of ADOs.  A handle made by
 * heom_create is a batch of one.  Fails with HEOM_E_ARG when the instances
 * do not share the above. */
int heom_create_batch(const heom_instance_desc* descs, int32_t count, const heom_options* opt,
                      heom_handle** out);
int32_t heom_instances(const heom_handle* h);
int64_t heom_instance_matrices(const heom_handle* h, int32_t inst);
/* First ADO of the instance in the concatenated state (reference uid order); -1 if out of range. */
int64_t heom_instance_offset(const heom_handle* h, int32_t inst);
int heom_set_instance_hamiltonian(heom_handle* h, int32_t inst, const double* hamiltonian);
int heom_set_instance_top(heom_handle* h, int32_t inst, const double* host_top);
int heom_get_instance_top(heom_handle* h, int32_t inst, double* host_top);

/* Ensembles: instances of any sizes (states, depth, Matsubara terms, baths).
 * Instances that can share a batch handle are grouped into one class (in
 * order of first appearance); each class is a batch handle.  With the product
 * or Horner scheme, 8 or more instances of one such group with at most 8
 * states and one depth (the realisations of a static-disorder ensemble) form
 * a class of their own in the lockstep layout: its state is stored
 * instance-minor, and its handle (heom_ensemble_class) refuses with
 * HEOM_E_UNSUPPORTED the calls that read or write a state in the
 * single-instance layout (heom_set_state, heom_get_state, masks, buffers,
 * flows, a field, the hierarchy norm); the ensemble calls below serve every
 * class.  One RK4 step of
 * the ensemble is one CUDA graph in which the classes' stage launches run as
 * concurrent branches; the grid of every class's stage kernel is chosen by
 * heom_ensemble_autotune, which times candidate shapes on the device (run
 * automatically before the first step unless already done).  Admission
 * computes the device footprint first and fails with HEOM_E_NOMEM, before
 * allocating anything, when it exceeds the device's free memory. */
typedef struct heom_ensemble heom_ensemble;
/* Device bytes an ensemble of these instances would hold (states, stage
 * buffers and tables); host-only, no device needed. */
int heom_ensemble_footprint(const heom_instance_desc* descs, int32_t count, const heom_options* opt,
                            size_t* bytes);
int heom_ensemble_create(const heom_instance_desc* descs, int32_t count, const heom_options* opt,
                         heom_ensemble** out);
int heom_ensemble_destroy(heom_ensemble* e);
int32_t heom_ensemble_instances(const heom_ensemble* e);
int32_t heom_ensemble_classes(const heom_ensemble* e);
/* class of an instance and its index inside that class's batch handle */
int heom_ensemble_locate(const heom_ensemble* e, int32_t inst, int32_t* cls, int32_t* index);
/* borrowed batch handle of a class (valid until heom_ensemble_destroy) */
heom_handle* heom_ensemble_class(heom_ensemble* e, int32_t cls);
int heom_ensemble_set_hamiltonian(heom_ensemble* e, int32_t inst, const double* hamiltonian);
/* Zero the whole hierarchy state of every instance (then set the tops). */
int heom_ensemble_clear(heom_ensemble* e);
int heom_ensemble_set_top(heom_ensemble* e, int32_t inst, const double* host_top);
int heom_ensemble_get_top(heom_ensemble* e, int32_t inst, double* host_top);
/* Time the candidate stage-kernel grids (on the stage buffers, not on the
 * states) and keep the fastest; *best_stage_us (may be NULL) receives the
 * time of one stage of all classes with the chosen grids. */
int heom_ensemble_autotune(heom_ensemble* e, double* best_stage_us);
int heom_ensemble_rk4_steps(heom_ensemble* e, double dt, int64_t steps);
/* As heom_propagate for every instance: host_tops holds rows of
 * heom_ensemble_top_row_len doubles; instance k's top (states_k^2 complex)
 * starts at heom_ensemble_top_offset(e, k) within each row. */
int heom_ensemble_propagate(heom_ensemble* e, double dt, int64_t steps, int64_t observe_every,
                            double* host_tops);
int64_t heom_ensemble_top_row_len(const heom_ensemble* e);
int64_t heom_ensemble_top_offset(const heom_ensemble* e, int32_t inst);
/* kernel launches of all classes, graph nodes counted one by one */
int64_t heom_ensemble_kernel_launches(const heom_ensemble* e);
/* the ensemble's CUDA stream (a cudaStream_t); steps are enqueued on it */
void* heom_ensemble_stream(heom_ensemble* e);

/* ------------------------------------------------------------------------
 * Host set-up: the reference's hierarchy_graph + instance construction
 * (dm-heom/src/heom/hierarchy_graph.cpp:30-181, instance.cpp:25-71,155-273)
 * and config parsing (config.cpp:20-191, population_dynamics_config.cpp).
 * ------------------------------------------------------------------------ */

/* A system in the reference's config units (config.cpp:37-67): energies in
 * cm^-1, bath correlation times invnu in fs, Omega in cm^-1; sites map to
 * states one to one (sites_to_states identity mode).  Converted to SI as in
 * config::post_process (config.cpp:182-191). */
typedef struct heom_system_desc {
    int32_t sites;
    int32_t ado_depth;
    const double* hamiltonian;     /* [sites*sites*2] cm^-1, interleaved re/im */
    int32_t baths;
    int32_t baths_max_per_site;
    const int32_t* baths_coupling; /* [sites * baths_max_per_site], < 0 = none */
    const double* lambda;          /* [baths] cm^-1 */
    const double* invnu;           /* [baths] fs */
    const double* omega;           /* [baths] cm^-1 */
    int32_t matsubaras;            /* includes the k = 0 term, 1..10 */
    double temperature;            /* K */
} heom_system_desc;

typedef struct heom_tables heom_tables;
/* Build the hierarchy graph and the bath tables of a system on the host. */
int heom_tables_build(const heom_system_desc* sys, heom_tables** out);
/* Borrowed view of the tables (valid until heom_tables_free). */
int heom_tables_view(const heom_tables* t, heom_instance_desc* view);
void heom_tables_free(heom_tables* t);
/* heom_tables_build + heom_create. */
int heom_create_from_system(const heom_system_desc* sys, const heom_options* opt, heom_handle** out);

typedef struct heom_config heom_config;
/* Parse and validate a population_dynamics or linear_absorption .cfg file
 * (program.task selects the task's own section: [population_dynamics] or
 * [dipole]). */
int heom_config_load(const char* path, heom_config** out);
void heom_config_free(heom_config* c);
/* Borrowed view of the [system]/[baths] values in config units. */
int heom_config_system(const heom_config* c, heom_system_desc* view);
/* population_dynamics.rho_init as sites*sites*2 interleaved doubles
 * (HEOM_E_ARG for a configuration of another task). */
int heom_config_rho_init(const heom_config* c, double* out);
/* Raw text of "section.key" copied into buf (NUL-terminated). */
int heom_config_get(const heom_config* c, const char* key, char* buf, size_t len);
/* The reference's binary instance file (instance::write_file / read_file,
 * instance.cpp:281-377, format version 1, native byte order): the tables, H
 * and a hierarchy state (NULL: zeros; top_only != 0 stores the top only) at
 * time `time`.  The bath coupling is not part of the format: heom_instance_read
 * takes it (states * baths_per_state, NULL for one bath per state), and
 * heom_tables_state returns the state and time read. */
int heom_instance_write(const heom_tables* t, const double* state, int32_t top_only, double time, const char* path);
int heom_instance_read(const char* path, const int32_t* coupling, heom_tables** out);
int heom_tables_state(const heom_tables* t, double* state, double* time);
/* Mask of a filtering strategy ("none" or "single_excitation",
 * hierarchy_mask.cpp:20-110) for the hierarchy of the tables, written to
 * mask[matrices]. */
int heom_tables_mask(const heom_tables* t, const char* strategy, int64_t first_layer, uint8_t* mask);

/* ------------------------------------------------------------------------
 * Adjoint gradients.  No counterpart in the reference.
 * ------------------------------------------------------------------------ */

/* Loss of a propagation from rho0 (the top ADO; all others zero) by RK4
 * steps of size dt (the product-form scheme):
 *     J = sum_{n=0}^{steps} weights[n] * Re(sum_ij conj(O_ij) rho_n(i,j))
 * with rho_n the top after n steps and O = observable (states^2 complex,
 * interleaved).  heom_adjoint_gradient returns J and its gradients from one
 * forward and one backward sweep (the transposed derivative L^H run backward
 * through the stages, checkpoints every ceil(sqrt(steps)) steps, each
 * segment recomputed from its checkpoint; when those states exceed the
 * memory limit, recursive checkpointing in the states that fit, each step
 * recomputed a few times more -- results are bit-identical either way):
 *   grad_h      [states*states*2]: dJ/dRe H_ij, dJ/dIm H_ij (per cm^-1), every
 *               entry independent (a symmetric coupling perturbation is the
 *               sum of the (i,j) and (j,i) entries)
 *   grad_lambda dJ/dlambda with lambda of every bath moved together (per cm^-1)
 *   grad_gamma  dJ/dgamma with gamma = 1/invnu of every bath moved together (per fs^-1)
 *   grad_rho0   [states*states*2]: dJ/dRe rho0_ij, dJ/dIm rho0_ij
 * Any output pointer may be NULL: the sweep then skips that gradient's
 * accumulation (grad_h: the Z reduction; grad_lambda and grad_gamma both
 * NULL: the bath-derivative terms).  Masks are not supported. */
typedef struct heom_adjoint heom_adjoint;
int heom_adjoint_create(const heom_system_desc* sys, const heom_options* opt, heom_adjoint** out);
/* A batch of K systems that share states, baths and bath parameters (they
 * may differ in H and depth) in one sweep: every array argument and output
 * of heom_adjoint_gradient then holds the K instances back to back (rho0,
 * observable, grad_h, grad_rho0: K x states^2 complex; loss, grad_lambda,
 * grad_gamma: K values, instance k's share of the shared-parameter
 * gradient); weights, dt and steps are common. */
int heom_adjoint_create_batch(const heom_system_desc* systems, int32_t count, const heom_options* opt,
                              heom_adjoint** out);
int32_t heom_adjoint_instances(const heom_adjoint* a);
int heom_adjoint_destroy(heom_adjoint* a);
/* the forward handle (borrowed): tables, stream, launch count */
heom_handle* heom_adjoint_handle(heom_adjoint* a);
int heom_adjoint_gradient(heom_adjoint* a, const double* rho0, const double* observable, const double* weights,
                          double dt, int64_t steps, double* loss, double* grad_h, double* grad_lambda,
                          double* grad_gamma, double* grad_rho0);
int64_t heom_adjoint_kernel_launches(const heom_adjoint* a);
/* Device memory heom_adjoint_gradient may hold for its states (checkpoints,
 * stage inputs, adjoint), in bytes; 0 (the default) = the device's free
 * memory at the call plus what the adjoint already holds.
 * heom_adjoint_recursive_slots: the step-state slots of the last call's
 * recursive checkpointing, 0 when it used the sqrt(steps) layout. */
int heom_adjoint_set_memory_limit(heom_adjoint* a, int64_t bytes);
int64_t heom_adjoint_recursive_slots(const heom_adjoint* a);

/* Adjoint gradients for an ensemble of systems of any sizes (an uneven
 * batch).  No counterpart in the reference.  heom_ensemble_adjoint_gradient
 * groups the systems into classes that share states, baths and bath
 * parameters; within a class it packs instances, smallest first, into groups
 * whose sqrt(steps) checkpoint layout fits in the memory budget (the limit
 * set below, else 85 % of the free device memory) and sweeps every group as
 * one batch adjoint, one group after another.  An instance whose layout alone
 * does not fit is swept alone with recursive checkpointing.  Per-instance
 * arrays hold the instances back to back in instance order: rho0,
 * observable, grad_h, grad_rho0 states_k^2 complex each (instance k starts at
 * complex element heom_ensemble_adjoint_offset(e, k)); loss, grad_lambda,
 * grad_gamma one value each.  weights, dt and steps are common; NULL outputs
 * are skipped as in heom_adjoint_gradient. */
typedef struct heom_ensemble_adjoint heom_ensemble_adjoint;
int heom_ensemble_adjoint_create(const heom_system_desc* systems, int32_t count, const heom_options* opt,
                                 heom_ensemble_adjoint** out);
int heom_ensemble_adjoint_destroy(heom_ensemble_adjoint* e);
int heom_ensemble_adjoint_set_memory_limit(heom_ensemble_adjoint* e, int64_t bytes);
int heom_ensemble_adjoint_gradient(heom_ensemble_adjoint* e, const double* rho0, const double* observable,
                                   const double* weights, double dt, int64_t steps, double* loss, double* grad_h,
                                   double* grad_lambda, double* grad_gamma, double* grad_rho0);
/* groups of the last gradient call; the group of an instance and its
 * recursive-checkpointing slots (0: the sqrt(steps) layout) */
int32_t heom_ensemble_adjoint_groups(const heom_ensemble_adjoint* e);
int heom_ensemble_adjoint_group_of(const heom_ensemble_adjoint* e, int32_t inst, int32_t* group,
                                   int64_t* recursive_slots);
int64_t heom_ensemble_adjoint_offset(const heom_ensemble_adjoint* e, int32_t inst);
int64_t heom_ensemble_adjoint_kernel_launches(const heom_ensemble_adjoint* e);
/* Derivatives of the bath tables (pf_same [baths*2], pf_circ [baths*2],
 * cbk [baths*matsubaras*2], SI units) with respect to theta = 0: lambda of
 * every bath together (per J), theta = 1: gamma = 1/invnu of every bath
 * together (per 1/s).  Host only. */
int heom_bath_derivatives(const heom_system_desc* sys, int32_t theta, double* d_pf_same, double* d_pf_circ,
                          double* d_cbk);

#ifdef __cplusplus
}
#endif
#endif
