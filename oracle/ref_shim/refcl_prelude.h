/* Forced include for compiling the reference's OpenCL kernels as host C++
 * (TEST INFRASTRUCTURE ONLY).  Maps the OpenCL C qualifiers to C++, provides
 * get_global_id()/get_global_size() for a host loop over work-items, and
 * turns the compile-time defines the reference generates per run
 * (dm-heom/include/heom/solver_base.hpp:179-195) into process-wide values
 * set by the host driver before each call. */
#pragma once
#include <cmath>
#include <cstddef>
using std::sqrt;
using std::hypot;

#define __kernel
#define __global
#define __constant static
#define constant static const
#define restrict __restrict

extern thread_local std::size_t refcl_gid;
extern std::size_t refcl_nodes;
static inline std::size_t get_global_id(int d) { return d == 1 ? refcl_gid : 0; }
static inline std::size_t get_global_size(int d) { return d == 0 ? 1 : refcl_nodes; }

extern int refcl_num_states;
extern int refcl_num_matsubaras;
extern int refcl_baths_max_per_state;
extern int refcl_ado_width;
extern int refcl_baths_coupling_storage[1024];
#define NUM_STATES refcl_num_states
#define NUM_MATRICES refcl_nodes
#define NUM_MATSUBARAS refcl_num_matsubaras
#define BATHS_MAX_PER_STATE refcl_baths_max_per_state
#define ADO_WIDTH refcl_ado_width
/* "__constant const int BATHS_COUPLING[] = BATHS_COUPLING_LIST;" becomes a
 * pointer to the run-time coupling table. */
#define BATHS_COUPLING (*refcl_baths_coupling)
#define BATHS_COUPLING_LIST (reinterpret_cast<const int(*)[]>(refcl_baths_coupling_storage))
