/* One translation unit that compiles the reference kernel
 * dm-heom/cl/heom/heom_ode.cl unmodified (found on the -I path) under the
 * name given by -Dheom_ode=..., with the write mode chosen by
 * -DNOMA_NUM_ODE_ACCUMULATE / -DNOMA_NUM_ODE_SUBDIAGONAL.
 * TEST INFRASTRUCTURE ONLY. */
#include "refcl_prelude.h"
#include "heom_ode.cl"
