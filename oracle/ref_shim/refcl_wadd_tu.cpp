/* Compiles the reference kernel dm-heom/cl/heom/rk_weighted_add.cl
 * unmodified.  TEST INFRASTRUCTURE ONLY. */
#include "refcl_prelude.h"
#include "rk_weighted_add.cl"
