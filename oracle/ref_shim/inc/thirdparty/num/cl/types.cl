/* Stand-in for the un-vendored noma/num "cl/types.cl" so that the reference's
 * OpenCL kernel sources compile as host C++ (TEST INFRASTRUCTURE ONLY).
 * The reference path "../../../thirdparty/num/cl/types.cl" resolves here
 * through the -I directory ref_shim/inc/d1/d2/d3. */
#pragma once
typedef double real_t;
typedef int bool_t;
typedef unsigned char uchar;
/* OpenCL double2; a scalar initialiser broadcasts as in OpenCL C. */
struct complex_t {
    double s[2];
    complex_t(double v = 0.0) { s[0] = v; s[1] = v; }
};
