// claw2_types.cuh -- plain-old-data types shared by the kernels and the C-ABI.
#pragma once

#include <cstdint>

#include "../../include/claw2.h"

namespace claw2 {

// Riemann-solver parameters (the reference's Fortran COMMON /cparam/,
// src/pyclaw/state.py:206-231), passed by value into every launch.
struct RPParams {
    double c[CLAW2_MAX_PARAMS];
    int flags;  // solver switch, e.g. the entropy fix of the Roe solvers
};

// Method switches (src/pyclaw/classic/solver.py:173-193: method(2), method(3))
// and the per-wave limiter codes (mthlim, limiter.f90 / philim.f90).
struct Method {
    int order;       // 1 = Godunov, 2 = high-resolution corrections
    int transverse;  // 0 none, 1 increment waves, 2 increment + correction waves
    int fwave;       // 1 if waves are f-waves (sign(s) instead of |s| in cqxx)
    int mthlim[CLAW2_MAX_WAVES];
};

// Device grid layout: structure-of-arrays planes, one per component.
// Element (m, c, r) with padded column c in [0, mx+4) and padded row r in
// [0, my+4) is at base[m * plane + r * pitch + c].  Padded index = Fortran
// index + 1 (num_ghost = 2): padded 0,1 are the lower ghost cells.
struct Layout {
    int mx, my;       // interior cells
    int pitch;        // doubles per row (>= mx + 4, multiple of 32)
    long long plane;  // doubles per component plane
};

// 1/a by Newton-Raphson refinement of PTX's approximate reciprocal
// (rcp.approx.ftz.f64): two steps of x <- x + x (1 - a x), each with the
// residual 1 - a x formed by one fused multiply-add, so the relative error
// squares per step (Newton's method for f(x) = 1/x - a; Markstein, IBM J.
// Res. Dev. 34 (1990) 111-119).  Not correctly rounded: within 1 ulp of the
// IEEE quotient (claw2_selftest_rcp).  Outside [1e-300, 1e300] in magnitude,
// where the approximation flushes or overflows, the IEEE division is used.
// Used for the limiter ratio and the reciprocal densities of the Roe solvers,
// whose results the parity tests hold to 1e-12 of the oracle's IEEE divisions.
__device__ __forceinline__ double rcp_nr(double a) {
    const double aa = fabs(a);
    if (!(aa > 1e-300 && aa < 1e300)) return 1.0 / a;
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(a));
    double e = fma(-a, r, 1.0);
    r = fma(r, e, r);
    e = fma(-a, r, 1.0);
    return fma(r, e, r);
}

}  // namespace claw2
