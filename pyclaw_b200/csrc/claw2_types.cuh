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
// IEEE quotient (claw2_selftest_rcp).  No branch: +-0, +-inf and NaN, whose
// residual is NaN, return the approximation itself (+-inf, +-0, NaN: the IEEE
// results); magnitudes outside the normal range are flushed like the
// approximation's (|a| < 2^-1022 gives +-inf, |a| > 2^1022 gives +-0).
// A range test with an IEEE-division fallback cost 12% of the fused step at
// 1024^2 Euler (the branch splits every Roe solve and limiter into blocks).
// Used for the limiter ratio and the reciprocal densities of the Roe solvers,
// whose results the parity tests hold to 1e-12 of the oracle's IEEE divisions.
__device__ __forceinline__ double rcp_nr(double a) {
    double r0;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r0) : "d"(a));
    double e = fma(-a, r0, 1.0);
    double r = fma(r0, e, r0);
    e = fma(-a, r, 1.0);
    r = fma(r, e, r);
    return (e == e) ? r : r0;
}

// sqrt(x) by Goldschmidt's coupled iteration from PTX's approximate
// reciprocal square root y ~ 1/sqrt(x) (rsqrt.approx.ftz.f64): g = x y ~
// sqrt(x) and h = y/2 are refined together, g <- g + g r, h <- h + h r with
// r = 1/2 - g h, twice; a last step adds the residual x - g^2 times h
// (Goldschmidt 1964; P. Markstein, IA-64 and Elementary Functions, 2000,
// ch. 9).  Within 1 ulp of the IEEE square root (claw2_selftest_sqrt).  No
// branch: +-0 and +inf, whose iterate is NaN, return x; negative arguments
// and NaN return NaN; subnormal arguments, flushed by the approximation,
// return x (the root of the flushed value being 0).  Used where the solvers
// take square roots per cell or per interface (sqrt(rho), sound speeds).
__device__ __forceinline__ double sqrt_nr(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double g = x * y, h = 0.5 * y;
    double r = fma(-g, h, 0.5);
    g = fma(g, r, g);
    h = fma(h, r, h);
    r = fma(-g, h, 0.5);
    g = fma(g, r, g);
    h = fma(h, r, h);
    const double e = fma(-g, g, x);
    g = fma(e, h, g);
    return (g == g) ? g : (x >= 0.0 ? x : g);
}

// 1/sqrt(x) by two Newton steps y <- y + (y/2)(1 - x y^2) on Newton's method
// for f(y) = 1/y^2 - x, from rsqrt.approx.ftz.f64 (the residual by one fused
// multiply-add).  Within 2 ulps of the IEEE 1.0 / sqrt(x) (claw2_selftest_rsqrt).
// No branch: +-0, +inf and NaN, whose residual is NaN, return the
// approximation itself (+-inf, +0, NaN); subnormal arguments flush to +inf.
// Used for the reciprocal sound speed of the Roe averages.
__device__ __forceinline__ double rsqrt_nr(double x) {
    double y0;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(x));
    double t = x * y0;
    double e = fma(-t, y0, 1.0);
    double y = fma(0.5 * y0, e, y0);
    t = x * y;
    e = fma(-t, y, 1.0);
    y = fma(0.5 * y, e, y);
    return (y == y) ? y : y0;
}

}  // namespace claw2
