// exact_euler.h -- exact Riemann solver of the 1D Euler equations (the normal
// direction of a 2D interface), used by the CUDA kernels (the CPU oracle
// restates it independently in oracle/claw_oracle.cpp).
//
// Method: Toro, Riemann Solvers and Numerical Methods for Fluid Dynamics, 3rd
// ed., Springer 2009, ch. 4: p* is the root of
//     f(p) = f_L(p) + f_R(p) + (u_R - u_L),
// f_K = shock branch (p > p_K) or rarefaction branch (p <= p_K) (eqs. 4.6-4.7,
// derivatives 4.37), found by Newton's method; u* from eq. 4.9; star densities
// from the shock / isentropic relations; the state at x/t = 0 by sampling the
// wave fan (sec. 4.5).  Initial guesses: the adaptive PVRS / two-rarefaction /
// two-shock choice of sec. 9.5.1 ("plain" guess), or a caller-supplied one
// (the learned guess), which is used only if finite and positive.
//
// Stopping rule: each Newton step |f/f'| is compared with tol * p; a step
// below it is the last one (applied, since f and f' are already at hand, which
// leaves p* at machine precision) and is not counted: `iters` counts the
// steps that were needed, so a guess already within tolerance costs none.
//
// Plain C++ with EX_HD on every function, so host code of the library can use
// it too.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define EX_HD __host__ __device__ __forceinline__
#else
#define EX_HD inline
#endif

#ifdef __CUDACC__
#include "claw2_types.cuh"
#endif

namespace exact_euler {

// Powers and square roots.  On the device x^y = exp(y ln x) (x > 0 wherever
// the solver takes a power) and the branch-free claw2::sqrt_nr: CUDA's pow
// handles every sign and integer case of its arguments in code that, inlined
// at the Newton, fan and sampling sites, outgrew the instruction cache of the
// step kernel (whose top stall was instruction fetch); the relative error of
// exp(y ln x) is about |y ln x| ulps, 1e-14 at most for the pressure and
// density ratios met here.  The host keeps the library functions.
EX_HD double ex_pow(double x, double y) {
#ifdef __CUDA_ARCH__
    return exp(y * log(x));
#else
    return pow(x, y);
#endif
}
EX_HD double ex_sqrt(double x) {
#ifdef __CUDA_ARCH__
    return claw2::sqrt_nr(x);
#else
    return sqrt(x);
#endif
}
// 1/x: the branch-free claw2::rcp_nr on the device (quotients in the Newton
// loop and the fan become products with it)
EX_HD double ex_rcp(double x) {
#ifdef __CUDA_ARCH__
    return claw2::rcp_nr(x);
#else
    return 1.0 / x;
#endif
}

struct Gas {
    double g, g1, g2, g3, g4, g5, g6, g7;  // gamma and Toro's constants G1..G7
};

EX_HD Gas make_gas(double gamma) {
    Gas G;
    G.g = gamma;
    G.g1 = (gamma - 1.0) / (2.0 * gamma);
    G.g2 = (gamma + 1.0) / (2.0 * gamma);
    G.g3 = 2.0 * gamma / (gamma - 1.0);
    G.g4 = 2.0 / (gamma - 1.0);
    G.g5 = 2.0 / (gamma + 1.0);
    G.g6 = (gamma - 1.0) / (gamma + 1.0);
    G.g7 = (gamma - 1.0) / 2.0;
    return G;
}

// f_K and f_K' at pressure p (Toro eqs. 4.6, 4.7, 4.37)
EX_HD void prefun(const Gas& G, double p, double rk, double pk, double ck, double& f, double& fd) {
    if (p <= pk) {
        const double prat = p * ex_rcp(pk);
        const double pw = ex_pow(prat, G.g1);
        f = G.g4 * ck * (pw - 1.0);
        fd = pw * ex_rcp(prat * rk * ck);  // (1/(rho c)) * prat^(-g2), with prat^(-g2) = prat^g1 / prat
    } else {
        const double ak = G.g5 * ex_rcp(rk);
        const double bk = G.g6 * pk;
        const double ibp = ex_rcp(bk + p);
        const double qrt = ex_sqrt(ak * ibp);
        f = (p - pk) * qrt;
        fd = (1.0 - 0.5 * (p - pk) * ibp) * qrt;
    }
}

// Adaptive noniterative guess (Toro sec. 9.5.1): PVRS when the pressure ratio
// is small and PVRS stays inside [pmin, pmax], else two-rarefaction (TRRS)
// below pmin or two-shock (TSRS) above.
EX_HD double guess_pvrs(const Gas& G, double rl, double ul, double pl, double cl, double rr, double ur, double pr,
                        double cr) {
    const double cup = 0.25 * (rl + rr) * (cl + cr);
    double ppv = 0.5 * (pl + pr) + 0.5 * (ul - ur) * cup;
    ppv = fmax(0.0, ppv);
    const double pmin = fmin(pl, pr), pmax = fmax(pl, pr);
    // (the pressure ratio pmax / pmin <= 2, compared without the quotient)
    if (pmax <= 2.0 * pmin && pmin <= ppv && ppv <= pmax) return ppv;
    if (ppv < pmin) {
        const double icl = ex_rcp(cl), icr = ex_rcp(cr);
        const double pq = ex_pow(pl * ex_rcp(pr), G.g1);
        const double um = (pq * ul * icl + ur * icr + G.g4 * (pq - 1.0)) * ex_rcp(pq * icl + icr);
        const double ptl = 1.0 + G.g7 * (ul - um) * icl;
        const double ptr = 1.0 + G.g7 * (um - ur) * icr;
        return 0.5 * (pl * ex_pow(ptl, G.g3) + pr * ex_pow(ptr, G.g3));
    }
    const double gel = ex_sqrt(G.g5 * ex_rcp(rl * (G.g6 * pl + ppv)));
    const double ger = ex_sqrt(G.g5 * ex_rcp(rr * (G.g6 * pr + ppv)));
    return (gel * pl + ger * pr - (ur - ul)) * ex_rcp(gel + ger);
}

// true if the data generate vacuum (Toro eq. 4.82)
EX_HD bool vacuum(const Gas& G, double ul, double cl, double ur, double cr) { return G.g4 * (cl + cr) <= ur - ul; }

// Newton iteration for p*; returns p*, u*; `iters` = updates applied.
// p0: starting pressure (<= 0 or non-finite: use the adaptive guess).
EX_HD void star(const Gas& G, double rl, double ul, double pl, double cl, double rr, double ur, double pr, double cr,
                double p0, double tol, int maxit, double& pstar, double& ustar, int& iters) {
    iters = 0;
    if (rl == rr && ul == ur && pl == pr) {
        pstar = pl;
        ustar = ul;
        return;
    }
    double p = p0;
    if (!(p > 0.0) || !(p < 1e300)) p = guess_pvrs(G, rl, ul, pl, cl, rr, ur, pr, cr);
    if (!(p > tol)) p = tol;
    const double du = ur - ul;
    double fl = 0.0, fr = 0.0;
    for (int k = 0; k <= maxit; ++k) {
        double fld, frd;
        prefun(G, p, rl, pl, cl, fl, fld);
        prefun(G, p, rr, pr, cr, fr, frd);
        const double step = (fl + fr + du) * ex_rcp(fld + frd);
        double pn = p - step;
        if (pn < 0.0) pn = tol;
        if (fabs(step) <= tol * p || k == maxit) {
            if (k < maxit) {
                p = pn;
                prefun(G, p, rl, pl, cl, fl, fld);
                prefun(G, p, rr, pr, cr, fr, frd);
            }
            break;
        }
        p = pn;
        ++iters;
    }
    pstar = p;
    ustar = 0.5 * (ul + ur + fr - fl);
}

// Primitive state at x/t = s of the solution with star values (ps, us)
// (Toro sec. 4.5, SAMPLE).  Also returns the star densities and the two
// acoustic wave speeds used by the wave-propagation correction (shock speed,
// or the mean of head and tail speeds of a rarefaction).
struct Fan {
    double rsl, rsr;  // rho*_L, rho*_R
    double s1, s3;    // left / right acoustic wave speeds (the shock speed of a shock)
    double cml, cmr;  // sound speeds behind a left / right rarefaction (0 for a shock)
};

EX_HD Fan fan(const Gas& G, double rl, double ul, double pl, double cl, double rr, double ur, double pr, double cr,
              double ps, double us) {
    Fan F;
    // (exactly 1 for ps equal to the side's pressure, as a quotient would be:
    // the record of two equal states stays the zero-jump shortcut's)
    const double pml = (ps == pl) ? 1.0 : ps * ex_rcp(pl), pmr = (ps == pr) ? 1.0 : ps * ex_rcp(pr);
    if (ps > pl) {
        F.rsl = rl * (pml + G.g6) * ex_rcp(pml * G.g6 + 1.0);
        F.s1 = ul - cl * ex_sqrt(G.g2 * pml + G.g1);
        F.cml = 0.0;
    } else {
        const double pw = ex_pow(pml, 1.0 / G.g);
        F.rsl = rl * pw;
        F.cml = cl * ex_pow(pml, G.g1);
        F.s1 = 0.5 * ((ul - cl) + (us - F.cml));
    }
    if (ps > pr) {
        F.rsr = rr * (pmr + G.g6) * ex_rcp(pmr * G.g6 + 1.0);
        F.s3 = ur + cr * ex_sqrt(G.g2 * pmr + G.g1);
        F.cmr = 0.0;
    } else {
        const double pw = ex_pow(pmr, 1.0 / G.g);
        F.rsr = rr * pw;
        F.cmr = cr * ex_pow(pmr, G.g1);
        F.s3 = 0.5 * ((ur + cr) + (us + F.cmr));
    }
    return F;
}

// Sample at x/t = 0: returns (rho, u, p) and whether the point is left of the contact.
// The shock speeds and the sound speeds behind the rarefactions are the fan's.
EX_HD void sample0(const Gas& G, double rl, double ul, double pl, double cl, double rr, double ur, double pr, double cr,
                   double ps, double us, const Fan& F, double& r, double& u, double& p, bool& left) {
    const double s = 0.0;
    left = s <= us;
    if (left) {
        if (ps <= pl) {
            const double shl = ul - cl;
            if (s <= shl) { r = rl; u = ul; p = pl; return; }
            const double stl = us - F.cml;
            if (s > stl) { r = F.rsl; u = us; p = ps; return; }
            u = G.g5 * (cl + G.g7 * ul + s);
            const double c = G.g5 * (cl + G.g7 * (ul - s));
            const double crat = c * ex_rcp(cl);
            r = rl * ex_pow(crat, G.g4);
            p = pl * ex_pow(crat, G.g3);
        } else {
            const double sl = F.s1;
            if (s <= sl) { r = rl; u = ul; p = pl; }
            else { r = F.rsl; u = us; p = ps; }
        }
    } else {
        if (ps > pr) {
            const double sr = F.s3;
            if (s >= sr) { r = rr; u = ur; p = pr; }
            else { r = F.rsr; u = us; p = ps; }
        } else {
            const double shr = ur + cr;
            if (s >= shr) { r = rr; u = ur; p = pr; return; }
            const double str = us + F.cmr;
            if (s <= str) { r = F.rsr; u = us; p = ps; return; }
            u = G.g5 * (-cr + G.g7 * ur + s);
            const double c = G.g5 * (cr - G.g7 * (ur - s));
            const double crat = c * ex_rcp(cr);
            r = rr * ex_pow(crat, G.g4);
            p = pr * ex_pow(crat, G.g3);
        }
    }
}

// The learned guess's input features and scaling (see pyclaw_b200/learned.py):
// x = (log rho_L/rb, log rho_R/rb, u_L/cb, u_R/cb, log p_L/pb, log p_R/pb) with
// rb = sqrt(rho_L rho_R), pb = sqrt(p_L p_R), cb = sqrt(gamma pb / rb); the
// network predicts y and the guess is p0 * exp(w y), w = J^2/(1+J^2),
// J^2 = (drho/rb)^2 + (dp/pb)^2 + (du/cb)^2, p0 the adaptive guess.
EX_HD void features(const Gas& G, double rl, double ul, double pl, double rr, double ur, double pr, float* x,
                    double& w) {
    const double rb = sqrt(rl * rr), pb = sqrt(pl * pr);
    const double cb = sqrt(G.g * pb / rb);
    const double lr = 0.5 * log(rl / rr), lp = 0.5 * log(pl / pr);
    x[0] = (float)lr;
    x[1] = (float)(-lr);
    x[2] = (float)(ul / cb);
    x[3] = (float)(ur / cb);
    x[4] = (float)lp;
    x[5] = (float)(-lp);
    const double dr = (rr - rl) / rb, dp = (pr - pl) / pb, du = (ur - ul) / cb;
    const double j2 = dr * dr + dp * dp + du * du;
    w = j2 / (1.0 + j2);
}

}  // namespace exact_euler
