// riemann.cuh -- pointwise device Riemann solvers for the classic 2D step.
//
// The reference calls Riemann solvers through the Fortran slice ABI
// rpn2(ixy,maxm,meqn,mwaves,maux,mbc,mx,ql,qr,auxl,auxr,wave,s,amdq,apdq) and
// rpt2(ixy,imp,...,asdq,bmasdq,bpasdq) (call sites src/pyclaw/classic/flux2.f90:101,
// 181, 194).  Here each solver is a struct of inline functions for ONE
// interface, with the direction (ixy) and the system size as compile-time
// constants so everything stays in registers:
//
//   prepare(q, p, c)            per-cell quantities (velocities, pressure,
//                               sqrt(density), sound speed ...) computed once
//                               per cell instead of once per interface side;
//                               c[0..MEQN) is q itself
//   solve<IXY>(cL, cR, p, f, amdq, apdq)
//                               rpn2: wave strengths + Roe state into the
//                               compact interface record f, and the
//                               fluctuations A-dq, A+dq (entropy fix included)
//   speeds<IXY>(f, p, s)        the wave speeds
//   waves<IXY>(f, p, w)         the waves, rebuilt from f (strength x eigenvector)
//   rpt2<IXY>(f, p, asdq, bm, bp)
//                               transverse split of asdq at the same Roe state,
//                               summed in eigen-coefficient form
//
// cL is the cell below/left of the interface, cR above/right.  Reusing the
// interface's Roe state in rpt2 is the reuse the reference's
// development/rp_approaches/report.tex:37-39 measures as a 10% gain.
//
// The formulas are the published ones (LeVeque, Finite Volume Methods for
// Hyperbolic Problems, 2002: advection sec. 20.5, acoustics sec. 18.2/21.7,
// Roe Euler sec. 15.3 and 18.8, Roe shallow water sec. 15.3, Harten-Hyman
// entropy fix sec. 15.3.5, transverse solvers sec. 21.6).  They equal the CPU
// oracle's (which keeps the reference's operation order) up to rounding:
// Roe averages are formed with one reciprocal and per-cell velocities, and
// 1/a comes from rsqrt.
#pragma once

#include "claw2_types.cuh"
#include "exact_euler.h"

namespace claw2 {

template <int IXY>
struct Dir {
    static constexpr int MU = (IXY == 1) ? 1 : 2;  // normal momentum component
    static constexpr int MV = (IXY == 1) ? 2 : 1;  // transverse momentum component
};

// Sum s*w over waves into amdq (s < 0) and apdq (s >= 0): no entropy fix.
template <int ME, int MW>
__device__ __forceinline__ void split_fluct(const double (&s)[MW], const double (&w)[MW][ME], double (&amdq)[ME],
                                            double (&apdq)[ME]) {
#pragma unroll
    for (int m = 0; m < ME; ++m) {
        double am = 0.0, ap = 0.0;
#pragma unroll
        for (int k = 0; k < MW; ++k) {
            if (s[k] < 0.0) am = am + s[k] * w[k][m];
            else ap = ap + s[k] * w[k][m];
        }
        amdq[m] = am;
        apdq[m] = ap;
    }
}

// One wave family K, rebuilt from the compact interface record.
template <class RP, int IXY, int K>
__device__ __forceinline__ void wave_k(const typename RP::Iface& f, const RPParams& p, double (&w)[RP::MEQN]) {
    double all[RP::MWAVES][RP::MEQN];
    RP::template waves<IXY>(f, p, all);
#pragma unroll
    for (int m = 0; m < RP::MEQN; ++m) w[m] = all[K][m];
}

// ---------------------------------------------------------------------------
// advection_2D: cparam = {u, v}
// ---------------------------------------------------------------------------
struct RPAdvection {
    static constexpr int MEQN = 1, MWAVES = 1, NC = 1, ID = CLAW2_RP_ADVECTION;
    struct Iface { double alpha[1]; };
    __device__ __forceinline__ static void prepare(const double (&q)[MEQN], const RPParams&, double (&c)[NC]) {
        c[0] = q[0];
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface&, const RPParams& p, double (&s)[MWAVES]) {
        s[0] = (IXY == 1) ? p.c[0] : p.c[1];
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams&, double (&w)[MWAVES][MEQN]) {
        w[0][0] = f.alpha[0];
    }
    template <int IXY>
    __device__ __forceinline__ static void zero_iface(const double (&)[NC], const double (&)[NC], const RPParams&,
                                                      Iface& f) {
        f.alpha[0] = 0.0;
    }
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        const double vel = (IXY == 1) ? p.c[0] : p.c[1];
        f.alpha[0] = cR[0] - cL[0];
        amdq[0] = fmin(vel, 0.0) * f.alpha[0];
        apdq[0] = fmax(vel, 0.0) * f.alpha[0];
    }
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Iface&, const RPParams& p, const double (&asdq)[MEQN],
                                                double (&bm)[MEQN], double (&bp)[MEQN]) {
        const double stran = (IXY == 1) ? p.c[1] : p.c[0];
        bm[0] = fmin(stran, 0.0) * asdq[0];
        bp[0] = fmax(stran, 0.0) * asdq[0];
    }
};

// ---------------------------------------------------------------------------
// acoustics_2D: cparam = {rho, bulk, cc, zz}; q = (p, u, v)
// Eigenvectors (-Z, 1, 0) at speed -c and (Z, 1, 0) at speed c.
// ---------------------------------------------------------------------------
struct RPAcoustics {
    static constexpr int MEQN = 3, MWAVES = 2, NC = 3, ID = CLAW2_RP_ACOUSTICS;
    struct Iface { double alpha[2]; };
    __device__ __forceinline__ static void prepare(const double (&q)[MEQN], const RPParams&, double (&c)[NC]) {
        c[0] = q[0]; c[1] = q[1]; c[2] = q[2];
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface&, const RPParams& p, double (&s)[MWAVES]) {
        s[0] = -p.c[2];
        s[1] = p.c[2];
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams& p, double (&w)[MWAVES][MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double zz = p.c[3];
        w[0][0] = -f.alpha[0] * zz; w[0][MU] = f.alpha[0]; w[0][MV] = 0.0;
        w[1][0] = f.alpha[1] * zz;  w[1][MU] = f.alpha[1]; w[1][MV] = 0.0;
    }
    template <int IXY>
    __device__ __forceinline__ static void zero_iface(const double (&)[NC], const double (&)[NC], const RPParams&,
                                                      Iface& f) {
        f.alpha[0] = f.alpha[1] = 0.0;
    }
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double cc = p.c[2], zz = p.c[3];
        const double delta1 = cR[0] - cL[0];
        const double delta2 = cR[MU] - cL[MU];
        const double i2z = rcp_nr(2.0 * zz);
        const double a1 = (-delta1 + zz * delta2) * i2z;
        const double a2 = (delta1 + zz * delta2) * i2z;
        f.alpha[0] = a1;
        f.alpha[1] = a2;
        amdq[0] = -cc * (-a1 * zz); amdq[MU] = -cc * a1; amdq[MV] = 0.0;
        apdq[0] = cc * (a2 * zz);   apdq[MU] = cc * a2;  apdq[MV] = 0.0;
    }
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Iface&, const RPParams& p, const double (&asdq)[MEQN],
                                                double (&bm)[MEQN], double (&bp)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double cc = p.c[2], zz = p.c[3];
        const double i2z = rcp_nr(2.0 * zz);
        const double a1 = (-asdq[0] + zz * asdq[MV]) * i2z;
        const double a2 = (asdq[0] + zz * asdq[MV]) * i2z;
        bm[0] = cc * a1 * zz; bm[MU] = 0.0; bm[MV] = -cc * a1;
        bp[0] = cc * a2 * zz; bp[MU] = 0.0; bp[MV] = cc * a2;
    }
};

// ---------------------------------------------------------------------------
// euler_4wave_2D (Roe): cparam = {gamma, efix}; q = (rho, rho u, rho v, E)
// Waves: 1 = u-c acoustic, 2 = entropy (u), 3 = shear (u), 4 = u+c acoustic.
// Cell: q, sqrt(rho), u, v, H = (E + p)/rho, c = sqrt(gamma p / rho).
// Iface: strengths in wave order + Roe state (normal u, transverse v, a, 1/a, H).
// ---------------------------------------------------------------------------
struct RPEulerRoe {
    static constexpr int MEQN = 4, MWAVES = 4, NC = 9, ID = CLAW2_RP_EULER_ROE;
    enum { RS = 4, UX = 5, UY = 6, HH = 7, CS = 8 };
    struct Iface { double alpha[4]; double u, v, a, ia, H; };

    __device__ __forceinline__ static void prepare(const double (&q)[MEQN], const RPParams& p, double (&c)[NC]) {
        const double gamma = p.c[0], gamma1 = gamma - 1.0;
        const double irho = rcp_nr(q[0]);
        const double u = q[1] * irho, v = q[2] * irho;
        const double pr = gamma1 * (q[3] - 0.5 * (q[1] * u + q[2] * v));
        c[0] = q[0]; c[1] = q[1]; c[2] = q[2]; c[3] = q[3];
        c[RS] = sqrt_nr(q[0]);
        c[UX] = u;
        c[UY] = v;
        c[HH] = (q[3] + pr) * irho;
        c[CS] = sqrt_nr(gamma * pr * irho);
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface& f, const RPParams&, double (&s)[MWAVES]) {
        s[0] = f.u - f.a;
        s[1] = f.u;
        s[2] = f.u;
        s[3] = f.u + f.a;
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams&, double (&w)[MWAVES][MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double u = f.u, v = f.v, a = f.a, H = f.H;
        const double b1 = f.alpha[0], b3 = f.alpha[1], b2 = f.alpha[2], b4 = f.alpha[3];
        w[0][0] = b1; w[0][MU] = b1 * (u - a); w[0][MV] = b1 * v; w[0][3] = b1 * (H - u * a);
        w[1][0] = b3; w[1][MU] = b3 * u; w[1][MV] = b3 * v; w[1][3] = b3 * 0.5 * (u * u + v * v);
        w[2][0] = 0.0; w[2][MU] = 0.0; w[2][MV] = b2; w[2][3] = b2 * v;
        w[3][0] = b4; w[3][MU] = b4 * (u + a); w[3][MV] = b4 * v; w[3][3] = b4 * (H + u * a);
    }

    // Roe averages with weights sqrt(rho) / (sqrt(rho_L) + sqrt(rho_R)): the
    // record's u, v, H, a, 1/a (everything but the wave strengths)
    template <int IXY>
    __device__ __forceinline__ static void roe_state(const double (&cL)[NC], const double (&cR)[NC],
                                                     const RPParams& p, Iface& f) {
        constexpr int UN = (IXY == 1) ? UX : UY, UT = (IXY == 1) ? UY : UX;
        // explicit roundings: the record comes out bit for bit the same in
        // every kernel that inlines this (the zero-jump shortcut and the full
        // solve build it in different places), whatever the contraction
        const double gamma1 = p.c[0] - 1.0;
        const double inv = rcp_nr(__dadd_rn(cL[RS], cR[RS]));
        const double wl = __dmul_rn(cL[RS], inv), wr = __dmul_rn(cR[RS], inv);
        const double u = __fma_rn(wl, cL[UN], __dmul_rn(wr, cR[UN]));
        const double v = __fma_rn(wl, cL[UT], __dmul_rn(wr, cR[UT]));
        const double H = __fma_rn(wl, cL[HH], __dmul_rn(wr, cR[HH]));
        const double a2 = __dmul_rn(gamma1, __fma_rn(-0.5, __fma_rn(u, u, __dmul_rn(v, v)), H));
        const double ia = rsqrt_nr(a2);
        f.u = u; f.v = v; f.H = H; f.a = __dmul_rn(a2, ia); f.ia = ia;
    }
    // The record of an interface whose two cells are equal: every strength is
    // zero (the jump is), the Roe state is solve's, so the speeds are too.
    template <int IXY>
    __device__ __forceinline__ static void zero_iface(const double (&cL)[NC], const double (&cR)[NC],
                                                      const RPParams& p, Iface& f) {
        roe_state<IXY>(cL, cR, p, f);
        f.alpha[0] = f.alpha[1] = f.alpha[2] = f.alpha[3] = 0.0;
    }

    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        constexpr int UN = (IXY == 1) ? UX : UY;
        const double gamma = p.c[0], gamma1 = gamma - 1.0;
        roe_state<IXY>(cL, cR, p, f);
        const double u = f.u, v = f.v, H = f.H, a = f.a, ia = f.ia;
        const double u2v2 = u * u + v * v;
        const double g1a2 = gamma1 * ia * ia;
        const double euv = H - u2v2;
        const double d0 = cR[0] - cL[0], d1 = cR[MU] - cL[MU], d2 = cR[MV] - cL[MV], d3 = cR[3] - cL[3];
        const double b3 = g1a2 * (euv * d0 + u * d1 + v * d2 - d3);
        const double b2 = d2 - v * d0;
        const double b4 = (d1 + (a - u) * d0 - a * b3) * (0.5 * ia);
        const double b1 = d0 - b3 - b4;
        f.alpha[0] = b1; f.alpha[1] = b3; f.alpha[2] = b2; f.alpha[3] = b4;

        double w[MWAVES][MEQN], s[MWAVES];
        waves<IXY>(f, p, w);
        speeds<IXY>(f, p, s);
        if (p.flags == 0) {
            split_fluct<MEQN, MWAVES>(s, w, amdq, apdq);
            return;
        }
        // Harten-Hyman entropy fix (branch structure of the oracle)
        bool done = false;
        {
            const double s0 = cL[UN] - cL[CS];  // u - c in the left state
            if (s0 >= 0.0 && s[0] > 0.0) {
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = 0.0;
                done = true;
            } else {
                const double rho1 = cL[0] + w[0][0];
                const double rhou1 = cL[MU] + w[0][MU];
                const double rhov1 = cL[MV] + w[0][MV];
                const double en1 = cL[3] + w[0][3];
                const double ir1 = rcp_nr(rho1);
                const double p1 = gamma1 * (en1 - 0.5 * (rhou1 * rhou1 + rhov1 * rhov1) * ir1);
                const double s1 = rhou1 * ir1 - sqrt_nr(gamma * p1 * ir1);  // u - c right of the 1-wave
                double sfract;
                if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s[0]) * rcp_nr(s1 - s0);
                else if (s[0] < 0.0) sfract = s[0];
                else sfract = 0.0;
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = sfract * w[0][m];
            }
        }
        if (!done && !(s[1] >= 0.0)) {
#pragma unroll
            for (int m = 0; m < MEQN; ++m) amdq[m] = amdq[m] + s[1] * w[1][m] + s[2] * w[2][m];
            const double s3 = cR[UN] + cR[CS];  // u + c in the right state
            const double rho2 = cR[0] - w[3][0];
            const double rhou2 = cR[MU] - w[3][MU];
            const double rhov2 = cR[MV] - w[3][MV];
            const double en2 = cR[3] - w[3][3];
            const double ir2 = rcp_nr(rho2);
            const double p2 = gamma1 * (en2 - 0.5 * (rhou2 * rhou2 + rhov2 * rhov2) * ir2);
            const double s2 = rhou2 * ir2 + sqrt_nr(gamma * p2 * ir2);  // u + c left of the 4-wave
            double sfract = 0.0;
            bool add = true;
            if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - s[3]) * rcp_nr(s3 - s2);
            else if (s[3] < 0.0) sfract = s[3];
            else add = false;
            if (add) {
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = amdq[m] + sfract * w[3][m];
            }
        }
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            double df = 0.0;
#pragma unroll
            for (int k = 0; k < MWAVES; ++k) df = df + s[k] * w[k][m];
            apdq[m] = df - amdq[m];
        }
    }

    // Transverse eigenvectors at the Roe state (v is now the "normal" speed):
    // r1 = (1, u, v-a, H-va), r2 = (1, u, v, |u|^2/2), r3 = (0, 1, 0, u), r4 = (1, u, v+a, H+va);
    // B-dq = sum min(s_k,0) b_k r_k, B+dq = sum max(s_k,0) b_k r_k.
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Iface& f, const RPParams& p, const double (&asdq)[MEQN],
                                                double (&bm)[MEQN], double (&bp)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double gamma1 = p.c[0] - 1.0;
        const double u = f.u, v = f.v, a = f.a, H = f.H;
        const double u2v2 = u * u + v * v;
        const double g1a2 = gamma1 * f.ia * f.ia;
        const double euv = H - u2v2;
        const double b3 = g1a2 * (euv * asdq[0] + u * asdq[MU] + v * asdq[MV] - asdq[3]);
        const double b2 = asdq[MU] - u * asdq[0];
        const double b4 = (asdq[MV] + (a - v) * asdq[0] - a * b3) * (0.5 * f.ia);
        const double b1 = asdq[0] - b3 - b4;
        const double s1 = v - a, s4 = v + a;
        const double m1 = fmin(s1, 0.0) * b1, m3 = fmin(v, 0.0) * b3, m2 = fmin(v, 0.0) * b2, m4 = fmin(s4, 0.0) * b4;
        const double p1 = fmax(s1, 0.0) * b1, p3 = fmax(v, 0.0) * b3, p2 = fmax(v, 0.0) * b2, p4 = fmax(s4, 0.0) * b4;
        const double va = v * a, hke = 0.5 * u2v2;
        double sm = m1 + m3 + m4, sp = p1 + p3 + p4;
        bm[0] = sm;
        bm[MU] = u * sm + m2;
        bm[MV] = v * sm + a * (m4 - m1);
        bm[3] = H * (m1 + m4) + va * (m4 - m1) + hke * m3 + u * m2;
        bp[0] = sp;
        bp[MU] = u * sp + p2;
        bp[MV] = v * sp + a * (p4 - p1);
        bp[3] = H * (p1 + p4) + va * (p4 - p1) + hke * p3 + u * p2;
    }
};

// ---------------------------------------------------------------------------
// shallow_hlle_2D: cparam = {grav}; q = (h, hu, hv).  Two waves through the
// HLL middle state q_m = (f(q_R) - f(q_L) - s2 q_R + s1 q_L) / (s1 - s2) with
// Einfeldt's speeds s1 = min(u_L - c_L, u_hat - c_hat), s2 = max(u_R + c_R,
// u_hat + c_hat), u_hat the Roe velocity, c_hat = sqrt(g (h_L + h_R) / 2)
// (Harten, Lax & van Leer 1983; Einfeldt 1988).  No transverse solve (split
// step or transverse_waves = 0; the host rejects anything else).
// Cell: q, sqrt(h), u, v, c = sqrt(g h).
// ---------------------------------------------------------------------------
struct RPShallowHLLE {
    static constexpr int MEQN = 3, MWAVES = 2, NC = 7, ID = CLAW2_RP_SHALLOW_HLLE;
    enum { RS = 3, UX = 4, UY = 5, CS = 6 };
    struct Iface { double w[2][3]; double s1, s2; };  // waves as (h, normal, transverse)

    __device__ __forceinline__ static void prepare(const double (&q)[MEQN], const RPParams& p, double (&c)[NC]) {
        c[0] = q[0]; c[1] = q[1]; c[2] = q[2];
        c[RS] = sqrt(q[0]);
        c[UX] = q[1] / q[0];
        c[UY] = q[2] / q[0];
        c[CS] = sqrt(p.c[0] * q[0]);
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface& f, const RPParams&, double (&s)[MWAVES]) {
        s[0] = f.s1;
        s[1] = f.s2;
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams&, double (&w)[MWAVES][MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            w[k][0] = f.w[k][0];
            w[k][MU] = f.w[k][1];
            w[k][MV] = f.w[k][2];
        }
    }
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        constexpr int UN = (IXY == 1) ? UX : UY, UT = (IXY == 1) ? UY : UX;
        const double g = p.c[0];
        const double hl = cL[0], hr = cR[0], hul = cL[MU], hur = cR[MU], hvl = cL[MV], hvr = cR[MV];
        const double ul = cL[UN], ur = cR[UN], vl = cL[UT], vr = cR[UT];
        const double u_hat = (cL[RS] * ul + cR[RS] * ur) / (cL[RS] + cR[RS]);
        const double c_hat = sqrt(0.5 * g * (hl + hr));
        const double s1 = fmin(ul - cL[CS], u_hat - c_hat);
        const double s2 = fmax(ur + cR[CS], u_hat + c_hat);
        const double den = s1 - s2;
        const double hm = (hur - hul - s2 * hr + s1 * hl) / den;
        const double hum = (hur * ur + 0.5 * g * hr * hr - hul * ul - 0.5 * g * hl * hl - s2 * hur + s1 * hul) / den;
        const double hvm = (hur * vr - hul * vl - s2 * hvr + s1 * hvl) / den;
        f.w[0][0] = hm - hl; f.w[0][1] = hum - hul; f.w[0][2] = hvm - hvl;
        f.w[1][0] = hr - hm; f.w[1][1] = hur - hum; f.w[1][2] = hvr - hvm;
        f.s1 = s1;
        f.s2 = s2;
        double w[MWAVES][MEQN];
        waves<IXY>(f, p, w);
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            amdq[m] = fmin(s1, 0.0) * w[0][m] + fmin(s2, 0.0) * w[1][m];
            apdq[m] = fmax(s1, 0.0) * w[0][m] + fmax(s2, 0.0) * w[1][m];
        }
    }
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Iface&, const RPParams&, const double (&)[MEQN],
                                                double (&bm)[MEQN], double (&bp)[MEQN]) {
#pragma unroll
        for (int m = 0; m < MEQN; ++m) bm[m] = bp[m] = 0.0;  // unreachable: the host rejects transverse solves
    }
};

// ---------------------------------------------------------------------------
// euler_5wave_2D: the Roe solver above with a passive tracer as fifth
// component (development/rp_approaches/rpn2_euler_5wave.f,
// rpt2_euler_5wave.f): the tracer jump is a fifth wave moving at the Roe
// normal velocity, in the transverse split at the Roe transverse velocity;
// the entropy fix treats it with the contact.  cparam = {gamma, efix}.
// Cell: the Euler cell, then the tracer.  The Euler parts run the 4-wave code.
// ---------------------------------------------------------------------------
struct RPEuler5 {
    using E = RPEulerRoe;
    // cell: q (the kernels read q from the first MEQN slots), then the Euler
    // cell's derived fields; ecell() rebuilds the Euler cell's layout
    static constexpr int MEQN = 5, MWAVES = 5, NC = E::NC + 1, ID = CLAW2_RP_EULER_5WAVE;
    struct Iface { E::Iface e; double dtr; };

    __device__ __forceinline__ static void ecell(const double (&c)[NC], double (&e)[E::NC]) {
        e[0] = c[0]; e[1] = c[1]; e[2] = c[2]; e[3] = c[3];
#pragma unroll
        for (int k = 4; k < E::NC; ++k) e[k] = c[k + 1];
    }
    __device__ __forceinline__ static void prepare(const double (&q)[MEQN], const RPParams& p, double (&c)[NC]) {
        const double q4[4] = {q[0], q[1], q[2], q[3]};
        double e[E::NC];
        E::prepare(q4, p, e);
        c[0] = e[0]; c[1] = e[1]; c[2] = e[2]; c[3] = e[3];
        c[4] = q[4];
#pragma unroll
        for (int k = 4; k < E::NC; ++k) c[k + 1] = e[k];
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface& f, const RPParams& p, double (&s)[MWAVES]) {
        double s4[4];
        E::template speeds<IXY>(f.e, p, s4);
        s[0] = s4[0]; s[1] = s4[1]; s[2] = s4[2]; s[3] = s4[3];
        s[4] = f.e.u;
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams& p, double (&w)[MWAVES][MEQN]) {
        // families in the 5-wave file's order: acoustic, shear, entropy,
        // acoustic, tracer (the 4-wave code keeps entropy before shear)
        double w4[4][4];
        E::template waves<IXY>(f.e, p, w4);
        constexpr int from[4] = {0, 2, 1, 3};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
#pragma unroll
            for (int m = 0; m < 4; ++m) w[k][m] = w4[from[k]][m];
            w[k][4] = 0.0;
        }
        w[4][0] = w[4][1] = w[4][2] = w[4][3] = 0.0;
        w[4][4] = f.dtr;
    }
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        double am4[4], ap4[4], eL[E::NC], eR[E::NC];
        ecell(cL, eL);
        ecell(cR, eR);
        E::template solve<IXY>(eL, eR, p, f.e, am4, ap4);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            amdq[m] = am4[m];
            apdq[m] = ap4[m];
        }
        // tracer: left-going exactly when the contact is (with or without the fix)
        f.dtr = cR[4] - cL[4];
        const double u = f.e.u;
        amdq[4] = (u < 0.0) ? u * f.dtr : 0.0;
        apdq[4] = (u < 0.0) ? 0.0 : u * f.dtr;
    }
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Iface& f, const RPParams& p, const double (&asdq)[MEQN],
                                                double (&bm)[MEQN], double (&bp)[MEQN]) {
        const double a4[4] = {asdq[0], asdq[1], asdq[2], asdq[3]};
        double bm4[4], bp4[4];
        E::template rpt2<IXY>(f.e, p, a4, bm4, bp4);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            bm[m] = bm4[m];
            bp[m] = bp4[m];
        }
        const double v = f.e.v;
        bm[4] = fmin(v, 0.0) * asdq[4];
        bp[4] = fmax(v, 0.0) * asdq[4];
    }
};

// ---------------------------------------------------------------------------
// shallow_roe_with_efix_2D: cparam = {grav, efix}; q = (h, hu, hv)
// Cell: q, sqrt(h), u, v, c = sqrt(g h).  Iface: strengths + (u, v, a, 1/a).
// ---------------------------------------------------------------------------
struct RPShallowRoe {
    static constexpr int MEQN = 3, MWAVES = 3, NC = 7, ID = CLAW2_RP_SHALLOW_ROE;
    enum { RS = 3, UX = 4, UY = 5, CS = 6 };
    struct Iface { double alpha[3]; double u, v, a, ia; };

    __device__ __forceinline__ static void prepare(const double (&q)[MEQN], const RPParams& p, double (&c)[NC]) {
        const double grav = p.c[0];
        const double ih = rcp_nr(q[0]);
        c[0] = q[0]; c[1] = q[1]; c[2] = q[2];
        c[RS] = sqrt_nr(q[0]);
        c[UX] = q[1] * ih;
        c[UY] = q[2] * ih;
        c[CS] = sqrt_nr(grav * q[0]);
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface& f, const RPParams&, double (&s)[MWAVES]) {
        s[0] = f.u - f.a;
        s[1] = f.u;
        s[2] = f.u + f.a;
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams&, double (&w)[MWAVES][MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double u = f.u, v = f.v, a = f.a;
        const double a1 = f.alpha[0], a2 = f.alpha[1], a3 = f.alpha[2];
        w[0][0] = a1; w[0][MU] = a1 * (u - a); w[0][MV] = a1 * v;
        w[1][0] = 0.0; w[1][MU] = 0.0; w[1][MV] = a2;
        w[2][0] = a3; w[2][MU] = a3 * (u + a); w[2][MV] = a3 * v;
    }

    // Roe averages (velocities weighted by sqrt(h)) and the celerity of the
    // mean depth: the record's u, v, a, 1/a
    template <int IXY>
    __device__ __forceinline__ static void roe_state(const double (&cL)[NC], const double (&cR)[NC],
                                                     const RPParams& p, Iface& f) {
        constexpr int UN = (IXY == 1) ? UX : UY, UT = (IXY == 1) ? UY : UX;
        // explicit roundings (see RPEulerRoe::roe_state)
        const double inv = rcp_nr(__dadd_rn(cL[RS], cR[RS]));
        const double wl = __dmul_rn(cL[RS], inv), wr = __dmul_rn(cR[RS], inv);
        const double gh = __dmul_rn(p.c[0], __dmul_rn(__dadd_rn(cL[0], cR[0]), 0.50));
        const double ia = rsqrt_nr(gh);
        f.u = __fma_rn(wl, cL[UN], __dmul_rn(wr, cR[UN]));
        f.v = __fma_rn(wl, cL[UT], __dmul_rn(wr, cR[UT]));
        f.a = __dmul_rn(gh, ia);
        f.ia = ia;
    }
    // equal cells: zero strengths, solve's Roe state (and so its speeds)
    template <int IXY>
    __device__ __forceinline__ static void zero_iface(const double (&cL)[NC], const double (&cR)[NC],
                                                      const RPParams& p, Iface& f) {
        roe_state<IXY>(cL, cR, p, f);
        f.alpha[0] = f.alpha[1] = f.alpha[2] = 0.0;
    }

    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        constexpr int UN = (IXY == 1) ? UX : UY;
        const double grav = p.c[0];
        roe_state<IXY>(cL, cR, p, f);
        const double u = f.u, v = f.v, a = f.a, ia = f.ia;
        const double d0 = cR[0] - cL[0], d1 = cR[MU] - cL[MU], d2 = cR[MV] - cL[MV];
        f.alpha[0] = ((u + a) * d0 - d1) * (0.50 * ia);
        f.alpha[1] = -v * d0 + d2;
        f.alpha[2] = (-(u - a) * d0 + d1) * (0.50 * ia);

        double w[MWAVES][MEQN], s[MWAVES];
        waves<IXY>(f, p, w);
        speeds<IXY>(f, p, s);
        if (p.flags == 0) {
            split_fluct<MEQN, MWAVES>(s, w, amdq, apdq);
            return;
        }
        bool done = false;
        {
            const double s0 = cL[UN] - cL[CS];
            if (s0 >= 0.0 && s[0] > 0.0) {
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = 0.0;
                done = true;
            } else {
                const double h1 = cL[0] + w[0][0];
                const double hu1 = cL[MU] + w[0][MU];
                const double s1 = hu1 * rcp_nr(h1) - sqrt_nr(grav * h1);  // speed just right of the 1-wave
                double sfract;
                if (s0 < 0.0 && s1 > 0.0) sfract = s0 * ((s1 - s[0]) * rcp_nr(s1 - s0));
                else if (s[0] < 0.0) sfract = s[0];
                else sfract = 0.0;
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = sfract * w[0][m];
            }
        }
        if (!done && !(s[1] > 0.0)) {
#pragma unroll
            for (int m = 0; m < MEQN; ++m) amdq[m] = amdq[m] + s[1] * w[1][m];
            const double s03 = cR[UN] + cR[CS];
            const double h3 = cR[0] - w[2][0];
            const double hu3 = cR[MU] - w[2][MU];
            const double s3 = hu3 * rcp_nr(h3) + sqrt_nr(grav * h3);  // speed just left of the 3-wave
            double sfract = 0.0;
            bool add = true;
            if (s3 < 0.0 && s03 > 0.0) sfract = s3 * ((s03 - s[2]) * rcp_nr(s03 - s3));
            else if (s[2] < 0.0) sfract = s[2];
            else add = false;
            if (add) {
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = amdq[m] + sfract * w[2][m];
            }
        }
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            double df = 0.0;
#pragma unroll
            for (int k = 0; k < MWAVES; ++k) df = df + s[k] * w[k][m];
            apdq[m] = df - amdq[m];
        }
    }

    // transverse eigenvectors r1 = (1, u, v-c), r2 = (0, 1, 0), r3 = (1, u, v+c)
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Iface& f, const RPParams&, const double (&asdq)[MEQN],
                                                double (&bm)[MEQN], double (&bp)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double u = f.u, v = f.v, a = f.a;
        const double a1 = (0.5 * f.ia) * ((v + a) * asdq[0] - asdq[MV]);
        const double a2 = -u * asdq[0] + asdq[MU];
        const double a3 = (0.5 * f.ia) * (-(v - a) * asdq[0] + asdq[MV]);
        const double s1 = v - a, s3 = v + a;
        const double m1 = fmin(s1, 0.0) * a1, m2 = fmin(v, 0.0) * a2, m3 = fmin(s3, 0.0) * a3;
        const double p1 = fmax(s1, 0.0) * a1, p2 = fmax(v, 0.0) * a2, p3 = fmax(s3, 0.0) * a3;
        bm[0] = m1 + m3;
        bm[MU] = u * (m1 + m3) + m2;
        bm[MV] = v * (m1 + m3) + a * (m3 - m1);
        bp[0] = p1 + p3;
        bp[MU] = u * (p1 + p3) + p2;
        bp[MV] = v * (p1 + p3) + a * (p3 - p1);
    }
};


// ---------------------------------------------------------------------------
// Exact Euler solver (no counterpart in the reference): cparam = {gamma, tol}.
// rpn2: p* by Newton (exact_euler.h) from the adaptive PVRS guess or from a
// per-interface guess (the learned one, computed by k_mlp_guess); three waves
// W1 = Q*L - QL, W2 = Q*R - Q*L (contact and shear), W3 = QR - Q*R with the
// shock speed or the fan's mean speed, and the Godunov fluctuations
// A-dq = F(Q(0)) - F(QL), A+dq = F(QR) - F(Q(0)) from the state at x/t = 0, so
// no entropy fix is needed.  rpt2: the Roe transverse split at the Roe state.
// Data that generate vacuum fall back to the Roe solver for that interface.
// ---------------------------------------------------------------------------
struct RPEulerExact {
    static constexpr int MEQN = 4, MWAVES = 3, NC = 10, ID = CLAW2_RP_EULER_EXACT;
    static constexpr bool USES_GUESS = true, COUNTS = true;
    enum { RS = 4, UX = 5, UY = 6, HH = 7, CS = 8, PP = 9 };
    struct Iface {
        double w[3][4];
        double s[3];
        double u, v, a, ia, H;  // Roe state for rpt2
        int iters;    // Newton steps needed (exact_euler::star's count)
        int applied;  // Newton steps applied: the needed ones plus the final sub-tolerance step
    };

    __device__ __forceinline__ static void prepare(const double (&q)[MEQN], const RPParams& p, double (&c)[NC]) {
        const double gamma = p.c[0], gamma1 = gamma - 1.0;
        // (k_exact_pstar_guess forms these the same way)
        const double irho = rcp_nr(q[0]);
        const double u = q[1] * irho, v = q[2] * irho;
        const double pr = gamma1 * (q[3] - 0.5 * (q[1] * u + q[2] * v));
        c[0] = q[0]; c[1] = q[1]; c[2] = q[2]; c[3] = q[3];
        c[RS] = sqrt_nr(q[0]);
        c[UX] = u;
        c[UY] = v;
        c[HH] = (q[3] + pr) * irho;
        c[CS] = sqrt_nr(gamma * pr * irho);
        c[PP] = pr;
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface& f, const RPParams&, double (&s)[MWAVES]) {
        s[0] = f.s[0]; s[1] = f.s[1]; s[2] = f.s[2];
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams&, double (&w)[MWAVES][MEQN]) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int m = 0; m < 4; ++m) w[k][m] = f.w[k][m];
    }
    // normal flux of a primitive state (rho, un, ut, p) in components (0, MU, MV, 3)
    template <int IXY>
    __device__ __forceinline__ static void flux(double r, double un, double ut, double pr, double g1inv,
                                                double (&F)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double E = pr * g1inv + 0.5 * r * (un * un + ut * ut);
        F[0] = r * un;
        F[MU] = r * un * un + pr;
        F[MV] = r * un * ut;
        F[3] = un * (E + pr);
    }
    template <int IXY>
    __device__ __forceinline__ static void cons(double r, double un, double ut, double pr, double g1inv,
                                                double (&Q)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        Q[0] = r;
        Q[MU] = r * un;
        Q[MV] = r * ut;
        Q[3] = pr * g1inv + 0.5 * r * (un * un + ut * ut);
    }

    template <int IXY>
    __device__ __forceinline__ static void solve_g(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                   double guess, Iface& f, double (&amdq)[MEQN],
                                                   double (&apdq)[MEQN]) {
        constexpr int UN = (IXY == 1) ? UX : UY, UT = (IXY == 1) ? UY : UX;
        const double gamma = p.c[0], gamma1 = gamma - 1.0, g1inv = 1.0 / gamma1;
        const double tol = p.c[1];
        // Roe state for the transverse solver
        {
            const double inv = rcp_nr(cL[RS] + cR[RS]);
            const double wl = cL[RS] * inv, wr = cR[RS] * inv;
            f.u = wl * cL[UN] + wr * cR[UN];
            f.v = wl * cL[UT] + wr * cR[UT];
            f.H = wl * cL[HH] + wr * cR[HH];
            const double a2 = gamma1 * (f.H - 0.5 * (f.u * f.u + f.v * f.v));
            f.ia = rsqrt_nr(a2);
            f.a = a2 * f.ia;
        }
        const exact_euler::Gas G = exact_euler::make_gas(gamma);
        const double rl = cL[0], ul = cL[UN], vl = cL[UT], pl = cL[PP], cl = cL[CS];
        const double rr = cR[0], ur = cR[UN], vr = cR[UT], pr = cR[PP], cr = cR[CS];
        if (exact_euler::vacuum(G, ul, cl, ur, cr)) {
            // vacuum: the Roe solution for this interface
            RPEulerRoe::Iface fr;
            double cl9[9], cr9[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) { cl9[k] = cL[k]; cr9[k] = cR[k]; }
            RPParams pp = p;
            pp.flags = 1;
            RPEulerRoe::template solve<IXY>(cl9, cr9, pp, fr, amdq, apdq);
            double w4[4][4];
            RPEulerRoe::template waves<IXY>(fr, pp, w4);
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                f.w[0][m] = w4[0][m];
                f.w[1][m] = w4[1][m] + w4[2][m];
                f.w[2][m] = w4[3][m];
            }
            f.s[0] = fr.u - fr.a; f.s[1] = fr.u; f.s[2] = fr.u + fr.a;
            f.iters = 0;
            f.applied = 0;
            return;
        }
        double ps, us;
        int it;
        exact_euler::star(G, rl, ul, pl, cl, rr, ur, pr, cr, guess, tol, 50, ps, us, it);
        f.iters = it;
        // star() returns at once for equal states; otherwise it also applies
        // the step that falls below the tolerance (unless it stopped at its cap)
        f.applied = (rl == rr && ul == ur && pl == pr) ? 0 : (it < 50 ? it + 1 : it);
        const exact_euler::Fan F = exact_euler::fan(G, rl, ul, pl, cl, rr, ur, pr, cr, ps, us);
        double QL[MEQN], QR[MEQN], QsL[MEQN], QsR[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; ++m) { QL[m] = cL[m]; QR[m] = cR[m]; }
        cons<IXY>(F.rsl, us, vl, ps, g1inv, QsL);
        cons<IXY>(F.rsr, us, vr, ps, g1inv, QsR);
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            f.w[0][m] = QsL[m] - QL[m];
            f.w[1][m] = QsR[m] - QsL[m];
            f.w[2][m] = QR[m] - QsR[m];
        }
        f.s[0] = F.s1;
        f.s[1] = us;
        f.s[2] = F.s3;
        double r0, u0, p0;
        bool left;
        exact_euler::sample0(G, rl, ul, pl, cl, rr, ur, pr, cr, ps, us, F, r0, u0, p0, left);
        double F0[MEQN], FL[MEQN], FR[MEQN];
        flux<IXY>(r0, u0, left ? vl : vr, p0, g1inv, F0);
        flux<IXY>(rl, ul, vl, pl, g1inv, FL);
        flux<IXY>(rr, ur, vr, pr, g1inv, FR);
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            amdq[m] = F0[m] - FL[m];
            apdq[m] = FR[m] - F0[m];
        }
    }
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        solve_g<IXY>(cL, cR, p, 0.0, f, amdq, apdq);
    }
    // Two equal states: star() returns p* = p, u* = u at once, the fan is two
    // rarefactions of zero width, so the waves and fluctuations are zero and
    // the speeds are solve_g's expressions at ps = p (pow(1, .) = 1):
    // 0.5 ((u - c) + (u* - c)) and 0.5 ((u + c) + (u* + c)).  (States that
    // generate vacuum -- c = 0 -- take the Roe fallback's record, as solve_g.)
    template <int IXY>
    __device__ __forceinline__ static void zero_iface(const double (&cL)[NC], const double (&cR)[NC],
                                                      const RPParams& p, Iface& f) {
        constexpr int UN = (IXY == 1) ? UX : UY;
        const exact_euler::Gas G = exact_euler::make_gas(p.c[0]);
        const double ul = cL[UN], cl = cL[CS], ur = cR[UN], cr = cR[CS];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int m = 0; m < 4; ++m) f.w[k][m] = 0.0;
        f.iters = 0;
        f.applied = 0;
        if (exact_euler::vacuum(G, ul, cl, ur, cr)) {
            double cl9[9], cr9[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) { cl9[k] = cL[k]; cr9[k] = cR[k]; }
            RPEulerRoe::Iface fr;
            RPEulerRoe::template zero_iface<IXY>(cl9, cr9, p, fr);
            f.s[0] = fr.u - fr.a; f.s[1] = fr.u; f.s[2] = fr.u + fr.a;
            return;
        }
        const double us = ul;
        f.s[0] = 0.5 * ((ul - cl) + (us - cl));
        f.s[1] = us;
        f.s[2] = 0.5 * ((ur + cr) + (us + cr));
    }
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Iface& f, const RPParams& p, const double (&asdq)[MEQN],
                                                double (&bm)[MEQN], double (&bp)[MEQN]) {
        RPEulerRoe::Iface r;
        r.u = f.u; r.v = f.v; r.a = f.a; r.ia = f.ia; r.H = f.H;
        RPEulerRoe::template rpt2<IXY>(r, p, asdq, bm, bp);
    }
    __device__ __forceinline__ static int count(const Iface& f) { return f.iters; }
    __device__ __forceinline__ static int count_applied(const Iface& f) { return f.applied; }
};

// ---------------------------------------------------------------------------
// vc_acoustics_2D: acoustics in a heterogeneous medium; aux = (rho, c) per
// cell, no cparam.  Cell: q, impedance Z = rho c, sound speed c.  The normal
// solve splits the jump between cells L and R into a left-going wave with
// L's impedance at speed -c_L and a right-going wave with R's impedance at
// speed c_R; the transverse solve sends the part of a fluctuation that enters
// cell k into the cells below and above k with their own impedances and
// speeds (LeVeque 2002, sec. 9.6 and 21.5.1).
// ---------------------------------------------------------------------------
struct RPVcAcoustics {
    static constexpr int MEQN = 3, MWAVES = 2, NC = 5, MAUX = 2, ID = CLAW2_RP_VC_ACOUSTICS;
    static constexpr bool TRANSVERSE_AUX = true;  // rpt2 needs the cells beside the receiving cell
    enum { ZZ = 3, CC = 4 };
    struct Iface { double alpha[2]; double zl, zr, cl, cr; };

    __device__ __forceinline__ static void prepare_aux(const double (&q)[MEQN], const double (&aux)[MAUX],
                                                       const RPParams&, double (&c)[NC]) {
        c[0] = q[0]; c[1] = q[1]; c[2] = q[2];
        c[ZZ] = aux[0] * aux[1];
        c[CC] = aux[1];
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface& f, const RPParams&, double (&s)[MWAVES]) {
        s[0] = -f.cl;
        s[1] = f.cr;
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams&, double (&w)[MWAVES][MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        w[0][0] = -f.alpha[0] * f.zl; w[0][MU] = f.alpha[0]; w[0][MV] = 0.0;
        w[1][0] = f.alpha[1] * f.zr;  w[1][MU] = f.alpha[1]; w[1][MV] = 0.0;
    }
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU;
        const double zr = cR[ZZ], zl = cL[ZZ];
        const double delta1 = cR[0] - cL[0];
        const double delta2 = cR[MU] - cL[MU];
        f.alpha[0] = (-delta1 + zr * delta2) / (zl + zr);
        f.alpha[1] = (delta1 + zl * delta2) / (zl + zr);
        f.zl = zl; f.zr = zr; f.cl = cL[CC]; f.cr = cR[CC];
        double w[MWAVES][MEQN], s[MWAVES];
        waves<IXY>(f, p, w);
        speeds<IXY>(f, p, s);
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            amdq[m] = s[0] * w[0][m];
            apdq[m] = s[1] * w[1][m];
        }
    }
    // asdq enters the cell c0; cm / cp are the cells below / above it in the
    // transverse direction (x for IXY = 2, y for IXY = 1)
    template <int IXY>
    __device__ __forceinline__ static void rpt2_aux(const double (&asdq)[MEQN], const double (&cm)[NC],
                                                    const double (&c0)[NC], const double (&cp)[NC],
                                                    double (&bm)[MEQN], double (&bp)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double zm = cm[ZZ], zz = c0[ZZ], zp = cp[ZZ];
        const double a1 = (-asdq[0] + asdq[MV] * zz) / (zm + zz);
        const double a2 = (asdq[0] + asdq[MV] * zz) / (zz + zp);
        bm[0] = cm[CC] * a1 * zm; bm[MU] = 0.0; bm[MV] = -cm[CC] * a1;
        bp[0] = cp[CC] * a2 * zp; bp[MU] = 0.0; bp[MV] = cp[CC] * a2;
    }
};

// ---------------------------------------------------------------------------
// vc_advection_2D: q_t + u q_x + v q_y = 0 with the velocities given on the
// cell edges, aux = (u at the left edge, v at the bottom edge) per cell, no
// cparam.  Cell: q, u, v.  The normal solve's one wave is the jump, moving at
// the velocity of its interface (the left / bottom edge of the right / upper
// cell); the transverse solve moves the part of a fluctuation that entered
// cell k out through k's own lower transverse edge (if that velocity is
// negative) and through the lower edge of the cell above k (if that one is
// positive) (LeVeque 2002, sec. 9.5 and 20.5).
// ---------------------------------------------------------------------------
struct RPVcAdvection {
    static constexpr int MEQN = 1, MWAVES = 1, NC = 3, MAUX = 2, ID = CLAW2_RP_VC_ADVECTION;
    static constexpr bool TRANSVERSE_AUX = true;
    struct Iface { double alpha[1]; double s; };

    __device__ __forceinline__ static void prepare_aux(const double (&q)[MEQN], const double (&aux)[MAUX],
                                                       const RPParams&, double (&c)[NC]) {
        c[0] = q[0];
        c[1] = aux[0];
        c[2] = aux[1];
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface& f, const RPParams&, double (&s)[MWAVES]) {
        s[0] = f.s;
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams&, double (&w)[MWAVES][MEQN]) {
        w[0][0] = f.alpha[0];
    }
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams&,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        const double vel = cR[IXY];  // the interface is the left (IXY = 1) / bottom (IXY = 2) edge of cR
        f.alpha[0] = cR[0] - cL[0];
        f.s = vel;
        amdq[0] = fmin(vel, 0.0) * f.alpha[0];
        apdq[0] = fmax(vel, 0.0) * f.alpha[0];
    }
    // asdq entered c0; cp is the cell above it in the transverse direction
    template <int IXY>
    __device__ __forceinline__ static void rpt2_aux(const double (&asdq)[MEQN], const double (&)[NC],
                                                    const double (&c0)[NC], const double (&cp)[NC],
                                                    double (&bm)[MEQN], double (&bp)[MEQN]) {
        constexpr int KT = (IXY == 1) ? 2 : 1;  // the transverse velocity
        bm[0] = fmin(c0[KT], 0.0) * asdq[0];
        bp[0] = fmax(cp[KT], 0.0) * asdq[0];
    }
};

// ---------------------------------------------------------------------------
// The advection-reaction example's own solver
// (examples/advection_reaction_2d/rpn2_vc_advection_vector.f90): the
// vc_advection_2D normal solve for each of the two components of q, edge
// velocities in aux.  No transverse solve (split step, or transverse_waves = 0;
// the host rejects anything else).  Cell: q0, q1, u, v.
// ---------------------------------------------------------------------------
struct RPVcAdvectionVec {
    static constexpr int MEQN = 2, MWAVES = 1, NC = 4, MAUX = 2, ID = CLAW2_RP_VC_ADVECTION_VEC;
    static constexpr bool TRANSVERSE_AUX = false;
    struct Iface { double alpha[2]; double s; };

    __device__ __forceinline__ static void prepare_aux(const double (&q)[MEQN], const double (&aux)[MAUX],
                                                       const RPParams&, double (&c)[NC]) {
        c[0] = q[0]; c[1] = q[1];
        c[2] = aux[0];
        c[3] = aux[1];
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface& f, const RPParams&, double (&s)[MWAVES]) {
        s[0] = f.s;
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams&, double (&w)[MWAVES][MEQN]) {
        w[0][0] = f.alpha[0];
        w[0][1] = f.alpha[1];
    }
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams&,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        const double vel = cR[1 + IXY];  // the velocity on the interface: the left / bottom edge of cR
        f.s = vel;
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            f.alpha[m] = cR[m] - cL[m];
            amdq[m] = fmin(vel, 0.0) * f.alpha[m];
            apdq[m] = fmax(vel, 0.0) * f.alpha[m];
        }
    }
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Iface&, const RPParams&, const double (&)[MEQN],
                                                double (&bm)[MEQN], double (&bp)[MEQN]) {
#pragma unroll
        for (int m = 0; m < MEQN; ++m) bm[m] = bp[m] = 0.0;  // unreachable: the host rejects transverse solves
    }
};

// ---------------------------------------------------------------------------
// psystem_2D: the p-system of nonlinear elasticity in a heterogeneous medium,
//   eps_t - u_x - v_y = 0,  (rho u)_t - sigma(eps)_x = 0,  (rho v)_t - sigma(eps)_y = 0,
// q = (eps, rho u, rho v), aux = (rho, K, stress-strain relation, strain at
// the start of the step), sigma = K eps (relation 1) or exp(K eps) - 1
// (relation 2).  f-wave solver: the flux difference across an interface is
// split into the left cell's eigenvector (1, Z, 0) at speed -c and the right
// cell's (1, -Z, 0) at speed c, c = sqrt(sigma'(eps) / rho), Z = rho c
// (LeVeque 2002, sec. 15.5).  The transverse solve splits a fluctuation
// into the cell below's down-going and the cell above's up-going eigenvector
// in one decomposition, with those cells' impedances from the strain in aux
// (the split that reproduces the reference's psystem_2d gauges).
// Cell: q, u, v, sigma, c, Z (from q) and c, Z (from the aux strain).
// ---------------------------------------------------------------------------
struct RPPsystem {
    static constexpr int MEQN = 3, MWAVES = 2, NC = 10, MAUX = 4, ID = CLAW2_RP_PSYSTEM;
    static constexpr bool TRANSVERSE_AUX = true;
    enum { U = 3, V = 4, SIG = 5, C = 6, Z = 7, CT = 8, ZT = 9 };
    struct Iface { double alpha[2]; double zl, zr, cl, cr; };

    __device__ __forceinline__ static void material(double eps, double K, double rel, double& sig, double& sigp) {
        if (rel == 1.0) {
            sig = K * eps;
            sigp = K;
        } else {
            const double e = exp(K * eps);
            sig = e - 1.0;
            sigp = K * e;
        }
    }
    __device__ __forceinline__ static void prepare_aux(const double (&q)[MEQN], const double (&aux)[MAUX],
                                                       const RPParams&, double (&c)[NC]) {
        const double rho = aux[0], K = aux[1], rel = aux[2];
        c[0] = q[0]; c[1] = q[1]; c[2] = q[2];
        c[U] = q[1] / rho;
        c[V] = q[2] / rho;
        double sig, sigp;
        material(q[0], K, rel, sig, sigp);
        c[SIG] = sig;
        c[C] = sqrt(sigp / rho);
        c[Z] = rho * c[C];
        double sig4, sigp4;
        material(aux[3], K, rel, sig4, sigp4);
        c[CT] = sqrt(sigp4 / rho);
        c[ZT] = rho * c[CT];
    }
    template <int IXY>
    __device__ __forceinline__ static void speeds(const Iface& f, const RPParams&, double (&s)[MWAVES]) {
        s[0] = -f.cl;
        s[1] = f.cr;
    }
    template <int IXY>
    __device__ __forceinline__ static void waves(const Iface& f, const RPParams&, double (&w)[MWAVES][MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        w[0][0] = f.alpha[0]; w[0][MU] = f.alpha[0] * f.zl;  w[0][MV] = 0.0;
        w[1][0] = f.alpha[1]; w[1][MU] = -f.alpha[1] * f.zr; w[1][MV] = 0.0;
    }
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[NC], const double (&cR)[NC], const RPParams& p,
                                                 Iface& f, double (&amdq)[MEQN], double (&apdq)[MEQN]) {
        constexpr int VN = (IXY == 1) ? U : V;  // the normal velocity
        const double zl = cL[Z], zr = cR[Z];
        const double df1 = -(cR[VN] - cL[VN]);
        const double df2 = -(cR[SIG] - cL[SIG]);
        f.alpha[0] = (df2 + zr * df1) / (zl + zr);
        f.alpha[1] = (zl * df1 - df2) / (zl + zr);
        f.zl = zl; f.zr = zr; f.cl = cL[C]; f.cr = cR[C];
        double w[MWAVES][MEQN];
        waves<IXY>(f, p, w);
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            amdq[m] = w[0][m];
            apdq[m] = w[1][m];
        }
    }
    template <int IXY>
    __device__ __forceinline__ static void rpt2_aux(const double (&asdq)[MEQN], const double (&cm)[NC],
                                                    const double (&)[NC], const double (&cp)[NC],
                                                    double (&bm)[MEQN], double (&bp)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        // one split of asdq into the cell below's down-going eigenvector
        // (1, 0, Zm) and the cell above's up-going one (1, 0, -Zp)
        const double zm = cm[ZT], zp = cp[ZT];
        const double bdown = (asdq[MV] + zp * asdq[0]) / (zm + zp);
        const double bup = (zm * asdq[0] - asdq[MV]) / (zm + zp);
        bm[0] = -cm[CT] * bdown; bm[MU] = 0.0; bm[MV] = -cm[CT] * bdown * zm;
        bp[0] = cp[CT] * bup;    bp[MU] = 0.0; bp[MV] = -cp[CT] * bup * zp;
    }
};

// Traits for solvers whose cells carry aux data (MAUX > 0, prepare_aux) and
// whose transverse solve needs the neighbouring cells (TRANSVERSE_AUX).
template <class RP, class = void>
struct AuxTraits {
    static constexpr int MAUX = 0;
    static constexpr bool TRANSVERSE_AUX = false;
    template <int N>
    __device__ __forceinline__ static void prep(const double (&q)[RP::MEQN], const double (&)[N], const RPParams& p,
                                                double (&c)[RP::NC]) {
        RP::prepare(q, p, c);
    }
};
template <class RP>
struct AuxTraits<RP, decltype((void)RP::MAUX, void())> {
    static constexpr int MAUX = RP::MAUX;
    static constexpr bool TRANSVERSE_AUX = RP::TRANSVERSE_AUX;
    template <int N>
    __device__ __forceinline__ static void prep(const double (&q)[RP::MEQN], const double (&aux)[N],
                                                const RPParams& p, double (&c)[RP::NC]) {
        static_assert(N == RP::MAUX, "aux vector of the wrong size");
        RP::prepare_aux(q, aux, p, c);
    }
};

// Traits for the zero-jump shortcut.  Solvers with `zero_iface` (no aux data,
// no guess) produce zero waves and zero fluctuations at an interface whose two
// cells hold bitwise-equal q: every strength is a difference of equal numbers
// (or a combination of such), so the limiter skips the waves (wnorm2 == 0,
// limiter.f90:42), the correction and transverse terms are zero, and only the
// speeds -- the Courant number -- remain; zero_iface builds that record.
template <class RP, class = void>
struct SkipTraits {
    static constexpr bool OK = false;
    template <int IXY>
    __device__ __forceinline__ static void zero_iface(const double (&)[RP::NC], const double (&)[RP::NC],
                                                      const RPParams&, typename RP::Iface&) {}
};
template <class RP>
struct SkipTraits<RP, decltype((void)&RP::template zero_iface<1>, void())> {
    static constexpr bool OK = true;
    template <int IXY>
    __device__ __forceinline__ static void zero_iface(const double (&cL)[RP::NC], const double (&cR)[RP::NC],
                                                      const RPParams& p, typename RP::Iface& f) {
        RP::template zero_iface<IXY>(cL, cR, p, f);
    }
};

// true when the first ME entries (q itself) of two prepared cells are equal bit for bit
template <int ME, int NC>
__device__ __forceinline__ bool same_q(const double (&a)[NC], const double (&b)[NC]) {
    bool eq = true;
#pragma unroll
    for (int m = 0; m < ME; ++m) eq = eq && (__double_as_longlong(a[m]) == __double_as_longlong(b[m]));
    return eq;
}

// Traits for the optional per-interface guess and iteration count.
template <class RP, class = void>
struct GuessTraits {
    static constexpr bool USES = false;
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[RP::NC], const double (&cR)[RP::NC],
                                                 const RPParams& p, double, typename RP::Iface& f,
                                                 double (&am)[RP::MEQN], double (&ap)[RP::MEQN]) {
        RP::template solve<IXY>(cL, cR, p, f, am, ap);
    }
    __device__ __forceinline__ static int count(const typename RP::Iface&) { return 0; }
    __device__ __forceinline__ static int count_applied(const typename RP::Iface&) { return 0; }
};
template <class RP>
struct GuessTraits<RP, decltype((void)RP::USES_GUESS, void())> {
    static constexpr bool USES = RP::USES_GUESS;
    template <int IXY>
    __device__ __forceinline__ static void solve(const double (&cL)[RP::NC], const double (&cR)[RP::NC],
                                                 const RPParams& p, double g, typename RP::Iface& f,
                                                 double (&am)[RP::MEQN], double (&ap)[RP::MEQN]) {
        RP::template solve_g<IXY>(cL, cR, p, g, f, am, ap);
    }
    __device__ __forceinline__ static int count(const typename RP::Iface& f) { return RP::count(f); }
    __device__ __forceinline__ static int count_applied(const typename RP::Iface& f) { return RP::count_applied(f); }
};

}  // namespace claw2
