// riemann.cuh -- pointwise device Riemann solvers for the classic 2D step.
//
// The reference calls Riemann solvers through the Fortran slice ABI
// rpn2(ixy,maxm,meqn,mwaves,maux,mbc,mx,ql,qr,auxl,auxr,wave,s,amdq,apdq) and
// rpt2(ixy,imp,...,asdq,bmasdq,bpasdq) (call sites src/pyclaw/classic/flux2.f90:101,
// 181, 194).  Here each solver is a struct of inline functions for ONE
// interface, with the direction (ixy) and the system size as compile-time
// constants so that waves, speeds and fluctuations stay in registers.
//
//   rpn2<IXY>(qL, qR, prm, wave, s, amdq, apdq, cache)
//       qL = state of the cell below/left of the interface, qR = above/right.
//   rpt2<IXY>(cache, qL, qR, prm, asdq, bmasdq, bpasdq)
//       split asdq into down-going and up-going parts; `cache` carries the
//       Roe-averaged state that rpn2 computed for the same interface so it is
//       not recomputed (the reuse the reference's
//       development/rp_approaches/report.tex:37-39 measures as a 10% gain).
//
// The formulas are the published ones (LeVeque, Finite Volume Methods for
// Hyperbolic Problems, 2002: advection sec. 20.5, acoustics sec. 18.2/21.7,
// Roe Euler sec. 15.3 and 18.8, Roe shallow water sec. 15.3, transverse
// solvers sec. 21.6) and match, operation for operation, the CPU oracle.
#pragma once

#include "claw2_types.cuh"

namespace claw2 {

template <int IXY>
struct Dir {
    static constexpr int MU = (IXY == 1) ? 1 : 2;  // normal momentum component
    static constexpr int MV = (IXY == 1) ? 2 : 1;  // transverse momentum component
};

// ---------------------------------------------------------------------------
// advection_2D: cparam = {u, v}
// ---------------------------------------------------------------------------
struct RPAdvection {
    static constexpr int MEQN = 1, MWAVES = 1, ID = CLAW2_RP_ADVECTION;
    struct Cache {};
    template <int IXY>
    __device__ __forceinline__ static void rpn2(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                const RPParams& p, double (&wave)[MWAVES][MEQN],
                                                double (&s)[MWAVES], double (&amdq)[MEQN],
                                                double (&apdq)[MEQN], Cache&) {
        const double vel = (IXY == 1) ? p.c[0] : p.c[1];
        wave[0][0] = qR[0] - qL[0];
        s[0] = vel;
        amdq[0] = fmin(s[0], 0.0) * wave[0][0];
        apdq[0] = fmax(s[0], 0.0) * wave[0][0];
    }
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Cache&, const RPParams& p,
                                                const double (&asdq)[MEQN], double (&bm)[MEQN],
                                                double (&bp)[MEQN]) {
        const double stran = (IXY == 1) ? p.c[1] : p.c[0];
        bm[0] = fmin(stran, 0.0) * asdq[0];
        bp[0] = fmax(stran, 0.0) * asdq[0];
    }
};

// ---------------------------------------------------------------------------
// acoustics_2D: cparam = {rho, bulk, cc, zz}; q = (p, u, v)
// ---------------------------------------------------------------------------
struct RPAcoustics {
    static constexpr int MEQN = 3, MWAVES = 2, ID = CLAW2_RP_ACOUSTICS;
    struct Cache {};
    template <int IXY>
    __device__ __forceinline__ static void rpn2(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                const RPParams& p, double (&wave)[MWAVES][MEQN],
                                                double (&s)[MWAVES], double (&amdq)[MEQN],
                                                double (&apdq)[MEQN], Cache&) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double cc = p.c[2], zz = p.c[3];
        const double delta1 = qR[0] - qL[0];
        const double delta2 = qR[MU] - qL[MU];
        const double a1 = (-delta1 + zz * delta2) / (2.0 * zz);
        const double a2 = (delta1 + zz * delta2) / (2.0 * zz);
        wave[0][0] = -a1 * zz; wave[0][MU] = a1; wave[0][MV] = 0.0; s[0] = -cc;
        wave[1][0] = a2 * zz;  wave[1][MU] = a2; wave[1][MV] = 0.0; s[1] = cc;
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            amdq[m] = s[0] * wave[0][m];
            apdq[m] = s[1] * wave[1][m];
        }
    }
    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Cache&, const RPParams& p,
                                                const double (&asdq)[MEQN], double (&bm)[MEQN],
                                                double (&bp)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double cc = p.c[2], zz = p.c[3];
        const double a1 = (-asdq[0] + zz * asdq[MV]) / (2.0 * zz);
        const double a2 = (asdq[0] + zz * asdq[MV]) / (2.0 * zz);
        bm[0] = cc * a1 * zz; bm[MU] = 0.0; bm[MV] = -cc * a1;
        bp[0] = cc * a2 * zz; bp[MU] = 0.0; bp[MV] = cc * a2;
    }
};

// ---------------------------------------------------------------------------
// euler_4wave_2D (Roe): cparam = {gamma, efix}; q = (rho, rho u, rho v, E)
// Waves: 1 = u-c acoustic, 2 = entropy (u), 3 = shear (u), 4 = u+c acoustic.
// ---------------------------------------------------------------------------
struct RPEulerRoe {
    static constexpr int MEQN = 4, MWAVES = 4, ID = CLAW2_RP_EULER_ROE;
    struct Cache { double u, v, a, enth, u2v2, g1a2, euv; };

    template <int IXY>
    __device__ __forceinline__ static void roe_state(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                     double gamma1, Cache& c) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double rhsqrtl = sqrt(qL[0]);
        const double rhsqrtr = sqrt(qR[0]);
        const double pl = gamma1 * (qL[3] - 0.5 * (qL[1] * qL[1] + qL[2] * qL[2]) / qL[0]);
        const double pr = gamma1 * (qR[3] - 0.5 * (qR[1] * qR[1] + qR[2] * qR[2]) / qR[0]);
        const double rhsq2 = rhsqrtl + rhsqrtr;
        c.u = (qL[MU] / rhsqrtl + qR[MU] / rhsqrtr) / rhsq2;
        c.v = (qL[MV] / rhsqrtl + qR[MV] / rhsqrtr) / rhsq2;
        c.enth = (((qL[3] + pl) / rhsqrtl + (qR[3] + pr) / rhsqrtr)) / rhsq2;
        c.u2v2 = c.u * c.u + c.v * c.v;
        const double a2 = gamma1 * (c.enth - 0.5 * c.u2v2);
        c.a = sqrt(a2);
        c.g1a2 = gamma1 / a2;
        c.euv = c.enth - c.u2v2;
    }

    template <int IXY>
    __device__ __forceinline__ static void rpn2(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                const RPParams& p, double (&wave)[MWAVES][MEQN],
                                                double (&s)[MWAVES], double (&amdq)[MEQN],
                                                double (&apdq)[MEQN], Cache& c) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double gamma = p.c[0];
        const double gamma1 = gamma - 1.0;
        roe_state<IXY>(qL, qR, gamma1, c);
        const double u = c.u, v = c.v, a = c.a, enth = c.enth;
        const double delta0 = qR[0] - qL[0];
        const double delta1 = qR[MU] - qL[MU];
        const double delta2 = qR[MV] - qL[MV];
        const double delta3 = qR[3] - qL[3];
        const double b3 = c.g1a2 * (c.euv * delta0 + u * delta1 + v * delta2 - delta3);
        const double b2 = delta2 - v * delta0;
        const double b4 = (delta1 + (a - u) * delta0 - a * b3) / (2.0 * a);
        const double b1 = delta0 - b3 - b4;

        wave[0][0] = b1; wave[0][MU] = b1 * (u - a); wave[0][MV] = b1 * v;
        wave[0][3] = b1 * (enth - u * a); s[0] = u - a;
        wave[1][0] = b3; wave[1][MU] = b3 * u; wave[1][MV] = b3 * v;
        wave[1][3] = b3 * 0.5 * c.u2v2; s[1] = u;
        wave[2][0] = 0.0; wave[2][MU] = 0.0; wave[2][MV] = b2;
        wave[2][3] = b2 * v; s[2] = u;
        wave[3][0] = b4; wave[3][MU] = b4 * (u + a); wave[3][MV] = b4 * v;
        wave[3][3] = b4 * (enth + u * a); s[3] = u + a;

        if (p.flags == 0) {
#pragma unroll
            for (int m = 0; m < MEQN; ++m) {
                double am = 0.0, ap = 0.0;
#pragma unroll
                for (int mw = 0; mw < MWAVES; ++mw) {
                    if (s[mw] < 0.0) am = am + s[mw] * wave[mw][m];
                    else ap = ap + s[mw] * wave[mw][m];
                }
                amdq[m] = am;
                apdq[m] = ap;
            }
            return;
        }
        // Harten-Hyman entropy fix (same branch structure as the oracle).
        bool done = false;
        {
            const double rhoim1 = qL[0];
            const double pim1 = gamma1 * (qL[3] - 0.5 * (qL[MU] * qL[MU] + qL[MV] * qL[MV]) / rhoim1);
            const double cim1 = sqrt(gamma * pim1 / rhoim1);
            const double s0 = qL[MU] / rhoim1 - cim1;
            if (s0 >= 0.0 && s[0] > 0.0) {
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = 0.0;
                done = true;
            } else {
                const double rho1 = qL[0] + wave[0][0];
                const double rhou1 = qL[MU] + wave[0][MU];
                const double rhov1 = qL[MV] + wave[0][MV];
                const double en1 = qL[3] + wave[0][3];
                const double p1 = gamma1 * (en1 - 0.5 * (rhou1 * rhou1 + rhov1 * rhov1) / rho1);
                const double c1 = sqrt(gamma * p1 / rho1);
                const double s1 = rhou1 / rho1 - c1;
                double sfract;
                if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s[0]) / (s1 - s0);
                else if (s[0] < 0.0) sfract = s[0];
                else sfract = 0.0;
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = sfract * wave[0][m];
            }
        }
        if (!done && !(s[1] >= 0.0)) {
#pragma unroll
            for (int m = 0; m < MEQN; ++m) amdq[m] = amdq[m] + s[1] * wave[1][m] + s[2] * wave[2][m];
            const double rhoi = qR[0];
            const double pi = gamma1 * (qR[3] - 0.5 * (qR[MU] * qR[MU] + qR[MV] * qR[MV]) / rhoi);
            const double ci = sqrt(gamma * pi / rhoi);
            const double s3 = qR[MU] / rhoi + ci;
            const double rho2 = qR[0] - wave[3][0];
            const double rhou2 = qR[MU] - wave[3][MU];
            const double rhov2 = qR[MV] - wave[3][MV];
            const double en2 = qR[3] - wave[3][3];
            const double p2 = gamma1 * (en2 - 0.5 * (rhou2 * rhou2 + rhov2 * rhov2) / rho2);
            const double c2 = sqrt(gamma * p2 / rho2);
            const double s2 = rhou2 / rho2 + c2;
            double sfract = 0.0;
            bool add = true;
            if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - s[3]) / (s3 - s2);
            else if (s[3] < 0.0) sfract = s[3];
            else add = false;
            if (add) {
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = amdq[m] + sfract * wave[3][m];
            }
        }
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            double df = 0.0;
#pragma unroll
            for (int mw = 0; mw < MWAVES; ++mw) df = df + s[mw] * wave[mw][m];
            apdq[m] = df - amdq[m];
        }
    }

    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Cache& c, const RPParams&,
                                                const double (&asdq)[MEQN], double (&bm)[MEQN],
                                                double (&bp)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double u = c.u, v = c.v, a = c.a, enth = c.enth;
        const double b3 = c.g1a2 * (c.euv * asdq[0] + u * asdq[MU] + v * asdq[MV] - asdq[3]);
        const double b2 = asdq[MU] - u * asdq[0];
        const double b4 = (asdq[MV] + (a - v) * asdq[0] - a * b3) / (2.0 * a);
        const double b1 = asdq[0] - b3 - b4;
        double wb[MWAVES][MEQN], sb[MWAVES];
        wb[0][0] = b1; wb[0][MU] = b1 * u; wb[0][MV] = b1 * (v - a); wb[0][3] = b1 * (enth - v * a); sb[0] = v - a;
        wb[1][0] = b3; wb[1][MU] = b3 * u; wb[1][MV] = b3 * v; wb[1][3] = b3 * 0.5 * c.u2v2; sb[1] = v;
        wb[2][0] = 0.0; wb[2][MU] = b2; wb[2][MV] = 0.0; wb[2][3] = b2 * u; sb[2] = v;
        wb[3][0] = b4; wb[3][MU] = b4 * u; wb[3][MV] = b4 * (v + a); wb[3][3] = b4 * (enth + v * a); sb[3] = v + a;
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            double xm = 0.0, xp = 0.0;
#pragma unroll
            for (int mw = 0; mw < MWAVES; ++mw) {
                xm = xm + fmin(sb[mw], 0.0) * wb[mw][m];
                xp = xp + fmax(sb[mw], 0.0) * wb[mw][m];
            }
            bm[m] = xm;
            bp[m] = xp;
        }
    }
};

// ---------------------------------------------------------------------------
// shallow_roe_with_efix_2D: cparam = {grav, efix}; q = (h, hu, hv)
// ---------------------------------------------------------------------------
struct RPShallowRoe {
    static constexpr int MEQN = 3, MWAVES = 3, ID = CLAW2_RP_SHALLOW_ROE;
    struct Cache { double u, v, a; };

    template <int IXY>
    __device__ __forceinline__ static void rpn2(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                const RPParams& p, double (&wave)[MWAVES][MEQN],
                                                double (&s)[MWAVES], double (&amdq)[MEQN],
                                                double (&apdq)[MEQN], Cache& c) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        const double grav = p.c[0];
        const double h = (qL[0] + qR[0]) * 0.50;
        const double hsqrtl = sqrt(qL[0]);
        const double hsqrtr = sqrt(qR[0]);
        const double hsq2 = hsqrtl + hsqrtr;
        const double u = (qL[MU] / hsqrtl + qR[MU] / hsqrtr) / hsq2;
        const double v = (qL[MV] / hsqrtl + qR[MV] / hsqrtr) / hsq2;
        const double a = sqrt(grav * h);
        c.u = u; c.v = v; c.a = a;
        const double delta0 = qR[0] - qL[0];
        const double delta1 = qR[MU] - qL[MU];
        const double delta2 = qR[MV] - qL[MV];
        const double a1 = ((u + a) * delta0 - delta1) * (0.50 / a);
        const double a2 = -v * delta0 + delta2;
        const double a3 = (-(u - a) * delta0 + delta1) * (0.50 / a);
        wave[0][0] = a1; wave[0][MU] = a1 * (u - a); wave[0][MV] = a1 * v; s[0] = u - a;
        wave[1][0] = 0.0; wave[1][MU] = 0.0; wave[1][MV] = a2; s[1] = u;
        wave[2][0] = a3; wave[2][MU] = a3 * (u + a); wave[2][MV] = a3 * v; s[2] = u + a;

        if (p.flags == 0) {
#pragma unroll
            for (int m = 0; m < MEQN; ++m) {
                double am = 0.0, ap = 0.0;
#pragma unroll
                for (int mw = 0; mw < MWAVES; ++mw) {
                    if (s[mw] < 0.0) am = am + s[mw] * wave[mw][m];
                    else ap = ap + s[mw] * wave[mw][m];
                }
                amdq[m] = am;
                apdq[m] = ap;
            }
            return;
        }
        bool done = false;
        {
            const double him1 = qL[0];
            const double s0 = qL[MU] / him1 - sqrt(grav * him1);
            if (s0 >= 0.0 && s[0] > 0.0) {
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = 0.0;
                done = true;
            } else {
                const double h1 = qL[0] + wave[0][0];
                const double hu1 = qL[MU] + wave[0][MU];
                const double s1 = hu1 / h1 - sqrt(grav * h1);
                double sfract;
                if (s0 < 0.0 && s1 > 0.0) sfract = s0 * ((s1 - s[0]) / (s1 - s0));
                else if (s[0] < 0.0) sfract = s[0];
                else sfract = 0.0;
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = sfract * wave[0][m];
            }
        }
        if (!done && !(s[1] > 0.0)) {
#pragma unroll
            for (int m = 0; m < MEQN; ++m) amdq[m] = amdq[m] + s[1] * wave[1][m];
            const double hi = qR[0];
            const double s03 = qR[MU] / hi + sqrt(grav * hi);
            const double h3 = qR[0] - wave[2][0];
            const double hu3 = qR[MU] - wave[2][MU];
            const double s3 = hu3 / h3 + sqrt(grav * h3);
            double sfract = 0.0;
            bool add = true;
            if (s3 < 0.0 && s03 > 0.0) sfract = s3 * ((s03 - s[2]) / (s03 - s3));
            else if (s[2] < 0.0) sfract = s[2];
            else add = false;
            if (add) {
#pragma unroll
                for (int m = 0; m < MEQN; ++m) amdq[m] = amdq[m] + sfract * wave[2][m];
            }
        }
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            double df = 0.0;
#pragma unroll
            for (int mw = 0; mw < MWAVES; ++mw) df = df + s[mw] * wave[mw][m];
            apdq[m] = df - amdq[m];
        }
    }

    template <int IXY>
    __device__ __forceinline__ static void rpt2(const Cache& c, const RPParams&,
                                                const double (&asdq)[MEQN], double (&bm)[MEQN],
                                                double (&bp)[MEQN]) {
        constexpr int MU = Dir<IXY>::MU, MV = Dir<IXY>::MV;
        // transverse speeds at the Roe state: v -+ c, v (cbar = sqrt(g*hbar))
        const double ubar = c.u, vbar = c.v, cbar = c.a;
        const double a1 = (0.5 / cbar) * ((vbar + cbar) * asdq[0] - asdq[MV]);
        const double a2 = -ubar * asdq[0] + asdq[MU];
        const double a3 = (0.5 / cbar) * (-(vbar - cbar) * asdq[0] + asdq[MV]);
        double wb[MWAVES][MEQN], sb[MWAVES];
        wb[0][0] = a1; wb[0][MU] = a1 * ubar; wb[0][MV] = a1 * (vbar - cbar); sb[0] = vbar - cbar;
        wb[1][0] = 0.0; wb[1][MU] = a2; wb[1][MV] = 0.0; sb[1] = vbar;
        wb[2][0] = a3; wb[2][MU] = a3 * ubar; wb[2][MV] = a3 * (vbar + cbar); sb[2] = vbar + cbar;
#pragma unroll
        for (int m = 0; m < MEQN; ++m) {
            double xm = 0.0, xp = 0.0;
#pragma unroll
            for (int mw = 0; mw < MWAVES; ++mw) {
                xm = xm + fmin(sb[mw], 0.0) * wb[mw][m];
                xp = xp + fmax(sb[mw], 0.0) * wb[mw][m];
            }
            bm[m] = xm;
            bp[m] = xp;
        }
    }
};

}  // namespace claw2
