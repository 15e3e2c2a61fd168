// claw_oracle.cpp -- CPU oracle (test infrastructure only; see claw_oracle.h).
//
// A restatement, in the reference's loop and operation order, of the classic
// Clawpack 2D kernels.  Index helpers below use the Fortran index ranges of the
// reference so each loop reads like the file:line it cites.  Component indices
// m and wave indices mw are 0-based; cell/interface indices i, j keep the
// Fortran ranges (1-mbc .. mx+mbc).
#include "claw_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

int g_threads = 1;

// ---------------------------------------------------------------------------
// Slice views with Fortran index ranges.
// ---------------------------------------------------------------------------
struct Slice {  // (meqn, 1-mbc:maxm+mbc)
    double* p; int meqn, mbc;
    double& operator()(int m, int i) const { return p[(size_t)(i + mbc - 1) * meqn + m]; }
};
struct CSlice {
    const double* p; int meqn, mbc;
    double operator()(int m, int i) const { return p[(size_t)(i + mbc - 1) * meqn + m]; }
};
struct Waves {  // (meqn, mwaves, 1-mbc:maxm+mbc)
    double* p; int meqn, mwaves, mbc;
    double& operator()(int m, int mw, int i) const {
        return p[((size_t)(i + mbc - 1) * mwaves + mw) * meqn + m];
    }
};
struct Speeds {  // (mwaves, 1-mbc:maxm+mbc)
    double* p; int mwaves, mbc;
    double& operator()(int mw, int i) const { return p[(size_t)(i + mbc - 1) * mwaves + mw]; }
};
struct Gadd {  // (meqn, 2, 1-mbc:maxm+mbc); k = 0 (below) or 1 (above)
    double* p; int meqn, mbc;
    double& operator()(int m, int k, int i) const {
        return p[((size_t)(i + mbc - 1) * 2 + k) * meqn + m];
    }
};
struct Grid2 {  // (meqn, 1-mbc:mx+mbc, 1-mbc:my+mbc), Fortran order
    double* p; int meqn, mbc, mx;
    double& operator()(int m, int i, int j) const {
        return p[((size_t)(j + mbc - 1) * (mx + 2 * mbc) + (i + mbc - 1)) * meqn + m];
    }
};

// ---------------------------------------------------------------------------
// philim.f90:16-35
// ---------------------------------------------------------------------------
double philim(double a, double b, int meth) {
    double r = b / a;
    switch (meth) {
        case 1: return std::max(0.0, std::min(1.0, r));                                   // minmod
        case 2: return std::max(0.0, std::max(std::min(1.0, 2.0 * r), std::min(2.0, r)));  // superbee
        case 3: return (r + std::fabs(r)) / (1.0 + std::fabs(r));                          // van Leer
        case 4: {                                                                          // MC
            double c = (1.0 + r) / 2.0;
            return std::max(0.0, std::min(c, std::min(2.0, 2.0 * r)));
        }
        case 5: return r;                                                                  // Beam-Warming
        default: return 0.0;
    }
}

// ---------------------------------------------------------------------------
// limiter.f90:29-53
// ---------------------------------------------------------------------------
void limiter(int mx, int meqn, int mwaves, const Waves& wave, const Speeds& s,
             const int* mthlim) {
    for (int mw = 0; mw < mwaves; ++mw) {
        if (mthlim[mw] == 0) continue;
        double dotr = 0.0;
        for (int i = 0; i <= mx + 1; ++i) {
            double wnorm2 = 0.0;
            double dotl = dotr;
            dotr = 0.0;
            for (int m = 0; m < meqn; ++m) {
                wnorm2 = wnorm2 + wave(m, mw, i) * wave(m, mw, i);
                dotr = dotr + wave(m, mw, i) * wave(m, mw, i + 1);
            }
            if (i == 0) continue;
            if (wnorm2 == 0.0) continue;
            double wlimitr;
            if (s(mw, i) > 0.0)
                wlimitr = philim(wnorm2, dotl, mthlim[mw]);
            else
                wlimitr = philim(wnorm2, dotr, mthlim[mw]);
            for (int m = 0; m < meqn; ++m) wave(m, mw, i) = wlimitr * wave(m, mw, i);
        }
    }
}

// ---------------------------------------------------------------------------
// Riemann solvers (external clawpack/riemann package; restated from the
// mathematics, Fortran slice ABI: interface i has left state qr(:,i-1) and
// right state ql(:,i); flux2 passes ql = qr = q1d).
// ---------------------------------------------------------------------------

// advection_2D: q_t + u q_x + v q_y = 0 (LeVeque 2002, sec. 20.5).
void rpn2_advection(int ixy, int mbc, int mx, int meqn, int mwaves, const CSlice& ql,
                    const CSlice& qr, const Waves& wave, const Speeds& s, const Slice& amdq,
                    const Slice& apdq, const double* cp) {
    const double vel = (ixy == 1) ? cp[0] : cp[1];
    (void)meqn; (void)mwaves;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        wave(0, 0, i) = ql(0, i) - qr(0, i - 1);
        s(0, i) = vel;
        amdq(0, i) = std::min(s(0, i), 0.0) * wave(0, 0, i);
        apdq(0, i) = std::max(s(0, i), 0.0) * wave(0, 0, i);
    }
}
void rpt2_advection(int ixy, int mbc, int mx, const Slice& asdq, const Slice& bmasdq,
                    const Slice& bpasdq, const double* cp) {
    const double stran = (ixy == 1) ? cp[1] : cp[0];
    const double stranm = std::min(stran, 0.0), stranp = std::max(stran, 0.0);
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        bmasdq(0, i) = stranm * asdq(0, i);
        bpasdq(0, i) = stranp * asdq(0, i);
    }
}

// acoustics_2D: p_t + K(u_x+v_y) = 0, rho u_t + p_x = 0, rho v_t + p_y = 0.
// Eigenvectors (-Z,1,0) with speed -c and (Z,1,0) with speed c in the normal
// direction (LeVeque 2002, sec. 18.2, 21.7).  cparam = rho, bulk, cc, zz.
void rpn2_acoustics(int ixy, int mbc, int mx, const CSlice& ql, const CSlice& qr,
                    const Waves& wave, const Speeds& s, const Slice& amdq, const Slice& apdq,
                    const double* cp, int meqn) {
    const double cc = cp[2], zz = cp[3];
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double delta1 = ql(0, i) - qr(0, i - 1);
        double delta2 = ql(mu, i) - qr(mu, i - 1);
        double a1 = (-delta1 + zz * delta2) / (2.0 * zz);
        double a2 = (delta1 + zz * delta2) / (2.0 * zz);
        wave(0, 0, i) = -a1 * zz;
        wave(mu, 0, i) = a1;
        wave(mv, 0, i) = 0.0;
        s(0, i) = -cc;
        wave(0, 1, i) = a2 * zz;
        wave(mu, 1, i) = a2;
        wave(mv, 1, i) = 0.0;
        s(1, i) = cc;
    }
    for (int m = 0; m < meqn; ++m)
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            amdq(m, i) = s(0, i) * wave(m, 0, i);
            apdq(m, i) = s(1, i) * wave(m, 1, i);
        }
}
void rpt2_acoustics(int ixy, int mbc, int mx, const Slice& asdq, const Slice& bmasdq,
                    const Slice& bpasdq, const double* cp) {
    const double cc = cp[2], zz = cp[3];
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double a1 = (-asdq(0, i) + zz * asdq(mv, i)) / (2.0 * zz);
        double a2 = (asdq(0, i) + zz * asdq(mv, i)) / (2.0 * zz);
        bmasdq(0, i) = cc * a1 * zz;
        bmasdq(mu, i) = 0.0;
        bmasdq(mv, i) = -cc * a1;
        bpasdq(0, i) = cc * a2 * zz;
        bpasdq(mu, i) = 0.0;
        bpasdq(mv, i) = cc * a2;
    }
}

// vc_acoustics_2D: acoustics in a heterogeneous medium, aux = (rho, c) per
// cell (LeVeque 2002, sec. 9.6 and 21.5.1).  Normal solve: the jump between
// cells i-1 and i splits into a left-going wave with cell i-1's impedance
// Z = rho c and speed -c(i-1) and a right-going wave with cell i's impedance
// and speed c(i).
void rpn2_vc_acoustics(int ixy, int mbc, int mx, int meqn, const CSlice& ql, const CSlice& qr,
                       const CSlice& auxl, const CSlice& auxr, const Waves& wave, const Speeds& s,
                       const Slice& amdq, const Slice& apdq) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double zi = auxl(0, i) * auxl(1, i);
        double zim = auxr(0, i - 1) * auxr(1, i - 1);
        double delta1 = ql(0, i) - qr(0, i - 1);
        double delta2 = ql(mu, i) - qr(mu, i - 1);
        double a1 = (-delta1 + zi * delta2) / (zim + zi);
        double a2 = (delta1 + zim * delta2) / (zim + zi);
        wave(0, 0, i) = -a1 * zim;
        wave(mu, 0, i) = a1;
        wave(mv, 0, i) = 0.0;
        s(0, i) = -auxr(1, i - 1);
        wave(0, 1, i) = a2 * zi;
        wave(mu, 1, i) = a2;
        wave(mv, 1, i) = 0.0;
        s(1, i) = auxl(1, i);
    }
    for (int m = 0; m < meqn; ++m)
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            amdq(m, i) = s(0, i) * wave(m, 0, i);
            apdq(m, i) = s(1, i) * wave(m, 1, i);
        }
}
// Transverse solve: asdq belongs to cell i1 (i-1 for imp = 1, i for imp = 2)
// with impedance zz; its down-going part is transmitted into the cell below
// (impedance zm, speed -cm) and its up-going part into the cell above (zp, cp).
void rpt2_vc_acoustics(int ixy, int imp, int mbc, int mx, const CSlice& aux1, const CSlice& aux2,
                       const CSlice& aux3, const Slice& asdq, const Slice& bmasdq, const Slice& bpasdq) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int i1 = (imp == 1) ? i - 1 : i;
        double zm = aux1(0, i1) * aux1(1, i1);
        double zz = aux2(0, i1) * aux2(1, i1);
        double zp = aux3(0, i1) * aux3(1, i1);
        double cm = aux1(1, i1), cp = aux3(1, i1);
        double a1 = (-asdq(0, i) + asdq(mv, i) * zz) / (zm + zz);
        double a2 = (asdq(0, i) + asdq(mv, i) * zz) / (zz + zp);
        bmasdq(0, i) = cm * a1 * zm;
        bmasdq(mu, i) = 0.0;
        bmasdq(mv, i) = -cm * a1;
        bpasdq(0, i) = cp * a2 * zp;
        bpasdq(mu, i) = 0.0;
        bpasdq(mv, i) = cp * a2;
    }
}

// vc_advection_2D: q_t + u q_x + v q_y = 0 with edge velocities in aux
// (LeVeque 2002, sec. 9.5 and 20.5): aux(1, i) is u at the left edge of cell
// i and aux(2, i) is v at its bottom edge.  Normal solve: one wave, the jump,
// moving at the velocity of the interface it sits on (the left edge of cell
// i for the interface i-1 | i).
void rpn2_vc_advection(int ixy, int mbc, int mx, const CSlice& ql, const CSlice& qr, const CSlice& auxl,
                       const Waves& wave, const Speeds& s, const Slice& amdq, const Slice& apdq) {
    const int kn = ixy - 1;  // the normal velocity's aux component
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        wave(0, 0, i) = ql(0, i) - qr(0, i - 1);
        s(0, i) = auxl(kn, i);
        amdq(0, i) = std::min(auxl(kn, i), 0.0) * wave(0, 0, i);
        apdq(0, i) = std::max(auxl(kn, i), 0.0) * wave(0, 0, i);
    }
}
// Transverse solve: asdq entered cell i1 (i-1 for imp = 1, i for imp = 2);
// its down-going part leaves through i1's own lower transverse edge (velocity
// in aux2) and its up-going part through the lower edge of the cell above
// (aux3), each at that edge's transverse velocity.
void rpt2_vc_advection(int ixy, int imp, int mbc, int mx, const CSlice& aux2, const CSlice& aux3,
                       const Slice& asdq, const Slice& bmasdq, const Slice& bpasdq) {
    const int kt = (ixy == 1) ? 1 : 0;  // the transverse velocity's aux component
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int i1 = (imp == 1) ? i - 1 : i;
        bmasdq(0, i) = std::min(aux2(kt, i1), 0.0) * asdq(0, i);
        bpasdq(0, i) = std::max(aux3(kt, i1), 0.0) * asdq(0, i);
    }
}

// The advection-reaction example's own solver
// (examples/advection_reaction_2d/rpn2_vc_advection_vector.f90:40-55): the
// vc_advection_2D normal solve applied to every component of q; no transverse
// solve (the example's rpt2 is a stub for the split step).
void rpn2_vc_advection_vector(int ixy, int mbc, int mx, int meqn, const CSlice& ql, const CSlice& qr,
                              const CSlice& auxl, const Waves& wave, const Speeds& s, const Slice& amdq,
                              const Slice& apdq) {
    const int kn = ixy - 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        s(0, i) = auxl(kn, i);
        for (int m = 0; m < meqn; ++m) {
            wave(m, 0, i) = ql(m, i) - qr(m, i - 1);
            amdq(m, i) = std::min(auxl(kn, i), 0.0) * wave(m, 0, i);
            apdq(m, i) = std::max(auxl(kn, i), 0.0) * wave(m, 0, i);
        }
    }
}

// psystem_2D: the two-dimensional p-system (nonlinear elasticity),
//   eps_t - u_x - v_y = 0,  (rho u)_t - sigma(eps)_x = 0,  (rho v)_t - sigma(eps)_y = 0,
// q = (eps, rho u, rho v), aux = (rho, K, stress-strain relation, eps at the
// start of the step), sigma = K eps (relation 1) or exp(K eps) - 1 (relation
// 2).  f-wave solver (LeVeque 2002, sec. 15.5; Ketcheson & LeVeque 2012 for
// the p-system in layered media): the flux difference is split into the
// left cell's eigenvector (1, Z, 0) at speed -c and the right cell's
// (1, -Z, 0) at speed c, c = sqrt(sigma'(eps) / rho), Z = rho c.
double psys_sigma(double eps, double K, double rel) { return rel == 1.0 ? K * eps : std::exp(K * eps) - 1.0; }
double psys_sigmap(double eps, double K, double rel) { return rel == 1.0 ? K : K * std::exp(K * eps); }

void rpn2_psystem(int ixy, int mbc, int mx, const CSlice& ql, const CSlice& qr, const CSlice& auxl,
                  const CSlice& auxr, const Waves& fwave, const Speeds& s, const Slice& amdq, const Slice& apdq) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double rhor = auxl(0, i), rhol = auxr(0, i - 1);
        const double Kr = auxl(1, i), Kl = auxr(1, i - 1);
        const double relr = auxl(2, i), rell = auxr(2, i - 1);
        const double epsr = ql(0, i), epsl = qr(0, i - 1);
        const double ur = ql(mu, i) / rhor, ul = qr(mu, i - 1) / rhol;
        const double cr = std::sqrt(psys_sigmap(epsr, Kr, relr) / rhor);
        const double cl = std::sqrt(psys_sigmap(epsl, Kl, rell) / rhol);
        const double zr = rhor * cr, zl = rhol * cl;
        const double df1 = -(ur - ul);
        const double df2 = -(psys_sigma(epsr, Kr, relr) - psys_sigma(epsl, Kl, rell));
        const double b1 = (df2 + zr * df1) / (zl + zr);
        const double b2 = (zl * df1 - df2) / (zl + zr);
        fwave(0, 0, i) = b1;
        fwave(mu, 0, i) = b1 * zl;
        fwave(mv, 0, i) = 0.0;
        s(0, i) = -cl;
        fwave(0, 1, i) = b2;
        fwave(mu, 1, i) = -b2 * zr;
        fwave(mv, 1, i) = 0.0;
        s(1, i) = cr;
        for (int m = 0; m < 3; ++m) {
            amdq(m, i) = fwave(m, 0, i);
            apdq(m, i) = fwave(m, 1, i);
        }
    }
}
// Transverse solve: asdq entered cell i1; it is split into the cell below's
// down-going eigenvector (1, 0, Zm) and the cell above's up-going one
// (1, 0, -Zp) -- one decomposition with the two neighbours' impedances -- and
// each part is multiplied by its cell's speed.  Sound speeds from the strain
// at the start of the step (aux component 4, set before each step).  This
// split reproduces the reference's psystem_2d gauges
// (examples/psystem_2d/test_2d_psystem.py:8-24) to their printed digits.
void rpt2_psystem(int ixy, int imp, int mbc, int mx, const CSlice& aux1, const CSlice& /*aux2*/, const CSlice& aux3,
                  const Slice& asdq, const Slice& bmasdq, const Slice& bpasdq) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int i1 = (imp == 1) ? i - 1 : i;
        const double rhom = aux1(0, i1), rhop = aux3(0, i1);
        const double cm = std::sqrt(psys_sigmap(aux1(3, i1), aux1(1, i1), aux1(2, i1)) / rhom);
        const double cp = std::sqrt(psys_sigmap(aux3(3, i1), aux3(1, i1), aux3(2, i1)) / rhop);
        const double zm = rhom * cm, zp = rhop * cp;
        const double bdown = (asdq(mv, i) + zp * asdq(0, i)) / (zm + zp);
        const double bup = (zm * asdq(0, i) - asdq(mv, i)) / (zm + zp);
        bmasdq(0, i) = -cm * bdown;
        bmasdq(mu, i) = 0.0;
        bmasdq(mv, i) = -cm * bdown * zm;
        bpasdq(0, i) = cp * bup;
        bpasdq(mu, i) = 0.0;
        bpasdq(mv, i) = -cp * bup * zp;
    }
}

// Euler equations, Roe solver with 4 waves (u-c, entropy, shear, u+c) and an
// optional Harten-Hyman entropy fix (LeVeque 2002, sec. 15.3.5 and 18.8;
// Roe 1981).  The wave layout follows the reference's vendored 5-wave solver
// development/rp_approaches/rpn2_euler_5wave.f:87-298 minus the tracer wave.
// cparam = gamma, efix.
void rpn2_euler_roe(int ixy, int mbc, int mx, int meqn, int mwaves, const CSlice& ql,
                    const CSlice& qr, const Waves& wave, const Speeds& s, const Slice& amdq,
                    const Slice& apdq, const double* cp) {
    const double gamma = cp[0];
    const bool efix = cp[1] != 0.0;
    const double gamma1 = gamma - 1.0;
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double rhsqrtl = std::sqrt(qr(0, i - 1));
        double rhsqrtr = std::sqrt(ql(0, i));
        double pl = gamma1 * (qr(3, i - 1) - 0.5 * (qr(1, i - 1) * qr(1, i - 1) +
                                                    qr(2, i - 1) * qr(2, i - 1)) / qr(0, i - 1));
        double pr = gamma1 * (ql(3, i) - 0.5 * (ql(1, i) * ql(1, i) + ql(2, i) * ql(2, i)) / ql(0, i));
        double rhsq2 = rhsqrtl + rhsqrtr;
        double u = (qr(mu, i - 1) / rhsqrtl + ql(mu, i) / rhsqrtr) / rhsq2;
        double v = (qr(mv, i - 1) / rhsqrtl + ql(mv, i) / rhsqrtr) / rhsq2;
        double enth = (((qr(3, i - 1) + pl) / rhsqrtl + (ql(3, i) + pr) / rhsqrtr)) / rhsq2;
        double u2v2 = u * u + v * v;
        double a2 = gamma1 * (enth - 0.5 * u2v2);
        double a = std::sqrt(a2);
        double g1a2 = gamma1 / a2;
        double euv = enth - u2v2;

        double delta0 = ql(0, i) - qr(0, i - 1);
        double delta1 = ql(mu, i) - qr(mu, i - 1);
        double delta2 = ql(mv, i) - qr(mv, i - 1);
        double delta3 = ql(3, i) - qr(3, i - 1);
        double b3 = g1a2 * (euv * delta0 + u * delta1 + v * delta2 - delta3);
        double b2 = delta2 - v * delta0;
        double b4 = (delta1 + (a - u) * delta0 - a * b3) / (2.0 * a);
        double b1 = delta0 - b3 - b4;

        wave(0, 0, i) = b1;
        wave(mu, 0, i) = b1 * (u - a);
        wave(mv, 0, i) = b1 * v;
        wave(3, 0, i) = b1 * (enth - u * a);
        s(0, i) = u - a;

        wave(0, 1, i) = b3;
        wave(mu, 1, i) = b3 * u;
        wave(mv, 1, i) = b3 * v;
        wave(3, 1, i) = b3 * 0.5 * u2v2;
        s(1, i) = u;

        wave(0, 2, i) = 0.0;
        wave(mu, 2, i) = 0.0;
        wave(mv, 2, i) = b2;
        wave(3, 2, i) = b2 * v;
        s(2, i) = u;

        wave(0, 3, i) = b4;
        wave(mu, 3, i) = b4 * (u + a);
        wave(mv, 3, i) = b4 * v;
        wave(3, 3, i) = b4 * (enth + u * a);
        s(3, i) = u + a;
    }

    if (!efix) {
        for (int m = 0; m < meqn; ++m)
            for (int i = 2 - mbc; i <= mx + mbc; ++i) {
                amdq(m, i) = 0.0;
                apdq(m, i) = 0.0;
                for (int mw = 0; mw < mwaves; ++mw) {
                    if (s(mw, i) < 0.0)
                        amdq(m, i) = amdq(m, i) + s(mw, i) * wave(m, mw, i);
                    else
                        apdq(m, i) = apdq(m, i) + s(mw, i) * wave(m, mw, i);
                }
            }
        return;
    }

    // Harten-Hyman entropy fix: split a transonic rarefaction's flux
    // difference using the characteristic speeds on either side of it.
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        // 1-wave (u - c)
        double rhoim1 = qr(0, i - 1);
        double pim1 = gamma1 * (qr(3, i - 1) - 0.5 * (qr(mu, i - 1) * qr(mu, i - 1) +
                                                      qr(mv, i - 1) * qr(mv, i - 1)) / rhoim1);
        double cim1 = std::sqrt(gamma * pim1 / rhoim1);
        double s0 = qr(mu, i - 1) / rhoim1 - cim1;
        if (s0 >= 0.0 && s(0, i) > 0.0) {
            for (int m = 0; m < meqn; ++m) amdq(m, i) = 0.0;
            goto done;
        }
        {
            double rho1 = qr(0, i - 1) + wave(0, 0, i);
            double rhou1 = qr(mu, i - 1) + wave(mu, 0, i);
            double rhov1 = qr(mv, i - 1) + wave(mv, 0, i);
            double en1 = qr(3, i - 1) + wave(3, 0, i);
            double p1 = gamma1 * (en1 - 0.5 * (rhou1 * rhou1 + rhov1 * rhov1) / rho1);
            double c1 = std::sqrt(gamma * p1 / rho1);
            double s1 = rhou1 / rho1 - c1;
            double sfract;
            if (s0 < 0.0 && s1 > 0.0)
                sfract = s0 * (s1 - s(0, i)) / (s1 - s0);
            else if (s(0, i) < 0.0)
                sfract = s(0, i);
            else
                sfract = 0.0;
            for (int m = 0; m < meqn; ++m) amdq(m, i) = sfract * wave(m, 0, i);
        }
        // 2- and 3-waves (speed u)
        if (s(1, i) >= 0.0) goto done;
        for (int m = 0; m < meqn; ++m)
            amdq(m, i) = amdq(m, i) + s(1, i) * wave(m, 1, i) + s(2, i) * wave(m, 2, i);
        {
            // 4-wave (u + c)
            double rhoi = ql(0, i);
            double pi = gamma1 * (ql(3, i) - 0.5 * (ql(mu, i) * ql(mu, i) + ql(mv, i) * ql(mv, i)) / rhoi);
            double ci = std::sqrt(gamma * pi / rhoi);
            double s3 = ql(mu, i) / rhoi + ci;
            double rho2 = ql(0, i) - wave(0, 3, i);
            double rhou2 = ql(mu, i) - wave(mu, 3, i);
            double rhov2 = ql(mv, i) - wave(mv, 3, i);
            double en2 = ql(3, i) - wave(3, 3, i);
            double p2 = gamma1 * (en2 - 0.5 * (rhou2 * rhou2 + rhov2 * rhov2) / rho2);
            double c2 = std::sqrt(gamma * p2 / rho2);
            double s2 = rhou2 / rho2 + c2;
            double sfract;
            if (s2 < 0.0 && s3 > 0.0)
                sfract = s2 * (s3 - s(3, i)) / (s3 - s2);
            else if (s(3, i) < 0.0)
                sfract = s(3, i);
            else
                goto done;
            for (int m = 0; m < meqn; ++m) amdq(m, i) = amdq(m, i) + sfract * wave(m, 3, i);
        }
    done:;
    }
    for (int m = 0; m < meqn; ++m)
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            double df = 0.0;
            for (int mw = 0; mw < mwaves; ++mw) df = df + s(mw, i) * wave(m, mw, i);
            apdq(m, i) = df - amdq(m, i);
        }
}

// Euler equations with a tracer, Roe solver with five waves (acoustic,
// shear, entropy, acoustic, tracer) and the Harten-Hyman entropy fix, in the
// order and form of development/rp_approaches/rpn2_euler_5wave.f:86-297
// (cparam = gamma, efix).  q = (rho, rho u, rho v, E, tracer); the tracer
// jump moves at the Roe-averaged normal velocity.
void rpn2_euler_5wave(int ixy, int mbc, int mx, int meqn, int mwaves, const CSlice& ql, const CSlice& qr,
                      const Waves& wave, const Speeds& s, const Slice& amdq, const Slice& apdq, const double* cp) {
    const double gamma = cp[0];
    const bool efix = cp[1] != 0.0;
    const double gamma1 = gamma - 1.0;
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double rhsqrtl = std::sqrt(qr(0, i - 1));
        double rhsqrtr = std::sqrt(ql(0, i));
        double pl = gamma1 * (qr(3, i - 1) - 0.5 * (qr(1, i - 1) * qr(1, i - 1) +
                                                    qr(2, i - 1) * qr(2, i - 1)) / qr(0, i - 1));
        double pr = gamma1 * (ql(3, i) - 0.5 * (ql(1, i) * ql(1, i) + ql(2, i) * ql(2, i)) / ql(0, i));
        double rhsq2 = rhsqrtl + rhsqrtr;
        double u = (qr(mu, i - 1) / rhsqrtl + ql(mu, i) / rhsqrtr) / rhsq2;
        double v = (qr(mv, i - 1) / rhsqrtl + ql(mv, i) / rhsqrtr) / rhsq2;
        double enth = (((qr(3, i - 1) + pl) / rhsqrtl + (ql(3, i) + pr) / rhsqrtr)) / rhsq2;
        double u2v2 = u * u + v * v;
        double a2 = gamma1 * (enth - 0.5 * u2v2);
        double a = std::sqrt(a2);
        double g1a2 = gamma1 / a2;
        double euv = enth - u2v2;
        double d0 = ql(0, i) - qr(0, i - 1), d1 = ql(mu, i) - qr(mu, i - 1);
        double d2 = ql(mv, i) - qr(mv, i - 1), d3 = ql(3, i) - qr(3, i - 1);
        double a3 = g1a2 * (euv * d0 + u * d1 + v * d2 - d3);
        double a2w = d2 - v * d0;
        double a4 = (d1 + (a - u) * d0 - a * a3) / (2.0 * a);
        double a1 = d0 - a3 - a4;
        wave(0, 0, i) = a1; wave(mu, 0, i) = a1 * (u - a); wave(mv, 0, i) = a1 * v;
        wave(3, 0, i) = a1 * (enth - u * a); wave(4, 0, i) = 0.0; s(0, i) = u - a;
        wave(0, 1, i) = 0.0; wave(mu, 1, i) = 0.0; wave(mv, 1, i) = a2w;
        wave(3, 1, i) = a2w * v; wave(4, 1, i) = 0.0; s(1, i) = u;
        wave(0, 2, i) = a3; wave(mu, 2, i) = a3 * u; wave(mv, 2, i) = a3 * v;
        wave(3, 2, i) = a3 * 0.5 * u2v2; wave(4, 2, i) = 0.0; s(2, i) = u;
        wave(0, 3, i) = a4; wave(mu, 3, i) = a4 * (u + a); wave(mv, 3, i) = a4 * v;
        wave(3, 3, i) = a4 * (enth + u * a); wave(4, 3, i) = 0.0; s(3, i) = u + a;
        wave(0, 4, i) = 0.0; wave(mu, 4, i) = 0.0; wave(mv, 4, i) = 0.0; wave(3, 4, i) = 0.0;
        wave(4, 4, i) = ql(4, i) - qr(4, i - 1); s(4, i) = u;
    }
    if (!efix) {
        for (int m = 0; m < meqn; ++m)
            for (int i = 2 - mbc; i <= mx + mbc; ++i) {
                amdq(m, i) = 0.0;
                apdq(m, i) = 0.0;
                for (int mw = 0; mw < mwaves; ++mw) {
                    if (s(mw, i) < 0.0) amdq(m, i) = amdq(m, i) + s(mw, i) * wave(m, mw, i);
                    else apdq(m, i) = apdq(m, i) + s(mw, i) * wave(m, mw, i);
                }
            }
        return;
    }
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double rhoim1 = qr(0, i - 1);
        double pim1 = gamma1 * (qr(3, i - 1) - 0.5 * (qr(mu, i - 1) * qr(mu, i - 1) +
                                                      qr(mv, i - 1) * qr(mv, i - 1)) / rhoim1);
        double cim1 = std::sqrt(gamma * pim1 / rhoim1);
        double s0 = qr(mu, i - 1) / rhoim1 - cim1;
        if (s0 >= 0.0 && s(0, i) > 0.0) {
            for (int m = 0; m < meqn; ++m) amdq(m, i) = 0.0;
            continue;
        }
        {
            double rho1 = qr(0, i - 1) + wave(0, 0, i);
            double rhou1 = qr(mu, i - 1) + wave(mu, 0, i);
            double rhov1 = qr(mv, i - 1) + wave(mv, 0, i);
            double en1 = qr(3, i - 1) + wave(3, 0, i);
            double p1 = gamma1 * (en1 - 0.5 * (rhou1 * rhou1 + rhov1 * rhov1) / rho1);
            double c1 = std::sqrt(gamma * p1 / rho1);
            double s1 = rhou1 / rho1 - c1;
            double sfract;
            if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s(0, i)) / (s1 - s0);
            else if (s(0, i) < 0.0) sfract = s(0, i);
            else sfract = 0.0;
            for (int m = 0; m < meqn; ++m) amdq(m, i) = sfract * wave(m, 0, i);
        }
        if (s(1, i) >= 0.0) continue;
        for (int m = 0; m < meqn; ++m) {
            amdq(m, i) = amdq(m, i) + s(1, i) * wave(m, 1, i);
            amdq(m, i) = amdq(m, i) + s(2, i) * wave(m, 2, i);
            amdq(m, i) = amdq(m, i) + s(4, i) * wave(m, 4, i);
        }
        {
            double rhoi = ql(0, i);
            double pi = gamma1 * (ql(3, i) - 0.5 * (ql(mu, i) * ql(mu, i) + ql(mv, i) * ql(mv, i)) / rhoi);
            double ci = std::sqrt(gamma * pi / rhoi);
            double s3 = ql(mu, i) / rhoi + ci;
            double rho2 = ql(0, i) - wave(0, 3, i);
            double rhou2 = ql(mu, i) - wave(mu, 3, i);
            double rhov2 = ql(mv, i) - wave(mv, 3, i);
            double en2 = ql(3, i) - wave(3, 3, i);
            double p2 = gamma1 * (en2 - 0.5 * (rhou2 * rhou2 + rhov2 * rhov2) / rho2);
            double c2 = std::sqrt(gamma * p2 / rho2);
            double s2 = rhou2 / rho2 + c2;
            double sfract;
            if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - s(3, i)) / (s3 - s2);
            else if (s(3, i) < 0.0) sfract = s(3, i);
            else continue;
            for (int m = 0; m < meqn; ++m) amdq(m, i) = amdq(m, i) + sfract * wave(m, 3, i);
        }
    }
    for (int m = 0; m < meqn; ++m)
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            double df = 0.0;
            for (int mw = 0; mw < mwaves; ++mw) df = df + s(mw, i) * wave(m, mw, i);
            apdq(m, i) = df - amdq(m, i);
        }
}

// Transverse split of the 5-wave solver (rpt2_euler_5wave.f:47-95): the Roe
// state of the interface, four transverse waves (acoustic, shear+entropy,
// acoustic, tracer).
void rpt2_euler_5wave(int ixy, int mbc, int mx, int meqn, const CSlice& ql, const CSlice& qr, const Slice& asdq,
                      const Slice& bmasdq, const Slice& bpasdq, const double* cp) {
    const double gamma1 = cp[0] - 1.0;
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    double waveb[4][5], sb[4];
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double rhsqrtl = std::sqrt(qr(0, i - 1));
        double rhsqrtr = std::sqrt(ql(0, i));
        double pl = gamma1 * (qr(3, i - 1) - 0.5 * (qr(1, i - 1) * qr(1, i - 1) +
                                                    qr(2, i - 1) * qr(2, i - 1)) / qr(0, i - 1));
        double pr = gamma1 * (ql(3, i) - 0.5 * (ql(1, i) * ql(1, i) + ql(2, i) * ql(2, i)) / ql(0, i));
        double rhsq2 = rhsqrtl + rhsqrtr;
        double u = (qr(mu, i - 1) / rhsqrtl + ql(mu, i) / rhsqrtr) / rhsq2;
        double v = (qr(mv, i - 1) / rhsqrtl + ql(mv, i) / rhsqrtr) / rhsq2;
        double enth = (((qr(3, i - 1) + pl) / rhsqrtl + (ql(3, i) + pr) / rhsqrtr)) / rhsq2;
        double u2v2 = u * u + v * v;
        double a2 = gamma1 * (enth - 0.5 * u2v2);
        double a = std::sqrt(a2);
        double g1a2 = gamma1 / a2;
        double euv = enth - u2v2;
        double a3 = g1a2 * (euv * asdq(0, i) + u * asdq(mu, i) + v * asdq(mv, i) - asdq(3, i));
        double a2w = asdq(mu, i) - u * asdq(0, i);
        double a4 = (asdq(mv, i) + (a - v) * asdq(0, i) - a * a3) / (2.0 * a);
        double a1 = asdq(0, i) - a3 - a4;
        waveb[0][0] = a1; waveb[0][mu] = a1 * u; waveb[0][mv] = a1 * (v - a);
        waveb[0][3] = a1 * (enth - v * a); waveb[0][4] = 0.0; sb[0] = v - a;
        waveb[1][0] = a3; waveb[1][mu] = a3 * u + a2w; waveb[1][mv] = a3 * v;
        waveb[1][3] = a3 * 0.5 * u2v2 + a2w * u; waveb[1][4] = 0.0; sb[1] = v;
        waveb[2][0] = a4; waveb[2][mu] = a4 * u; waveb[2][mv] = a4 * (v + a);
        waveb[2][3] = a4 * (enth + v * a); waveb[2][4] = 0.0; sb[2] = v + a;
        waveb[3][0] = 0.0; waveb[3][mu] = 0.0; waveb[3][mv] = 0.0; waveb[3][3] = 0.0;
        waveb[3][4] = asdq(4, i); sb[3] = v;
        for (int m = 0; m < meqn; ++m) {
            bmasdq(m, i) = 0.0;
            bpasdq(m, i) = 0.0;
            for (int mw = 0; mw < 4; ++mw) {
                bmasdq(m, i) = bmasdq(m, i) + std::min(sb[mw], 0.0) * waveb[mw][m];
                bpasdq(m, i) = bpasdq(m, i) + std::max(sb[mw], 0.0) * waveb[mw][m];
            }
        }
    }
}

// HLLE solver (Harten, Lax & van Leer 1983 with Einfeldt's 1988 speed
// estimates): two waves through the HLL middle state
//   q_m = (f(q_r) - f(q_l) - s2 q_r + s1 q_l) / (s1 - s2),
// s1 = min(u_l - c_l, u_hat - c_hat), s2 = max(u_r + c_r, u_hat + c_hat) with
// the Roe velocity u_hat and c_hat = sqrt(g (h_l + h_r) / 2); fluctuations =
// sum of s^-/s^+ times the waves.
// shallow_hlle_2D: cparam = grav.  No transverse solve (split step).
void rpn2_shallow_hlle(int ixy, int mbc, int mx, int meqn, const CSlice& ql, const CSlice& qr, const Waves& wave,
                       const Speeds& s, const Slice& amdq, const Slice& apdq, const double* cp) {
    const double g = cp[0];
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double h_l = qr(0, i - 1), hu_l = qr(mu, i - 1), hv_l = qr(mv, i - 1);
        const double h_r = ql(0, i), hu_r = ql(mu, i), hv_r = ql(mv, i);
        const double u_l = hu_l / h_l, v_l = hv_l / h_l, u_r = hu_r / h_r, v_r = hv_r / h_r;
        const double c_l = std::sqrt(g * h_l), c_r = std::sqrt(g * h_r);
        const double rsl = std::sqrt(h_l), rsr = std::sqrt(h_r);
        const double u_hat = (rsl * u_l + rsr * u_r) / (rsl + rsr);
        const double c_hat = std::sqrt(0.5 * g * (h_l + h_r));
        const double s1 = std::min(u_l - c_l, u_hat - c_hat);
        const double s2 = std::max(u_r + c_r, u_hat + c_hat);
        const double den = s1 - s2;
        const double h_m = (hu_r - hu_l - s2 * h_r + s1 * h_l) / den;
        const double hu_m = (hu_r * u_r + 0.5 * g * h_r * h_r - hu_l * u_l - 0.5 * g * h_l * h_l - s2 * hu_r +
                             s1 * hu_l) / den;
        const double hv_m = (hu_r * v_r - hu_l * v_l - s2 * hv_r + s1 * hv_l) / den;
        wave(0, 0, i) = h_m - h_l; wave(mu, 0, i) = hu_m - hu_l; wave(mv, 0, i) = hv_m - hv_l; s(0, i) = s1;
        wave(0, 1, i) = h_r - h_m; wave(mu, 1, i) = hu_r - hu_m; wave(mv, 1, i) = hv_r - hv_m; s(1, i) = s2;
        for (int m = 0; m < meqn; ++m) {
            amdq(m, i) = std::min(s1, 0.0) * wave(m, 0, i) + std::min(s2, 0.0) * wave(m, 1, i);
            apdq(m, i) = std::max(s1, 0.0) * wave(m, 0, i) + std::max(s2, 0.0) * wave(m, 1, i);
        }
    }
}

// Transverse Roe split for Euler: decompose asdq on the eigenvectors of the
// transverse Jacobian at the same Roe-averaged state and keep the down- and
// up-going parts (LeVeque 2002, sec. 21.6; reference structure
// development/rp_approaches/rpt2_euler_5wave.f:47-95 minus the tracer).
void rpt2_euler_roe(int ixy, int mbc, int mx, int meqn, int mwaves, const CSlice& ql,
                    const CSlice& qr, const Slice& asdq, const Slice& bmasdq,
                    const Slice& bpasdq, const double* cp) {
    const double gamma = cp[0];
    const double gamma1 = gamma - 1.0;
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    double waveb[4][4], sb[4];
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double rhsqrtl = std::sqrt(qr(0, i - 1));
        double rhsqrtr = std::sqrt(ql(0, i));
        double pl = gamma1 * (qr(3, i - 1) - 0.5 * (qr(1, i - 1) * qr(1, i - 1) +
                                                    qr(2, i - 1) * qr(2, i - 1)) / qr(0, i - 1));
        double pr = gamma1 * (ql(3, i) - 0.5 * (ql(1, i) * ql(1, i) + ql(2, i) * ql(2, i)) / ql(0, i));
        double rhsq2 = rhsqrtl + rhsqrtr;
        double u = (qr(mu, i - 1) / rhsqrtl + ql(mu, i) / rhsqrtr) / rhsq2;
        double v = (qr(mv, i - 1) / rhsqrtl + ql(mv, i) / rhsqrtr) / rhsq2;
        double enth = (((qr(3, i - 1) + pl) / rhsqrtl + (ql(3, i) + pr) / rhsqrtr)) / rhsq2;
        double u2v2 = u * u + v * v;
        double a2 = gamma1 * (enth - 0.5 * u2v2);
        double a = std::sqrt(a2);
        double g1a2 = gamma1 / a2;
        double euv = enth - u2v2;

        double b3 = g1a2 * (euv * asdq(0, i) + u * asdq(mu, i) + v * asdq(mv, i) - asdq(3, i));
        double b2 = asdq(mu, i) - u * asdq(0, i);
        double b4 = (asdq(mv, i) + (a - v) * asdq(0, i) - a * b3) / (2.0 * a);
        double b1 = asdq(0, i) - b3 - b4;

        waveb[0][0] = b1; waveb[0][mu] = b1 * u; waveb[0][mv] = b1 * (v - a);
        waveb[0][3] = b1 * (enth - v * a); sb[0] = v - a;
        waveb[1][0] = b3; waveb[1][mu] = b3 * u; waveb[1][mv] = b3 * v;
        waveb[1][3] = b3 * 0.5 * u2v2; sb[1] = v;
        waveb[2][0] = 0.0; waveb[2][mu] = b2; waveb[2][mv] = 0.0;
        waveb[2][3] = b2 * u; sb[2] = v;
        waveb[3][0] = b4; waveb[3][mu] = b4 * u; waveb[3][mv] = b4 * (v + a);
        waveb[3][3] = b4 * (enth + v * a); sb[3] = v + a;

        for (int m = 0; m < meqn; ++m) {
            bmasdq(m, i) = 0.0;
            bpasdq(m, i) = 0.0;
            for (int mw = 0; mw < mwaves; ++mw) {
                bmasdq(m, i) = bmasdq(m, i) + std::min(sb[mw], 0.0) * waveb[mw][m];
                bpasdq(m, i) = bpasdq(m, i) + std::max(sb[mw], 0.0) * waveb[mw][m];
            }
        }
    }
}

// Shallow water equations, Roe solver with Harten-Hyman entropy fix
// (LeVeque 2002, sec. 15.3 and 21.6).  cparam = grav, efix.
void rpn2_shallow_roe(int ixy, int mbc, int mx, int meqn, int mwaves, const CSlice& ql,
                      const CSlice& qr, const Waves& wave, const Speeds& s, const Slice& amdq,
                      const Slice& apdq, const double* cp) {
    const double grav = cp[0];
    const bool efix = cp[1] != 0.0;
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double h = (qr(0, i - 1) + ql(0, i)) * 0.50;
        double hsqrtl = std::sqrt(qr(0, i - 1));
        double hsqrtr = std::sqrt(ql(0, i));
        double hsq2 = hsqrtl + hsqrtr;
        double u = (qr(mu, i - 1) / hsqrtl + ql(mu, i) / hsqrtr) / hsq2;
        double v = (qr(mv, i - 1) / hsqrtl + ql(mv, i) / hsqrtr) / hsq2;
        double a = std::sqrt(grav * h);

        double delta0 = ql(0, i) - qr(0, i - 1);
        double delta1 = ql(mu, i) - qr(mu, i - 1);
        double delta2 = ql(mv, i) - qr(mv, i - 1);
        double a1 = ((u + a) * delta0 - delta1) * (0.50 / a);
        double a2 = -v * delta0 + delta2;
        double a3 = (-(u - a) * delta0 + delta1) * (0.50 / a);

        wave(0, 0, i) = a1;
        wave(mu, 0, i) = a1 * (u - a);
        wave(mv, 0, i) = a1 * v;
        s(0, i) = u - a;
        wave(0, 1, i) = 0.0;
        wave(mu, 1, i) = 0.0;
        wave(mv, 1, i) = a2;
        s(1, i) = u;
        wave(0, 2, i) = a3;
        wave(mu, 2, i) = a3 * (u + a);
        wave(mv, 2, i) = a3 * v;
        s(2, i) = u + a;
    }

    if (!efix) {
        for (int m = 0; m < meqn; ++m)
            for (int i = 2 - mbc; i <= mx + mbc; ++i) {
                amdq(m, i) = 0.0;
                apdq(m, i) = 0.0;
                for (int mw = 0; mw < mwaves; ++mw) {
                    if (s(mw, i) < 0.0)
                        amdq(m, i) = amdq(m, i) + s(mw, i) * wave(m, mw, i);
                    else
                        apdq(m, i) = apdq(m, i) + s(mw, i) * wave(m, mw, i);
                }
            }
        return;
    }

    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        // 1-wave
        double him1 = qr(0, i - 1);
        double s0 = qr(mu, i - 1) / him1 - std::sqrt(grav * him1);
        if (s0 >= 0.0 && s(0, i) > 0.0) {
            for (int m = 0; m < meqn; ++m) amdq(m, i) = 0.0;
            continue;
        }
        {
            double h1 = qr(0, i - 1) + wave(0, 0, i);
            double hu1 = qr(mu, i - 1) + wave(mu, 0, i);
            double s1 = hu1 / h1 - std::sqrt(grav * h1);
            double sfract;
            if (s0 < 0.0 && s1 > 0.0)
                sfract = s0 * ((s1 - s(0, i)) / (s1 - s0));
            else if (s(0, i) < 0.0)
                sfract = s(0, i);
            else
                sfract = 0.0;
            for (int m = 0; m < meqn; ++m) amdq(m, i) = sfract * wave(m, 0, i);
        }
        // 2-wave
        if (s(1, i) > 0.0) continue;
        for (int m = 0; m < meqn; ++m) amdq(m, i) = amdq(m, i) + s(1, i) * wave(m, 1, i);
        {
            // 3-wave
            double hi = ql(0, i);
            double s03 = ql(mu, i) / hi + std::sqrt(grav * hi);
            double h3 = ql(0, i) - wave(0, 2, i);
            double hu3 = ql(mu, i) - wave(mu, 2, i);
            double s3 = hu3 / h3 + std::sqrt(grav * h3);
            double sfract;
            if (s3 < 0.0 && s03 > 0.0)
                sfract = s3 * ((s03 - s(2, i)) / (s03 - s3));
            else if (s(2, i) < 0.0)
                sfract = s(2, i);
            else
                continue;
            for (int m = 0; m < meqn; ++m) amdq(m, i) = amdq(m, i) + sfract * wave(m, 2, i);
        }
    }
    for (int m = 0; m < meqn; ++m)
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            double df = 0.0;
            for (int mw = 0; mw < mwaves; ++mw) df = df + s(mw, i) * wave(m, mw, i);
            apdq(m, i) = df - amdq(m, i);
        }
}

void rpt2_shallow_roe(int ixy, int mbc, int mx, int meqn, int mwaves, const CSlice& ql,
                      const CSlice& qr, const Slice& asdq, const Slice& bmasdq,
                      const Slice& bpasdq, const double* cp) {
    const double grav = cp[0];
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    double waveb[3][3], sb[3];
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double hsqrtl = std::sqrt(qr(0, i - 1));
        double hsqrtr = std::sqrt(ql(0, i));
        double hsq2 = hsqrtl + hsqrtr;
        double ubar = (qr(mu, i - 1) / hsqrtl + ql(mu, i) / hsqrtr) / hsq2;
        double vbar = (qr(mv, i - 1) / hsqrtl + ql(mv, i) / hsqrtr) / hsq2;
        double cbar = std::sqrt(0.5 * grav * (qr(0, i - 1) + ql(0, i)));

        double a1 = (0.5 / cbar) * ((vbar + cbar) * asdq(0, i) - asdq(mv, i));
        double a2 = -ubar * asdq(0, i) + asdq(mu, i);
        double a3 = (0.5 / cbar) * (-(vbar - cbar) * asdq(0, i) + asdq(mv, i));

        waveb[0][0] = a1; waveb[0][mu] = a1 * ubar; waveb[0][mv] = a1 * (vbar - cbar);
        sb[0] = vbar - cbar;
        waveb[1][0] = 0.0; waveb[1][mu] = a2; waveb[1][mv] = 0.0;
        sb[1] = vbar;
        waveb[2][0] = a3; waveb[2][mu] = a3 * ubar; waveb[2][mv] = a3 * (vbar + cbar);
        sb[2] = vbar + cbar;

        for (int m = 0; m < meqn; ++m) {
            bmasdq(m, i) = 0.0;
            bpasdq(m, i) = 0.0;
            for (int mw = 0; mw < mwaves; ++mw) {
                bmasdq(m, i) = bmasdq(m, i) + std::min(sb[mw], 0.0) * waveb[mw][m];
                bpasdq(m, i) = bpasdq(m, i) + std::max(sb[mw], 0.0) * waveb[mw][m];
            }
        }
    }
}


// ---------------------------------------------------------------------------
// Exact Euler Riemann solver (no reference counterpart), restated from Toro,
// Riemann Solvers and Numerical Methods for Fluid Dynamics (3rd ed., 2009):
// guess (sec. 9.5.1 adaptive PVRS / TRRS / TSRS), pressure functions
// (eqs. 4.6-4.7, 4.37), Newton with the relative-change test of sec. 4.3.2,
// star velocity (eq. 4.9) and sampling at x/t = 0 (sec. 4.5).
// ---------------------------------------------------------------------------
struct ExGas {
    double g, g1, g2, g3, g4, g5, g6, g7;
    explicit ExGas(double gamma) : g(gamma) {
        g1 = (g - 1.0) / (2.0 * g); g2 = (g + 1.0) / (2.0 * g); g3 = 2.0 * g / (g - 1.0);
        g4 = 2.0 / (g - 1.0); g5 = 2.0 / (g + 1.0); g6 = (g - 1.0) / (g + 1.0); g7 = (g - 1.0) / 2.0;
    }
};

void ex_prefun(const ExGas& G, double p, double dk, double pk, double ck, double& f, double& fd) {
    if (p <= pk) {
        double prat = p / pk;
        f = G.g4 * ck * (std::pow(prat, G.g1) - 1.0);
        fd = (1.0 / (dk * ck)) * std::pow(prat, -G.g2);
    } else {
        double ak = G.g5 / dk, bk = G.g6 * pk, qrt = std::sqrt(ak / (bk + p));
        f = (p - pk) * qrt;
        fd = (1.0 - 0.5 * (p - pk) / (bk + p)) * qrt;
    }
}

double ex_guess(const ExGas& G, double dl, double ul, double pl, double cl, double dr, double ur, double pr, double cr) {
    double cup = 0.25 * (dl + dr) * (cl + cr);
    double ppv = std::max(0.0, 0.5 * (pl + pr) + 0.5 * (ul - ur) * cup);
    double pmin = std::min(pl, pr), pmax = std::max(pl, pr), qmax = pmax / pmin;
    if (qmax <= 2.0 && pmin <= ppv && ppv <= pmax) return ppv;
    if (ppv < pmin) {
        double pq = std::pow(pl / pr, G.g1);
        double um = (pq * ul / cl + ur / cr + G.g4 * (pq - 1.0)) / (pq / cl + 1.0 / cr);
        double ptl = 1.0 + G.g7 * (ul - um) / cl, ptr = 1.0 + G.g7 * (um - ur) / cr;
        return 0.5 * (pl * std::pow(ptl, G.g3) + pr * std::pow(ptr, G.g3));
    }
    double gel = std::sqrt((G.g5 / dl) / (G.g6 * pl + ppv));
    double ger = std::sqrt((G.g5 / dr) / (G.g6 * pr + ppv));
    return (gel * pl + ger * pr - (ur - ul)) / (gel + ger);
}

// returns false on vacuum
bool ex_starpu(const ExGas& G, double dl, double ul, double pl, double dr, double ur, double pr, double tol,
               double& p, double& u, int& iters) {
    double cl = std::sqrt(G.g * pl / dl), cr = std::sqrt(G.g * pr / dr);
    iters = 0;
    if (G.g4 * (cl + cr) <= ur - ul) return false;
    if (dl == dr && ul == ur && pl == pr) { p = pl; u = ul; return true; }
    double pold = std::max(ex_guess(G, dl, ul, pl, cl, dr, ur, pr, cr), tol);
    double udiff = ur - ul, fl = 0, fr = 0, fld, frd;
    for (int i = 1; i <= 100; ++i) {
        ex_prefun(G, pold, dl, pl, cl, fl, fld);
        ex_prefun(G, pold, dr, pr, cr, fr, frd);
        p = pold - (fl + fr + udiff) / (fld + frd);
        double change = 2.0 * std::fabs((p - pold) / (p + pold));
        ++iters;
        if (change <= tol) break;
        if (p < 0.0) p = tol;
        pold = p;
    }
    ex_prefun(G, p, dl, pl, cl, fl, fld);
    ex_prefun(G, p, dr, pr, cr, fr, frd);
    u = 0.5 * (ul + ur + fr - fl);
    return true;
}

// state at x/t = 0 (Toro SAMPLE with S = 0); left = point left of the contact
void ex_sample0(const ExGas& G, double pm, double um, double dl, double ul, double pl, double dr, double ur, double pr,
                double& d, double& u, double& p, bool& left) {
    double cl = std::sqrt(G.g * pl / dl), cr = std::sqrt(G.g * pr / dr);
    const double s = 0.0;
    left = s <= um;
    if (left) {
        if (pm <= pl) {
            double shl = ul - cl;
            if (s <= shl) { d = dl; u = ul; p = pl; return; }
            double cml = cl * std::pow(pm / pl, G.g1), stl = um - cml;
            if (s > stl) { d = dl * std::pow(pm / pl, 1.0 / G.g); u = um; p = pm; return; }
            u = G.g5 * (cl + G.g7 * ul + s);
            double c = G.g5 * (cl + G.g7 * (ul - s));
            d = dl * std::pow(c / cl, G.g4);
            p = pl * std::pow(c / cl, G.g3);
        } else {
            double pml = pm / pl, sl = ul - cl * std::sqrt(G.g2 * pml + G.g1);
            if (s <= sl) { d = dl; u = ul; p = pl; }
            else { d = dl * (pml + G.g6) / (pml * G.g6 + 1.0); u = um; p = pm; }
        }
    } else {
        if (pm > pr) {
            double pmr = pm / pr, sr = ur + cr * std::sqrt(G.g2 * pmr + G.g1);
            if (s >= sr) { d = dr; u = ur; p = pr; }
            else { d = dr * (pmr + G.g6) / (pmr * G.g6 + 1.0); u = um; p = pm; }
        } else {
            double shr = ur + cr;
            if (s >= shr) { d = dr; u = ur; p = pr; return; }
            double cmr = cr * std::pow(pm / pr, G.g1), str = um + cmr;
            if (s <= str) { d = dr * std::pow(pm / pr, 1.0 / G.g); u = um; p = pm; return; }
            u = G.g5 * (-cr + G.g7 * ur + s);
            double c = G.g5 * (cr - G.g7 * (ur - s));
            d = dr * std::pow(c / cr, G.g4);
            p = pr * std::pow(c / cr, G.g3);
        }
    }
}

int g_exact_vacuum = 0;

// Wave-propagation form of the exact solver on a slice: waves Q*L - QL,
// Q*R - Q*L, QR - Q*R; speeds = shock speed or the fan's mean speed, u*;
// fluctuations from the Godunov flux F(Q(0)).  cparam = gamma, tol.
void rpn2_euler_exact(int ixy, int mbc, int mx, int meqn, int mwaves, const CSlice& ql, const CSlice& qr,
                      const Waves& wave, const Speeds& s, const Slice& amdq, const Slice& apdq, const double* cp) {
    (void)meqn; (void)mwaves;
    const double gamma = cp[0], tol = cp[1], g1 = gamma - 1.0;
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    ExGas G(gamma);
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double QL[4], QR[4];
        for (int m = 0; m < 4; ++m) { QL[m] = qr(m, i - 1); QR[m] = ql(m, i); }
        double dl = QL[0], ul = QL[mu] / dl, vl = QL[mv] / dl, pl = g1 * (QL[3] - 0.5 * dl * (ul * ul + vl * vl));
        double dr = QR[0], ur = QR[mu] / dr, vr = QR[mv] / dr, pr = g1 * (QR[3] - 0.5 * dr * (ur * ur + vr * vr));
        double pm, um;
        int it;
        if (!ex_starpu(G, dl, ul, pl, dr, ur, pr, tol, pm, um, it)) {
            g_exact_vacuum = 1;
            pm = 0.5 * (pl + pr); um = 0.5 * (ul + ur);
        }
        double cl = std::sqrt(gamma * pl / dl), cr = std::sqrt(gamma * pr / dr);
        double dsl, dsr, s1, s3;
        if (pm > pl) {
            double pml = pm / pl;
            dsl = dl * (pml + G.g6) / (pml * G.g6 + 1.0);
            s1 = ul - cl * std::sqrt(G.g2 * pml + G.g1);
        } else {
            dsl = dl * std::pow(pm / pl, 1.0 / gamma);
            s1 = 0.5 * ((ul - cl) + (um - cl * std::pow(pm / pl, G.g1)));
        }
        if (pm > pr) {
            double pmr = pm / pr;
            dsr = dr * (pmr + G.g6) / (pmr * G.g6 + 1.0);
            s3 = ur + cr * std::sqrt(G.g2 * pmr + G.g1);
        } else {
            dsr = dr * std::pow(pm / pr, 1.0 / gamma);
            s3 = 0.5 * ((ur + cr) + (um + cr * std::pow(pm / pr, G.g1)));
        }
        auto cons = [&](double d, double un, double ut, double p, double* Q) {
            Q[0] = d; Q[mu] = d * un; Q[mv] = d * ut; Q[3] = p / g1 + 0.5 * d * (un * un + ut * ut);
        };
        auto flux = [&](double d, double un, double ut, double p, double* F) {
            double E = p / g1 + 0.5 * d * (un * un + ut * ut);
            F[0] = d * un; F[mu] = d * un * un + p; F[mv] = d * un * ut; F[3] = un * (E + p);
        };
        double QsL[4], QsR[4];
        cons(dsl, um, vl, pm, QsL);
        cons(dsr, um, vr, pm, QsR);
        for (int m = 0; m < 4; ++m) {
            wave(m, 0, i) = QsL[m] - QL[m];
            wave(m, 1, i) = QsR[m] - QsL[m];
            wave(m, 2, i) = QR[m] - QsR[m];
        }
        s(0, i) = s1; s(1, i) = um; s(2, i) = s3;
        double d0, u0, p0;
        bool left;
        ex_sample0(G, pm, um, dl, ul, pl, dr, ur, pr, d0, u0, p0, left);
        double F0[4], FL[4], FR[4];
        flux(d0, u0, left ? vl : vr, p0, F0);
        flux(dl, ul, vl, pl, FL);
        flux(dr, ur, vr, pr, FR);
        for (int m = 0; m < 4; ++m) {
            amdq(m, i) = F0[m] - FL[m];
            apdq(m, i) = FR[m] - F0[m];
        }
    }
}

// ---------------------------------------------------------------------------
// Dispatch
// ---------------------------------------------------------------------------
bool rp_known(int rp) {
    return rp == ORC_RP_ADVECTION || rp == ORC_RP_ACOUSTICS || rp == ORC_RP_EULER_ROE ||
           rp == ORC_RP_SHALLOW_ROE || rp == ORC_RP_EULER_EXACT || rp == ORC_RP_VC_ACOUSTICS ||
           rp == ORC_RP_VC_ADVECTION || rp == ORC_RP_PSYSTEM || rp == ORC_RP_VC_ADVECTION_VEC ||
           rp == ORC_RP_EULER_5WAVE || rp == ORC_RP_SHALLOW_HLLE;
}

// aux components per cell the solver reads (the leading ones of the aux array)
int rp_maux(int rp) {
    if (rp == ORC_RP_PSYSTEM) return 4;
    return (rp == ORC_RP_VC_ACOUSTICS || rp == ORC_RP_VC_ADVECTION || rp == ORC_RP_VC_ADVECTION_VEC) ? 2 : 0;
}

void call_rpn2(int rp, int ixy, int mbc, int mx, int meqn, int mwaves, const CSlice& q, const CSlice& aux2,
               const Waves& wave, const Speeds& s, const Slice& amdq, const Slice& apdq,
               const double* cp) {
    switch (rp) {
        case ORC_RP_ADVECTION: rpn2_advection(ixy, mbc, mx, meqn, mwaves, q, q, wave, s, amdq, apdq, cp); break;
        case ORC_RP_ACOUSTICS: rpn2_acoustics(ixy, mbc, mx, q, q, wave, s, amdq, apdq, cp, meqn); break;
        case ORC_RP_EULER_ROE: rpn2_euler_roe(ixy, mbc, mx, meqn, mwaves, q, q, wave, s, amdq, apdq, cp); break;
        case ORC_RP_SHALLOW_ROE: rpn2_shallow_roe(ixy, mbc, mx, meqn, mwaves, q, q, wave, s, amdq, apdq, cp); break;
        case ORC_RP_EULER_EXACT: rpn2_euler_exact(ixy, mbc, mx, meqn, mwaves, q, q, wave, s, amdq, apdq, cp); break;
        case ORC_RP_VC_ACOUSTICS: rpn2_vc_acoustics(ixy, mbc, mx, meqn, q, q, aux2, aux2, wave, s, amdq, apdq); break;
        case ORC_RP_VC_ADVECTION: rpn2_vc_advection(ixy, mbc, mx, q, q, aux2, wave, s, amdq, apdq); break;
        case ORC_RP_PSYSTEM: rpn2_psystem(ixy, mbc, mx, q, q, aux2, aux2, wave, s, amdq, apdq); break;
        case ORC_RP_VC_ADVECTION_VEC: rpn2_vc_advection_vector(ixy, mbc, mx, meqn, q, q, aux2, wave, s, amdq, apdq); break;
        case ORC_RP_EULER_5WAVE: rpn2_euler_5wave(ixy, mbc, mx, meqn, mwaves, q, q, wave, s, amdq, apdq, cp); break;
        case ORC_RP_SHALLOW_HLLE: rpn2_shallow_hlle(ixy, mbc, mx, meqn, q, q, wave, s, amdq, apdq, cp); break;
    }
}
void call_rpt2(int rp, int ixy, int imp, int mbc, int mx, int meqn, int mwaves, const CSlice& q,
               const CSlice& aux1, const CSlice& aux2, const CSlice& aux3,
               const Slice& asdq, const Slice& bm, const Slice& bp, const double* cp) {
    switch (rp) {
        case ORC_RP_VC_ACOUSTICS: rpt2_vc_acoustics(ixy, imp, mbc, mx, aux1, aux2, aux3, asdq, bm, bp); break;
        case ORC_RP_VC_ADVECTION: rpt2_vc_advection(ixy, imp, mbc, mx, aux2, aux3, asdq, bm, bp); break;
        case ORC_RP_PSYSTEM: rpt2_psystem(ixy, imp, mbc, mx, aux1, aux2, aux3, asdq, bm, bp); break;
        case ORC_RP_EULER_5WAVE: rpt2_euler_5wave(ixy, mbc, mx, meqn, q, q, asdq, bm, bp, cp); break;
        case ORC_RP_ADVECTION: rpt2_advection(ixy, mbc, mx, asdq, bm, bp, cp); break;
        case ORC_RP_ACOUSTICS: rpt2_acoustics(ixy, mbc, mx, asdq, bm, bp, cp); break;
        case ORC_RP_EULER_ROE: rpt2_euler_roe(ixy, mbc, mx, meqn, mwaves, q, q, asdq, bm, bp, cp); break;
        case ORC_RP_SHALLOW_ROE: rpt2_shallow_roe(ixy, mbc, mx, meqn, mwaves, q, q, asdq, bm, bp, cp); break;
        case ORC_RP_EULER_EXACT: rpt2_euler_roe(ixy, mbc, mx, meqn, 4, q, q, asdq, bm, bp, cp); break;
    }
}

// Per-slice scratch (the reference's `work` partition, step2.f90:53-71, plus
// the optional q1d/qadd/fadd/gadd/dtdx1d arrays).
struct Work {
    int n;     // maxm + 2*mbc
    int maux;  // aux components per cell (>= 1 so the slices exist)
    std::vector<double> q1d, qadd, fadd, gadd, dtdx1d, dtdy1d, wave, s, amdq, apdq, cqxx,
        bmasdq, bpasdq, aux1, aux2, aux3;
    Work(int maxm, int mbc, int meqn, int mwaves, int maux_ = 0) {
        n = maxm + 2 * mbc;
        maux = maux_ > 0 ? maux_ : 1;
        aux1.assign((size_t)n * maux, 0.0);
        aux2.assign((size_t)n * maux, 0.0);
        aux3.assign((size_t)n * maux, 0.0);
        q1d.assign((size_t)n * meqn, 0.0);
        qadd.assign((size_t)n * meqn, 0.0);
        fadd.assign((size_t)n * meqn, 0.0);
        gadd.assign((size_t)n * meqn * 2, 0.0);
        dtdx1d.assign(n, 0.0);
        dtdy1d.assign(n, 0.0);
        wave.assign((size_t)n * meqn * mwaves, 0.0);
        s.assign((size_t)n * mwaves, 0.0);
        amdq.assign((size_t)n * meqn, 0.0);
        apdq.assign((size_t)n * meqn, 0.0);
        cqxx.assign((size_t)n * meqn, 0.0);
        bmasdq.assign((size_t)n * meqn, 0.0);
        bpasdq.assign((size_t)n * meqn, 0.0);
    }
};

// ---------------------------------------------------------------------------
// flux2.f90:82-204.  dtdx1d has the Fortran range 1-mbc:maxm+mbc.
// ---------------------------------------------------------------------------
void flux2(int ixy, int mbc, int mx, int meqn, int mwaves, Work& w, const int* method,
           const int* mthlim, double* cfl1d, bool use_fwave, int rp, const double* cp) {
    Slice q1d{w.q1d.data(), meqn, mbc};
    Slice qadd{w.qadd.data(), meqn, mbc};
    Slice fadd{w.fadd.data(), meqn, mbc};
    Gadd gadd{w.gadd.data(), meqn, mbc};
    Slice amdq{w.amdq.data(), meqn, mbc}, apdq{w.apdq.data(), meqn, mbc};
    Slice cqxx{w.cqxx.data(), meqn, mbc};
    Slice bmasdq{w.bmasdq.data(), meqn, mbc}, bpasdq{w.bpasdq.data(), meqn, mbc};
    Waves wave{w.wave.data(), meqn, mwaves, mbc};
    Speeds s{w.s.data(), mwaves, mbc};
    auto dtdx1d = [&](int i) -> double& { return w.dtdx1d[(size_t)(i + mbc - 1)]; };
    CSlice q{w.q1d.data(), meqn, mbc};
    CSlice a1{w.aux1.data(), w.maux, mbc}, a2{w.aux2.data(), w.maux, mbc}, a3{w.aux3.data(), w.maux, mbc};

    bool limit = false;
    for (int mw = 0; mw < mwaves; ++mw)
        if (mthlim[mw] > 0) limit = true;

    // flux2.f90:90-95
    for (int i = 1 - mbc; i <= mx + mbc; ++i)
        for (int m = 0; m < meqn; ++m) {
            qadd(m, i) = 0.0;
            fadd(m, i) = 0.0;
            gadd(m, 0, i) = 0.0;
            gadd(m, 1, i) = 0.0;
        }
    (void)q1d;

    // flux2.f90:101
    call_rpn2(rp, ixy, mbc, mx, meqn, mwaves, q, a2, wave, s, amdq, apdq, cp);

    // flux2.f90:104-108 (forall: first statement over all i, then the second)
    for (int i = 1; i <= mx + 1; ++i)
        for (int m = 0; m < meqn; ++m) qadd(m, i) = qadd(m, i) - dtdx1d(i) * apdq(m, i);
    for (int i = 1; i <= mx + 1; ++i)
        for (int m = 0; m < meqn; ++m) qadd(m, i - 1) = qadd(m, i - 1) - dtdx1d(i - 1) * amdq(m, i);

    // flux2.f90:111-119
    double c = 0.0;
    for (int mw = 0; mw < mwaves; ++mw)
        for (int i = 1; i <= mx + 1; ++i)
            c = std::max(c, std::max(dtdx1d(i) * s(mw, i), -dtdx1d(i - 1) * s(mw, i)));
    *cfl1d = c;

    if (method[1] != 1) {
        // flux2.f90:127
        if (limit) limiter(mx, meqn, mwaves, wave, s, mthlim);
        // flux2.f90:134-160
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            double dtdxave = 0.5 * (dtdx1d(i - 1) + dtdx1d(i));
            for (int m = 0; m < meqn; ++m) {
                cqxx(m, i) = 0.0;
                for (int mw = 0; mw < mwaves; ++mw) {
                    double sc = use_fwave ? std::copysign(1.0, s(mw, i)) : std::fabs(s(mw, i));
                    cqxx(m, i) = cqxx(m, i) + sc * (1.0 - std::fabs(s(mw, i)) * dtdxave) * wave(m, mw, i);
                }
                fadd(m, i) = fadd(m, i) + 0.5 * cqxx(m, i);
            }
        }
    }

    // flux2.f90:163
    if (method[2] <= 0) return;

    // flux2.f90:165-172
    if (method[1] > 1 && method[2] == 2) {
        for (int i = 1; i <= mx + 1; ++i)
            for (int m = 0; m < meqn; ++m) {
                amdq(m, i) = amdq(m, i) + cqxx(m, i);
                apdq(m, i) = apdq(m, i) - cqxx(m, i);
            }
    }

    // flux2.f90:181-190
    call_rpt2(rp, ixy, 1, mbc, mx, meqn, mwaves, q, a1, a2, a3, amdq, bmasdq, bpasdq, cp);
    for (int i = 1; i <= mx + 1; ++i)
        for (int m = 0; m < meqn; ++m) gadd(m, 0, i - 1) = gadd(m, 0, i - 1) - 0.5 * dtdx1d(i - 1) * bmasdq(m, i);
    for (int i = 1; i <= mx + 1; ++i)
        for (int m = 0; m < meqn; ++m) gadd(m, 1, i - 1) = gadd(m, 1, i - 1) - 0.5 * dtdx1d(i - 1) * bpasdq(m, i);

    // flux2.f90:194-203
    call_rpt2(rp, ixy, 2, mbc, mx, meqn, mwaves, q, a1, a2, a3, apdq, bmasdq, bpasdq, cp);
    for (int i = 1; i <= mx + 1; ++i)
        for (int m = 0; m < meqn; ++m) gadd(m, 0, i) = gadd(m, 0, i) - 0.5 * dtdx1d(i) * bmasdq(m, i);
    for (int i = 1; i <= mx + 1; ++i)
        for (int m = 0; m < meqn; ++m) gadd(m, 1, i) = gadd(m, 1, i) - 0.5 * dtdx1d(i) * bpasdq(m, i);
}

int check_args(int meqn, int mwaves, int mbc, int mx, int my, int rp) {
    if (meqn < 1 || mwaves < 1 || mbc != 2 || mx < 1 || my < 1) return 1;
    if (!rp_known(rp)) return 2;
    return 0;
}

}  // namespace

extern "C" {

void oracle_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int oracle_get_threads(void) { return g_threads; }

// step2.f90:74-247
int oracle_step2(int maxm, int meqn, int mwaves, int maux, int mbc, int mx, int my,
                 const double* qold_p, double* qnew_p, const double* aux_p, double dx,
                 double dy, double dt, const int* method, const int* mthlim, double* cfl_out,
                 int use_fwave, int rp, const double* cp) {
    int e = check_args(meqn, mwaves, mbc, mx, my, rp);
    if (e) return e;
    if (maxm < std::max(mx, my)) return 3;
    const int index_capa = method[5];
    if (index_capa > 0 && (aux_p == nullptr || maux < index_capa)) return 4;
    if (rp_maux(rp) > 0 && (aux_p == nullptr || maux < rp_maux(rp))) return 4;
    if ((rp == ORC_RP_VC_ADVECTION_VEC || rp == ORC_RP_SHALLOW_HLLE) && method[2] > 0)
        return 5;  // no transverse solve
    Grid2 qold{const_cast<double*>(qold_p), meqn, mbc, mx};
    Grid2 qnew{qnew_p, meqn, mbc, mx};
    Grid2 aux{const_cast<double*>(aux_p), maux > 0 ? maux : 1, mbc, mx};
    const double dtdx = dt / dx, dtdy = dt / dy;
    double cfl = 0.0;

    // Rows interact through the j-1/j+1 scatter, so a parallel x-sweep colours
    // rows by j mod 3 (any row set with distinct colours has disjoint targets).
    // With one thread this is exactly the reference's sequential order.
    const int nthr = g_threads;
    auto sweep = [&](int ixy) {
        const int nslab = (ixy == 1) ? my + 2 : mx + 2;  // j (or i) = 0 .. n+1
        const int n = (ixy == 1) ? mx : my;
        const double d_norm = (ixy == 1) ? dtdx : dtdy;
        const int ncolor = nthr > 1 ? 3 : 1;
        double cfl_s = 0.0;
        for (int color = 0; color < ncolor; ++color) {
#ifdef _OPENMP
#pragma omp parallel num_threads(nthr) reduction(max : cfl_s) if (nthr > 1)
#endif
            {
                Work w(maxm, mbc, meqn, mwaves, maux);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
                for (int k = 0; k < nslab; ++k) {
                    if (ncolor > 1 && (k % 3) != color) continue;
                    const int js = k;  // slice index 0 .. n_other+1
                    for (int i = 1 - mbc; i <= maxm + mbc; ++i) {
                        w.dtdx1d[(size_t)(i + mbc - 1)] = d_norm;
                    }
                    for (int m = 0; m < meqn; ++m)
                        for (int i = 1 - mbc; i <= n + mbc; ++i)
                            w.q1d[(size_t)(i + mbc - 1) * meqn + m] =
                                (ixy == 1) ? qold(m, i, js) : qold(m, js, i);
                    if (index_capa > 0)
                        for (int i = 1 - mbc; i <= n + mbc; ++i)
                            w.dtdx1d[(size_t)(i + mbc - 1)] =
                                d_norm / ((ixy == 1) ? aux(index_capa - 1, i, js) : aux(index_capa - 1, js, i));
                    // step2.f90: aux1/aux2/aux3 = the aux slices below, at and above this one
                    if (maux > 0)
                        for (int ma = 0; ma < maux; ++ma)
                            for (int i = 1 - mbc; i <= n + mbc; ++i) {
                                const size_t o = (size_t)(i + mbc - 1) * w.maux + ma;
                                w.aux1[o] = (ixy == 1) ? aux(ma, i, js - 1) : aux(ma, js - 1, i);
                                w.aux2[o] = (ixy == 1) ? aux(ma, i, js) : aux(ma, js, i);
                                w.aux3[o] = (ixy == 1) ? aux(ma, i, js + 1) : aux(ma, js + 1, i);
                            }
                    double c1d = 0.0;
                    flux2(ixy, mbc, n, meqn, mwaves, w, method, mthlim, &c1d, use_fwave != 0, rp, cp);
                    cfl_s = std::max(cfl_s, c1d);
                    Slice qadd{w.qadd.data(), meqn, mbc};
                    Slice fadd{w.fadd.data(), meqn, mbc};
                    Gadd gadd{w.gadd.data(), meqn, mbc};
                    for (int m = 0; m < meqn; ++m)
                        for (int i = 1; i <= n; ++i) {
                            if (ixy == 1) {
                                const int j = js;
                                if (index_capa == 0) {
                                    qnew(m, i, j) = qnew(m, i, j) + qadd(m, i) - dtdx * (fadd(m, i + 1) - fadd(m, i)) -
                                                    dtdy * (gadd(m, 1, i) - gadd(m, 0, i));
                                    qnew(m, i, j - 1) = qnew(m, i, j - 1) - dtdy * gadd(m, 0, i);
                                    qnew(m, i, j + 1) = qnew(m, i, j + 1) + dtdy * gadd(m, 1, i);
                                } else {
                                    qnew(m, i, j) = qnew(m, i, j) + qadd(m, i) -
                                                    (dtdx * (fadd(m, i + 1) - fadd(m, i)) +
                                                     dtdy * (gadd(m, 1, i) - gadd(m, 0, i))) /
                                                        aux(index_capa - 1, i, j);
                                    qnew(m, i, j - 1) = qnew(m, i, j - 1) - dtdy * gadd(m, 0, i) / aux(index_capa - 1, i, j - 1);
                                    qnew(m, i, j + 1) = qnew(m, i, j + 1) + dtdy * gadd(m, 1, i) / aux(index_capa - 1, i, j + 1);
                                }
                            } else {
                                const int ii = js, j = i;
                                if (index_capa == 0) {
                                    qnew(m, ii, j) = qnew(m, ii, j) + (qadd(m, j) - dtdy * (fadd(m, j + 1) - fadd(m, j)) -
                                                                       dtdx * (gadd(m, 1, j) - gadd(m, 0, j)));
                                    qnew(m, ii - 1, j) = qnew(m, ii - 1, j) - dtdx * gadd(m, 0, j);
                                    qnew(m, ii + 1, j) = qnew(m, ii + 1, j) + dtdx * gadd(m, 1, j);
                                } else {
                                    qnew(m, ii, j) = qnew(m, ii, j) + qadd(m, j) -
                                                     (dtdy * (fadd(m, j + 1) - fadd(m, j)) +
                                                      dtdx * (gadd(m, 1, j) - gadd(m, 0, j))) /
                                                         aux(index_capa - 1, ii, j);
                                    qnew(m, ii - 1, j) = qnew(m, ii - 1, j) - dtdx * gadd(m, 0, j) / aux(index_capa - 1, ii - 1, j);
                                    qnew(m, ii + 1, j) = qnew(m, ii + 1, j) + dtdx * gadd(m, 1, j) / aux(index_capa - 1, ii + 1, j);
                                }
                            }
                        }
                }
            }
        }
        cfl = std::max(cfl, cfl_s);
    };
    sweep(1);
    sweep(2);
    *cfl_out = cfl;
    return 0;
}

// step2ds.f90:72-261 (no transverse terms; method[2] is -1 for split runs)
int oracle_step2ds(int maxm, int meqn, int mwaves, int maux, int mbc, int mx, int my,
                   const double* qold_p, double* qnew_p, const double* aux_p, double dx,
                   double dy, double dt, const int* method, const int* mthlim, double* cfl_out,
                   int ids, int use_fwave, int rp, const double* cp) {
    int e = check_args(meqn, mwaves, mbc, mx, my, rp);
    if (e) return e;
    if (maxm < std::max(mx, my)) return 3;
    if (ids != 1 && ids != 2) return 5;
    const int index_capa = method[5];
    if (index_capa > 0 && (aux_p == nullptr || maux < index_capa)) return 4;
    if (rp_maux(rp) > 0 && (aux_p == nullptr || maux < rp_maux(rp))) return 4;
    Grid2 qold{const_cast<double*>(qold_p), meqn, mbc, mx};
    Grid2 qnew{qnew_p, meqn, mbc, mx};
    Grid2 aux{const_cast<double*>(aux_p), maux > 0 ? maux : 1, mbc, mx};
    const double dtdx = dt / dx, dtdy = dt / dy;
    double cfl = 0.0;
    const int ixy = ids;
    const int n = (ixy == 1) ? mx : my;
    const int nother = (ixy == 1) ? my : mx;
    const double d_norm = (ixy == 1) ? dtdx : dtdy;
    // Slices are independent in a split sweep.  The q1d gather copies the whole
    // slice before any write, so qold may alias qnew as in the reference.
    const int nthr = g_threads;
#ifdef _OPENMP
#pragma omp parallel num_threads(nthr) reduction(max : cfl) if (nthr > 1)
#endif
    {
        Work w(maxm, mbc, meqn, mwaves, maux);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int k = 1 - mbc; k <= nother + mbc; ++k) {
            for (int i = 1 - mbc; i <= maxm + mbc; ++i) w.dtdx1d[(size_t)(i + mbc - 1)] = d_norm;
            for (int m = 0; m < meqn; ++m)
                for (int i = 1 - mbc; i <= n + mbc; ++i)
                    w.q1d[(size_t)(i + mbc - 1) * meqn + m] = (ixy == 1) ? qold(m, i, k) : qold(m, k, i);
            if (index_capa > 0)
                for (int i = 1 - mbc; i <= n + mbc; ++i)
                    w.dtdx1d[(size_t)(i + mbc - 1)] =
                        d_norm / ((ixy == 1) ? aux(index_capa - 1, i, k) : aux(index_capa - 1, k, i));
            // the split sweep's Riemann solves see this slice's aux (no transverse solves)
            if (maux > 0)
                for (int ma = 0; ma < maux; ++ma)
                    for (int i = 1 - mbc; i <= n + mbc; ++i)
                        w.aux2[(size_t)(i + mbc - 1) * w.maux + ma] = (ixy == 1) ? aux(ma, i, k) : aux(ma, k, i);
            double c1d = 0.0;
            flux2(ixy, mbc, n, meqn, mwaves, w, method, mthlim, &c1d, use_fwave != 0, rp, cp);
            cfl = std::max(cfl, c1d);
            Slice qadd{w.qadd.data(), meqn, mbc};
            Slice fadd{w.fadd.data(), meqn, mbc};
            for (int m = 0; m < meqn; ++m)
                for (int i = 1; i <= n; ++i) {
                    double* t = (ixy == 1) ? &qnew(m, i, k) : &qnew(m, k, i);
                    const double dd = (ixy == 1) ? dtdx : dtdy;
                    if (index_capa == 0)
                        *t = *t + qadd(m, i) - dd * (fadd(m, i + 1) - fadd(m, i));
                    else
                        *t = *t + qadd(m, i) - dd * (fadd(m, i + 1) - fadd(m, i)) /
                                                   ((ixy == 1) ? aux(index_capa - 1, i, k) : aux(index_capa - 1, k, i));
                }
        }
    }
    *cfl_out = cfl;
    return 0;
}

// solver.py:351-519 for q: dimension 0 lower, upper, then dimension 1 lower,
// upper; each dimension fills its ghost layers across the full extent of the
// other index (so corners come from the dimension-1 pass).
}  // extern "C"

namespace {
// negate: q (a wall negates the normal momentum) or aux (plain mirror)
int bc_fill(int meqn, int mbc, int mx, int my, double* qbc, const int* bcl, const int* bcu, bool negate) {
    Grid2 q{qbc, meqn, mbc, mx};
    const int reflect[2] = {negate ? 1 : -1, negate ? 2 : -1};
    for (int idim = 0; idim < 2; ++idim) {
        const int n = idim == 0 ? mx : my;
        const int lo_other = 1 - mbc, hi_other = (idim == 0 ? my : mx) + mbc;
        auto at = [&](int m, int a, int b) -> double& {  // a along idim, b along the other
            return idim == 0 ? q(m, a, b) : q(m, b, a);
        };
        for (int side = 0; side < 2; ++side) {
            const int bc = side == 0 ? bcl[idim] : bcu[idim];
            if (bc == -1) continue;  // ghost cells filled by the caller (a neighbour's halo)
            for (int b = lo_other; b <= hi_other; ++b) {
                for (int g = 0; g < mbc; ++g) {
                    // Python index g along the rolled axis: cell 1-mbc+g (lower) or n+mbc-g (upper)
                    const int ghost = side == 0 ? (1 - mbc + g) : (n + mbc - g);
                    int src;
                    if (bc == 1) {
                        src = side == 0 ? 1 : n;
                    } else if (bc == 2) {
                        src = side == 0 ? (n - mbc + 1 + g) : (mbc - g);
                    } else if (bc == 3) {
                        src = side == 0 ? (mbc - g) : (n - mbc + 1 + g);
                    } else {
                        return 6;
                    }
                    for (int m = 0; m < meqn; ++m) {
                        double v = at(m, src, b);
                        if (bc == 3 && m == reflect[idim]) v = -v;
                        at(m, ghost, b) = v;
                    }
                }
            }
        }
    }
    return 0;
}
}  // namespace

extern "C" {

int oracle_bc_fill(int meqn, int mbc, int mx, int my, double* qbc, const int* bcl, const int* bcu) {
    return bc_fill(meqn, mbc, mx, my, qbc, bcl, bcu, true);
}

int oracle_bc_fill_aux(int maux, int mbc, int mx, int my, double* auxbc, const int* bcl, const int* bcu) {
    return bc_fill(maux, mbc, mx, my, auxbc, bcl, bcu, false);
}

int oracle_rpn2_aux(int rp, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx, const double* q,
                    const double* aux, double* wave, double* s, double* amdq, double* apdq, const double* cp) {
    if (!rp_known(rp) || mx > maxm || maux < 1) return 2;
    CSlice ql{q, meqn, mbc}, a{aux, maux, mbc};
    Waves w{wave, meqn, mwaves, mbc};
    Speeds sp{s, mwaves, mbc};
    Slice am{amdq, meqn, mbc}, ap{apdq, meqn, mbc};
    call_rpn2(rp, ixy, mbc, mx, meqn, mwaves, ql, a, w, sp, am, ap, cp);
    return 0;
}

int oracle_rpt2_aux(int rp, int ixy, int imp, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                    const double* q, const double* aux1, const double* aux2, const double* aux3, const double* asdq,
                    double* bmasdq, double* bpasdq, const double* cp) {
    if (!rp_known(rp) || mx > maxm || maux < 1 || (imp != 1 && imp != 2)) return 2;
    CSlice ql{q, meqn, mbc}, a1{aux1, maux, mbc}, a2{aux2, maux, mbc}, a3{aux3, maux, mbc};
    Slice as{const_cast<double*>(asdq), meqn, mbc}, bm{bmasdq, meqn, mbc}, bp{bpasdq, meqn, mbc};
    call_rpt2(rp, ixy, imp, mbc, mx, meqn, mwaves, ql, a1, a2, a3, as, bm, bp, cp);
    return 0;
}

int oracle_rpn2(int rp, int ixy, int maxm, int meqn, int mwaves, int mbc, int mx, const double* ql,
                const double* qr, double* wave, double* s, double* amdq, double* apdq, const double* cp) {
    if (!rp_known(rp) || mx > maxm) return 2;
    CSlice l{ql, meqn, mbc}, r{qr, meqn, mbc};
    Waves w{wave, meqn, mwaves, mbc};
    Speeds sp{s, mwaves, mbc};
    Slice am{amdq, meqn, mbc}, ap{apdq, meqn, mbc};
    switch (rp) {
        case ORC_RP_ADVECTION: rpn2_advection(ixy, mbc, mx, meqn, mwaves, l, r, w, sp, am, ap, cp); break;
        case ORC_RP_ACOUSTICS: rpn2_acoustics(ixy, mbc, mx, l, r, w, sp, am, ap, cp, meqn); break;
        case ORC_RP_EULER_ROE: rpn2_euler_roe(ixy, mbc, mx, meqn, mwaves, l, r, w, sp, am, ap, cp); break;
        case ORC_RP_SHALLOW_ROE: rpn2_shallow_roe(ixy, mbc, mx, meqn, mwaves, l, r, w, sp, am, ap, cp); break;
        case ORC_RP_EULER_EXACT: rpn2_euler_exact(ixy, mbc, mx, meqn, mwaves, l, r, w, sp, am, ap, cp); break;
    }
    return 0;
}

int oracle_rpt2(int rp, int ixy, int imp, int maxm, int meqn, int mwaves, int mbc, int mx,
                const double* ql, const double* qr, const double* asdq, double* bmasdq, double* bpasdq,
                const double* cp) {
    (void)imp;
    if (!rp_known(rp) || mx > maxm) return 2;
    CSlice l{ql, meqn, mbc}, r{qr, meqn, mbc};
    Slice as{const_cast<double*>(asdq), meqn, mbc}, bm{bmasdq, meqn, mbc}, bp{bpasdq, meqn, mbc};
    switch (rp) {
        case ORC_RP_ADVECTION: rpt2_advection(ixy, mbc, mx, as, bm, bp, cp); break;
        case ORC_RP_ACOUSTICS: rpt2_acoustics(ixy, mbc, mx, as, bm, bp, cp); break;
        case ORC_RP_EULER_ROE: rpt2_euler_roe(ixy, mbc, mx, meqn, mwaves, l, r, as, bm, bp, cp); break;
        case ORC_RP_SHALLOW_ROE: rpt2_shallow_roe(ixy, mbc, mx, meqn, mwaves, l, r, as, bm, bp, cp); break;
    }
    return 0;
}

int oracle_exact_star(double gamma, double rl, double ul, double pl, double rr, double ur, double pr, double tol,
                      int guess, double* pstar, double* ustar, int* iters) {
    (void)guess;
    ExGas G(gamma);
    return ex_starpu(G, rl, ul, pl, rr, ur, pr, tol, *pstar, *ustar, *iters) ? 0 : 7;
}

}  // extern "C"
