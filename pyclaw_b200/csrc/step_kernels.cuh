// step_kernels.cuh -- the classic 2D wave-propagation step on sm_100a.
//
// Reference: src/pyclaw/classic/step2.f90:74-247 (unsplit), step2ds.f90:72-261
// (split), flux2.f90:82-204, limiter.f90:29-53, philim.f90:16-35.
//
// Design ("column march").  A CTA owns a strip of NT padded columns and a
// block of H interior rows.  Thread t owns padded column cp = strip*W + t,
// W = NT - 4 (2 halo columns each side).  The CTA marches down the rows; at
// row R every thread
//   * solves the x-interface between (cp-1, R) and (cp, R)   [rpn2, ixy = 1]
//   * solves the y-interface between (cp, R-1) and (cp, R)    [rpn2, ixy = 2]
//   * finishes the y-interface between (cp, R-2) and (cp, R-1) (limiter with
//     the waves below and above it, second-order correction, rpt2 x 2)
//   * finishes its x-interface (limiter with the neighbours' waves, read from
//     shared memory; correction; rpt2 x 2)
//   * routes every increment to the cell that receives it: its own column's
//     increments stay in registers (4 rows in flight), the left/right
//     neighbours' go through shared memory,
// and writes qnew for row R-2, whose increments are then complete.  Every
// interface is solved once per CTA; the only recomputation is the 2-column
// halo of the strip and 2-3 halo rows of the row block.
//
// The reference reads qold for both sweeps (step2.f90:97,177), so the x and y
// increments are independent and one pass over qold gives exactly its update;
// only the order in which the increments of a cell are summed differs.
#pragma once

#include <cuda.h>

#include "riemann.cuh"

namespace claw2 {

// Device-resident time loop (claw2_patch_evolve): the loop's state lives in
// device memory; each step reads its dt/dx, dt/dy from it and does nothing
// once the loop is done.  Field meanings as in claw2_evolve_state.
struct EvolveDev {
    double t, tstart, tend, dt, dtdx, dtdy, cfl, cfl_desired, cfl_max, dt_max, dtmin, dtmax, cflmax, dx, dy;
    int dt_variable, dt_old_set, max_steps, attempts, num_steps, cfl_error, done, reject, fault;
};

struct StepArgs {
    const double* __restrict__ qold;
    double* __restrict__ qnew;
    Layout L;
    double dtdx, dtdy;
    int H;  // interior rows per CTA
    RPParams rp;
    Method meth;
    unsigned long long* cfl_bits;  // atomicMax of non-negative double bit patterns
    int* status;                   // bit 0: non-finite output
    const double* guess;           // optional per-interface p* guesses: x plane, then y plane
    unsigned long long* counters;  // optional: [0] Newton iterations, [1] Riemann solves
    // optional tile schedule of k_step_unsplit (1D grid of nstrips * row blocks):
    // CTA b runs tile tile_order[b] and, with tile_cost, records its cost in
    // SM clock cycles there (see k_lpt_order)
    const int* tile_order = nullptr;
    unsigned int* tile_cost = nullptr;
    int nstrips = 0;
    // a launch over a subset of the tiles (no schedule): CTA b runs tile
    // b + tile_offset, plus tile_jump from CTA tile_jump_at on (the interior
    // row blocks, or the first and last ones, of a slab's overlapped step)
    int tile_offset = 0, tile_jump_at = 1 << 30, tile_jump = 0, tile_count = 0;
    // aux planes (same layout as q) for solvers with aux data, else nullptr
    const double* __restrict__ aux = nullptr;
    // device-resident time loop: dt from here, no work once it is done (else nullptr)
    const EvolveDev* evo = nullptr;
    // capacity function kappa (one plane, same layout), else nullptr: every
    // increment of a cell is divided by its kappa, a transverse increment also
    // by the kappa of the cell its fluctuation entered (step2.f90:132-160,
    // flux2.f90:104-119,134-203 with dtdx1d = dtdx / kappa)
    const double* __restrict__ capa = nullptr;
};

// The tile a CTA of a step launch runs (see StepArgs::tile_order, tile_offset).
__device__ __forceinline__ int tile_index(const StepArgs& a) {
    int tile = blockIdx.x;
    if (a.tile_order) {
        const int t = a.tile_order[blockIdx.x];
        if (t >= 0 && t < (int)gridDim.x) tile = t;  // a schedule is a permutation; anything else is ignored
    } else {
        tile += a.tile_offset + ((int)blockIdx.x >= a.tile_jump_at ? a.tile_jump : 0);
    }
    return tile;
}

// philim.f90:16-35
__device__ __forceinline__ double philim(double a, double b, int meth) {
    const double r = b * rcp_nr(a);
    switch (meth) {
        case 1: return fmax(0.0, fmin(1.0, r));
        case 2: return fmax(0.0, fmax(fmin(1.0, 2.0 * r), fmin(2.0, r)));
        case 3: return (r + fabs(r)) / (1.0 + fabs(r));
        case 4: return fmax(0.0, fmin((1.0 + r) / 2.0, fmin(2.0, 2.0 * r)));
        case 5: return r;
        default: return 0.0;
    }
}

__device__ __forceinline__ void cfl_commit(double cfl, double* s_red, unsigned long long* slot) {
    // warp max, then block max, then one 64-bit atomicMax per CTA
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cfl = fmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_red[warp] = cfl;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, s_red[w]);
        // non-negative doubles order like their bit patterns
        atomicMax(slot, (unsigned long long)__double_as_longlong(m));
    }
}

// Warp-sum three counters (Newton steps needed, solves, Newton steps
// applied) and add them once per warp.
__device__ __forceinline__ void counter_commit(unsigned long long* c, unsigned long long a, unsigned long long b,
                                               unsigned long long d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        d += __shfl_xor_sync(0xffffffffu, d, o);
    }
    if ((threadIdx.x & 31) == 0 && c) {
        atomicAdd(c, a);
        atomicAdd(c + 1, b);
        atomicAdd(c + 2, d);
    }
}

template <int ME>
__device__ __forceinline__ bool all_finite(const double (&v)[ME]) {
    bool ok = true;
#pragma unroll
    for (int m = 0; m < ME; ++m) ok = ok && isfinite(v[m]);
    return ok;
}

// ---------------------------------------------------------------------------
// Shared pieces of the interface work
// ---------------------------------------------------------------------------

// Method specialisations of the step kernels.  SPEC_ANY reads order,
// transverse mode, limiters and f-wave flag at run time; SPEC_MC2 is the
// high-resolution method with transverse correction waves and the MC limiter
// on every family (order 2, trans_cor, mthlim = 4, no f-waves), fixed at
// compile time so the limiter switch and the method branches fold away.
// SPEC_MM2 (order 2, minmod on every family, no f-waves: the reference's
// default limiter) specialises the split sweeps the same way.
enum { SPEC_ANY = 0, SPEC_MC2 = 1, SPEC_MM2 = 2 };

// Limiter (limiter.f90:29-53 / philim.f90) and second-order correction
// cqxx = sum_k coef_k * phi_k * w_k (flux2.f90:134-160) for one interface.
// dl / dr are the dot products of each unlimited wave with the same family's
// unlimited wave at the interface below/left and above/right.
template <class RP, int IXY, int SPEC = SPEC_ANY>
__device__ __forceinline__ void correction(const typename RP::Iface& f, const RPParams& p, const Method& meth,
                                           double dtdx, const double (&dl)[RP::MWAVES],
                                           const double (&dr)[RP::MWAVES], double (&cq)[RP::MEQN]) {
    constexpr int ME = RP::MEQN, MW = RP::MWAVES;
    double s[MW];
    RP::template speeds<IXY>(f, p, s);
    double w[MW][ME];
    RP::template waves<IXY>(f, p, w);
#pragma unroll
    for (int m = 0; m < ME; ++m) cq[m] = 0.0;
#pragma unroll
    for (int k = 0; k < MW; ++k) {
        const int lim = (SPEC == SPEC_MC2) ? 4 : (SPEC == SPEC_MM2) ? 1 : meth.mthlim[k];
        double wn2 = 0.0;
#pragma unroll
        for (int m = 0; m < ME; ++m) wn2 = wn2 + w[k][m] * w[k][m];
        double phi = 1.0;
        if (lim != 0 && wn2 != 0.0) phi = philim(wn2, (s[k] > 0.0) ? dl[k] : dr[k], lim);
        const double as = fabs(s[k]);
        const bool fw = (SPEC != SPEC_ANY) ? false : (meth.fwave != 0);
        const double coef = (fw ? copysign(1.0, s[k]) : as) * (1.0 - as * dtdx);
#pragma unroll
        for (int m = 0; m < ME; ++m) cq[m] = cq[m] + coef * (phi * w[k][m]);
    }
}

template <class RP, int IXY>
__device__ __forceinline__ double iface_cfl(const typename RP::Iface& f, const RPParams& p, double dtdx) {
    double s[RP::MWAVES];
    RP::template speeds<IXY>(f, p, s);
    double c = 0.0;
#pragma unroll
    for (int k = 0; k < RP::MWAVES; ++k) c = fmax(c, fabs(dtdx * s[k]));
    return c;
}

// With a capacity function the two sides of an interface have their own
// dt/(dx kappa): the Courant number is max(dtdx_r s, -dtdx_l s) over the
// waves (flux2.f90:111-119).
template <class RP, int IXY>
__device__ __forceinline__ double iface_cfl2(const typename RP::Iface& f, const RPParams& p, double dtdx_l,
                                             double dtdx_r) {
    double s[RP::MWAVES];
    RP::template speeds<IXY>(f, p, s);
    double c = 0.0;
#pragma unroll
    for (int k = 0; k < RP::MWAVES; ++k) c = fmax(c, fmax(dtdx_r * s[k], -dtdx_l * s[k]));
    return c;
}

// aux of the cell at column pointer ap (already offset by the column), row R
template <class RP, int MAD>
__device__ __forceinline__ void load_aux(const double* ap, long long plane, int pitch, int R, double (&av)[MAD]) {
#pragma unroll
    for (int k = 0; k < MAD; ++k) av[k] = (AuxTraits<RP>::MAUX > 0) ? __ldg(ap + k * plane + (long long)R * pitch) : 0.0;
}

// ---------------------------------------------------------------------------
// TMA row staging: one thread per CTA copies the next row of a strip (NT
// columns x 1 row x num_eqn planes) from a 3D tensor map of the q planes into
// shared memory; an mbarrier (one arrival + the copy's bytes) signals it.
// Waits are bounded: a copy that does not land within the bound sets status
// bit 1 (the host reports CLAW2_ETIMEOUT) and the kernel carries on.
// ---------------------------------------------------------------------------
constexpr int MBAR_SPIN_LIMIT = 1 << 20;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// true when the phase with the given parity has completed
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    const unsigned addr = smem_u32(bar);
    for (int i = 0; i < MBAR_SPIN_LIMIT; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Issue the copy of the box at (x, y, 0) into dst and arm the barrier with its
// size.  x must be a multiple of 2 (16 bytes of doubles); dst 128-byte aligned.
__device__ __forceinline__ void tma_row(const CUtensorMap* tm, double* dst, unsigned long long* bar, int x, int y,
                                        unsigned bytes) {
    const unsigned b = smem_u32(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(x), "r"(y), "r"(0), "r"(b)
        : "memory");
}

// ---------------------------------------------------------------------------
// Unsplit step (step2.f90), fused x + y sweeps.
// ---------------------------------------------------------------------------
template <class RP, int NT, bool CAPA = false>
struct UnsplitSmem {
    static constexpr int ME = RP::MEQN, MW = RP::MWAVES, NC = RP::NC;
    // solvers with a large interface record (the exact solver's carries its
    // waves) keep the y-interface being finished in shared memory between
    // rows, so it does not occupy registers during the x work
    static constexpr int NF = (int)(sizeof(typename RP::Iface) / sizeof(double));
    static constexpr bool YS = NF > 12;
    double cell[3][NC][NT];  // prepared cells of rows R-2, R-1, R (ring)
    double w[MW][ME][NT];    // unlimited x-waves of row R
    double xl[4][ME][NT];    // increments for column cp-1: rows R-2, R-1, R, R+1
    double yr[2][ME][NT];    // increments for column cp+1: rows R-2, R-1
    double icap[CAPA ? 3 : 1][CAPA ? NT : 1];  // 1 / kappa of the ring's cells (capacity form)
    double yrec[YS ? NF + 2 * ME + MW : 1][YS ? NT : 1];  // (YS) record, A-dq, A+dq, dots of (R-2 | R-1)
    double red[NT / 32];
};

// The TMA form's extra shared memory: the staged row (first, 128-byte
// aligned for the copy) and its barrier.
template <class RP, int NT>
struct UnsplitSmemTma {
    alignas(128) double qrow[RP::MEQN][NT];
    unsigned long long bar;
    UnsplitSmem<RP, NT> s;
};

// One tile: the strip `strip` (columns strip*W .. strip*W+NT-1, padded) and
// the interior rows [rb, rb + H) of one grid.  Returns this thread's CFL
// contribution in `cfl`; the caller reduces it (the tile ends with every
// shared-memory read done, so a persistent CTA can start the next tile).
// With a tensor map (tm != nullptr; qrow and bar in shared memory) the rows
// are staged by TMA, else each thread loads its column a row ahead.
//
// CAPA: the capacity form.  Increments are summed without the receiving
// cell's 1/kappa, which multiplies the sum when the cell is written (every
// term of a cell carries that one factor); transverse increments carry in
// addition the 1/kappa of the cell their fluctuation entered, the
// second-order correction the mean of the two cells' dt/(dx kappa).
template <class RP, int NT, int SPEC = SPEC_ANY, bool CAPA = false, bool EVO = false>
__device__ __forceinline__ void unsplit_tile(const StepArgs& a, int strip, int rb, UnsplitSmem<RP, NT, CAPA>& S,
                                             double& cfl, const CUtensorMap* tm = nullptr, double* qrow = nullptr,
                                             unsigned long long* bar = nullptr) {
    constexpr int ME = RP::MEQN, MW = RP::MWAVES, NC = RP::NC, W = NT - 4;
    using Iface = typename RP::Iface;

    const int t = threadIdx.x;
    const int mx = a.L.mx, my = a.L.my;
    const int pitch = a.L.pitch;
    const long long plane = a.L.plane;
    const int cp = strip * W + t;
    const int cpl = min(cp, mx + 3);
    const int Hb = min(a.H, my - rb);
    const int R0 = rb, R1 = rb + Hb + 3;
    const bool out_col = (t >= 2) && (t < W + 2) && (cp <= mx + 1);
    const bool xcfl_col = (t >= 2) && (t <= W + 2) && (cp <= mx + 2);
    const bool ycfl_col = (t >= 1) && (t <= W + 2) && (cp <= mx + 2);
    const int tl = (t > 0) ? t - 1 : 0;
    const int tr = (t < NT - 1) ? t + 1 : NT - 1;
    // dt/dx, dt/dy: kernel parameters, or (EVO, the device time loop) the
    // loop's record; a compile-time choice, so ordinary steps keep the
    // parameters as operands of the FP64 instructions instead of registers
    const double dtdx = EVO ? a.evo->dtdx : a.dtdx, dtdy = EVO ? a.evo->dtdy : a.dtdy;
    const RPParams& P = a.rp;
    const int order = (SPEC == SPEC_MC2) ? 2 : a.meth.order;
    const int trans = (SPEC == SPEC_MC2) ? 2 : a.meth.transverse;
    const bool tc = (order > 1) && (trans == 2);
    const double* qo = a.qold + cpl;
    double* qn = a.qnew + cpl;

    // aux data: loaded with q a row ahead (MA planes); solvers whose transverse
    // solve needs the cells above and below (TAUX) run the x-interface's
    // transverse solve one row late, when the row above is prepared
    constexpr int MA = AuxTraits<RP>::MAUX, MAD = MA > 0 ? MA : 1;
    constexpr bool TAUX = AuxTraits<RP>::TRANSVERSE_AUX;
    const double* ao = a.aux + cpl;
    double pfa[MAD];
    double cxa1[ME], cxa2[ME];  // deferred x-transverse inputs (A-dq and A+dq of the row above's interface)
    bool cx_valid = false;
#pragma unroll
    for (int m = 0; m < ME; ++m) cxa1[m] = cxa2[m] = 0.0;
#pragma unroll
    for (int k = 0; k < MAD; ++k) pfa[k] = (MA > 0) ? __ldg(ao + k * plane + (long long)R0 * pitch) : 0.0;
    const double* ko = CAPA ? a.capa + cpl : nullptr;
    double pfk = CAPA ? __ldg(ko + (long long)R0 * pitch) : 1.0;

    // Zero-jump shortcut (solvers without aux data, q-waves): when
    // every lane of a warp has equal cells on both sides of its interface, the
    // warp builds the interface's record with zero strengths and only the Roe
    // state the Courant number needs, and skips the finish (limiter,
    // correction, transverse solves), whose increments are all zero.  Warp-
    // uniform decisions, so no lane diverges; the results equal the full
    // path's up to the sign of zero terms.
    constexpr bool ZS = SkipTraits<RP>::OK && MA == 0 && !CAPA;
    const bool zs = ZS && (SPEC != SPEC_ANY || a.meth.fwave == 0);
    bool zY = false;  // the y-interface being finished, (R-2 | R-1), is zero in the whole warp

    // (the copy needs a 128-byte aligned destination; anything else loads
    // directly; solvers with aux data load directly)
    const bool tma = (MA == 0) && !CAPA && (tm != nullptr) && ((smem_u32(qrow) & 127u) == 0);
    const int x0 = strip * W;                                     // first column of the strip
    const unsigned row_bytes = (unsigned)(ME * NT * sizeof(double));
    const int tq = cpl - x0;                                      // this thread's staged column
    double pf[ME];
    double accA[ME], accB[ME], accC[ME], accD[ME];  // rows R-2, R-1, R, R+1
    Iface fY;                                       // y-interface (R-2 | R-1)
    double amY[ME], apY[ME], dY[MW];
    unsigned long long n_it = 0, n_solve = 0, n_app = 0;
    if (tma) {
        if (t == 0) mbar_init(bar);
        __syncthreads();
        if (t == 0) tma_row(tm, qrow, bar, x0, R0, row_bytes);
    }
#pragma unroll
    for (int m = 0; m < ME; ++m) {
        pf[m] = tma ? 0.0 : __ldg(qo + m * plane + (long long)R0 * pitch);
        accA[m] = accB[m] = accC[m] = accD[m] = 0.0;
        amY[m] = apY[m] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < MW; ++k) dY[k] = 0.0;
    memset(&fY, 0, sizeof(fY));
    constexpr bool YS = UnsplitSmem<RP, NT, CAPA>::YS;
    constexpr int NFY = UnsplitSmem<RP, NT, CAPA>::NF;
    if constexpr (YS) {
#pragma unroll
        for (int k = 0; k < NFY + 2 * ME + MW; ++k) S.yrec[k][t] = 0.0;
    }

    int s2 = 0, s1 = 2, s0 = 1;  // ring slots of rows R, R-1, R-2
    for (int R = R0; R <= R1; ++R) {
        // ---- row R: prepare this column's cell, prefetch the next row ----
        {
            double q[ME], c[NC];
            if (tma) {
                if (!mbar_wait(bar, (unsigned)(R - R0) & 1u)) atomicOr(a.status, 2);
#pragma unroll
                for (int m = 0; m < ME; ++m) q[m] = qrow[m * NT + tq];
            } else {
#pragma unroll
                for (int m = 0; m < ME; ++m) q[m] = pf[m];
                if (R < R1) {
#pragma unroll
                    for (int m = 0; m < ME; ++m) pf[m] = __ldg(qo + m * plane + (long long)(R + 1) * pitch);
                }
            }
            double av[MAD];
#pragma unroll
            for (int k = 0; k < MAD; ++k) av[k] = pfa[k];
            if (MA > 0 && R < R1) {
#pragma unroll
                for (int k = 0; k < MAD; ++k) pfa[k] = __ldg(ao + k * plane + (long long)(R + 1) * pitch);
            }
            AuxTraits<RP>::prep(q, av, P, c);
#pragma unroll
            for (int k = 0; k < NC; ++k) S.cell[s2][k][t] = c[k];
            if constexpr (CAPA) {
                S.icap[s2][t] = 1.0 / pfk;
                if (R < R1) pfk = __ldg(ko + (long long)(R + 1) * pitch);
            }
        }
        __syncthreads();  // S1: cells of row R visible; previous exchange consumed
        if (tma && t == 0 && R < R1) {
            // every thread has read row R from the staging buffer (before S1)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tma_row(tm, qrow, bar, x0, R + 1, row_bytes);
        }

        // ---- the x-interface of row R-1, deferred transverse solve (TAUX) ----
        // Its receiving cells (cp-1 or cp, row R-1) and their neighbours in
        // rows R-2 and R are now in the ring; the increments go to rows R-2,
        // R-1, R of column cp-1 (exchange slots 0..2) and of this column.
        double dxl0[ME], dxl1[ME], dxl2[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) dxl0[m] = dxl1[m] = dxl2[m] = 0.0;
        if constexpr (TAUX) {
            if (cx_valid) {
                const double h = 0.5 * dtdx * dtdy;
                const double hl = CAPA ? h * S.icap[s1][tl] : h, hr = CAPA ? h * S.icap[s1][t] : h;
                double cm[NC], c0[NC], cu[NC], bm[ME], bp[ME];
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    cm[k] = S.cell[s0][k][tl];
                    c0[k] = S.cell[s1][k][tl];
                    cu[k] = S.cell[s2][k][tl];
                }
                RP::template rpt2_aux<1>(cxa1, cm, c0, cu, bm, bp);  // imp = 1 -> column cp-1
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    dxl1[m] = hl * (bp[m] - bm[m]);
                    dxl0[m] = hl * bm[m];
                    dxl2[m] = -hl * bp[m];
                }
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    cm[k] = S.cell[s0][k][t];
                    c0[k] = S.cell[s1][k][t];
                    cu[k] = S.cell[s2][k][t];
                }
                RP::template rpt2_aux<1>(cxa2, cm, c0, cu, bm, bp);  // imp = 2 -> column cp
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    accB[m] = accB[m] + hr * (bp[m] - bm[m]);
                    accA[m] = accA[m] + hr * bm[m];
                    accC[m] = accC[m] - hr * bp[m];
                }
            }
            cx_valid = false;
        }

        double ylB[ME], ylA[ME], yrB[ME], yrA[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) ylB[m] = ylA[m] = yrB[m] = yrA[m] = 0.0;

        // ---- y: solve (R-1 | R), finish (R-2 | R-1) ----
        if (R > R0) {
            if constexpr (YS) {  // the record of (R-2 | R-1) back from shared memory
                double* fp = reinterpret_cast<double*>(&fY);
#pragma unroll
                for (int k = 0; k < NFY; ++k) fp[k] = S.yrec[k][t];
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    amY[m] = S.yrec[NFY + m][t];
                    apY[m] = S.yrec[NFY + ME + m][t];
                }
#pragma unroll
                for (int k = 0; k < MW; ++k) dY[k] = S.yrec[NFY + 2 * ME + k][t];
            }
            double cB[NC], cA[NC];
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                cB[k] = S.cell[s1][k][t];
                cA[k] = S.cell[s2][k][t];
            }
            Iface fN;
            double amN[ME], apN[ME];
            double dn[MW];
            const bool zN = zs && __all_sync(0xffffffffu, same_q<ME, NC>(cB, cA));
            if (ZS && zN) {
                SkipTraits<RP>::template zero_iface<2>(cB, cA, P, fN);
#pragma unroll
                for (int m = 0; m < ME; ++m) amN[m] = apN[m] = 0.0;
#pragma unroll
                for (int k = 0; k < MW; ++k) dn[k] = 0.0;
                if (GuessTraits<RP>::USES && cp <= mx + 3) n_solve += 1;  // a solve with no Newton step
            } else {
                double gy = 0.0;
                if (GuessTraits<RP>::USES && a.guess) gy = a.guess[plane + (long long)R * pitch + cpl];
                GuessTraits<RP>::template solve<2>(cB, cA, P, gy, fN, amN, apN);
                if (GuessTraits<RP>::USES && cp <= mx + 3) {
                    n_it += GuessTraits<RP>::count(fN);
                    n_app += GuessTraits<RP>::count_applied(fN);
                    n_solve += 1;
                }
                double wY[MW][ME], wN[MW][ME];
                RP::template waves<2>(fY, P, wY);
                RP::template waves<2>(fN, P, wN);
#pragma unroll
                for (int k = 0; k < MW; ++k) {
                    double d = 0.0;
#pragma unroll
                    for (int m = 0; m < ME; ++m) d = d + wY[k][m] * wN[k][m];
                    dn[k] = d;
                }
            }
            if (R >= R0 + 3) {
                // capacity form: dt/(dy kappa) of the cells below (R-2) and above (R-1)
                const double ydl = CAPA ? dtdy * S.icap[s0][t] : dtdy, ydr = CAPA ? dtdy * S.icap[s1][t] : dtdy;
                if (ycfl_col)
                    cfl = fmax(cfl, CAPA ? iface_cfl2<RP, 2>(fY, P, ydl, ydr) : iface_cfl<RP, 2>(fY, P, dtdy));
            }
            if (R >= R0 + 3 && !(ZS && zY)) {
                const double ydl = CAPA ? dtdy * S.icap[s0][t] : dtdy, ydr = CAPA ? dtdy * S.icap[s1][t] : dtdy;
                double cq[ME];
                if (order != 1) {
                    correction<RP, 2, SPEC>(fY, P, a.meth, CAPA ? 0.5 * (ydl + ydr) : dtdy, dY, dn, cq);
                } else {
#pragma unroll
                    for (int m = 0; m < ME; ++m) cq[m] = 0.0;
                }
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    const double f = 0.5 * cq[m];
                    accA[m] = accA[m] - dtdy * (amY[m] + f);
                    accB[m] = accB[m] - dtdy * (apY[m] - f);
                }
                if (trans > 0) {
                    const double h = 0.5 * dtdy * dtdx;
                    const double hl = CAPA ? h * S.icap[s0][t] : h, hr = CAPA ? h * S.icap[s1][t] : h;
                    double as2[ME], bm[ME], bp[ME];
#pragma unroll
                    for (int m = 0; m < ME; ++m) as2[m] = tc ? amY[m] + cq[m] : amY[m];
                    if constexpr (TAUX) {  // cell (cp, R-2) between columns cp-1 and cp+1
                        double cm[NC], c0[NC], cu[NC];
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            cm[k] = S.cell[s0][k][tl];
                            c0[k] = S.cell[s0][k][t];
                            cu[k] = S.cell[s0][k][tr];
                        }
                        RP::template rpt2_aux<2>(as2, cm, c0, cu, bm, bp);
                    } else {
                        RP::template rpt2<2>(fY, P, as2, bm, bp);  // imp = 1 -> row R-2
                    }
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        accA[m] = accA[m] + hl * (bp[m] - bm[m]);
                        ylB[m] = hl * bm[m];
                        yrB[m] = -hl * bp[m];
                    }
#pragma unroll
                    for (int m = 0; m < ME; ++m) as2[m] = tc ? apY[m] - cq[m] : apY[m];
                    if constexpr (TAUX) {  // cell (cp, R-1)
                        double cm[NC], c0[NC], cu[NC];
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            cm[k] = S.cell[s1][k][tl];
                            c0[k] = S.cell[s1][k][t];
                            cu[k] = S.cell[s1][k][tr];
                        }
                        RP::template rpt2_aux<2>(as2, cm, c0, cu, bm, bp);
                    } else {
                        RP::template rpt2<2>(fY, P, as2, bm, bp);  // imp = 2 -> row R-1
                    }
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        accB[m] = accB[m] + hr * (bp[m] - bm[m]);
                        ylA[m] = hr * bm[m];
                        yrA[m] = -hr * bp[m];
                    }
                }
            }
            zY = zN;
            if constexpr (YS) {
                const double* fp = reinterpret_cast<const double*>(&fN);
#pragma unroll
                for (int k = 0; k < NFY; ++k) S.yrec[k][t] = fp[k];
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    S.yrec[NFY + m][t] = amN[m];
                    S.yrec[NFY + ME + m][t] = apN[m];
                }
#pragma unroll
                for (int k = 0; k < MW; ++k) S.yrec[NFY + 2 * ME + k][t] = dn[k];
            } else {
                fY = fN;
#pragma unroll
                for (int m = 0; m < ME; ++m) { amY[m] = amN[m]; apY[m] = apN[m]; }
#pragma unroll
                for (int k = 0; k < MW; ++k) dY[k] = dn[k];
            }
        }
        // Publish the y sweep's neighbour increments now, which ends their live
        // range before the x work (fewer registers); every read of the previous
        // row's exchange slots came before S1.
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            S.xl[0][m][t] = ylB[m] + dxl0[m];
            S.yr[0][m][t] = yrB[m];
            S.yr[1][m][t] = yrA[m];
        }

        // ---- x: the interface (cp-1 | cp) on row R ----
        const bool xrow = (R > R0) && (R < R1);  // rows R0+1 .. R1-1
        Iface fX;
        double amX[ME], apX[ME];
        bool zX = false;
        {
            double cL[NC], cR[NC];
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                cL[k] = S.cell[s2][k][tl];
                cR[k] = S.cell[s2][k][t];
            }
            // (the first and last rows' x-interfaces are never finished: no solve)
            zX = ZS && (!xrow || (zs && __all_sync(0xffffffffu, same_q<ME, NC>(cL, cR))));
            if (ZS && zX) {
                SkipTraits<RP>::template zero_iface<1>(cL, cR, P, fX);
                if (GuessTraits<RP>::USES && xrow && cp <= mx + 3 && t > 0) n_solve += 1;
#pragma unroll
                for (int m = 0; m < ME; ++m) amX[m] = apX[m] = 0.0;
#pragma unroll
                for (int k = 0; k < MW; ++k)
#pragma unroll
                    for (int m = 0; m < ME; ++m) S.w[k][m][t] = 0.0;
            } else {
            double gx = 0.0;
            if (GuessTraits<RP>::USES && a.guess) gx = a.guess[(long long)R * pitch + cpl];
            GuessTraits<RP>::template solve<1>(cL, cR, P, gx, fX, amX, apX);
            if (GuessTraits<RP>::USES && cp <= mx + 3 && t > 0) {
                n_it += GuessTraits<RP>::count(fX);
                n_app += GuessTraits<RP>::count_applied(fX);
                n_solve += 1;
            }
            double wX[MW][ME];
            RP::template waves<1>(fX, P, wX);
#pragma unroll
            for (int k = 0; k < MW; ++k)
#pragma unroll
                for (int m = 0; m < ME; ++m) S.w[k][m][t] = wX[k][m];
            }
        }
        __syncthreads();  // S2: x-waves of row R visible

        double xcL[ME], xbL[ME], xaL[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) xcL[m] = xbL[m] = xaL[m] = 0.0;
        if (xrow) {
            // capacity form: dt/(dx kappa) of the cells left (cp-1) and right (cp)
            const double xdl = CAPA ? dtdx * S.icap[s2][tl] : dtdx, xdr = CAPA ? dtdx * S.icap[s2][t] : dtdx;
            if (xcfl_col) cfl = fmax(cfl, CAPA ? iface_cfl2<RP, 1>(fX, P, xdl, xdr) : iface_cfl<RP, 1>(fX, P, dtdx));
        }
        if (xrow && !(ZS && zX)) {
            const double xdl = CAPA ? dtdx * S.icap[s2][tl] : dtdx, xdr = CAPA ? dtdx * S.icap[s2][t] : dtdx;
            double cq[ME];
            if (order != 1) {
                double dl[MW], dr[MW];
#pragma unroll
                for (int k = 0; k < MW; ++k) {
                    double x = 0.0, y = 0.0;
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        const double w = S.w[k][m][t];
                        x = x + S.w[k][m][tl] * w;
                        y = y + w * S.w[k][m][tr];
                    }
                    dl[k] = x;
                    dr[k] = y;
                }
                correction<RP, 1, SPEC>(fX, P, a.meth, CAPA ? 0.5 * (xdl + xdr) : dtdx, dl, dr, cq);
            } else {
#pragma unroll
                for (int m = 0; m < ME; ++m) cq[m] = 0.0;
            }
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                const double f = 0.5 * cq[m];
                accC[m] = accC[m] - dtdx * (apX[m] - f);
                xcL[m] = -dtdx * (amX[m] + f);
            }
            if constexpr (TAUX) {
                if (trans > 0) {  // the transverse solve runs with the next row
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        cxa1[m] = tc ? amX[m] + cq[m] : amX[m];
                        cxa2[m] = tc ? apX[m] - cq[m] : apX[m];
                    }
                    cx_valid = true;
                }
            } else if (trans > 0) {
                const double h = 0.5 * dtdx * dtdy;
                const double hl = CAPA ? h * S.icap[s2][tl] : h, hr = CAPA ? h * S.icap[s2][t] : h;
                double as2[ME], bm[ME], bp[ME];
#pragma unroll
                for (int m = 0; m < ME; ++m) as2[m] = tc ? amX[m] + cq[m] : amX[m];
                RP::template rpt2<1>(fX, P, as2, bm, bp);  // imp = 1 -> column cp-1
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    xcL[m] = xcL[m] + hl * (bp[m] - bm[m]);
                    xbL[m] = hl * bm[m];
                    xaL[m] = -hl * bp[m];
                }
#pragma unroll
                for (int m = 0; m < ME; ++m) as2[m] = tc ? apX[m] - cq[m] : apX[m];
                RP::template rpt2<1>(fX, P, as2, bm, bp);  // imp = 2 -> column cp
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    accC[m] = accC[m] + hr * (bp[m] - bm[m]);
                    accB[m] = accB[m] + hr * bm[m];
                    accD[m] = accD[m] - hr * bp[m];
                }
            }
        }
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            S.xl[1][m][t] = xbL[m] + ylA[m] + dxl1[m];
            S.xl[2][m][t] = xcL[m] + dxl2[m];
            S.xl[3][m][t] = xaL[m];
        }
        __syncthreads();  // S3: neighbour increments visible
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            accA[m] = accA[m] + S.xl[0][m][tr] + S.yr[0][m][tl];
            accB[m] = accB[m] + S.xl[1][m][tr] + S.yr[1][m][tl];
            accC[m] = accC[m] + S.xl[2][m][tr];
            accD[m] = accD[m] + S.xl[3][m][tr];
        }

        // ---- row R-2 is complete ----
        if (R >= R0 + 4 && out_col) {
            double v[ME];
            const double ik = CAPA ? S.icap[s0][t] : 1.0;
#pragma unroll
            for (int m = 0; m < ME; ++m) v[m] = CAPA ? S.cell[s0][m][t] + ik * accA[m] : S.cell[s0][m][t] + accA[m];
#pragma unroll
            for (int m = 0; m < ME; ++m) qn[m * plane + (long long)(R - 2) * pitch] = v[m];
            if (!all_finite<ME>(v)) atomicOr(a.status, 1);
        }
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            accA[m] = accB[m];
            accB[m] = accC[m];
            accC[m] = accD[m];
            accD[m] = 0.0;
        }
        const int tmp = s0;
        s0 = s1;
        s1 = s2;
        s2 = tmp;
    }
    if (GuessTraits<RP>::USES && a.counters) counter_commit(a.counters, n_it, n_solve, n_app);
}

// ---------------------------------------------------------------------------
// The two-barrier form of the tile ("deferred x finish").  Each x-interface
// is solved on its row R as before, but finished (limiter with the
// neighbours' waves, correction, transverse solves) one row later, together
// with the y work of that row: at row R every thread
//   * finishes the x-interface (cp-1 | cp) of row R-1 (its waves and those of
//     the neighbours wait in a double-buffered shared array, its own record
//     in shared memory), with the cells of rows R-2, R-1, R in the ring, so
//     solvers whose transverse solve reads the neighbouring cells need no
//     extra deferral,
//   * solves the y-interface (R-1 | R) and finishes (R-2 | R-1),
//   * solves the x-interface of row R and stores its waves,
// all between the same two barriers (cells visible; increments visible).  The
// three independent chains in one block give the scheduler independent
// FP64 work, and a barrier per row is saved.  Every increment lands in the
// same cell with the same factors as in unsplit_tile; row R-2 is still
// complete and written at the end of row R.
// ---------------------------------------------------------------------------
template <class RP, int NT, bool CAPA = false>
struct UnsplitSmem2 {
    static constexpr int ME = RP::MEQN, MW = RP::MWAVES, NC = RP::NC;
    static constexpr int NF = (int)(sizeof(typename RP::Iface) / sizeof(double)) + 2 * ME;  // record + A-dq, A+dq
    double cell[3][NC][NT];   // prepared cells of rows R-2, R-1, R (ring)
    double w[2][MW][ME][NT];  // unlimited x-waves of rows R-1 and R (by row parity)
    double fx[NF][NT];        // this column's x-interface of row R-1: record, A-dq, A+dq
    double xl[3][ME][NT];     // increments for column cp-1: rows R-2, R-1, R
    double yr[2][ME][NT];     // increments for column cp+1: rows R-2, R-1
    double icap[CAPA ? 3 : 1][CAPA ? NT : 1];
    double red[NT / 32];
};

template <class RP, int NT, int SPEC = SPEC_ANY, bool CAPA = false, bool EVO = false>
__device__ __forceinline__ void unsplit_tile2(const StepArgs& a, int strip, int rb, UnsplitSmem2<RP, NT, CAPA>& S,
                                              double& cfl) {
    constexpr int ME = RP::MEQN, MW = RP::MWAVES, NC = RP::NC, W = NT - 4;
    constexpr int NI = (int)(sizeof(typename RP::Iface) / sizeof(double));
    using Iface = typename RP::Iface;
    static_assert(sizeof(Iface) % sizeof(double) == 0, "interface records are made of doubles");

    const int t = threadIdx.x;
    const int mx = a.L.mx, my = a.L.my;
    const int pitch = a.L.pitch;
    const long long plane = a.L.plane;
    const int cp = strip * W + t;
    const int cpl = min(cp, mx + 3);
    const int Hb = min(a.H, my - rb);
    const int R0 = rb, R1 = rb + Hb + 3;
    const bool out_col = (t >= 2) && (t < W + 2) && (cp <= mx + 1);
    const bool xcfl_col = (t >= 2) && (t <= W + 2) && (cp <= mx + 2);
    const bool ycfl_col = (t >= 1) && (t <= W + 2) && (cp <= mx + 2);
    const int tl = (t > 0) ? t - 1 : 0;
    const int tr = (t < NT - 1) ? t + 1 : NT - 1;
    // dt/dx, dt/dy: kernel parameters, or (EVO, the device time loop) the
    // loop's record; a compile-time choice, so ordinary steps keep the
    // parameters as operands of the FP64 instructions instead of registers
    const double dtdx = EVO ? a.evo->dtdx : a.dtdx, dtdy = EVO ? a.evo->dtdy : a.dtdy;
    const RPParams& P = a.rp;
    const int order = (SPEC == SPEC_MC2) ? 2 : a.meth.order;
    const int trans = (SPEC == SPEC_MC2) ? 2 : a.meth.transverse;
    const bool tc = (order > 1) && (trans == 2);
    const double* qo = a.qold + cpl;
    double* qn = a.qnew + cpl;

    constexpr int MA = AuxTraits<RP>::MAUX, MAD = MA > 0 ? MA : 1;
    constexpr bool TAUX = AuxTraits<RP>::TRANSVERSE_AUX;
    const double* ao = a.aux + cpl;
    double pfa[MAD];
#pragma unroll
    for (int k = 0; k < MAD; ++k) pfa[k] = (MA > 0) ? __ldg(ao + k * plane + (long long)R0 * pitch) : 0.0;
    const double* ko = CAPA ? a.capa + cpl : nullptr;
    double pfk = CAPA ? __ldg(ko + (long long)R0 * pitch) : 1.0;

    double pf[ME];
    double accA[ME], accB[ME], accC[ME];  // rows R-2, R-1, R
    Iface fY;                             // y-interface (R-2 | R-1)
    double amY[ME], apY[ME], dY[MW];
    unsigned long long n_it = 0, n_solve = 0, n_app = 0;
#pragma unroll
    for (int m = 0; m < ME; ++m) {
        pf[m] = __ldg(qo + m * plane + (long long)R0 * pitch);
        accA[m] = accB[m] = accC[m] = 0.0;
        amY[m] = apY[m] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < MW; ++k) dY[k] = 0.0;
    memset(&fY, 0, sizeof(fY));

    int s2 = 0, s1 = 2, s0 = 1;  // ring slots of rows R, R-1, R-2
    for (int R = R0; R <= R1; ++R) {
        // ---- row R: prepare this column's cell, prefetch the next row ----
        {
            double q[ME], c[NC];
#pragma unroll
            for (int m = 0; m < ME; ++m) q[m] = pf[m];
            if (R < R1) {
#pragma unroll
                for (int m = 0; m < ME; ++m) pf[m] = __ldg(qo + m * plane + (long long)(R + 1) * pitch);
            }
            double av[MAD];
#pragma unroll
            for (int k = 0; k < MAD; ++k) av[k] = pfa[k];
            if (MA > 0 && R < R1) {
#pragma unroll
                for (int k = 0; k < MAD; ++k) pfa[k] = __ldg(ao + k * plane + (long long)(R + 1) * pitch);
            }
            AuxTraits<RP>::prep(q, av, P, c);
#pragma unroll
            for (int k = 0; k < NC; ++k) S.cell[s2][k][t] = c[k];
            if constexpr (CAPA) {
                S.icap[s2][t] = 1.0 / pfk;
                if (R < R1) pfk = __ldg(ko + (long long)(R + 1) * pitch);
            }
        }
        __syncthreads();  // S1: cells of row R and x-waves of row R-1 visible; previous exchange consumed

        double xl0[ME], xl1[ME], xl2[ME], yr0[ME], yr1[ME];  // this row's increments for the neighbours
#pragma unroll
        for (int m = 0; m < ME; ++m) xl0[m] = xl1[m] = xl2[m] = yr0[m] = yr1[m] = 0.0;

        // ---- x: finish the interface (cp-1 | cp) of row R-1 ----
        if (R - 1 > R0 && R - 1 < R1) {  // rows R0+1 .. R1-1 carry x-interfaces
            const int pb = (R - 1) & 1;
            Iface fX;
            double amX[ME], apX[ME];
            {
                double* fr = reinterpret_cast<double*>(&fX);
#pragma unroll
                for (int k = 0; k < NI; ++k) fr[k] = S.fx[k][t];
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    amX[m] = S.fx[NI + m][t];
                    apX[m] = S.fx[NI + ME + m][t];
                }
            }
            const double xdl = CAPA ? dtdx * S.icap[s1][tl] : dtdx, xdr = CAPA ? dtdx * S.icap[s1][t] : dtdx;
            if (xcfl_col) cfl = fmax(cfl, CAPA ? iface_cfl2<RP, 1>(fX, P, xdl, xdr) : iface_cfl<RP, 1>(fX, P, dtdx));
            double cq[ME];
            if (order != 1) {
                double dl[MW], dr[MW];
#pragma unroll
                for (int k = 0; k < MW; ++k) {
                    double x = 0.0, y = 0.0;
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        const double w = S.w[pb][k][m][t];
                        x = x + S.w[pb][k][m][tl] * w;
                        y = y + w * S.w[pb][k][m][tr];
                    }
                    dl[k] = x;
                    dr[k] = y;
                }
                correction<RP, 1, SPEC>(fX, P, a.meth, CAPA ? 0.5 * (xdl + xdr) : dtdx, dl, dr, cq);
            } else {
#pragma unroll
                for (int m = 0; m < ME; ++m) cq[m] = 0.0;
            }
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                const double f = 0.5 * cq[m];
                accB[m] = accB[m] - dtdx * (apX[m] - f);
                xl1[m] = -dtdx * (amX[m] + f);
            }
            if (trans > 0) {
                const double h = 0.5 * dtdx * dtdy;
                const double hl = CAPA ? h * S.icap[s1][tl] : h, hr = CAPA ? h * S.icap[s1][t] : h;
                double as2[ME], bm[ME], bp[ME];
#pragma unroll
                for (int m = 0; m < ME; ++m) as2[m] = tc ? amX[m] + cq[m] : amX[m];
                if constexpr (TAUX) {  // cell (cp-1, R-1) between rows R-2 and R
                    double cm[NC], c0[NC], cu[NC];
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        cm[k] = S.cell[s0][k][tl];
                        c0[k] = S.cell[s1][k][tl];
                        cu[k] = S.cell[s2][k][tl];
                    }
                    RP::template rpt2_aux<1>(as2, cm, c0, cu, bm, bp);
                } else {
                    RP::template rpt2<1>(fX, P, as2, bm, bp);  // imp = 1 -> column cp-1
                }
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    xl1[m] = xl1[m] + hl * (bp[m] - bm[m]);
                    xl0[m] = hl * bm[m];
                    xl2[m] = -hl * bp[m];
                }
#pragma unroll
                for (int m = 0; m < ME; ++m) as2[m] = tc ? apX[m] - cq[m] : apX[m];
                if constexpr (TAUX) {  // cell (cp, R-1)
                    double cm[NC], c0[NC], cu[NC];
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        cm[k] = S.cell[s0][k][t];
                        c0[k] = S.cell[s1][k][t];
                        cu[k] = S.cell[s2][k][t];
                    }
                    RP::template rpt2_aux<1>(as2, cm, c0, cu, bm, bp);
                } else {
                    RP::template rpt2<1>(fX, P, as2, bm, bp);  // imp = 2 -> column cp
                }
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    accB[m] = accB[m] + hr * (bp[m] - bm[m]);
                    accA[m] = accA[m] + hr * bm[m];
                    accC[m] = accC[m] - hr * bp[m];
                }
            }
        }

        // ---- y: solve (R-1 | R), finish (R-2 | R-1) ----
        if (R > R0) {
            double cB[NC], cA[NC];
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                cB[k] = S.cell[s1][k][t];
                cA[k] = S.cell[s2][k][t];
            }
            Iface fN;
            double amN[ME], apN[ME];
            double gy = 0.0;
            if (GuessTraits<RP>::USES && a.guess) gy = a.guess[plane + (long long)R * pitch + cpl];
            GuessTraits<RP>::template solve<2>(cB, cA, P, gy, fN, amN, apN);
            if (GuessTraits<RP>::USES && cp <= mx + 3) {
                n_it += GuessTraits<RP>::count(fN);
                n_app += GuessTraits<RP>::count_applied(fN);
                n_solve += 1;
            }
            double dn[MW];
            {
                double wY[MW][ME], wN[MW][ME];
                RP::template waves<2>(fY, P, wY);
                RP::template waves<2>(fN, P, wN);
#pragma unroll
                for (int k = 0; k < MW; ++k) {
                    double d = 0.0;
#pragma unroll
                    for (int m = 0; m < ME; ++m) d = d + wY[k][m] * wN[k][m];
                    dn[k] = d;
                }
            }
            if (R >= R0 + 3) {
                const double ydl = CAPA ? dtdy * S.icap[s0][t] : dtdy, ydr = CAPA ? dtdy * S.icap[s1][t] : dtdy;
                if (ycfl_col)
                    cfl = fmax(cfl, CAPA ? iface_cfl2<RP, 2>(fY, P, ydl, ydr) : iface_cfl<RP, 2>(fY, P, dtdy));
                double cq[ME];
                if (order != 1) {
                    correction<RP, 2, SPEC>(fY, P, a.meth, CAPA ? 0.5 * (ydl + ydr) : dtdy, dY, dn, cq);
                } else {
#pragma unroll
                    for (int m = 0; m < ME; ++m) cq[m] = 0.0;
                }
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    const double f = 0.5 * cq[m];
                    accA[m] = accA[m] - dtdy * (amY[m] + f);
                    accB[m] = accB[m] - dtdy * (apY[m] - f);
                }
                if (trans > 0) {
                    const double h = 0.5 * dtdy * dtdx;
                    const double hl = CAPA ? h * S.icap[s0][t] : h, hr = CAPA ? h * S.icap[s1][t] : h;
                    double as2[ME], bm[ME], bp[ME];
#pragma unroll
                    for (int m = 0; m < ME; ++m) as2[m] = tc ? amY[m] + cq[m] : amY[m];
                    if constexpr (TAUX) {  // cell (cp, R-2) between columns cp-1 and cp+1
                        double cm[NC], c0[NC], cu[NC];
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            cm[k] = S.cell[s0][k][tl];
                            c0[k] = S.cell[s0][k][t];
                            cu[k] = S.cell[s0][k][tr];
                        }
                        RP::template rpt2_aux<2>(as2, cm, c0, cu, bm, bp);
                    } else {
                        RP::template rpt2<2>(fY, P, as2, bm, bp);  // imp = 1 -> row R-2
                    }
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        accA[m] = accA[m] + hl * (bp[m] - bm[m]);
                        xl0[m] = xl0[m] + hl * bm[m];
                        yr0[m] = -hl * bp[m];
                    }
#pragma unroll
                    for (int m = 0; m < ME; ++m) as2[m] = tc ? apY[m] - cq[m] : apY[m];
                    if constexpr (TAUX) {  // cell (cp, R-1)
                        double cm[NC], c0[NC], cu[NC];
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            cm[k] = S.cell[s1][k][tl];
                            c0[k] = S.cell[s1][k][t];
                            cu[k] = S.cell[s1][k][tr];
                        }
                        RP::template rpt2_aux<2>(as2, cm, c0, cu, bm, bp);
                    } else {
                        RP::template rpt2<2>(fY, P, as2, bm, bp);  // imp = 2 -> row R-1
                    }
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        accB[m] = accB[m] + hr * (bp[m] - bm[m]);
                        xl1[m] = xl1[m] + hr * bm[m];
                        yr1[m] = -hr * bp[m];
                    }
                }
            }
            fY = fN;
#pragma unroll
            for (int m = 0; m < ME; ++m) { amY[m] = amN[m]; apY[m] = apN[m]; }
#pragma unroll
            for (int k = 0; k < MW; ++k) dY[k] = dn[k];
        }

        // ---- x: solve the interface (cp-1 | cp) of row R, keep it for the next row ----
        if (R > R0 && R < R1) {
            double cL[NC], cR[NC];
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                cL[k] = S.cell[s2][k][tl];
                cR[k] = S.cell[s2][k][t];
            }
            Iface fX;
            double amX[ME], apX[ME];
            double gx = 0.0;
            if (GuessTraits<RP>::USES && a.guess) gx = a.guess[(long long)R * pitch + cpl];
            GuessTraits<RP>::template solve<1>(cL, cR, P, gx, fX, amX, apX);
            if (GuessTraits<RP>::USES && cp <= mx + 3 && t > 0) {
                n_it += GuessTraits<RP>::count(fX);
                n_app += GuessTraits<RP>::count_applied(fX);
                n_solve += 1;
            }
            double wX[MW][ME];
            RP::template waves<1>(fX, P, wX);
            const int pb = R & 1;
#pragma unroll
            for (int k = 0; k < MW; ++k)
#pragma unroll
                for (int m = 0; m < ME; ++m) S.w[pb][k][m][t] = wX[k][m];
            const double* fr = reinterpret_cast<const double*>(&fX);
#pragma unroll
            for (int k = 0; k < NI; ++k) S.fx[k][t] = fr[k];
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                S.fx[NI + m][t] = amX[m];
                S.fx[NI + ME + m][t] = apX[m];
            }
        }
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            S.xl[0][m][t] = xl0[m];
            S.xl[1][m][t] = xl1[m];
            S.xl[2][m][t] = xl2[m];
            S.yr[0][m][t] = yr0[m];
            S.yr[1][m][t] = yr1[m];
        }
        __syncthreads();  // S2: neighbour increments (and this row's x-waves) visible
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            accA[m] = accA[m] + S.xl[0][m][tr] + S.yr[0][m][tl];
            accB[m] = accB[m] + S.xl[1][m][tr] + S.yr[1][m][tl];
            accC[m] = accC[m] + S.xl[2][m][tr];
        }

        // ---- row R-2 is complete ----
        if (R >= R0 + 4 && out_col) {
            double v[ME];
            const double ik = CAPA ? S.icap[s0][t] : 1.0;
#pragma unroll
            for (int m = 0; m < ME; ++m) v[m] = CAPA ? S.cell[s0][m][t] + ik * accA[m] : S.cell[s0][m][t] + accA[m];
#pragma unroll
            for (int m = 0; m < ME; ++m) qn[m * plane + (long long)(R - 2) * pitch] = v[m];
            if (!all_finite<ME>(v)) atomicOr(a.status, 1);
        }
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            accA[m] = accB[m];
            accB[m] = accC[m];
            accC[m] = 0.0;
        }
        const int tmp = s0;
        s0 = s1;
        s1 = s2;
        s2 = tmp;
    }
    if (GuessTraits<RP>::USES && a.counters) counter_commit(a.counters, n_it, n_solve, n_app);
}

template <class RP, int NT, int MINB, int SPEC, bool CAPA = false, bool EVO = false>
__global__ void __launch_bounds__(NT, MINB) k_step_unsplit2(const StepArgs a) {
    if (EVO && a.evo->done) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    UnsplitSmem2<RP, NT, CAPA>& S = *reinterpret_cast<UnsplitSmem2<RP, NT, CAPA>*>(smem_raw);
    const int tile = tile_index(a);
    long long t0 = 0;
    if (a.tile_cost && threadIdx.x == 0) t0 = clock64();
    double cfl = 0.0;
    unsplit_tile2<RP, NT, SPEC, CAPA, EVO>(a, tile % a.nstrips, (tile / a.nstrips) * a.H, S, cfl);
    cfl_commit(cfl, S.red, a.cfl_bits);
    if (a.tile_cost && threadIdx.x == 0) {
        const long long c = clock64() - t0;
        a.tile_cost[tile] = (unsigned int)(c < 0 ? 0 : (c > 0xffffffffll ? 0xffffffffll : c));
    }
}

// ---------------------------------------------------------------------------
// The direction-split tile: two threads per column.  The CTA has 2*NT
// threads; the first NT (the Y warps) own the y-interfaces of their column
// and the second NT (the X warps) its x-interfaces, so each thread carries
// half the live state of unsplit_tile and twice as many warps fit on an SM
// (16 instead of 8 for Euler), which is what the FP64 pipe of a latency-bound
// step needs.  The two warp groups meet only through named barriers used by
// row parity, so the x work of a row overlaps the y work of the same row:
//   Y, row R: [wait EMPTY(R-1)] prepare the column's cell of row R into a
//      4-row ring, prefetch row R+1, [arrive CELLS(R)]; solve (R-1 | R);
//      finish (R-2 | R-1) (limiter with the waves below and above,
//      correction, two transverse solves); [Y] exchange with the neighbour
//      columns [Y]; write row R-3 = q + (its y total + the X group's total);
//      after the last row, [wait EMPTY(R1)] and write row R1-2.
//   X, row R: [wait CELLS(R)] solve (cp-1 | cp) of row R, store its waves
//      [X]; gather the neighbour's increments of row R-1, publish its total of
//      row R-2; finish row R (limiter with the neighbours' waves, correction,
//      two transverse solves), publish column cp-1's increments [X];
//      [arrive EMPTY(R)].
// CELLS(R): row R's cells are in the ring.  EMPTY(R): the X group is done
// with row R (so the ring slot that row R+1 reuses, rows R-3's, and the
// total buffer Y reads next are free).  Both are pairs of barriers used by
// row parity, each with all 2*NT threads; [X] and [Y] are the groups' own
// barriers.  Every arrival has its wait: Y arrives CELLS on every row and X
// waits on every row; X arrives EMPTY on every row and Y waits on rows
// R0+1..R1 and once after the loop.  The y-interface being finished, its
// fluctuations and its dot products wait in shared memory (per column,
// touched only by that column's Y thread).  The increments are the same
// terms as in unsplit_tile; only the order of the per-cell sum differs (the
// x and y parts are summed apart and then added).  Solvers without aux data
// or guesses, no capacity form.
// ---------------------------------------------------------------------------
template <class RP, int NT>
struct UnsplitSmemWS {
    static constexpr int ME = RP::MEQN, MW = RP::MWAVES, NC = RP::NC;
    static constexpr int NF = (int)(sizeof(typename RP::Iface) / sizeof(double));
    double cell[4][NC][NT];          // prepared cells, row R in slot R & 3 (Y writes)
    double w[MW][ME][NT];            // unlimited x-waves of the current row (X)
    double xl[3][ME][NT];            // X -> column cp-1: rows R-1, R, R+1
    double yl[2][ME][NT];            // Y -> column cp-1: rows R-2, R-1
    double yr[2][ME][NT];            // Y -> column cp+1: rows R-2, R-1
    double xs[2][ME][NT];            // X's total of row R-2, by row parity (X -> Y)
    double fy[NF][NT];               // Y: the y-interface being finished, (R-2 | R-1)
    double amy[ME][NT], apy[ME][NT];  // its fluctuations
    double dy[MW][NT];               // its waves' dot products with the waves below it
    double red[2 * NT / 32];
};

// named barriers of the direction-split tile (0 is __syncthreads)
enum { NB_X = 1, NB_Y = 2, NB_CELLS = 3, NB_EMPTY = 5 };

template <int ID, int N>
__device__ __forceinline__ void nb_sync() {
    asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(N) : "memory");
}
template <int ID, int N>
__device__ __forceinline__ void nb_arrive() {
    asm volatile("bar.arrive %0, %1;" ::"n"(ID), "n"(N) : "memory");
}
// the barrier of a pair chosen by row parity (compile-time ids)
template <int ID, int N>
__device__ __forceinline__ void nb_sync_parity(int R) {
    if (R & 1) nb_sync<ID + 1, N>();
    else nb_sync<ID, N>();
}
template <int ID, int N>
__device__ __forceinline__ void nb_arrive_parity(int R) {
    if (R & 1) nb_arrive<ID + 1, N>();
    else nb_arrive<ID, N>();
}

template <class RP, int NT, int SPEC = SPEC_ANY, bool EVO = false, int REG_Y = 0, int REG_X = 0>
__device__ __forceinline__ void unsplit_tile_ws(const StepArgs& a, int strip, int rb, UnsplitSmemWS<RP, NT>& S,
                                                double& cfl) {
    constexpr int ME = RP::MEQN, MW = RP::MWAVES, NC = RP::NC, W = NT - 4;
    constexpr int NF = UnsplitSmemWS<RP, NT>::NF;
    using Iface = typename RP::Iface;
    static_assert(AuxTraits<RP>::MAUX == 0 && !GuessTraits<RP>::USES, "direction-split tile: no aux, no guess");

    const bool yrole = threadIdx.x < NT;
    const int t = yrole ? threadIdx.x : threadIdx.x - NT;
    const int mx = a.L.mx, my = a.L.my;
    const int pitch = a.L.pitch;
    const long long plane = a.L.plane;
    const int cp = strip * W + t;
    const int cpl = min(cp, mx + 3);
    const int Hb = min(a.H, my - rb);
    const int R0 = rb, R1 = rb + Hb + 3;
    const bool out_col = (t >= 2) && (t < W + 2) && (cp <= mx + 1);
    const bool xcfl_col = (t >= 2) && (t <= W + 2) && (cp <= mx + 2);
    const bool ycfl_col = (t >= 1) && (t <= W + 2) && (cp <= mx + 2);
    const int tl = (t > 0) ? t - 1 : 0;
    const int tr = (t < NT - 1) ? t + 1 : NT - 1;
    const double dtdx = EVO ? a.evo->dtdx : a.dtdx, dtdy = EVO ? a.evo->dtdy : a.dtdy;
    const RPParams& P = a.rp;
    const int order = (SPEC == SPEC_MC2) ? 2 : a.meth.order;
    const int trans = (SPEC == SPEC_MC2) ? 2 : a.meth.transverse;
    const bool tc = (order > 1) && (trans == 2);
    constexpr bool ZS = SkipTraits<RP>::OK;
    const bool zs = ZS && (SPEC != SPEC_ANY || a.meth.fwave == 0);
    constexpr int N2 = 2 * NT;

    if (yrole) {
        // ================= Y warps =================
        if (REG_Y > 0) asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(REG_Y));
        const double* qo = a.qold + cpl;
        double* qn = a.qnew + cpl;
        double pf[ME], yA[ME], yB[ME], yC[ME];  // prefetched row; increments of rows R-2, R-1; total of R-3
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            pf[m] = __ldg(qo + m * plane + (long long)R0 * pitch);
            yA[m] = yB[m] = yC[m] = 0.0;
        }
        bool zY = false;
        for (int R = R0; R <= R1; ++R) {
            const int s2 = R & 3, s1 = (R - 1) & 3;
            if (R >= R0 + 1) nb_sync_parity<NB_EMPTY, N2>(R - 1);  // X done with row R-1: the slot of R-4 is free
            {
                double q[ME], c[NC];
#pragma unroll
                for (int m = 0; m < ME; ++m) q[m] = pf[m];
                if (R < R1) {
#pragma unroll
                    for (int m = 0; m < ME; ++m) pf[m] = __ldg(qo + m * plane + (long long)(R + 1) * pitch);
                }
                RP::prepare(q, P, c);
#pragma unroll
                for (int k = 0; k < NC; ++k) S.cell[s2][k][t] = c[k];
            }
            nb_arrive_parity<NB_CELLS, N2>(R);  // row R prepared
            double ylB[ME], ylA[ME], yrB[ME], yrA[ME];
#pragma unroll
            for (int m = 0; m < ME; ++m) ylB[m] = ylA[m] = yrB[m] = yrA[m] = 0.0;
            if (R > R0) {
                double cB[NC], cA[NC];
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    cB[k] = S.cell[s1][k][t];
                    cA[k] = S.cell[s2][k][t];
                }
                Iface fN, fY;
                double amN[ME], apN[ME], dn[MW];
                const bool zN = zs && __all_sync(0xffffffffu, same_q<ME, NC>(cB, cA));
                {
                    double* fp = reinterpret_cast<double*>(&fY);
#pragma unroll
                    for (int k = 0; k < NF; ++k) fp[k] = S.fy[k][t];
                }
                if (ZS && zN) {
                    SkipTraits<RP>::template zero_iface<2>(cB, cA, P, fN);
#pragma unroll
                    for (int m = 0; m < ME; ++m) amN[m] = apN[m] = 0.0;
#pragma unroll
                    for (int k = 0; k < MW; ++k) dn[k] = 0.0;
                } else {
                    RP::template solve<2>(cB, cA, P, fN, amN, apN);
                    double wY[MW][ME], wN[MW][ME];
                    RP::template waves<2>(fY, P, wY);
                    RP::template waves<2>(fN, P, wN);
#pragma unroll
                    for (int k = 0; k < MW; ++k) {
                        double d = 0.0;
#pragma unroll
                        for (int m = 0; m < ME; ++m) d = d + wY[k][m] * wN[k][m];
                        dn[k] = d;
                    }
                }
                if (R >= R0 + 3) {
                    if (ycfl_col) cfl = fmax(cfl, iface_cfl<RP, 2>(fY, P, dtdy));
                    if (!(ZS && zY)) {
                        double amY[ME], apY[ME], dY[MW], cq[ME];
#pragma unroll
                        for (int m = 0; m < ME; ++m) {
                            amY[m] = S.amy[m][t];
                            apY[m] = S.apy[m][t];
                        }
#pragma unroll
                        for (int k = 0; k < MW; ++k) dY[k] = S.dy[k][t];
                        if (order != 1) {
                            correction<RP, 2, SPEC>(fY, P, a.meth, dtdy, dY, dn, cq);
                        } else {
#pragma unroll
                            for (int m = 0; m < ME; ++m) cq[m] = 0.0;
                        }
#pragma unroll
                        for (int m = 0; m < ME; ++m) {
                            const double f = 0.5 * cq[m];
                            yA[m] = yA[m] - dtdy * (amY[m] + f);
                            yB[m] = yB[m] - dtdy * (apY[m] - f);
                        }
                        if (trans > 0) {
                            const double h = 0.5 * dtdy * dtdx;
                            double as2[ME], bm[ME], bp[ME];
#pragma unroll
                            for (int m = 0; m < ME; ++m) as2[m] = tc ? amY[m] + cq[m] : amY[m];
                            RP::template rpt2<2>(fY, P, as2, bm, bp);  // imp = 1 -> row R-2
#pragma unroll
                            for (int m = 0; m < ME; ++m) {
                                yA[m] = yA[m] + h * (bp[m] - bm[m]);
                                ylB[m] = h * bm[m];
                                yrB[m] = -h * bp[m];
                            }
#pragma unroll
                            for (int m = 0; m < ME; ++m) as2[m] = tc ? apY[m] - cq[m] : apY[m];
                            RP::template rpt2<2>(fY, P, as2, bm, bp);  // imp = 2 -> row R-1
#pragma unroll
                            for (int m = 0; m < ME; ++m) {
                                yB[m] = yB[m] + h * (bp[m] - bm[m]);
                                ylA[m] = h * bm[m];
                                yrA[m] = -h * bp[m];
                            }
                        }
                    }
                }
                {
                    const double* fp = reinterpret_cast<const double*>(&fN);
#pragma unroll
                    for (int k = 0; k < NF; ++k) S.fy[k][t] = fp[k];
                }
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    S.amy[m][t] = amN[m];
                    S.apy[m][t] = apN[m];
                }
#pragma unroll
                for (int k = 0; k < MW; ++k) S.dy[k][t] = dn[k];
                zY = zN;
            } else {
                // the first row: an empty record below it (zero waves, zero dots)
#pragma unroll
                for (int k = 0; k < NF; ++k) S.fy[k][t] = 0.0;
            }
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                S.yl[0][m][t] = ylB[m];
                S.yl[1][m][t] = ylA[m];
                S.yr[0][m][t] = yrB[m];
                S.yr[1][m][t] = yrA[m];
            }
            nb_sync<NB_Y, NT>();  // the Y warps' neighbour increments visible
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                yA[m] = yA[m] + S.yl[0][m][tr] + S.yr[0][m][tl];
                yB[m] = yB[m] + S.yl[1][m][tr] + S.yr[1][m][tl];
            }
            nb_sync<NB_Y, NT>();  // every read of the exchange done before the next row's writes
            if (R >= R0 + 5 && out_col) {  // row R-3: both totals complete (X's since its row R-1)
                double v[ME];
#pragma unroll
                for (int m = 0; m < ME; ++m) v[m] = S.cell[(R - 3) & 3][m][t] + (yC[m] + S.xs[(R - 3) & 1][m][t]);
#pragma unroll
                for (int m = 0; m < ME; ++m) qn[m * plane + (long long)(R - 3) * pitch] = v[m];
                if (!all_finite<ME>(v)) atomicOr(a.status, 1);
            }
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                yC[m] = yA[m];  // row R-2 complete on the y side
                yA[m] = yB[m];
                yB[m] = 0.0;
            }
        }
        nb_sync_parity<NB_EMPTY, N2>(R1);  // X done with the last row: its total of row R1-2
        if (R1 >= R0 + 4 && out_col) {
            double v[ME];
#pragma unroll
            for (int m = 0; m < ME; ++m) v[m] = S.cell[(R1 - 2) & 3][m][t] + (yC[m] + S.xs[(R1 - 2) & 1][m][t]);
#pragma unroll
            for (int m = 0; m < ME; ++m) qn[m * plane + (long long)(R1 - 2) * pitch] = v[m];
            if (!all_finite<ME>(v)) atomicOr(a.status, 1);
        }
    } else {
        // ================= X warps =================
        if (REG_X > 0) asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REG_X));
        double x0[ME], x1[ME], x2[ME];  // increments of rows R-2, R-1, R (this column)
#pragma unroll
        for (int m = 0; m < ME; ++m) x0[m] = x1[m] = x2[m] = 0.0;
        for (int R = R0; R <= R1; ++R) {
            const int s2 = R & 3;
            nb_sync_parity<NB_CELLS, N2>(R);  // row R prepared
            Iface fX;
            double amX[ME], apX[ME];
            bool zX;
            const bool xrow = (R > R0) && (R < R1);
            {
                double cL[NC], cR[NC];
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    cL[k] = S.cell[s2][k][tl];
                    cR[k] = S.cell[s2][k][t];
                }
                // (the first and last rows' x-interfaces are never finished: no solve)
                zX = ZS && (!xrow || (zs && __all_sync(0xffffffffu, same_q<ME, NC>(cL, cR))));
                if (ZS && zX) {
                    SkipTraits<RP>::template zero_iface<1>(cL, cR, P, fX);
#pragma unroll
                    for (int m = 0; m < ME; ++m) amX[m] = apX[m] = 0.0;
#pragma unroll
                    for (int k = 0; k < MW; ++k)
#pragma unroll
                        for (int m = 0; m < ME; ++m) S.w[k][m][t] = 0.0;
                } else {
                    RP::template solve<1>(cL, cR, P, fX, amX, apX);
                    double wX[MW][ME];
                    RP::template waves<1>(fX, P, wX);
#pragma unroll
                    for (int k = 0; k < MW; ++k)
#pragma unroll
                        for (int m = 0; m < ME; ++m) S.w[k][m][t] = wX[k][m];
                }
            }
            nb_sync<NB_X, NT>();  // x-waves of row R and column cp-1's increments of row R-1 visible
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                x0[m] = x0[m] + S.xl[0][m][tr];  // rows R-2, R-1, R from the neighbour's row R-1
                x1[m] = x1[m] + S.xl[1][m][tr];
                x2[m] = x2[m] + S.xl[2][m][tr];
                S.xs[R & 1][m][t] = x0[m];  // row R-2 complete on the x side
            }
            double x3[ME], xbL[ME], xcL[ME], xaL[ME];
#pragma unroll
            for (int m = 0; m < ME; ++m) x3[m] = xbL[m] = xcL[m] = xaL[m] = 0.0;
            if (xrow && xcfl_col) cfl = fmax(cfl, iface_cfl<RP, 1>(fX, P, dtdx));
            if (xrow && !(ZS && zX)) {
                double cq[ME];
                if (order != 1) {
                    double dl[MW], dr[MW];
#pragma unroll
                    for (int k = 0; k < MW; ++k) {
                        double x = 0.0, y = 0.0;
#pragma unroll
                        for (int m = 0; m < ME; ++m) {
                            const double w = S.w[k][m][t];
                            x = x + S.w[k][m][tl] * w;
                            y = y + w * S.w[k][m][tr];
                        }
                        dl[k] = x;
                        dr[k] = y;
                    }
                    correction<RP, 1, SPEC>(fX, P, a.meth, dtdx, dl, dr, cq);
                } else {
#pragma unroll
                    for (int m = 0; m < ME; ++m) cq[m] = 0.0;
                }
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    const double f = 0.5 * cq[m];
                    x2[m] = x2[m] - dtdx * (apX[m] - f);
                    xcL[m] = -dtdx * (amX[m] + f);
                }
                if (trans > 0) {
                    const double h = 0.5 * dtdx * dtdy;
                    double as2[ME], bm[ME], bp[ME];
#pragma unroll
                    for (int m = 0; m < ME; ++m) as2[m] = tc ? amX[m] + cq[m] : amX[m];
                    RP::template rpt2<1>(fX, P, as2, bm, bp);  // imp = 1 -> column cp-1
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        xcL[m] = xcL[m] + h * (bp[m] - bm[m]);
                        xbL[m] = h * bm[m];
                        xaL[m] = -h * bp[m];
                    }
#pragma unroll
                    for (int m = 0; m < ME; ++m) as2[m] = tc ? apX[m] - cq[m] : apX[m];
                    RP::template rpt2<1>(fX, P, as2, bm, bp);  // imp = 2 -> column cp
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        x2[m] = x2[m] + h * (bp[m] - bm[m]);
                        x1[m] = x1[m] + h * bm[m];
                        x3[m] = x3[m] - h * bp[m];
                    }
                }
            }
            nb_sync<NB_X, NT>();  // every read of the waves and of the exchange slots done
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                S.xl[0][m][t] = xbL[m];
                S.xl[1][m][t] = xcL[m];
                S.xl[2][m][t] = xaL[m];
                x0[m] = x1[m];
                x1[m] = x2[m];
                x2[m] = x3[m];
            }
            nb_arrive_parity<NB_EMPTY, N2>(R);  // done with row R; its total of row R-2 published
        }
    }
}

// Grid: 1D over the tiles as k_step_unsplit, 2*NT threads per CTA.
template <class RP, int NT, int MINB, int SPEC, bool EVO = false, int REG_Y = 0, int REG_X = 0>
__global__ void __launch_bounds__(2 * NT, MINB) k_step_unsplit_ws(const StepArgs a) {
    if (EVO && a.evo->done) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    UnsplitSmemWS<RP, NT>& S = *reinterpret_cast<UnsplitSmemWS<RP, NT>*>(smem_raw);
    const int tile = tile_index(a);
    long long t0 = 0;
    if (a.tile_cost && threadIdx.x == 0) t0 = clock64();
    double cfl = 0.0;
    unsplit_tile_ws<RP, NT, SPEC, EVO, REG_Y, REG_X>(a, tile % a.nstrips, (tile / a.nstrips) * a.H, S, cfl);
    cfl_commit(cfl, S.red, a.cfl_bits);
    if (a.tile_cost && threadIdx.x == 0) {
        const long long c = clock64() - t0;
        a.tile_cost[tile] = (unsigned int)(c < 0 ? 0 : (c > 0xffffffffll ? 0xffffffffll : c));
    }
}

// The same kernel with its rows staged by TMA from the tensor map of qold.
template <class RP, int NT, int MINB, int SPEC>
__global__ void __launch_bounds__(NT, MINB) k_step_unsplit_tma(const StepArgs a, const __grid_constant__ CUtensorMap tm) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    UnsplitSmemTma<RP, NT>& S = *reinterpret_cast<UnsplitSmemTma<RP, NT>*>(smem_raw);
    const int tile = tile_index(a);
    long long t0 = 0;
    if (a.tile_cost && threadIdx.x == 0) t0 = clock64();
    double cfl = 0.0;
    unsplit_tile<RP, NT, SPEC>(a, tile % a.nstrips, (tile / a.nstrips) * a.H, S.s, cfl, &tm, &S.qrow[0][0], &S.bar);
    cfl_commit(cfl, S.s.red, a.cfl_bits);
    if (a.tile_cost && threadIdx.x == 0) {
        const long long c = clock64() - t0;
        a.tile_cost[tile] = (unsigned int)(c < 0 ? 0 : (c > 0xffffffffll ? 0xffffffffll : c));
    }
}

// Grid: 1D over the tiles (strip fastest).  Tile t = (strip t % nstrips, row
// block t / nstrips); CTA b runs tile_order[b] when a schedule is given.
// EVO: launched by the device time loop (dt from a.evo, nothing to do once
// the loop is done).
template <class RP, int NT, int MINB, int SPEC, bool CAPA = false, bool EVO = false>
__global__ void __launch_bounds__(NT, MINB) k_step_unsplit(const StepArgs a) {
    if (EVO && a.evo->done) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    UnsplitSmem<RP, NT, CAPA>& S = *reinterpret_cast<UnsplitSmem<RP, NT, CAPA>*>(smem_raw);
    const int tile = tile_index(a);
    long long t0 = 0;
    if (a.tile_cost && threadIdx.x == 0) t0 = clock64();
    double cfl = 0.0;
    unsplit_tile<RP, NT, SPEC, CAPA, EVO>(a, tile % a.nstrips, (tile / a.nstrips) * a.H, S, cfl);
    cfl_commit(cfl, S.red, a.cfl_bits);
    if (a.tile_cost && threadIdx.x == 0) {
        const long long c = clock64() - t0;
        a.tile_cost[tile] = (unsigned int)(c < 0 ? 0 : (c > 0xffffffffll ? 0xffffffffll : c));
    }
}

// Longest-first tile schedule for the next step from this step's tile costs:
// one CTA sorts (cost, tile) pairs, n <= LPT_MAX_TILES, descending by cost
// (ties: lower tile first) with a bitonic network in shared memory, and
// writes the tile order.  The hardware starts CTAs in block order, so the
// most expensive tiles (the developed parts of the flow; the cost pattern
// moves slowly from step to step) start first and the cheap ones fill the
// tail, which evens out the SMs' finishing times.  The order changes only
// which SM runs a tile: every result is independent of it.
constexpr int LPT_MAX_TILES = 8192;
// Up to 1024 tiles (one key per thread): the stages whose partner is in the
// same warp (j < 32, 40 of the 55 stages at 1024) exchange keys by shuffles,
// the others through two alternating shared-memory buffers, one barrier each.
static __global__ void __launch_bounds__(1024) k_lpt_order(const unsigned int* cost, int* order, int n) {
    extern __shared__ unsigned long long keys[];
    int N = 1;
    while (N < n) N <<= 1;
    if (N >= 32 && N <= (int)blockDim.x) {
        const int i = threadIdx.x;
        unsigned long long x = 0ull;
        if (i < n) x = ((unsigned long long)cost[i] << 32) | (unsigned long long)(0xffffffffu - (unsigned)i);
        int pb = 0;
        for (int k = 2; k <= N; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                unsigned long long y;
                if (j >= 32) {
                    if (i < N) keys[pb * N + i] = x;
                    __syncthreads();
                    y = (i < N) ? keys[pb * N + (i ^ j)] : 0ull;
                    pb ^= 1;
                } else {
                    y = __shfl_xor_sync(0xffffffffu, x, j);
                }
                // descending blocks ((i & k) == 0) keep the larger key at the
                // lower index of the pair, ascending blocks the smaller
                const bool keep_max = ((i & j) == 0) == ((i & k) == 0);
                x = keep_max ? (x > y ? x : y) : (x > y ? y : x);
            }
        }
        if (i < n) order[i] = (int)(0xffffffffu - (unsigned)(x & 0xffffffffull));
        return;
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x)
        keys[i] = (i < n) ? (((unsigned long long)cost[i] << 32) | (unsigned long long)(0xffffffffu - (unsigned)i))
                          : 0ull;
    __syncthreads();
    for (int k = 2; k <= N; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < N; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long x = keys[i], y = keys[ixj];
                    // descending overall: blocks with (i & k) == 0 descend, the others ascend
                    const bool swap = ((i & k) == 0) ? (x < y) : (x > y);
                    if (swap) {
                        keys[i] = y;
                        keys[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        order[i] = (int)(0xffffffffu - (unsigned)(keys[i] & 0xffffffffull));
}

static __global__ void k_iota(int* a, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// ---------------------------------------------------------------------------
// Split step, x-sweep (step2ds.f90:86-172): every padded row, no transverse
// terms.  Writes the interior columns of qtmp and copies the ghost columns.
// ---------------------------------------------------------------------------
template <class RP, int NT>
struct SplitXSmem {
    static constexpr int ME = RP::MEQN, MW = RP::MWAVES, NC = RP::NC;
    double cell[2][NC][NT];
    double icap[2][NT];  // 1 / kappa (1 without a capacity function)
    double w[MW][ME][NT];
    double xl[ME][NT];
    double red[NT / 32];
};

template <class RP, int NT, int SPEC = SPEC_ANY, bool EVO = false>
__global__ void __launch_bounds__(NT) k_split_x(const StepArgs a) {
    if (EVO && a.evo->done) return;
    constexpr int ME = RP::MEQN, MW = RP::MWAVES, NC = RP::NC, W = NT - 4;
    constexpr int MAD = AuxTraits<RP>::MAUX > 0 ? AuxTraits<RP>::MAUX : 1;
    using Iface = typename RP::Iface;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    SplitXSmem<RP, NT>& S = *reinterpret_cast<SplitXSmem<RP, NT>*>(smem_raw);

    const int t = threadIdx.x;
    const int mx = a.L.mx, my = a.L.my;
    const int pitch = a.L.pitch;
    const long long plane = a.L.plane;
    const int cp = blockIdx.x * W + t;
    const int cpl = min(cp, mx + 3);
    const int rb = blockIdx.y * a.H;       // first padded row of this block
    const int re = min(rb + a.H, my + 4);  // one past the last
    const bool out_col = (t >= 2) && (t < W + 2) && (cp <= mx + 1);
    const bool ghost_copy = (cp <= mx + 3) && ((cp < 2 && t == cp) || (cp >= mx + 2 && t >= 2));
    const bool xcfl_col = (t >= 2) && (t <= W + 2) && (cp <= mx + 2);
    const int tl = (t > 0) ? t - 1 : 0;
    const int tr = (t < NT - 1) ? t + 1 : NT - 1;
    const double dtdx = EVO ? a.evo->dtdx : a.dtdx;  // (compile-time choice, as in unsplit_tile)
    const RPParams& P = a.rp;
    const double* qo = a.qold + cpl;
    double* qn = a.qnew + cpl;
    double cfl = 0.0;
    // zero-jump shortcut (q-wave solvers without aux data), as in unsplit_tile
    constexpr bool ZS = SkipTraits<RP>::OK && AuxTraits<RP>::MAUX == 0;
    const bool zs = ZS && (SPEC != SPEC_ANY || a.meth.fwave == 0);

    for (int R = rb; R < re; ++R) {
        const int buf = R & 1;
        double q[ME];
        {
            double c[NC];
#pragma unroll
            for (int m = 0; m < ME; ++m) q[m] = __ldg(qo + m * plane + (long long)R * pitch);
            double av[MAD];
            load_aux<RP, MAD>(a.aux + cpl, plane, pitch, R, av);
            AuxTraits<RP>::prep(q, av, P, c);
#pragma unroll
            for (int k = 0; k < NC; ++k) S.cell[buf][k][t] = c[k];
            S.icap[buf][t] = a.capa ? 1.0 / __ldg(a.capa + cpl + (long long)R * pitch) : 1.0;
        }
        __syncthreads();
        Iface fX;
        double amX[ME], apX[ME];
        bool zX = false;  // every lane of the warp has equal cells on both sides
        {
            double cL[NC], cR[NC];
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                cL[k] = S.cell[buf][k][tl];
                cR[k] = S.cell[buf][k][t];
            }
            zX = ZS && zs && __all_sync(0xffffffffu, same_q<ME, NC>(cL, cR));
            if (ZS && zX) {
                SkipTraits<RP>::template zero_iface<1>(cL, cR, P, fX);
#pragma unroll
                for (int m = 0; m < ME; ++m) amX[m] = apX[m] = 0.0;
#pragma unroll
                for (int k = 0; k < MW; ++k)
#pragma unroll
                    for (int m = 0; m < ME; ++m) S.w[k][m][t] = 0.0;
            } else {
                RP::template solve<1>(cL, cR, P, fX, amX, apX);
                double wX[MW][ME];
                RP::template waves<1>(fX, P, wX);
#pragma unroll
                for (int k = 0; k < MW; ++k)
#pragma unroll
                    for (int m = 0; m < ME; ++m) S.w[k][m][t] = wX[k][m];
            }
        }
        __syncthreads();
        // dt/(dx kappa) left and right of the interface (both dtdx without capacity)
        const double xdl = dtdx * S.icap[buf][tl], xdr = dtdx * S.icap[buf][t];
        if (xcfl_col) cfl = fmax(cfl, iface_cfl2<RP, 1>(fX, P, xdl, xdr));
        double cq[ME];
        if (!(ZS && zX) && ((SPEC != SPEC_ANY) || a.meth.order != 1)) {
            double dl[MW], dr[MW];
#pragma unroll
            for (int k = 0; k < MW; ++k) {
                double x = 0.0, y = 0.0;
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    const double w = S.w[k][m][t];
                    x = x + S.w[k][m][tl] * w;
                    y = y + w * S.w[k][m][tr];
                }
                dl[k] = x;
                dr[k] = y;
            }
            correction<RP, 1, SPEC>(fX, P, a.meth, 0.5 * (xdl + xdr), dl, dr, cq);
        } else {
#pragma unroll
            for (int m = 0; m < ME; ++m) cq[m] = 0.0;
        }
#pragma unroll
        for (int m = 0; m < ME; ++m) S.xl[m][t] = -dtdx * (amX[m] + 0.5 * cq[m]);
        __syncthreads();
        if (out_col) {
            double v[ME];
            const double ik = S.icap[buf][t];
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                v[m] = q[m] + ik * (-dtdx * (apX[m] - 0.5 * cq[m]) + S.xl[m][tr]);
                qn[m * plane + (long long)R * pitch] = v[m];
            }
            if (!all_finite<ME>(v)) atomicOr(a.status, 1);
        } else if (ghost_copy) {
#pragma unroll
            for (int m = 0; m < ME; ++m) qn[m * plane + (long long)R * pitch] = q[m];
        }
    }
    cfl_commit(cfl, S.red, a.cfl_bits);
}

// ---------------------------------------------------------------------------
// Split step, y-sweep (step2ds.f90:174-261): every padded column, one thread
// per column marching down the rows; limiter neighbours come from the
// register pipeline.  Writes the interior cells of qnew.
// ---------------------------------------------------------------------------
template <class RP, int NT, int SPEC = SPEC_ANY, bool EVO = false>
__global__ void __launch_bounds__(NT) k_split_y(const StepArgs a) {
    if (EVO && a.evo->done) return;
    constexpr int ME = RP::MEQN, MW = RP::MWAVES, NC = RP::NC;
    constexpr int MAD = AuxTraits<RP>::MAUX > 0 ? AuxTraits<RP>::MAUX : 1;
    using Iface = typename RP::Iface;
    __shared__ double sRed[NT / 32];
    const int mx = a.L.mx, my = a.L.my;
    const int pitch = a.L.pitch;
    const long long plane = a.L.plane;
    const int cp = blockIdx.x * NT + threadIdx.x;
    const int cpl = min(cp, mx + 3);
    const bool valid = cp <= mx + 3;
    const bool out_col = (cp >= 2) && (cp <= mx + 1);
    const int rb = blockIdx.y * a.H;
    const int Hb = min(a.H, my - rb);
    const int R0 = rb, R1 = rb + Hb + 3;
    const double dtdy = EVO ? a.evo->dtdy : a.dtdy;
    const RPParams& P = a.rp;
    const double* qo = a.qold + cpl;
    double* qn = a.qnew + cpl;

    // zero-jump shortcut (q-wave solvers without aux data), as in unsplit_tile
    constexpr bool ZS = SkipTraits<RP>::OK && AuxTraits<RP>::MAUX == 0;
    const bool zs = ZS && (SPEC != SPEC_ANY || a.meth.fwave == 0);
    bool zY = false;  // the interface (R-2 | R-1) being finished is zero in the whole warp
    double q0[ME], q1[ME], cB[NC], acc0[ME], acc1[ME];
    Iface fY;
    double amY[ME], apY[ME], dY[MW];
    double cfl = 0.0;
    // 1 / kappa of rows R-2 and R-1 (1 without a capacity function)
    const double* ko = a.capa ? a.capa + cpl : nullptr;
    double ic0 = ko ? 1.0 / __ldg(ko + (long long)R0 * pitch) : 1.0, ic1 = ic0;
    {
        double q[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) q[m] = __ldg(qo + m * plane + (long long)R0 * pitch);
        double av[MAD];
        load_aux<RP, MAD>(a.aux + cpl, plane, pitch, R0, av);
        AuxTraits<RP>::prep(q, av, P, cB);
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            q0[m] = q1[m] = q[m];
            acc0[m] = acc1[m] = 0.0;
            amY[m] = apY[m] = 0.0;
        }
    }
#pragma unroll
    for (int k = 0; k < MW; ++k) dY[k] = 0.0;
    memset(&fY, 0, sizeof(fY));
    for (int R = R0 + 1; R <= R1; ++R) {
        double q2[ME], cA[NC];
#pragma unroll
        for (int m = 0; m < ME; ++m) q2[m] = __ldg(qo + m * plane + (long long)R * pitch);
        double av[MAD];
        load_aux<RP, MAD>(a.aux + cpl, plane, pitch, R, av);
        AuxTraits<RP>::prep(q2, av, P, cA);
        const double ic2 = ko ? 1.0 / __ldg(ko + (long long)R * pitch) : 1.0;
        Iface fN;
        double amN[ME], apN[ME];
        double dn[MW];
        const bool zN = ZS && zs && __all_sync(0xffffffffu, same_q<ME, NC>(cB, cA));
        if (ZS && zN) {
            SkipTraits<RP>::template zero_iface<2>(cB, cA, P, fN);
#pragma unroll
            for (int m = 0; m < ME; ++m) amN[m] = apN[m] = 0.0;
#pragma unroll
            for (int k = 0; k < MW; ++k) dn[k] = 0.0;
        } else {
            RP::template solve<2>(cB, cA, P, fN, amN, apN);
            double wY[MW][ME], wN[MW][ME];
            RP::template waves<2>(fY, P, wY);
            RP::template waves<2>(fN, P, wN);
#pragma unroll
            for (int k = 0; k < MW; ++k) {
                double d = 0.0;
#pragma unroll
                for (int m = 0; m < ME; ++m) d = d + wY[k][m] * wN[k][m];
                dn[k] = d;
            }
        }
        // acc0 <-> row R-2, acc1 <-> row R-1
        if (R >= R0 + 3) {
            const double ydl = dtdy * ic0, ydr = dtdy * ic1;
            if (valid) cfl = fmax(cfl, iface_cfl2<RP, 2>(fY, P, ydl, ydr));
        }
        if (R >= R0 + 3 && !(ZS && zY)) {
            const double ydl = dtdy * ic0, ydr = dtdy * ic1;
            double cq[ME];
            if ((SPEC != SPEC_ANY) || a.meth.order != 1) {
                correction<RP, 2, SPEC>(fY, P, a.meth, 0.5 * (ydl + ydr), dY, dn, cq);
            } else {
#pragma unroll
                for (int m = 0; m < ME; ++m) cq[m] = 0.0;
            }
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                acc0[m] = acc0[m] - dtdy * (amY[m] + 0.5 * cq[m]);
                acc1[m] = acc1[m] - dtdy * (apY[m] - 0.5 * cq[m]);
            }
        }
        if (R >= R0 + 4 && out_col) {
            double v[ME];
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                v[m] = q0[m] + ic0 * acc0[m];
                qn[m * plane + (long long)(R - 2) * pitch] = v[m];
            }
            if (!all_finite<ME>(v)) atomicOr(a.status, 1);
        }
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            acc0[m] = acc1[m];
            acc1[m] = 0.0;
            amY[m] = amN[m];
            apY[m] = apN[m];
            q0[m] = q1[m];
            q1[m] = q2[m];
        }
        ic0 = ic1;
        ic1 = ic2;
#pragma unroll
        for (int k = 0; k < NC; ++k) cB[k] = cA[k];
#pragma unroll
        for (int k = 0; k < MW; ++k) dY[k] = dn[k];
        fY = fN;
        zY = zN;
    }
    cfl_commit(cfl, sRed, a.cfl_bits);
}

// ---------------------------------------------------------------------------
// Ghost-cell fill (solver.py:351-519) in one pass: a ghost cell takes its
// value from the interior source its x rule and/or y rule name, with the
// normal-momentum sign flips of a wall.  Sources are always interior cells, so
// the fill runs in place.  Also clears the CFL word of the step that follows.
// ---------------------------------------------------------------------------
struct BCArgs {
    double* q;
    Layout L;
    int meqn;
    int bcl[2], bcu[2];
    unsigned long long* cfl_bits;
    int negate = 1;  // a wall negates the normal momentum (q); 0 for aux (plain mirror)
    // 0: every ghost cell; 1: all but the ghost rows of internal sides
    // (CLAW2_BC_NONE), which a halo exchange may be writing; 2: only the
    // ghost columns of those rows (their corners), after the exchange
    int part = 0;
};

__device__ __forceinline__ int bc_src(int c, int n, int lo, int up, bool& flip) {
    // c padded index in [0, n+4); returns the padded source index
    flip = false;
    if (c < 2) {
        if (lo == CLAW2_BC_NONE) return c;
        if (lo == CLAW2_BC_EXTRAP) return 2;
        if (lo == CLAW2_BC_PERIODIC) return c + n;
        flip = true;
        return 3 - c;  // wall
    }
    if (c >= n + 2) {
        if (up == CLAW2_BC_NONE) return c;
        if (up == CLAW2_BC_EXTRAP) return n + 1;
        if (up == CLAW2_BC_PERIODIC) return c - n;
        flip = true;
        return 2 * n + 3 - c;  // wall
    }
    return c;
}

static __global__ void k_bc_fill(const BCArgs a) {
    const int mx = a.L.mx, my = a.L.my;
    const int nrow = 4 * (mx + 4);   // cells of the 4 ghost rows
    const int ncol = 4 * my;         // ghost-column cells of interior rows
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0 && a.cfl_bits && a.part != 2) *a.cfl_bits = 0ull;
    if (k >= nrow + ncol) return;
    int c, r;
    if (k < nrow) {
        const int g = k / (mx + 4);
        c = k - g * (mx + 4);
        r = (g < 2) ? g : my + g;  // 0, 1, my+2, my+3
    } else {
        const int kk = k - nrow;
        const int g = kk & 3;
        r = 2 + (kk >> 2);
        c = (g < 2) ? g : mx + g;
    }
    if (a.part != 0) {
        const bool halo_row = (r < 2 && a.bcl[1] == CLAW2_BC_NONE) || (r >= my + 2 && a.bcu[1] == CLAW2_BC_NONE);
        if (a.part == 1 && halo_row) return;
        if (a.part == 2 && !(halo_row && (c < 2 || c >= mx + 2))) return;
    }
    bool fx, fy;
    const int cs = bc_src(c, mx, a.bcl[0], a.bcu[0], fx);
    const int rs = bc_src(r, my, a.bcl[1], a.bcu[1], fy);
    const long long src = (long long)rs * a.L.pitch + cs, dst = (long long)r * a.L.pitch + c;
    // all loads of a group before its stores: the planes are one array, so a
    // store could alias the next load and would otherwise serialise the
    // (cold, after an L2 flush) DRAM round trips one component at a time
    constexpr int G = 4;
    for (int m0 = 0; m0 < a.meqn; m0 += G) {
        double v[G];
#pragma unroll
        for (int k = 0; k < G; ++k)
            if (m0 + k < a.meqn) v[k] = a.q[(m0 + k) * a.L.plane + src];
#pragma unroll
        for (int k = 0; k < G; ++k) {
            const int m = m0 + k;
            if (m >= a.meqn) break;
            double x = v[k];
            if (a.negate && fx && m == 1) x = -x;
            if (a.negate && fy && m == 2) x = -x;
            a.q[m * a.L.plane + dst] = x;
        }
    }
}

// ---------------------------------------------------------------------------
// Layout conversion between the host's Fortran-ordered arrays (component
// fastest) and the device planes.  `ghost` = 2 when the host array is qbc
// (with ghost cells), 0 when it is State.q (interior only).
// ---------------------------------------------------------------------------
static __global__ void k_aos_to_planes(const double* __restrict__ src, double* __restrict__ dst, Layout L,
                                int meqn, int ghost) {
    const int nx = L.mx + 2 * ghost, ny = L.my + 2 * ghost;
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k % nx), j = (int)(k / nx);
        const long long d = (long long)(j + 2 - ghost) * L.pitch + (i + 2 - ghost);
        for (int m = 0; m < meqn; ++m) dst[m * L.plane + d] = src[k * meqn + m];
    }
}

static __global__ void k_planes_to_aos(const double* __restrict__ src, double* __restrict__ dst, Layout L,
                                int meqn, int ghost) {
    const int nx = L.mx + 2 * ghost, ny = L.my + 2 * ghost;
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k % nx), j = (int)(k / nx);
        const long long s = (long long)(j + 2 - ghost) * L.pitch + (i + 2 - ghost);
        for (int m = 0; m < meqn; ++m) dst[k * meqn + m] = src[m * L.plane + s];
    }
}

// q at n interior cells (i, j) (0-based, pairs in ij) into out[k * meqn + m]:
// the gauge values of solver.py:680-715 without moving the whole array.
static __global__ void k_gather_cells(const double* __restrict__ q, Layout L, int meqn, int n,
                                      const int* __restrict__ ij, double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * meqn) return;
    const int g = k / meqn, m = k - g * meqn;
    const int i = ij[2 * g], j = ij[2 * g + 1];
    out[k] = q[m * L.plane + (long long)(j + 2) * L.pitch + (i + 2)];
}

// Linear source step q <- q + (dt M) q_old in every interior cell, terms with
// M[m][k] = 0 skipped, each product and sum rounded on its own (no fused
// multiply-add), so the result is bit for bit the forward-Euler source step a
// host function computes as q + (M dt) q_k.
constexpr int SRC_MAX = CLAW2_MAX_WAVES;
struct LinearSourceArgs {
    double m[SRC_MAX * SRC_MAX];  // row-major, n x n
    int n;
    double dt;
};
static __global__ void k_linear_source(double* __restrict__ q, Layout L, const LinearSourceArgs a) {
    const long long ncell = (long long)L.mx * L.my;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < ncell;
         k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k % L.mx), j = (int)(k / L.mx);
        double* c = q + (long long)(j + 2) * L.pitch + (i + 2);
        double old[SRC_MAX];
        for (int m = 0; m < a.n; ++m) old[m] = c[m * L.plane];
        for (int m = 0; m < a.n; ++m) {
            double v = old[m];
            for (int kk = 0; kk < a.n; ++kk) {
                const double mk = a.m[m * a.n + kk];
                if (mk != 0.0) v = __dadd_rn(v, __dmul_rn(__dmul_rn(mk, a.dt), old[kk]));
            }
            c[m * L.plane] = v;
        }
    }
}

// Geometric source of the axisymmetric Euler equations (r = the radius plane)
// in every interior cell: two-stage Runge-Kutta,
//   q* = q - (dt/2) S(q) / r,  q <- q - dt S(q*) / r,
//   S = (rho v, rho u v, rho v^2, v (E + p)), p = (gamma-1)(E - rho |u|^2 / 2),
// components past the fourth unchanged; every operation rounded on its own,
// in the order of the host function it replaces, so the two agree bit for bit.
static __global__ void k_euler_axisym_source(double* __restrict__ q, const double* __restrict__ rad, Layout L,
                                             double gamma, double dt) {
    const long long ncell = (long long)L.mx * L.my;
    const double g1 = gamma - 1.0, dt2 = dt / 2.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < ncell;
         k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k % L.mx), j = (int)(k / L.mx);
        const long long o = (long long)(j + 2) * L.pitch + (i + 2);
        const double r = rad[o];
        const double q0 = q[o], q1 = q[L.plane + o], q2 = q[2 * L.plane + o], q3 = q[3 * L.plane + o];
        auto pressure = [&](double rho, double u, double v, double e) {
            const double ke = __dmul_rn(__dmul_rn(0.5, rho), __dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)));
            return __dmul_rn(g1, __dsub_rn(e, ke));
        };
        double rho = q0, u = __ddiv_rn(q1, rho), v = __ddiv_rn(q2, rho);
        double pr = pressure(rho, u, v, q3);
        const double h = __ddiv_rn(dt2, r);
        const double s0 = __dsub_rn(q0, __dmul_rn(h, q2));
        const double s1 = __dsub_rn(q1, __dmul_rn(__dmul_rn(__dmul_rn(h, rho), u), v));
        const double s2 = __dsub_rn(q2, __dmul_rn(__dmul_rn(__dmul_rn(h, rho), v), v));
        const double s3 = __dsub_rn(q3, __dmul_rn(__dmul_rn(h, v), __dadd_rn(q3, pr)));
        rho = s0;
        u = __ddiv_rn(s1, rho);
        v = __ddiv_rn(s2, rho);
        pr = pressure(rho, u, v, s3);
        const double f = __ddiv_rn(dt, r);
        q[o] = __dsub_rn(q0, __dmul_rn(f, s2));
        q[L.plane + o] = __dsub_rn(q1, __dmul_rn(__dmul_rn(__dmul_rn(f, rho), u), v));
        q[2 * L.plane + o] = __dsub_rn(q2, __dmul_rn(__dmul_rn(__dmul_rn(f, rho), v), v));
        q[3 * L.plane + o] = __dsub_rn(q3, __dmul_rn(__dmul_rn(f, v), __dadd_rn(s3, pr)));
    }
}

// Interior-only copy of qbc-layout planes (for the "ghosts unchanged" rule of
// claw2_step2: qnew starts as a copy of qold).
static __global__ void k_copy_planes(const double* __restrict__ src, double* __restrict__ dst, long long n) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        dst[k] = src[k];
}

// FP64 FMA throughput probe: 16 independent dependency chains per thread.
static __global__ void k_fp64_fma(double* out, int iters, double b) {
    double a[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = 1.0 + 1e-3 * (threadIdx.x + k);
    const double c = 1e-9 * blockIdx.x;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 16; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Self-test of rcp_nr: a = +-(1 + u) 2^e, e uniform in [-1000, 1000], u in
// [0, 1) from a counter hash of (seed, i); the largest distance in units in
// the last place between rcp_nr(a) and the IEEE quotient 1.0 / a.  The first
// threads also check the special values against the documented results
// (+-0 -> +-inf, +-inf -> +-0, NaN -> NaN, a subnormal -> +inf, 1e308 ->
// +0); a mismatch reports the largest distance there is.
static __global__ void k_selftest_rcp(int n, unsigned long long seed, unsigned long long* worst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 7) {
        const double inf = __longlong_as_double(0x7ff0000000000000ll);
        const double in[7] = {0.0, -0.0, inf, -inf, __longlong_as_double(0x7ff8000000000000ll), 1e-310, 1e308};
        const double want[7] = {inf, -inf, 0.0, -0.0, 0.0, inf, 0.0};
        const double r = rcp_nr(in[i]);
        const bool ok = (i == 4) ? (r != r) : (__double_as_longlong(r) == __double_as_longlong(want[i]));
        if (!ok) atomicMax(worst, ~0ull);
    }
    if (i >= n) return;
    unsigned long long z = seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1));
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    const int e = (int)((z & 2047ull) % 2001ull) - 1000;
    const double a = ((z >> 63) ? -1.0 : 1.0) * ldexp(1.0 + u, e);
    const double r = rcp_nr(a), q = 1.0 / a;
    const long long d = __double_as_longlong(r) - __double_as_longlong(q);
    atomicMax(worst, (unsigned long long)(d < 0 ? -d : d));
}

// Self-test of sqrt_nr: x = (1 + u) 2^e as above (positive), the largest
// distance in ulps from CUDA's IEEE sqrt(x); the first threads check +-0,
// +inf, -1, NaN and a subnormal against the documented results.
static __global__ void k_selftest_sqrt(int n, unsigned long long seed, unsigned long long* worst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 6) {
        const double inf = __longlong_as_double(0x7ff0000000000000ll);
        const double in[6] = {0.0, -0.0, inf, -1.0, __longlong_as_double(0x7ff8000000000000ll), 1e-310};
        const double r = sqrt_nr(in[i]);
        const bool ok = (i == 3 || i == 4) ? (r != r) : (__double_as_longlong(r) == __double_as_longlong(in[i]));
        if (!ok) atomicMax(worst, ~0ull);
    }
    if (i >= n) return;
    unsigned long long z = seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1));
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    const int e = (int)((z & 2047ull) % 2001ull) - 1000;
    const double x = ldexp(1.0 + u, e);
    const long long d = __double_as_longlong(sqrt_nr(x)) - __double_as_longlong(sqrt(x));
    atomicMax(worst, (unsigned long long)(d < 0 ? -d : d));
}

// Self-test of rsqrt_nr against the IEEE 1.0 / sqrt(x) (two roundings, so a
// distance of up to 2 ulps is expected), same arguments; the first threads
// check +-0, +inf, -1 and NaN against the documented results.
static __global__ void k_selftest_rsqrt(int n, unsigned long long seed, unsigned long long* worst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 5) {
        const double inf = __longlong_as_double(0x7ff0000000000000ll);
        const double in[5] = {0.0, -0.0, inf, -1.0, __longlong_as_double(0x7ff8000000000000ll)};
        const double want[5] = {inf, -inf, 0.0, 0.0, 0.0};
        const double r = rsqrt_nr(in[i]);
        const bool ok = (i >= 3) ? (r != r) : (__double_as_longlong(r) == __double_as_longlong(want[i]));
        if (!ok) atomicMax(worst, ~0ull);
    }
    if (i >= n) return;
    unsigned long long z = seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1));
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    const int e = (int)((z & 2047ull) % 2001ull) - 1000;
    const double x = ldexp(1.0 + u, e);
    const long long d = __double_as_longlong(rsqrt_nr(x)) - __double_as_longlong(1.0 / sqrt(x));
    atomicMax(worst, (unsigned long long)(d < 0 ? -d : d));
}

}  // namespace claw2
