// batch.cuh -- many independent problems of uneven size stepped together.
//
// Each instance is one ClawSolver2D problem (same Riemann solver and method,
// its own grid size, cell sizes, dt and time).  One step of the whole batch is
// three launches, all device-side so a multi-step loop can be captured in a
// CUDA graph with no host round trip:
//   k_batch_bc        ghost cells of every active instance (solver.py:351-519)
//   k_batch_step      a persistent kernel: the CTAs walk one flat work list of
//                     (instance, strip, row block) tiles -- largest instances
//                     first -- and run the unsplit tile of step_kernels.cuh on
//                     each; the CFL of a tile goes to its instance's word
//   k_batch_finalize  per instance, the reference's accept/reject and dt rule
//                     (solver.py:524-552, 619-651): accept swaps the q buffers,
//                     reject keeps them; dt <- min(dt_max, dt*cfl_desired/cfl),
//                     clipped to tend; an instance that reached tend is done
//                     and its tiles are skipped.  A step with a non-finite
//                     result is discarded and its instance retired (status
//                     bit 0), so one failing problem does not stop the rest.
#pragma once

#include "step_kernels.cuh"

namespace claw2 {

struct BatchInst {       // static per-instance data
    double* q[2];        // ping-pong planes
    Layout L;
    double dx, dy;
    int nstrips, H;      // tiling of this instance
};

struct BatchState {      // dynamic per-instance data
    double dt, t, cfl_last;
    unsigned long long cfl_bits;
    int cur, done, nsteps, nreject, status;
    int pad;
};

struct BatchCtl {
    double cfl_desired, cfl_max, dt_max, tend;
};

struct BatchArgs {
    const BatchInst* inst;
    BatchState* st;
    const int2* tiles;   // (instance, tile index within the instance)
    int ntiles, ninst;
    RPParams rp;
    Method meth;
    BatchCtl ctl;
};

// ghost cells: blockIdx.y = instance
static __global__ void k_batch_bc(const BatchArgs b, int first, int bcl0, int bcl1, int bcu0, int bcu1, int meqn) {
    const int i = first + blockIdx.y;
    BatchState& s = b.st[i];
    if (s.done) return;
    const BatchInst& in = b.inst[i];
    const int mx = in.L.mx, my = in.L.my;
    const int nrow = 4 * (mx + 4), ncol = 4 * my;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) s.cfl_bits = 0ull;
    if (k >= nrow + ncol) return;
    int c, r;
    if (k < nrow) {
        const int g = k / (mx + 4);
        c = k - g * (mx + 4);
        r = (g < 2) ? g : my + g;
    } else {
        const int kk = k - nrow;
        const int g = kk & 3;
        r = 2 + (kk >> 2);
        c = (g < 2) ? g : mx + g;
    }
    bool fx, fy;
    const int cs = bc_src(c, mx, bcl0, bcu0, fx);
    const int rs = bc_src(r, my, bcl1, bcu1, fy);
    double* q = in.q[s.cur];
    const long long src = (long long)rs * in.L.pitch + cs, dst = (long long)r * in.L.pitch + c;
    // loads of a group before its stores (see k_bc_fill)
    constexpr int G = 4;
    for (int m0 = 0; m0 < meqn; m0 += G) {
        double v[G];
#pragma unroll
        for (int k = 0; k < G; ++k)
            if (m0 + k < meqn) v[k] = q[(m0 + k) * in.L.plane + src];
#pragma unroll
        for (int k = 0; k < G; ++k) {
            const int m = m0 + k;
            if (m >= meqn) break;
            double x = v[k];
            if (fx && m == 1) x = -x;
            if (fy && m == 2) x = -x;
            q[m * in.L.plane + dst] = x;
        }
    }
}

template <class RP, int NT, int MINB, int SPEC>
__global__ void __launch_bounds__(NT, MINB) k_batch_step(const BatchArgs b, int first, int count) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    UnsplitSmem<RP, NT>& S = *reinterpret_cast<UnsplitSmem<RP, NT>*>(smem_raw);
    const int end = min(first + count, b.ntiles);
    for (int w = first + blockIdx.x; w < end; w += gridDim.x) {
        const int2 tl = b.tiles[w];
        const BatchInst& in = b.inst[tl.x];
        BatchState& s = b.st[tl.x];
        if (s.done) continue;  // uniform across the CTA
        StepArgs a;
        a.qold = in.q[s.cur];
        a.qnew = in.q[s.cur ^ 1];
        a.L = in.L;
        a.dtdx = s.dt / in.dx;
        a.dtdy = s.dt / in.dy;
        a.H = in.H;
        a.rp = b.rp;
        a.meth = b.meth;
        a.cfl_bits = &s.cfl_bits;
        a.status = &s.status;
        a.guess = nullptr;
        a.counters = nullptr;
        const int strip = tl.y % in.nstrips, rblk = tl.y / in.nstrips;
        double cfl = 0.0;
        unsplit_tile<RP, NT, SPEC>(a, strip, rblk * in.H, S, cfl);
        cfl_commit(cfl, S.red, a.cfl_bits);
    }
}

// one thread per instance (solver.py:524-552, 604-651)
static __global__ void k_batch_finalize(const BatchArgs b, int first, int count) {
    const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= first + count || i >= b.ninst) return;
    BatchState& s = b.st[i];
    if (s.done) return;
    if (s.status & 1) {  // non-finite result: keep the last good state, retire the problem
        s.done = 1;
        return;
    }
    const double cfl = __longlong_as_double((long long)s.cfl_bits);
    s.cfl_last = cfl;
    if (cfl <= b.ctl.cfl_max) {
        s.cur ^= 1;
        s.t += s.dt;
        s.nsteps += 1;
    } else {
        s.nreject += 1;
    }
    double dt = (cfl > 0.0) ? fmin(b.ctl.dt_max, s.dt * b.ctl.cfl_desired / cfl) : b.ctl.dt_max;
    if (s.t + dt > b.ctl.tend) dt = b.ctl.tend - s.t;
    if (b.ctl.tend - s.t - dt < 1.e-14 * s.t) dt = b.ctl.tend - s.t;
    s.dt = dt;
    if (s.t >= b.ctl.tend) s.done = 1;
}

}  // namespace claw2
