// claw2_noalloc.cu -- the dimensionally split step for callers that cannot
// allocate device memory.
//
// Some callers own every byte of device memory themselves: a host framework
// that reserves the GPU's memory up front in its own pool (a cudaMalloc from a
// library would fail or fragment that pool), or a time-critical loop that
// cannot afford the implicit device synchronisation of cudaMalloc/cudaFree.
// The split step needs scratch memory (the state after the x-sweep, which the
// y-sweep reads, plus the Courant-number and status words), which every other
// entry point of this library allocates.  claw2_step2ds_noalloc instead keeps
// that scratch in one file-scope device array of fixed size, which the driver
// creates when the library is loaded onto a device and which stays there
// until the process exits.
//
// Rules that follow from sharing one array:
//   * the problem must fit: num_eqn * plane doubles of intermediate state (see
//     CLAW2_NOALLOC_SCRATCH_BYTES); larger problems are rejected with
//     CLAW2_EINVAL before any GPU work;
//   * every call reuses the array and finds the previous call's contents in
//     it; the words that must start at zero are cleared by each call, and the
//     intermediate state is fully written by the x-sweep before it is read;
//   * calls whose GPU work overlaps (on different streams, or from several
//     threads) race on the array: serialise them;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture;
//   * each call waits for its stream to finish the step (it copies the
//     Courant number back to the host before it returns).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "step_kernels.cuh"

using namespace claw2;

extern "C" void claw2_internal_set_error(const char* msg);  // claw2.cu, not exported
// claw2.cu, not exported: claw2_step2ds's two sweeps on the given buffers
int claw2_internal_launch_split(int rp, const StepArgs& ax, const StepArgs& ay, cudaStream_t st);

namespace {

// [0] CFL bit pattern, [1] status word, intermediate state from kHeader on.
constexpr long long kScratchDoubles = CLAW2_NOALLOC_SCRATCH_BYTES / 8;
constexpr long long kHeader = 32;  // 256 bytes, so the planes stay 256-byte aligned
constexpr int kMaxSide = 1 << 28;  // mx, my bound (the scratch limit is far below it anyway)
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_scratch_ptr[64] = {nullptr};

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    claw2_internal_set_error(buf);  // reported by claw2_last_error()
    return code;
}

// Device address of the scratch array on the current device (looked up once
// per device; the host-side name is only a stand-in for it).
int scratch_on_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(CLAW2_ECUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail(CLAW2_EUNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fail(CLAW2_ECUDA, "cudaGetSymbolAddress of the scratch array failed: %s", cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return CLAW2_OK;
}

}  // namespace

extern "C" {

int claw2_step2ds_noalloc(const claw2_desc* d, const double* qold, double* qnew, long long pitch,
                          long long plane, double dt, double* cfl, void* stream) {
    if (!d || !qold || !qnew || !cfl) return fail(CLAW2_EINVAL, "null pointer argument");
    int meqn = 0, mwaves = 0;
    switch (d->riemann) {
        case CLAW2_RP_ADVECTION: meqn = 1; mwaves = 1; break;
        case CLAW2_RP_ACOUSTICS: meqn = 3; mwaves = 2; break;
        case CLAW2_RP_EULER_ROE: meqn = 4; mwaves = 4; break;
        case CLAW2_RP_SHALLOW_ROE: meqn = 3; mwaves = 3; break;
        default: return fail(CLAW2_EINVAL, "unknown Riemann solver id %d", d->riemann);
    }
    if (d->num_eqn != meqn || d->num_waves != mwaves)
        return fail(CLAW2_EINVAL, "solver %d has num_eqn=%d num_waves=%d (got %d, %d)", d->riemann, meqn,
                    mwaves, d->num_eqn, d->num_waves);
    if (d->num_ghost != 2 || d->num_aux != 0 || d->mcapa != 0 || d->fwave)
        return fail(CLAW2_EUNSUPPORTED, "num_ghost must be 2, without aux arrays, capacity or f-waves");
    // bounded first, so that mx + 4, my + 4 and the products below cannot overflow
    if (d->mx < 1 || d->my < 1 || d->mx > kMaxSide || d->my > kMaxSide)
        return fail(CLAW2_EINVAL, "bad sizes mx=%d my=%d (1..%d each)", d->mx, d->my, kMaxSide);
    if (d->order != 1 && d->order != 2) return fail(CLAW2_EINVAL, "order must be 1 or 2");
    if (!(d->dx > 0.0) || !(d->dy > 0.0) || !(dt >= 0.0)) return fail(CLAW2_EINVAL, "dx, dy > 0 and dt >= 0 required");
    for (int k = 0; k < mwaves; ++k)
        if (d->mthlim[k] < 0 || d->mthlim[k] > 5) return fail(CLAW2_EINVAL, "limiter %d out of range", d->mthlim[k]);
    if (pitch < d->mx + 4 || pitch > (1ll << 30) || plane < pitch * (long long)(d->my + 4))
        return fail(CLAW2_EINVAL, "layout too small: pitch=%lld plane=%lld for %dx%d cells", pitch, plane, d->mx,
                    d->my);
    if (((uintptr_t)qold | (uintptr_t)qnew) & 7) return fail(CLAW2_EINVAL, "q planes must be 8-byte aligned");
    // plane is compared before it is multiplied: meqn * plane cannot overflow
    if (plane > (kScratchDoubles - kHeader) / meqn)
        return fail(CLAW2_EINVAL,
                    "problem too large for the fixed scratch array: needs %lld planes of %lld doubles, the maximum "
                    "is %lld bytes (CLAW2_NOALLOC_SCRATCH_BYTES) including a %lld-byte header; use claw2_patch_* "
                    "for larger grids",
                    (long long)meqn, plane, kScratchDoubles * 8, kHeader * 8);

    double* scr = nullptr;
    int rc = scratch_on_device(&scr);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long* cfl_bits = reinterpret_cast<unsigned long long*>(scr);
    int* status = reinterpret_cast<int*>(scr + 1);
    double* qtmp = scr + kHeader;

    // the CFL word (atomicMax) and the status word (atomicOr) must start at zero
    cudaError_t e = cudaMemsetAsync(scr, 0, 2 * sizeof(double), st);
    if (e != cudaSuccess) return fail(CLAW2_ECUDA, "clearing the scratch words failed: %s", cudaGetErrorString(e));

    StepArgs a;
    a.L.mx = d->mx;
    a.L.my = d->my;
    a.L.pitch = (int)pitch;
    a.L.plane = plane;
    a.dtdx = dt / d->dx;
    a.dtdy = dt / d->dy;
    a.H = 0;
    for (int k = 0; k < CLAW2_MAX_PARAMS; ++k) a.rp.c[k] = k < d->ncparam ? d->cparam[k] : 0.0;
    a.rp.flags = (d->riemann == CLAW2_RP_EULER_ROE || d->riemann == CLAW2_RP_SHALLOW_ROE) && a.rp.c[1] != 0.0;
    a.meth.order = d->order;
    a.meth.transverse = -1;
    a.meth.fwave = 0;
    for (int k = 0; k < CLAW2_MAX_WAVES; ++k) a.meth.mthlim[k] = k < mwaves ? d->mthlim[k] : 0;
    a.cfl_bits = cfl_bits;
    a.status = status;
    a.guess = nullptr;
    a.counters = nullptr;
    StepArgs ax = a, ay = a;
    ax.qold = qold;
    ax.qnew = qtmp;  // x-sweep: every row of the interior columns, ghost columns copied
    ay.qold = qtmp;
    ay.qnew = qnew;  // y-sweep: interior cells

    if (claw2_internal_launch_split(d->riemann, ax, ay, st) != 0)
        return fail(CLAW2_EINVAL, "unknown Riemann solver id %d", d->riemann);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CLAW2_ECUDA, "launch failed: %s", cudaGetErrorString(e));
    unsigned long long bits = 0;
    int stat = 0;
    e = cudaMemcpyAsync(&bits, cfl_bits, sizeof bits, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&stat, status, sizeof stat, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(CLAW2_ECUDA, "split step failed: %s", cudaGetErrorString(e));
    std::memcpy(cfl, &bits, sizeof(double));
    if (stat & 1) return fail(CLAW2_ENONFINITE, "the step produced a non-finite value");
    return CLAW2_OK;
}

}  // extern "C"
