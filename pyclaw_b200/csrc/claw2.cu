// claw2.cu -- C ABI of the classic 2D step (declarations: include/claw2.h).
//
// Host side of the drop-in: argument checks with the reference's error
// behaviour mapped to status codes, the device-resident patch (two q buffers,
// CFL and status words, one stream), and the stateless replacements of the
// f2py step2/step2ds routines.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "batch.cuh"
#include "mlp.cuh"
#include "step_kernels.cuh"

#include <vector>
#include <numeric>

using namespace claw2;

// frame_io.cpp: the ascii frame writer
__attribute__((visibility("hidden"))) int claw2_internal_write_ascii(const char* path, int append,
                                                                     const char* header, const double* q,
                                                                     int nvar, int mx, int my, int nthreads);

namespace {

thread_local std::string g_err = "no error";

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(CLAW2_ECUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));      \
    } while (0)

constexpr int NT_UNSPLIT = 128;  // threads per strip (124 output columns)
constexpr int NT_SPLIT_X = 128;
constexpr int NT_SPLIT_Y = 128;

int rp_shape(int rp, int* meqn, int* mwaves) {
    switch (rp) {
        case CLAW2_RP_ADVECTION: *meqn = 1; *mwaves = 1; return 0;
        case CLAW2_RP_ACOUSTICS: *meqn = 3; *mwaves = 2; return 0;
        case CLAW2_RP_EULER_ROE: *meqn = 4; *mwaves = 4; return 0;
        case CLAW2_RP_SHALLOW_ROE: *meqn = 3; *mwaves = 3; return 0;
        case CLAW2_RP_EULER_EXACT: *meqn = 4; *mwaves = 3; return 0;
        case CLAW2_RP_VC_ACOUSTICS: *meqn = 3; *mwaves = 2; return 0;
        case CLAW2_RP_VC_ADVECTION: *meqn = 1; *mwaves = 1; return 0;
        case CLAW2_RP_PSYSTEM: *meqn = 3; *mwaves = 2; return 0;
        case CLAW2_RP_VC_ADVECTION_VEC: *meqn = 2; *mwaves = 1; return 0;
        case CLAW2_RP_EULER_5WAVE: *meqn = 5; *mwaves = 5; return 0;
        case CLAW2_RP_SHALLOW_HLLE: *meqn = 3; *mwaves = 2; return 0;
        default: return -1;
    }
}

// aux components a solver reads per cell (the leading ones of the aux array)
int rp_maux(int rp) {
    if (rp == CLAW2_RP_PSYSTEM) return 4;
    return (rp == CLAW2_RP_VC_ACOUSTICS || rp == CLAW2_RP_VC_ADVECTION || rp == CLAW2_RP_VC_ADVECTION_VEC) ? 2 : 0;
}

RPParams make_params(int rp, const double* cparam, int n) {
    RPParams p;
    for (int k = 0; k < CLAW2_MAX_PARAMS; ++k) p.c[k] = (cparam && k < n) ? cparam[k] : 0.0;
    p.flags = 0;
    if (rp == CLAW2_RP_EULER_ROE || rp == CLAW2_RP_SHALLOW_ROE || rp == CLAW2_RP_EULER_5WAVE)
        p.flags = (p.c[1] != 0.0) ? 1 : 0;
    return p;
}

Layout make_layout(int mx, int my) {
    Layout L;
    L.mx = mx;
    L.my = my;
    L.pitch = ((mx + 4 + 31) / 32) * 32;
    L.plane = (long long)L.pitch * (my + 4);
    L.plane = ((L.plane + 31) / 32) * 32;  // 256-byte aligned planes
    return L;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links only the CUDA runtime); nullptr when unavailable.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::mutex mu;
    static bool tried = false;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!tried) {
        tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
        else
            cudaGetLastError();
    }
    return fn;
}

// TMA descriptor of one q buffer for the row staging of the unsplit kernel:
// 3D (columns mx+4, rows my+4, components) with the padded layout's strides,
// box = one row of one strip (NT columns) over all components; columns past
// mx+3 read as zeros.  The kernel's box x coordinates are strip*(NT-4), so
// x * 8 bytes is a multiple of 16 as a tiled copy requires.
template <int NT>
bool make_row_tmap(CUtensorMap* tm, double* q, const Layout& L, int meqn) {
    static_assert(((NT - 4) * 8) % 16 == 0, "strip starts must be 16-byte aligned");
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || ((unsigned long long)q & 15ull)) return false;
    cuuint64_t dims[3] = {(cuuint64_t)(L.mx + 4), (cuuint64_t)(L.my + 4), (cuuint64_t)meqn};
    cuuint64_t strides[2] = {(cuuint64_t)L.pitch * 8, (cuuint64_t)L.plane * 8};
    cuuint32_t box[3] = {(cuuint32_t)NT, 1, (cuuint32_t)meqn};
    cuuint32_t estr[3] = {1, 1, 1};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, q, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// SM count of the current device (queried once per device; 148 on a B200).
int device_sms() {
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n <= 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

int pick_rows(int nstrips, int nrows, int nsm) {
    // about three CTAs per SM, 2..64 rows per CTA: a small grid gets short
    // row blocks, since its time is one tile's march down its rows (measured
    // at 100^2-300^2: 2-3 rows 1.5-1.8x faster than 8)
    const int want_blocks = std::max(1, (3 * nsm + nstrips - 1) / nstrips);
    int H = (nrows + want_blocks - 1) / want_blocks;
    return std::max(2, std::min(64, H));
}

// ---- launches, one instantiation per Riemann solver -----------------------
// Opt a kernel into more than 48 KB of dynamic shared memory, once per device.
template <class K>
void smem_attr(K kernel, int bytes, unsigned long long& done) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(done & (1ull << dev))) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        done |= 1ull << dev;
    }
}

// Launch shapes of the unsplit kernel.  A variant fixes the register budget
// (blocks per SM the kernel is compiled for); `rows` is the row-block height
// (0 = heuristic).  Chosen per call by the tuning table (claw2_tune_set /
// claw2_autotune) or the heuristic default.
struct UnsplitShape {
    int variant;  // bit 0: 3 blocks/SM (register cap) instead of 2; bit 1: TMA row staging;
                  // 4: the two-barrier tile (deferred x finish); 8: the direction-split
                  // tile (two threads per column)
    int rows;
};

constexpr int TUNE_SLOTS = 16;  // indexed by Riemann solver id
UnsplitShape g_tune[TUNE_SLOTS] = {};
std::atomic<unsigned> g_tune_gen{0};  // bumped by every claw2_tune_set (cached graphs go stale)

// true for the method the SPEC_MC2 kernels are compiled for
bool is_mc2(const Method& m, int mwaves) {
    if (m.order != 2 || m.transverse != 2 || m.fwave != 0) return false;
    for (int k = 0; k < mwaves; ++k)
        if (m.mthlim[k] != 4) return false;
    return true;
}

// tm: the tensor map of qold for the TMA-staged kernel, or nullptr
template <class RP, int MB, int SPEC, bool EVO>
void launch_unsplit_s(const StepArgs& b, dim3 grid, cudaStream_t st, const CUtensorMap* tm) {
    if (!EVO && tm) {
        constexpr int smem = (int)sizeof(UnsplitSmemTma<RP, NT_UNSPLIT>);
        static unsigned long long attr = 0;
        smem_attr(k_step_unsplit_tma<RP, NT_UNSPLIT, MB, SPEC>, smem, attr);
        k_step_unsplit_tma<RP, NT_UNSPLIT, MB, SPEC><<<grid, NT_UNSPLIT, smem, st>>>(b, *tm);
        return;
    }
    constexpr int smem = (int)sizeof(UnsplitSmem<RP, NT_UNSPLIT>);
    static unsigned long long attr = 0;
    smem_attr(k_step_unsplit<RP, NT_UNSPLIT, MB, SPEC, false, EVO>, smem, attr);
    k_step_unsplit<RP, NT_UNSPLIT, MB, SPEC, false, EVO><<<grid, NT_UNSPLIT, smem, st>>>(b);
}

// Tiling of the unsplit kernel: strips of NT_UNSPLIT - 4 output columns,
// row blocks of H rows (the tuned height, else the heuristic).
void unsplit_tiling(int riemann, int mx, int my, int& nstrips, int& H, int& nblocks) {
    constexpr int W = NT_UNSPLIT - 4;
    nstrips = (mx + W - 1) / W;
    const int rows = g_tune[riemann & (TUNE_SLOTS - 1)].rows;
    H = rows > 0 ? rows : pick_rows(nstrips, my, device_sms());
    nblocks = (my + H - 1) / H;
}

// The two-barrier tile (deferred x finish), any method, with or without capacity.
template <class RP, int SPEC, bool CAPA, bool EVO>
void launch_unsplit2_s(const StepArgs& b, dim3 grid, cudaStream_t st) {
    constexpr int smem = (int)sizeof(UnsplitSmem2<RP, NT_UNSPLIT, CAPA>);
    static unsigned long long attr = 0;
    smem_attr(k_step_unsplit2<RP, NT_UNSPLIT, 2, SPEC, CAPA, EVO>, smem, attr);
    k_step_unsplit2<RP, NT_UNSPLIT, 2, SPEC, CAPA, EVO><<<grid, NT_UNSPLIT, smem, st>>>(b);
}

// The direction-split tile (two threads per column, 2 CTAs of 256 threads
// per SM).  For the Euler solvers the Y warps take 136 registers and the X
// warps 120 (setmaxnreg), which needs exactly 128 registers per thread at
// launch: checked once per kernel, and a kernel built otherwise is not
// launched (the caller falls back to the one-thread tile).
template <class RP> struct WSRegs { static constexpr int Y = 0, X = 0; };
template <> struct WSRegs<RPEulerRoe> { static constexpr int Y = 136, X = 120; };
static_assert(WSRegs<RPEulerRoe>::Y * NT_UNSPLIT + WSRegs<RPEulerRoe>::X * NT_UNSPLIT == 2 * NT_UNSPLIT * 128,
              "the warpgroups' register shares must add up to the launch's 128 per thread");

template <class RP, int SPEC, bool EVO>
bool launch_unsplit_ws_s(const StepArgs& b, dim3 grid, cudaStream_t st) {
    constexpr int smem = (int)sizeof(UnsplitSmemWS<RP, NT_UNSPLIT>);
    constexpr int RY = WSRegs<RP>::Y, RX = WSRegs<RP>::X;
    auto kern = k_step_unsplit_ws<RP, NT_UNSPLIT, 2, SPEC, EVO, RY, RX>;
    if (RY > 0) {
        static int regs = -1;
        if (regs < 0) {
            cudaFuncAttributes fa;
            regs = (cudaFuncGetAttributes(&fa, kern) == cudaSuccess) ? fa.numRegs : 0;
        }
        if (regs != 128) return false;
    }
    static unsigned long long attr = 0;
    smem_attr(kern, smem, attr);
    kern<<<grid, 2 * NT_UNSPLIT, smem, st>>>(b);
    return true;
}

// The capacity form (any method, rows loaded directly).
template <class RP, bool EVO>
void launch_unsplit_capa(const StepArgs& b, dim3 grid, cudaStream_t st) {
    constexpr int smem = (int)sizeof(UnsplitSmem<RP, NT_UNSPLIT, true>);
    static unsigned long long attr = 0;
    smem_attr(k_step_unsplit<RP, NT_UNSPLIT, 2, SPEC_ANY, true, EVO>, smem, attr);
    k_step_unsplit<RP, NT_UNSPLIT, 2, SPEC_ANY, true, EVO><<<grid, NT_UNSPLIT, smem, st>>>(b);
}

// EVO: a launch of the device time loop (dt read from a.evo; rows loaded
// directly, never by TMA).
template <class RP, int MB, bool EVO>
void launch_unsplit_v(const StepArgs& a, cudaStream_t st, const CUtensorMap* tm) {
    StepArgs b = a;
    int ns, H, nb;
    unsplit_tiling(RP::ID, a.L.mx, a.L.my, ns, H, nb);
    if (b.tile_order == nullptr) {  // a caller with a schedule has fixed H and nstrips already
        b.H = H;
        b.nstrips = ns;
    }
    const int nbk = (a.L.my + b.H - 1) / b.H;
    dim3 grid(b.tile_count > 0 ? b.tile_count : b.nstrips * nbk);
    if constexpr (AuxTraits<RP>::MAUX == 0 && !GuessTraits<RP>::USES) {
        if ((g_tune[RP::ID & (TUNE_SLOTS - 1)].variant & 8) && !a.capa) {  // the direction-split tile
            const bool ok = is_mc2(a.meth, RP::MWAVES) ? launch_unsplit_ws_s<RP, SPEC_MC2, EVO>(b, grid, st)
                                                       : launch_unsplit_ws_s<RP, SPEC_ANY, EVO>(b, grid, st);
            if (ok) return;
        }
    }
    if (g_tune[RP::ID & (TUNE_SLOTS - 1)].variant & 4) {  // the two-barrier tile
        if (a.capa) launch_unsplit2_s<RP, SPEC_ANY, true, EVO>(b, grid, st);
        else if (is_mc2(a.meth, RP::MWAVES)) launch_unsplit2_s<RP, SPEC_MC2, false, EVO>(b, grid, st);
        else launch_unsplit2_s<RP, SPEC_ANY, false, EVO>(b, grid, st);
        return;
    }
    if (a.capa) launch_unsplit_capa<RP, EVO>(b, grid, st);
    else if (is_mc2(a.meth, RP::MWAVES)) launch_unsplit_s<RP, MB, SPEC_MC2, EVO>(b, grid, st, tm);
    else launch_unsplit_s<RP, MB, SPEC_ANY, EVO>(b, grid, st, tm);
}

// Variants: 4 = the two-barrier tile (k_step_unsplit2); otherwise bit 0 = 3
// blocks per SM (register cap) instead of 2, bit 1 = rows
// staged by TMA (only where the caller has a tensor map of qold).
template <class RP>
void launch_unsplit(const StepArgs& a, cudaStream_t st, const CUtensorMap* tm) {
    const UnsplitShape sh = g_tune[RP::ID & (TUNE_SLOTS - 1)];
    if (a.evo) {
        if (sh.variant & 1) launch_unsplit_v<RP, 3, true>(a, st, nullptr);
        else launch_unsplit_v<RP, 2, true>(a, st, nullptr);
        return;
    }
    const CUtensorMap* use = (sh.variant & 2) ? tm : nullptr;
    if (sh.variant & 1) launch_unsplit_v<RP, 3, false>(a, st, use);
    else launch_unsplit_v<RP, 2, false>(a, st, use);
}

// the split sweeps' specialisation: order 2 with one limiter on every family
int split_spec(const Method& m, int mwaves) {
    if (m.order != 2 || m.fwave != 0) return SPEC_ANY;
    for (int k = 1; k < mwaves; ++k)
        if (m.mthlim[k] != m.mthlim[0]) return SPEC_ANY;
    return m.mthlim[0] == 4 ? SPEC_MC2 : m.mthlim[0] == 1 ? SPEC_MM2 : SPEC_ANY;
}

template <class RP, int SPEC, bool EVO>
void launch_split_s(const StepArgs& ax, const StepArgs& ay, cudaStream_t st, int which) {
    if (which & 1) {
        constexpr int W = NT_SPLIT_X - 4;
        const int ns = (ax.L.mx + W - 1) / W;
        StepArgs b = ax;
        b.H = pick_rows(ns, ax.L.my + 4, device_sms());
        dim3 grid(ns, (ax.L.my + 4 + b.H - 1) / b.H);
        constexpr int smem = (int)sizeof(SplitXSmem<RP, NT_SPLIT_X>);
        static unsigned long long attr = 0;
        smem_attr(k_split_x<RP, NT_SPLIT_X, SPEC, EVO>, smem, attr);
        k_split_x<RP, NT_SPLIT_X, SPEC, EVO><<<grid, NT_SPLIT_X, smem, st>>>(b);
    }
    if (which & 2) {
        const int ns = (ay.L.mx + 4 + NT_SPLIT_Y - 1) / NT_SPLIT_Y;
        StepArgs b = ay;
        b.H = pick_rows(ns, ay.L.my, device_sms());
        dim3 grid(ns, (ay.L.my + b.H - 1) / b.H);
        k_split_y<RP, NT_SPLIT_Y, SPEC, EVO><<<grid, NT_SPLIT_Y, 0, st>>>(b);
    }
}

template <class RP, bool EVO>
void launch_split_e(const StepArgs& ax, const StepArgs& ay, cudaStream_t st, int which) {
    switch (split_spec(ax.meth, RP::MWAVES)) {
        case SPEC_MC2: launch_split_s<RP, SPEC_MC2, EVO>(ax, ay, st, which); break;
        case SPEC_MM2: launch_split_s<RP, SPEC_MM2, EVO>(ax, ay, st, which); break;
        default: launch_split_s<RP, SPEC_ANY, EVO>(ax, ay, st, which); break;
    }
}

// (a.evo: the device time loop's launch, dt read from its record)
template <class RP>
void launch_split(const StepArgs& ax, const StepArgs& ay, cudaStream_t st, int which) {
    if (ax.evo) launch_split_e<RP, true>(ax, ay, st, which);
    else launch_split_e<RP, false>(ax, ay, st, which);
}

template <template <class> class F, class... A>
int dispatch(int rp, A&&... args) {
    switch (rp) {
        case CLAW2_RP_ADVECTION: F<RPAdvection>::run(args...); return 0;
        case CLAW2_RP_ACOUSTICS: F<RPAcoustics>::run(args...); return 0;
        case CLAW2_RP_EULER_ROE: F<RPEulerRoe>::run(args...); return 0;
        case CLAW2_RP_SHALLOW_ROE: F<RPShallowRoe>::run(args...); return 0;
        case CLAW2_RP_EULER_EXACT: F<RPEulerExact>::run(args...); return 0;
        case CLAW2_RP_VC_ACOUSTICS: F<RPVcAcoustics>::run(args...); return 0;
        case CLAW2_RP_VC_ADVECTION: F<RPVcAdvection>::run(args...); return 0;
        case CLAW2_RP_PSYSTEM: F<RPPsystem>::run(args...); return 0;
        case CLAW2_RP_VC_ADVECTION_VEC: F<RPVcAdvectionVec>::run(args...); return 0;
        case CLAW2_RP_EULER_5WAVE: F<RPEuler5>::run(args...); return 0;
        case CLAW2_RP_SHALLOW_HLLE: F<RPShallowHLLE>::run(args...); return 0;
        default: return -1;
    }
}
template <class RP>
struct UnsplitF {
    static void run(const StepArgs& a, cudaStream_t st, const CUtensorMap* tm = nullptr) {
        launch_unsplit<RP>(a, st, tm);
    }
};
template <class RP>
struct SplitF {
    static void run(const StepArgs& ax, const StepArgs& ay, cudaStream_t st, int which) {
        launch_split<RP>(ax, ay, st, which);
    }
};

void launch_bc(double* q, const Layout& L, int meqn, const int* bcl, const int* bcu,
               unsigned long long* cfl_bits, cudaStream_t st, int negate = 1, int part = 0) {
    BCArgs b;
    b.negate = negate;
    b.part = part;
    b.q = q;
    b.L = L;
    b.meqn = meqn;
    b.bcl[0] = bcl[0]; b.bcl[1] = bcl[1];
    b.bcu[0] = bcu[0]; b.bcu[1] = bcu[1];
    b.cfl_bits = cfl_bits;
    const int n = 4 * (L.mx + 4) + 4 * L.my;
    k_bc_fill<<<(n + 255) / 256, 256, 0, st>>>(b);
}

int check_method(int rp, int order, int trans, const int* mthlim, int mwaves, int fwave) {
    if (order != 1 && order != 2) return fail(CLAW2_EINVAL, "order must be 1 or 2 (got %d)", order);
    if (trans < -1 || trans > 2) return fail(CLAW2_EINVAL, "transverse must be -1..2 (got %d)", trans);
    if ((rp == CLAW2_RP_VC_ADVECTION_VEC || rp == CLAW2_RP_SHALLOW_HLLE) && trans > 0)
        return fail(CLAW2_EINVAL, "solver %d has no transverse solve: use the split step or transverse 0", rp);
    if (fwave != 0 && fwave != 1) return fail(CLAW2_EINVAL, "use_fwave must be 0 or 1 (got %d)", fwave);
    for (int k = 0; k < mwaves; ++k)
        if (mthlim[k] < 0 || mthlim[k] > 5) return fail(CLAW2_EINVAL, "limiter %d out of range", mthlim[k]);
    return CLAW2_OK;
}

int check_bc(const int* bcl, const int* bcu, int mx, int my) {
    for (int d = 0; d < 2; ++d) {
        const int n = d == 0 ? mx : my;
        // a wall or periodic ghost cell copies one of the first/last two
        // interior cells; with one cell that source would itself be a ghost
        const bool lo_ok = bcl[d] == CLAW2_BC_EXTRAP || bcl[d] == CLAW2_BC_NONE;
        const bool up_ok = bcu[d] == CLAW2_BC_EXTRAP || bcu[d] == CLAW2_BC_NONE;
        if (n < 2 && !(lo_ok && up_ok))
            return fail(CLAW2_EINVAL, "wall/periodic BCs need at least 2 cells in dimension %d", d);
        for (int v : {bcl[d], bcu[d]}) {
            if (v == CLAW2_BC_CUSTOM)
                return fail(CLAW2_EUNSUPPORTED, "custom BCs are applied by the host (dimension %d)", d);
            if (v == CLAW2_BC_NONE && d == 0)
                return fail(CLAW2_EINVAL, "caller-filled ghost cells are supported in dimension 1 only");
            if (v != CLAW2_BC_NONE && (v < 1 || v > 3))
                return fail(CLAW2_EINVAL, "boundary condition %d not implemented", v);
        }
        if ((bcl[d] == CLAW2_BC_PERIODIC) != (bcu[d] == CLAW2_BC_PERIODIC))
            return fail(CLAW2_EINVAL, "periodic BC must be set on both sides of dimension %d", d);
    }
    return CLAW2_OK;
}

// Scratch used by the stateless entry points (grown on demand, reused).
struct Scratch {
    std::mutex mu;
    int device = -1;
    size_t cap = 0;  // doubles per buffer
    double *a = nullptr, *b = nullptr, *c = nullptr, *stage = nullptr;
    size_t stage_cap = 0;
    unsigned long long* cfl = nullptr;
    int* status = nullptr;
    double* aux = nullptr;  // aux planes of the stateless step
    size_t aux_cap = 0;
    cudaStream_t st = nullptr;
};
Scratch g_scr;

int scratch_reserve(size_t n, size_t nstage) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (g_scr.device != dev) {
        g_scr.cap = g_scr.stage_cap = 0;
        g_scr.a = g_scr.b = g_scr.c = g_scr.stage = nullptr;
        g_scr.cfl = nullptr;
        g_scr.status = nullptr;
        g_scr.aux = nullptr;
        g_scr.aux_cap = 0;
        g_scr.st = nullptr;
        g_scr.device = dev;
    }
    if (!g_scr.st) CUDA_TRY(cudaStreamCreateWithFlags(&g_scr.st, cudaStreamNonBlocking));
    if (!g_scr.cfl) {
        CUDA_TRY(cudaMalloc(&g_scr.cfl, sizeof(unsigned long long)));
        CUDA_TRY(cudaMalloc(&g_scr.status, sizeof(int)));
    }
    if (n > g_scr.cap) {
        cudaFree(g_scr.a); cudaFree(g_scr.b); cudaFree(g_scr.c);
        g_scr.a = g_scr.b = g_scr.c = nullptr;
        g_scr.cap = 0;
        if (cudaMalloc(&g_scr.a, n * 8) != cudaSuccess || cudaMalloc(&g_scr.b, n * 8) != cudaSuccess ||
            cudaMalloc(&g_scr.c, n * 8) != cudaSuccess)
            return fail(CLAW2_ENOMEM, "device allocation of %zu doubles failed", n);
        g_scr.cap = n;
    }
    if (nstage > g_scr.stage_cap) {
        cudaFree(g_scr.stage);
        g_scr.stage = nullptr;
        g_scr.stage_cap = 0;
        if (cudaMalloc(&g_scr.stage, nstage * 8) != cudaSuccess)
            return fail(CLAW2_ENOMEM, "device allocation of %zu doubles failed", nstage);
        g_scr.stage_cap = nstage;
    }
    return CLAW2_OK;
}

int grid_blocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 16LL * device_sms()); }

// Shared body of claw2_step2 / claw2_step2ds: host qbc -> device planes ->
// kernels -> host qbc (interior cells).
int host_step(int maxm, int meqn, int mwaves, int maux, int mbc, int mx, int my, const double* qold,
              double* qnew, const double* aux, double dx, double dy, double dt, const int* method,
              const int* mthlim, double* cfl, int ids, int use_fwave, int rp, const double* cparam, int ncparam) {
    if (!qold || !qnew || !method || !mthlim || !cfl) return fail(CLAW2_EINVAL, "null pointer argument");
    int me = 0, mw = 0;
    if (rp_shape(rp, &me, &mw) != 0) return fail(CLAW2_EINVAL, "unknown Riemann solver id %d", rp);
    if (me != meqn || mw != mwaves)
        return fail(CLAW2_EINVAL, "solver %d has num_eqn=%d num_waves=%d (got %d, %d)", rp, me, mw, meqn, mwaves);
    if (mbc != 2) return fail(CLAW2_EINVAL, "num_ghost must be 2 (got %d)", mbc);
    if (mx < 1 || my < 1 || maxm < std::max(mx, my))
        return fail(CLAW2_EINVAL, "bad sizes mx=%d my=%d maxm=%d", mx, my, maxm);
    const int need_aux = rp_maux(rp);  // solvers without aux data ignore an aux array
    if (need_aux > 0 && (maux < need_aux || !aux))
        return fail(CLAW2_EINVAL, "solver %d reads %d aux components per cell (got %d%s)", rp, need_aux, maux,
                    aux ? "" : ", no aux array");
    const int mcapa = method[5];  // method(6): 1 + the aux component of kappa, or 0
    if (mcapa < 0 || (mcapa > 0 && (mcapa > maux || !aux)))
        return fail(CLAW2_EINVAL, "method(6) = %d names no component of the aux array (num_aux = %d)", mcapa, maux);
    const int nup = (need_aux > 0 || mcapa > 0) ? maux : 0;  // aux components uploaded
    if (!(dx > 0.0) || !(dy > 0.0)) return fail(CLAW2_EINVAL, "dx, dy must be positive");
    int rc = check_method(rp, method[1], method[2], mthlim, mwaves, use_fwave);
    if (rc) return rc;

    std::lock_guard<std::mutex> lock(g_scr.mu);
    const Layout L = make_layout(mx, my);
    const size_t nplanes = (size_t)meqn * L.plane;
    const size_t nqbc = (size_t)meqn * (mx + 4) * (my + 4);
    const size_t nstage = (size_t)std::max(meqn, nup) * (mx + 4) * (my + 4);
    rc = scratch_reserve(nplanes, nstage);
    if (rc) return rc;
    cudaStream_t st = g_scr.st;

    if (nup > 0) {  // auxbc as the caller filled it, ghost cells included
        const size_t naux = (size_t)nup * L.plane;
        if (naux > g_scr.aux_cap) {
            cudaFree(g_scr.aux);
            g_scr.aux = nullptr;
            g_scr.aux_cap = 0;
            if (cudaMalloc(&g_scr.aux, naux * 8) != cudaSuccess)
                return fail(CLAW2_ENOMEM, "device allocation of %zu doubles failed", naux);
            g_scr.aux_cap = naux;
        }
        const size_t na = (size_t)nup * (mx + 4) * (my + 4);
        CUDA_TRY(cudaMemcpyAsync(g_scr.stage, aux, na * 8, cudaMemcpyHostToDevice, st));
        k_aos_to_planes<<<grid_blocks((long long)(mx + 4) * (my + 4)), 256, 0, st>>>(g_scr.stage, g_scr.aux, L,
                                                                                    nup, 2);
    }
    CUDA_TRY(cudaMemcpyAsync(g_scr.stage, qold, nqbc * 8, cudaMemcpyHostToDevice, st));
    k_aos_to_planes<<<grid_blocks((long long)(mx + 4) * (my + 4)), 256, 0, st>>>(g_scr.stage, g_scr.a, L, meqn, 2);
    CUDA_TRY(cudaMemsetAsync(g_scr.cfl, 0, sizeof(unsigned long long), st));
    CUDA_TRY(cudaMemsetAsync(g_scr.status, 0, sizeof(int), st));

    StepArgs a;
    a.L = L;
    a.dtdx = dt / dx;
    a.dtdy = dt / dy;
    a.H = 0;
    a.rp = make_params(rp, cparam, ncparam);
    a.meth.order = method[1];
    a.meth.transverse = method[2];
    a.meth.fwave = use_fwave;
    for (int k = 0; k < CLAW2_MAX_WAVES; ++k) a.meth.mthlim[k] = k < mwaves ? mthlim[k] : 0;
    a.cfl_bits = g_scr.cfl;
    a.status = g_scr.status;
    a.guess = nullptr;
    a.counters = nullptr;
    a.aux = need_aux > 0 ? g_scr.aux : nullptr;
    a.capa = mcapa > 0 ? g_scr.aux + (size_t)(mcapa - 1) * L.plane : nullptr;

    a.qold = g_scr.a;
    a.qnew = g_scr.b;
    const int bad = (ids == 0) ? dispatch<UnsplitF>(rp, a, st) : dispatch<SplitF>(rp, a, a, st, ids);
    if (bad) return fail(CLAW2_EINVAL, "unknown Riemann solver id %d", rp);
    CUDA_TRY(cudaGetLastError());
    k_planes_to_aos<<<grid_blocks((long long)(mx + 4) * (my + 4)), 256, 0, st>>>(g_scr.b, g_scr.stage, L, meqn, 2);
    CUDA_TRY(cudaGetLastError());
    unsigned long long bits = 0;
    int status = 0;
    CUDA_TRY(cudaMemcpyAsync(&bits, g_scr.cfl, sizeof bits, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(&status, g_scr.status, sizeof status, cudaMemcpyDeviceToHost, st));
    if (ids == 1) {
        // the x-sweep of the split step updates every row, ghost rows included,
        // and leaves ghost columns as they were: the whole qbc is the result
        CUDA_TRY(cudaMemcpyAsync(qnew, g_scr.stage, nqbc * 8, cudaMemcpyDeviceToHost, st));
    } else {
        // interior cells only; ghost cells of qnew keep their entry values
        const size_t rowb = (size_t)meqn * (mx + 4) * 8;
        const size_t off = (size_t)meqn * ((size_t)(mx + 4) * 2 + 2);
        CUDA_TRY(cudaMemcpy2DAsync(qnew + off, rowb, g_scr.stage + off, rowb, (size_t)meqn * mx * 8, my,
                                   cudaMemcpyDeviceToHost, st));
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    double c;
    std::memcpy(&c, &bits, sizeof c);
    *cfl = c;
    if (status & 1) return fail(CLAW2_ENONFINITE, "the step produced a non-finite value");
    return CLAW2_OK;
}

}  // namespace


// ===========================================================================
// The learned Newton guess (mlp.cuh)
// ===========================================================================
struct claw2_mlp {
    int device = 0;
    float* P = nullptr;      // parameters (FP32)
    float* G = nullptr;      // gradient accumulator
    float* M1 = nullptr;     // Adam moments
    float* M2 = nullptr;
    float* loss = nullptr;
    MlpPacked* packed = nullptr;   // mma.sync fragments
    MlpTcImage* tc = nullptr;      // tcgen05 operand image
    int engine = CLAW2_MLP_TCGEN05;
    int* status = nullptr;         // bit 1: an MMA completion wait gave up (claw2_mlp_infer)
    int nsm = 148;
    int guess_per_sm = 0, eval_per_sm = 0;  // resident CTAs of the tcgen05 kernels (0: not yet queried)
    int adam_step = 0;
    float* x = nullptr;      // samples: 8 floats each
    float* y = nullptr;
    int* ok = nullptr;
    long long nsamples = 0, cap = 0;
    cudaStream_t st = nullptr;
};

namespace {

int mlp_repack(claw2_mlp* m) {
    std::vector<float> h(MLP_NPARAM);
    CUDA_TRY(cudaMemcpy(h.data(), m->P, MLP_NPARAM * 4, cudaMemcpyDeviceToHost));
    MlpPacked pk;
    mlp_pack(h.data(), pk);
    CUDA_TRY(cudaMemcpy(m->packed, &pk, sizeof pk, cudaMemcpyHostToDevice));
    MlpTcImage ti;
    mlp_pack_tc(h.data(), ti);
    CUDA_TRY(cudaMemcpy(m->tc, &ti, sizeof ti, cudaMemcpyHostToDevice));
    return CLAW2_OK;
}

// CTAs of a tcgen05 kernel: the resident ones only (each allocates TMEM once
// and loops over its tiles).  Residency per SM (cached in *per_sm) from the
// kernel's registers and static shared memory against the SM's register
// file, shared memory (with the per-CTA reservation) and thread slots, for
// 128-thread CTAs.
template <class K>
int mlp_tc_grid(const claw2_mlp* m, K kernel, int* per_sm, long long tiles) {
    if (*per_sm <= 0) {
        int b = 1;
        cudaFuncAttributes fa;
        cudaDeviceProp pr;
        if (cudaFuncGetAttributes(&fa, kernel) == cudaSuccess && cudaGetDeviceProperties(&pr, m->device) == cudaSuccess) {
            const int regs = std::max(8, (fa.numRegs + 7) / 8 * 8);
            const int by_regs = pr.regsPerMultiprocessor / (regs * 128);
            const int by_smem = (int)(pr.sharedMemPerMultiprocessor /
                                      (fa.sharedSizeBytes + std::max<size_t>(pr.reservedSharedMemPerBlock, 1)));
            const int by_threads = pr.maxThreadsPerMultiProcessor / 128;
            b = std::max(1, std::min(std::min(by_regs, by_smem), std::min(by_threads, 32)));
        } else {
            cudaGetLastError();
        }
        *per_sm = b;
    }
    return (int)std::max(1ll, std::min(tiles, (long long)m->nsm * *per_sm));
}

void mlp_guess_launch(claw2_mlp* m, const double* q, const Layout& L, double gamma, double* guess, int* status,
                      cudaStream_t st) {
    if (m->engine == CLAW2_MLP_TCGEN05) {
        const long long tiles = (long long)((L.mx + 4 + 31) / 32) * ((L.my + 4 + 3) / 4);
        const int grid = mlp_tc_grid(m, k_mlp_guess_tc, &m->guess_per_sm, tiles);
        k_mlp_guess_tc<<<grid, 128, 0, st>>>(m->tc, q, L, gamma, guess, status);
        return;
    }
    dim3 grid((L.mx + 4 + 31) / 32, (L.my + 4 + 3) / 4);
    k_mlp_guess<<<grid, 128, 0, st>>>(m->packed, q, L, gamma, guess);
}

}  // namespace

extern "C" {

int claw2_mlp_create(int device, unsigned long long seed, claw2_mlp** out) {
    if (!out) return fail(CLAW2_EINVAL, "null pointer argument");
    *out = nullptr;
    claw2_mlp* m = new claw2_mlp();
    m->device = device;
    DeviceGuard g(device);
    bool ok = cudaMalloc(&m->P, MLP_NPARAM * 4) == cudaSuccess && cudaMalloc(&m->G, MLP_NPARAM * 4) == cudaSuccess &&
              cudaMalloc(&m->M1, MLP_NPARAM * 4) == cudaSuccess && cudaMalloc(&m->M2, MLP_NPARAM * 4) == cudaSuccess &&
              cudaMalloc(&m->loss, 4) == cudaSuccess && cudaMalloc(&m->packed, sizeof(MlpPacked)) == cudaSuccess &&
              cudaMalloc(&m->tc, sizeof(MlpTcImage)) == cudaSuccess && cudaMalloc(&m->status, 4) == cudaSuccess &&
              cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        claw2_mlp_destroy(m);
        return fail(CLAW2_ENOMEM, "device allocation for the network failed");
    }
    if (cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || m->nsm <= 0)
        m->nsm = 148;
    // the tcgen05 kernels' residency, found here (not inside a stream capture),
    // with the whole shared-memory carveout asked for so it is reached
    cudaFuncSetAttribute(k_mlp_guess_tc, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(k_mlp_eval_tc, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaGetLastError();
    mlp_tc_grid(m, k_mlp_guess_tc, &m->guess_per_sm, 1);
    mlp_tc_grid(m, k_mlp_eval_tc, &m->eval_per_sm, 1);
    // Glorot-uniform weights from the counter RNG, zero biases
    std::vector<float> h(MLP_NPARAM, 0.f);
    auto fill = [&](int off, int fan_out, int fan_in) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for (int k = 0; k < fan_out * fan_in; ++k) h[off + k] = (float)(a * (2.0 * u01(seed, off + k, 7) - 1.0));
    };
    fill(OFF_W1, MLP_H, MLP_IN);
    fill(OFF_W2, MLP_H, MLP_H);
    fill(OFF_W3, 1, MLP_H);
    cudaMemcpy(m->P, h.data(), MLP_NPARAM * 4, cudaMemcpyHostToDevice);
    cudaMemset(m->G, 0, MLP_NPARAM * 4);
    cudaMemset(m->M1, 0, MLP_NPARAM * 4);
    cudaMemset(m->M2, 0, MLP_NPARAM * 4);
    int rc = mlp_repack(m);
    if (rc) {
        claw2_mlp_destroy(m);
        return rc;
    }
    *out = m;
    return CLAW2_OK;
}

int claw2_mlp_destroy(claw2_mlp* m) {
    if (!m) return CLAW2_OK;
    {
        DeviceGuard g(m->device);
        if (m->st) cudaStreamSynchronize(m->st);
        cudaFree(m->P); cudaFree(m->G); cudaFree(m->M1); cudaFree(m->M2); cudaFree(m->loss);
        cudaFree(m->packed); cudaFree(m->tc); cudaFree(m->status); cudaFree(m->x); cudaFree(m->y); cudaFree(m->ok);
        if (m->st) cudaStreamDestroy(m->st);
    }
    delete m;
    return CLAW2_OK;
}

int claw2_mlp_set_params(claw2_mlp* m, const float* p, int n) {
    if (!m || !p || n != MLP_NPARAM) return fail(CLAW2_EINVAL, "need %d parameters", MLP_NPARAM);
    DeviceGuard g(m->device);
    CUDA_TRY(cudaMemcpy(m->P, p, MLP_NPARAM * 4, cudaMemcpyHostToDevice));
    return mlp_repack(m);
}

int claw2_mlp_get_params(claw2_mlp* m, float* p, int n) {
    if (!m || !p || n != MLP_NPARAM) return fail(CLAW2_EINVAL, "need %d parameters", MLP_NPARAM);
    DeviceGuard g(m->device);
    CUDA_TRY(cudaMemcpy(p, m->P, MLP_NPARAM * 4, cudaMemcpyDeviceToHost));
    return CLAW2_OK;
}

int claw2_mlp_generate(claw2_mlp* m, unsigned long long seed, long long n, double gamma, double tol,
                       long long* nvalid) {
    if (!m || n < 1 || n > (1ll << 28)) return fail(CLAW2_EINVAL, "bad sample count");
    DeviceGuard g(m->device);
    if (n > m->cap) {
        cudaFree(m->x); cudaFree(m->y); cudaFree(m->ok);
        m->x = nullptr; m->y = nullptr; m->ok = nullptr; m->cap = 0;
        if (cudaMalloc(&m->x, n * 8 * 4) != cudaSuccess || cudaMalloc(&m->y, n * 4) != cudaSuccess ||
            cudaMalloc(&m->ok, n * 4) != cudaSuccess)
            return fail(CLAW2_ENOMEM, "device allocation for %lld samples failed", n);
        m->cap = n;
    }
    const int chunk = 1 << 22;
    for (long long f = 0; f < n; f += chunk) {
        const int c = (int)std::min<long long>(chunk, n - f);
        k_gen_samples<<<(c + 255) / 256, 256, 0, m->st>>>(seed, f, c, gamma, tol, m->x + f * 8, m->y + f,
                                                          m->ok + f, nullptr);
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(m->st));
    m->nsamples = n;
    if (nvalid) {
        std::vector<int> h(n);
        CUDA_TRY(cudaMemcpy(h.data(), m->ok, n * 4, cudaMemcpyDeviceToHost));
        long long s = 0;
        for (long long k = 0; k < n; ++k) s += h[k];
        *nvalid = s;
    }
    return CLAW2_OK;
}

int claw2_mlp_samples(claw2_mlp* m, long long first, int count, float* x8, float* y, int* ok) {
    if (!m || first < 0 || count < 0 || first + count > m->nsamples) return fail(CLAW2_EINVAL, "bad sample range");
    DeviceGuard g(m->device);
    if (x8) CUDA_TRY(cudaMemcpy(x8, m->x + first * 8, (size_t)count * 32, cudaMemcpyDeviceToHost));
    if (y) CUDA_TRY(cudaMemcpy(y, m->y + first, (size_t)count * 4, cudaMemcpyDeviceToHost));
    if (ok) CUDA_TRY(cudaMemcpy(ok, m->ok + first, (size_t)count * 4, cudaMemcpyDeviceToHost));
    return CLAW2_OK;
}

int claw2_mlp_gradient(claw2_mlp* m, long long first, int count, float* grad, float* loss) {
    if (!m || !grad || first < 0 || count < 1 || first + count > m->nsamples)
        return fail(CLAW2_EINVAL, "bad sample range");
    DeviceGuard g(m->device);
    CUDA_TRY(cudaMemsetAsync(m->G, 0, MLP_NPARAM * 4, m->st));
    CUDA_TRY(cudaMemsetAsync(m->loss, 0, 4, m->st));
    k_train_grad<<<(count + 255) / 256, 256, 0, m->st>>>(m->P, m->x, m->y, m->ok, first, count, 1.f / count, m->G,
                                                         m->loss);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(grad, m->G, MLP_NPARAM * 4, cudaMemcpyDeviceToHost, m->st));
    if (loss) CUDA_TRY(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->st));
    CUDA_TRY(cudaStreamSynchronize(m->st));
    CUDA_TRY(cudaMemset(m->G, 0, MLP_NPARAM * 4));
    return CLAW2_OK;
}

int claw2_mlp_train(claw2_mlp* m, int epochs, int batch, float lr, float* last_loss) {
    if (!m || epochs < 0 || batch < 32 || m->nsamples < batch) return fail(CLAW2_EINVAL, "bad training arguments");
    DeviceGuard g(m->device);
    const long long nb = m->nsamples / batch;
    float l = 0.f;
    for (int e = 0; e < epochs; ++e) {
        CUDA_TRY(cudaMemsetAsync(m->loss, 0, 4, m->st));
        for (long long b = 0; b < nb; ++b) {
            k_train_grad<<<(batch + 255) / 256, 256, 0, m->st>>>(m->P, m->x, m->y, m->ok, b * batch, batch,
                                                                 1.f / batch, m->G, m->loss);
            ++m->adam_step;
            // step size decays linearly to a tenth over the run
            const float frac = (float)(e * nb + b) / (float)(epochs * nb);
            k_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, m->st>>>(m->P, m->G, m->M1, m->M2, lr * (1.f - 0.9f * frac),
                                                                0.9f, 0.999f, 1e-8f, m->adam_step);
        }
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(&l, m->loss, 4, cudaMemcpyDeviceToHost, m->st));
        CUDA_TRY(cudaStreamSynchronize(m->st));
        l /= (float)nb;
    }
    if (last_loss) *last_loss = l;
    return mlp_repack(m);
}

int claw2_mlp_infer(claw2_mlp* m, const float* x8, int n, float* y) {
    if (!m || !x8 || !y || n < 1) return fail(CLAW2_EINVAL, "bad arguments");
    DeviceGuard g(m->device);
    float *dx = nullptr, *dy = nullptr;
    if (cudaMalloc(&dx, (size_t)n * 32) != cudaSuccess || cudaMalloc(&dy, (size_t)n * 4) != cudaSuccess) {
        cudaFree(dx);
        return fail(CLAW2_ENOMEM, "device allocation failed");
    }
    cudaMemcpy(dx, x8, (size_t)n * 32, cudaMemcpyHostToDevice);
    cudaMemsetAsync(m->status, 0, 4, m->st);
    if (m->engine == CLAW2_MLP_TCGEN05)
        k_mlp_eval_tc<<<mlp_tc_grid(m, k_mlp_eval_tc, &m->eval_per_sm, (n + 255) / 256), 128, 0, m->st>>>(
            m->tc, dx, n, dy, m->status);
    else
        k_mlp_eval<<<(n + 255) / 256, 128, 0, m->st>>>(m->packed, dx, n, dy);
    cudaError_t e = cudaStreamSynchronize(m->st);
    int st = 0;
    if (e == cudaSuccess) e = cudaMemcpy(y, dy, (size_t)n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&st, m->status, 4, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dy);
    if (e != cudaSuccess) return fail(CLAW2_ECUDA, "inference failed: %s", cudaGetErrorString(e));
    if (st & 2) return fail(CLAW2_ETIMEOUT, "a tensor-core completion wait gave up");
    return CLAW2_OK;
}

int claw2_mlp_set_engine(claw2_mlp* m, int engine) {
    if (!m || (engine != CLAW2_MLP_TCGEN05 && engine != CLAW2_MLP_MMA_SYNC))
        return fail(CLAW2_EINVAL, "engine must be CLAW2_MLP_TCGEN05 or CLAW2_MLP_MMA_SYNC");
    m->engine = engine;
    return CLAW2_OK;
}

}  // extern "C"

// ===========================================================================
// Device-resident patch
// ===========================================================================
struct claw2_mlp;
struct claw2_patch {
    claw2_desc d;
    Layout L;
    RPParams rp;
    Method meth;
    int device = 0;
    double* q[2] = {nullptr, nullptr};  // current / pending (ping-pong)
    double* tmp = nullptr;              // intermediate of the split step
    double* aux = nullptr;              // aux planes (solvers with aux data), ghost cells filled at upload
    double* stage = nullptr;            // AoS staging for host copies
    size_t stage_n = 0;                 // its size in doubles
    unsigned long long* cfl = nullptr;
    int* status = nullptr;
    unsigned long long* h_cfl = nullptr;  // pinned
    int* h_status = nullptr;              // pinned
    cudaStream_t st = nullptr;      // the stream work is issued on
    cudaStream_t own_st = nullptr;  // the patch's own stream
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timing = false;
    double* guess = nullptr;                  // exact solver: learned guesses, x and y planes
    unsigned long long* counters = nullptr;   // exact solver: Newton steps needed, solves, steps applied
    int exact_guess = 0;                      // exact solver: 1 = start from the converged p* (measurement)
    double exact_guess_err = 0.0;             // mode 1: relative error put on the converged p*
    int split_part = 0;                       // 1 after claw2_patch_step_part(.., 1): part 2 must follow
    claw2_mlp* mlp = nullptr;
    // claw2_patch_evolve's captured attempts, one graph per starting buffer
    // parity, reused while nothing they captured changed: graph_gen counts
    // changes of the patch's parameters, network and tile schedule arrays
    cudaGraphExec_t evo_exec[2] = {nullptr, nullptr};
    unsigned long long evo_stamp[2] = {0, 0};
    unsigned graph_gen = 1;
    // longest-first tile schedule of the unsplit kernel (k_lpt_order)
    unsigned int* tile_cost = nullptr;
    int* tile_order = nullptr;
    int tile_cap = 0, tile_n = 0, tile_H = 0;
    unsigned int tile_steps = 0;  // steps run on the current tiling
    long long step_launches = 0;  // kernels enqueued by patch_enqueue_step (claw2_patch_launch_count)
    // host pipeline of claw2_patch_run_host
    cudaStream_t cst = nullptr, dst = nullptr;  // upload and download streams
    double* stage_in[2] = {nullptr, nullptr};
    double* stage_out1 = nullptr;
    cudaEvent_t h2d_done[2] = {nullptr, nullptr}, in_free[2] = {nullptr, nullptr};
    cudaEvent_t out_ready[2] = {nullptr, nullptr}, out_free[2] = {nullptr, nullptr};
    unsigned long long* cfl_hist = nullptr;
    unsigned long long* h_cfl_hist = nullptr;
    int cfl_hist_cap = 0;
    int nsm = 0;                  // SMs of the patch's device
    bool ghosts_supplied = false; // claw2_patch_upload_qbc: the next step keeps the uploaded ghost cells
    // claw2_patch_write_ascii_async: pinned copy of a frame, its event, the writer thread
    double* out_host = nullptr;
    cudaEvent_t out_ev = nullptr;
    // claw2_patch_evolve: the time loop's state on the device and a pinned copy
    EvolveDev* evo = nullptr;
    EvolveDev* h_evo = nullptr;
    std::thread* writer = nullptr;
    int writer_rc = 0;
    void* gather_buf = nullptr;   // claw2_patch_gather_q: values, then cell indices
    size_t gather_cap = 0;
    CUtensorMap tmap[2];          // TMA descriptors of q[0], q[1]
    bool has_tmap = false;
    int cur = 0;
    bool pending = false;
};

namespace {


// Buffers of the longest-first schedule for n tiles of height H; a new
// tiling starts from the identity order.  Returns non-OK (no schedule) when
// the tiling is too large for the one-CTA sort or the buffers cannot be had.
int lpt_prepare(claw2_patch* p, int n, int H) {
    if (n < 1 || n > LPT_MAX_TILES) return CLAW2_EINVAL;
    if (n > p->tile_cap) {
        // (the patch's stream may still run a step on the old arrays)
        cudaStreamSynchronize(p->st);
        cudaFree(p->tile_cost);
        cudaFree(p->tile_order);
        p->tile_cost = nullptr;
        p->tile_order = nullptr;
        p->tile_cap = 0;
        if (cudaMalloc(&p->tile_cost, sizeof(unsigned int) * n) != cudaSuccess ||
            cudaMalloc(&p->tile_order, sizeof(int) * n) != cudaSuccess) {
            cudaFree(p->tile_cost);
            cudaFree(p->tile_order);
            p->tile_cost = nullptr;
            p->tile_order = nullptr;
            cudaGetLastError();
            return CLAW2_ENOMEM;
        }
        p->tile_cap = n;
        p->tile_n = 0;
    }
    if (p->tile_n != n || p->tile_H != H) {
        ++p->graph_gen;
        k_iota<<<(n + 255) / 256, 256, 0, p->st>>>(p->tile_order, n);
        cudaMemsetAsync(p->tile_cost, 0, sizeof(unsigned int) * n, p->st);
        p->tile_n = n;
        p->tile_H = H;
        p->tile_steps = 0;
    }
    return CLAW2_OK;
}

// The tile costs drift slowly with the flow, so the schedule is re-sorted
// after the first step on a tiling and then every LPT_EVERY steps.
constexpr unsigned int LPT_EVERY = 4;

void launch_lpt(const unsigned int* cost, int* order, int n, cudaStream_t st) {
    int N = 1;
    while (N < n) N <<= 1;
    static unsigned long long attr = 0;
    smem_attr(k_lpt_order, (int)sizeof(unsigned long long) * LPT_MAX_TILES, attr);
    // (the sort of up to 1024 keys double-buffers its shared-memory stages)
    const size_t smem = sizeof(unsigned long long) * (N >= 32 && N <= 1024 ? 2 * N : N);
    k_lpt_order<<<1, 1024, smem, st>>>(cost, order, n);
}

StepArgs patch_args(claw2_patch* p, double dt) {
    StepArgs a;
    a.L = p->L;
    a.dtdx = dt / p->d.dx;
    a.dtdy = dt / p->d.dy;
    a.H = 0;
    a.rp = p->rp;
    a.meth = p->meth;
    a.cfl_bits = p->cfl;
    a.aux = p->aux;
    a.capa = p->d.mcapa > 0 ? p->aux + (size_t)(p->d.mcapa - 1) * p->L.plane : nullptr;
    a.status = p->status;
    a.guess = nullptr;
    a.counters = p->counters;
    a.qold = p->q[p->cur];
    a.qnew = p->q[p->cur ^ 1];
    return a;
}

}  // namespace

// The split sweeps on caller-owned buffers, for claw2_step2ds_noalloc
// (claw2_noalloc.cu): the launches claw2_step2ds makes (same kernels, method
// specialisations and row heights).  Hidden: not part of the exported ABI.
__attribute__((visibility("hidden"))) int claw2_internal_launch_split(int rp, const StepArgs& ax, const StepArgs& ay,
                                                                      cudaStream_t st) {
    return dispatch<SplitF>(rp, ax, ay, st, 3);
}

extern "C" {

// Lets other translation units of this library report errors through
// claw2_last_error(); hidden, so it is not part of the exported ABI.
__attribute__((visibility("hidden"))) void claw2_internal_set_error(const char* msg) { g_err = msg; }

const char* claw2_last_error(void) { return g_err.c_str(); }
const char* claw2_version(void) { return "claw2 0.1 (sm_100a, FP64)"; }

int claw2_step2(int maxm, int num_eqn, int num_waves, int num_aux, int num_ghost, int mx, int my,
                const double* qold, double* qnew, const double* aux, double dx, double dy, double dt,
                const int* method, const int* mthlim, double* cfl, int use_fwave, int riemann,
                const double* cparam, int ncparam) {
    if (method && method[2] < 0)
        return fail(CLAW2_EINVAL, "method(3) = -1 selects the split step: call claw2_step2ds");
    return host_step(maxm, num_eqn, num_waves, num_aux, num_ghost, mx, my, qold, qnew, aux, dx, dy, dt, method,
                     mthlim, cfl, 0, use_fwave, riemann, cparam, ncparam);
}

int claw2_step2ds(int maxm, int num_eqn, int num_waves, int num_aux, int num_ghost, int mx, int my,
                  const double* qold, double* qnew, const double* aux, double dx, double dy, double dt,
                  const int* method, const int* mthlim, double* cfl, int ids, int use_fwave, int riemann,
                  const double* cparam, int ncparam) {
    if (ids != 1 && ids != 2) return fail(CLAW2_EINVAL, "ids must be 1 or 2 (got %d)", ids);
    return host_step(maxm, num_eqn, num_waves, num_aux, num_ghost, mx, my, qold, qnew, aux, dx, dy, dt, method,
                     mthlim, cfl, ids, use_fwave, riemann, cparam, ncparam);
}

int claw2_bc_fill(int num_eqn, int num_ghost, int mx, int my, double* qbc, const int* bcl, const int* bcu) {
    if (!qbc || !bcl || !bcu) return fail(CLAW2_EINVAL, "null pointer argument");
    if (num_ghost != 2 || mx < 1 || my < 1 || num_eqn < 1)
        return fail(CLAW2_EINVAL, "bad sizes num_eqn=%d num_ghost=%d mx=%d my=%d", num_eqn, num_ghost, mx, my);
    int rc = check_bc(bcl, bcu, mx, my);
    if (rc) return rc;
    std::lock_guard<std::mutex> lock(g_scr.mu);
    const Layout L = make_layout(mx, my);
    const size_t nplanes = (size_t)num_eqn * L.plane;
    const size_t nstage = (size_t)num_eqn * (mx + 4) * (my + 4);
    rc = scratch_reserve(nplanes, nstage);
    if (rc) return rc;
    cudaStream_t st = g_scr.st;
    CUDA_TRY(cudaMemcpyAsync(g_scr.stage, qbc, nstage * 8, cudaMemcpyHostToDevice, st));
    k_aos_to_planes<<<grid_blocks((long long)(mx + 4) * (my + 4)), 256, 0, st>>>(g_scr.stage, g_scr.a, L, num_eqn, 2);
    launch_bc(g_scr.a, L, num_eqn, bcl, bcu, nullptr, st);
    k_planes_to_aos<<<grid_blocks((long long)(mx + 4) * (my + 4)), 256, 0, st>>>(g_scr.a, g_scr.stage, L, num_eqn, 2);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(qbc, g_scr.stage, nstage * 8, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return CLAW2_OK;
}

int claw2_patch_create(const claw2_desc* d, claw2_patch** out) {
    if (!d || !out) return fail(CLAW2_EINVAL, "null pointer argument");
    *out = nullptr;
    int me = 0, mw = 0;
    if (rp_shape(d->riemann, &me, &mw) != 0) return fail(CLAW2_EINVAL, "unknown Riemann solver id %d", d->riemann);
    if (d->num_eqn != me || d->num_waves != mw)
        return fail(CLAW2_EINVAL, "solver %d has num_eqn=%d num_waves=%d (got %d, %d)", d->riemann, me, mw,
                    d->num_eqn, d->num_waves);
    if (d->num_ghost != 2) return fail(CLAW2_EINVAL, "num_ghost must be 2 (got %d)", d->num_ghost);
    if (d->num_aux < rp_maux(d->riemann))
        return fail(CLAW2_EINVAL, "solver %d reads %d aux components per cell (num_aux=%d)", d->riemann,
                    rp_maux(d->riemann), d->num_aux);
    if (d->mcapa < 0 || d->mcapa > d->num_aux)
        return fail(CLAW2_EINVAL, "mcapa = %d names no component of the aux array (num_aux = %d)", d->mcapa,
                    d->num_aux);
    if (d->mx < 1 || d->my < 1) return fail(CLAW2_EINVAL, "bad sizes mx=%d my=%d", d->mx, d->my);
    if (!(d->dx > 0.0) || !(d->dy > 0.0)) return fail(CLAW2_EINVAL, "dx, dy must be positive");
    const int trans = d->dimensional_split ? -1 : d->transverse;
    int rc = check_method(d->riemann, d->order, trans, d->mthlim, mw, d->fwave);
    if (rc) return rc;
    rc = check_bc(d->bc_lower, d->bc_upper, d->mx, d->my);
    if (rc) return rc;
    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (d->device < 0 || d->device >= ndev) return fail(CLAW2_EINVAL, "device %d not present", d->device);

    claw2_patch* p = new claw2_patch();
    p->d = *d;
    p->device = d->device;
    p->L = make_layout(d->mx, d->my);
    p->rp = make_params(d->riemann, d->cparam, d->ncparam);
    p->meth.order = d->order;
    p->meth.transverse = trans;
    p->meth.fwave = d->fwave;
    for (int k = 0; k < CLAW2_MAX_WAVES; ++k) p->meth.mthlim[k] = k < mw ? d->mthlim[k] : 0;
    DeviceGuard g(p->device);
    cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, p->device);
    const size_t nb = (size_t)me * p->L.plane * 8;
    // staging: q or the aux array, with ghost cells
    const size_t ns = (size_t)std::max(me, d->num_aux) * (d->mx + 4) * (d->my + 4) * 8;
    p->stage_n = ns / 8;
    bool ok = cudaMalloc(&p->q[0], nb) == cudaSuccess && cudaMalloc(&p->q[1], nb) == cudaSuccess &&
              cudaMalloc(&p->stage, ns) == cudaSuccess &&
              cudaMalloc(&p->cfl, sizeof(unsigned long long)) == cudaSuccess &&
              cudaMalloc(&p->status, sizeof(int)) == cudaSuccess &&
              cudaMallocHost(&p->h_cfl, sizeof(unsigned long long)) == cudaSuccess &&
              cudaMallocHost(&p->h_status, sizeof(int)) == cudaSuccess &&
              cudaStreamCreateWithFlags(&p->own_st, cudaStreamNonBlocking) == cudaSuccess;
    p->st = p->own_st;
    if (ok && d->dimensional_split) ok = cudaMalloc(&p->tmp, nb) == cudaSuccess;
    if (ok && d->num_aux > 0) {
        ok = cudaMalloc(&p->aux, (size_t)d->num_aux * p->L.plane * 8) == cudaSuccess;
        if (ok) cudaMemsetAsync(p->aux, 0, (size_t)d->num_aux * p->L.plane * 8, p->st);
    }
    if (ok && d->riemann == CLAW2_RP_EULER_EXACT)
        ok = cudaMalloc(&p->guess, 2 * (size_t)p->L.plane * 8) == cudaSuccess &&
             cudaMalloc(&p->counters, 3 * sizeof(unsigned long long)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        claw2_patch_destroy(p);
        return fail(CLAW2_ENOMEM, "device allocation for a %dx%d patch failed", d->mx, d->my);
    }
    p->has_tmap = make_row_tmap<NT_UNSPLIT>(&p->tmap[0], p->q[0], p->L, me) &&
                  make_row_tmap<NT_UNSPLIT>(&p->tmap[1], p->q[1], p->L, me);
    // zero everything once so padding and ghost cells are defined
    cudaMemsetAsync(p->q[0], 0, nb, p->st);
    cudaMemsetAsync(p->q[1], 0, nb, p->st);
    if (p->tmp) cudaMemsetAsync(p->tmp, 0, nb, p->st);
    if (p->counters) cudaMemsetAsync(p->counters, 0, 3 * sizeof(unsigned long long), p->st);
    cudaMemsetAsync(p->cfl, 0, sizeof(unsigned long long), p->st);
    cudaMemsetAsync(p->status, 0, sizeof(int), p->st);
    if (cudaStreamSynchronize(p->st) != cudaSuccess) {
        claw2_patch_destroy(p);
        return fail(CLAW2_ECUDA, "patch initialisation failed");
    }
    *out = p;
    return CLAW2_OK;
}

int claw2_patch_destroy(claw2_patch* p) {
    if (!p) return CLAW2_OK;
    if (p->writer) {
        p->writer->join();
        delete p->writer;
        p->writer = nullptr;
    }
    {
        DeviceGuard g(p->device);
        if (p->st) cudaStreamSynchronize(p->st);
        cudaFree(p->q[0]);
        cudaFree(p->q[1]);
        cudaFree(p->tmp);
        cudaFree(p->aux);
        cudaFree(p->guess);
        cudaFree(p->counters);
        cudaFree(p->tile_cost);
        cudaFree(p->tile_order);
        // the host pipeline of claw2_patch_run_host
        if (p->cst) cudaStreamSynchronize(p->cst);
        if (p->dst) cudaStreamSynchronize(p->dst);
        for (int i = 0; i < 2; ++i) {
            cudaFree(p->stage_in[i]);
            if (p->h2d_done[i]) cudaEventDestroy(p->h2d_done[i]);
            if (p->in_free[i]) cudaEventDestroy(p->in_free[i]);
            if (p->out_ready[i]) cudaEventDestroy(p->out_ready[i]);
            if (p->out_free[i]) cudaEventDestroy(p->out_free[i]);
        }
        cudaFree(p->stage_out1);
        cudaFree(p->cfl_hist);
        cudaFreeHost(p->h_cfl_hist);
        if (p->cst) cudaStreamDestroy(p->cst);
        if (p->dst) cudaStreamDestroy(p->dst);
        cudaFree(p->stage);
        cudaFree(p->gather_buf);
        cudaFreeHost(p->out_host);
        if (p->out_ev) cudaEventDestroy(p->out_ev);
        for (int i = 0; i < 2; ++i)
            if (p->evo_exec[i]) cudaGraphExecDestroy(p->evo_exec[i]);
        cudaFree(p->evo);
        cudaFreeHost(p->h_evo);
        cudaFree(p->cfl);
        cudaFree(p->status);
        cudaFreeHost(p->h_cfl);
        cudaFreeHost(p->h_status);
        if (p->ev0) cudaEventDestroy(p->ev0);
        if (p->ev1) cudaEventDestroy(p->ev1);
        if (p->own_st) cudaStreamDestroy(p->own_st);
    }
    delete p;
    return CLAW2_OK;
}

int claw2_patch_set_cparam(claw2_patch* p, const double* cparam, int n) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    if (n < 0 || n > CLAW2_MAX_PARAMS) return fail(CLAW2_EINVAL, "ncparam %d out of range", n);
    p->rp = make_params(p->d.riemann, cparam, n);
    ++p->graph_gen;
    return CLAW2_OK;
}

int claw2_patch_upload_q(claw2_patch* p, const double* q) {
    if (!p || !q) return fail(CLAW2_EINVAL, "null pointer argument");
    DeviceGuard g(p->device);
    const size_t n = (size_t)p->d.num_eqn * p->d.mx * p->d.my;
    CUDA_TRY(cudaMemcpyAsync(p->stage, q, n * 8, cudaMemcpyHostToDevice, p->st));
    k_aos_to_planes<<<grid_blocks((long long)p->d.mx * p->d.my), 256, 0, p->st>>>(p->stage, p->q[p->cur], p->L,
                                                                                   p->d.num_eqn, 0);
    CUDA_TRY(cudaGetLastError());
    p->pending = false;
    return CLAW2_OK;
}

int claw2_patch_upload_aux(claw2_patch* p, const double* aux, const int* aux_bc_lower, const int* aux_bc_upper) {
    if (!p || !aux || !aux_bc_lower || !aux_bc_upper) return fail(CLAW2_EINVAL, "null pointer argument");
    if (p->d.num_aux < 1) return fail(CLAW2_EINVAL, "this patch has no aux arrays (num_aux = 0)");
    int rc = check_bc(aux_bc_lower, aux_bc_upper, p->d.mx, p->d.my);
    if (rc) return rc;
    DeviceGuard g(p->device);
    const size_t n = (size_t)p->d.num_aux * p->d.mx * p->d.my;
    CUDA_TRY(cudaMemcpyAsync(p->stage, aux, n * 8, cudaMemcpyHostToDevice, p->st));
    k_aos_to_planes<<<grid_blocks((long long)p->d.mx * p->d.my), 256, 0, p->st>>>(p->stage, p->aux, p->L,
                                                                                   p->d.num_aux, 0);
    // ghost cells of aux (solver.py:439-519 with name != 'q': a wall mirrors without sign change)
    launch_bc(p->aux, p->L, p->d.num_aux, aux_bc_lower, aux_bc_upper, nullptr, p->st, 0);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(p->st));
    return CLAW2_OK;
}

int claw2_patch_upload_qbc(claw2_patch* p, const double* qbc) {
    if (!p || !qbc) return fail(CLAW2_EINVAL, "null pointer argument");
    if (p->pending) return fail(CLAW2_EINVAL, "a step is pending: accept or reject it first");
    DeviceGuard g(p->device);
    const size_t n = (size_t)p->d.num_eqn * (p->d.mx + 4) * (p->d.my + 4);
    if (n > p->stage_n) return fail(CLAW2_EINVAL, "staging buffer too small for qbc");
    CUDA_TRY(cudaMemcpyAsync(p->stage, qbc, n * 8, cudaMemcpyHostToDevice, p->st));
    k_aos_to_planes<<<grid_blocks((long long)(p->d.mx + 4) * (p->d.my + 4)), 256, 0, p->st>>>(p->stage, p->q[p->cur],
                                                                                           p->L, p->d.num_eqn, 2);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(p->st));
    p->ghosts_supplied = true;
    return CLAW2_OK;
}

int claw2_patch_upload_auxbc(claw2_patch* p, const double* auxbc) {
    if (!p || !auxbc) return fail(CLAW2_EINVAL, "null pointer argument");
    if (p->d.num_aux < 1) return fail(CLAW2_EINVAL, "this patch has no aux arrays (num_aux = 0)");
    DeviceGuard g(p->device);
    const size_t n = (size_t)p->d.num_aux * (p->d.mx + 4) * (p->d.my + 4);
    CUDA_TRY(cudaMemcpyAsync(p->stage, auxbc, n * 8, cudaMemcpyHostToDevice, p->st));
    k_aos_to_planes<<<grid_blocks((long long)(p->d.mx + 4) * (p->d.my + 4)), 256, 0, p->st>>>(p->stage, p->aux, p->L,
                                                                                           p->d.num_aux, 2);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(p->st));
    return CLAW2_OK;
}

int claw2_patch_gather_q(claw2_patch* p, int n, const int* ij, double* out) {
    if (!p || (n > 0 && (!ij || !out))) return fail(CLAW2_EINVAL, "null pointer argument");
    if (n < 0 || n > (1 << 20)) return fail(CLAW2_EINVAL, "gather of %d cells out of range", n);
    if (n == 0) return CLAW2_OK;
    for (int g = 0; g < n; ++g)
        if (ij[2 * g] < 0 || ij[2 * g] >= p->d.mx || ij[2 * g + 1] < 0 || ij[2 * g + 1] >= p->d.my)
            return fail(CLAW2_EINVAL, "cell (%d, %d) outside the %dx%d grid", ij[2 * g], ij[2 * g + 1], p->d.mx,
                        p->d.my);
    DeviceGuard g(p->device);
    const int me = p->d.num_eqn;
    const size_t need = (size_t)n * 2 * sizeof(int) + (size_t)n * me * sizeof(double);
    if (need > p->gather_cap) {
        cudaFree(p->gather_buf);
        p->gather_buf = nullptr;
        p->gather_cap = 0;
        if (cudaMalloc(&p->gather_buf, need) != cudaSuccess) {
            cudaGetLastError();
            return fail(CLAW2_ENOMEM, "gather buffer of %zu bytes could not be allocated", need);
        }
        p->gather_cap = need;
    }
    double* dout = reinterpret_cast<double*>(p->gather_buf);  // doubles first: 8-byte aligned
    int* dij = reinterpret_cast<int*>(dout + (size_t)n * me);
    CUDA_TRY(cudaMemcpyAsync(dij, ij, (size_t)n * 2 * sizeof(int), cudaMemcpyHostToDevice, p->st));
    k_gather_cells<<<(n * me + 127) / 128, 128, 0, p->st>>>(p->q[p->cur], p->L, me, n, dij, dout);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, dout, (size_t)n * me * sizeof(double), cudaMemcpyDeviceToHost, p->st));
    CUDA_TRY(cudaStreamSynchronize(p->st));
    return CLAW2_OK;
}

int claw2_patch_linear_source(claw2_patch* p, const double* m, int n, double dt) {
    if (!p || !m) return fail(CLAW2_EINVAL, "null pointer argument");
    if (n != p->d.num_eqn || n > SRC_MAX)
        return fail(CLAW2_EINVAL, "source matrix of order %d for num_eqn = %d", n, p->d.num_eqn);
    if (p->pending) return fail(CLAW2_EINVAL, "a step is pending: accept or reject it first");
    LinearSourceArgs a;
    for (int k = 0; k < n * n; ++k) a.m[k] = m[k];
    a.n = n;
    a.dt = dt;
    DeviceGuard g(p->device);
    k_linear_source<<<grid_blocks((long long)p->d.mx * p->d.my), 256, 0, p->st>>>(p->q[p->cur], p->L, a);
    CUDA_TRY(cudaGetLastError());
    return CLAW2_OK;
}

int claw2_patch_euler_axisymmetric_source(claw2_patch* p, double gamma, int radius_aux, double dt) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    if (p->d.num_eqn < 4) return fail(CLAW2_EINVAL, "the Euler source needs num_eqn >= 4 (got %d)", p->d.num_eqn);
    if (radius_aux < 0 || radius_aux >= p->d.num_aux || !p->aux)
        return fail(CLAW2_EINVAL, "aux component %d (the radius) is not on the device (num_aux = %d)", radius_aux,
                    p->d.num_aux);
    if (p->pending) return fail(CLAW2_EINVAL, "a step is pending: accept or reject it first");
    DeviceGuard g(p->device);
    k_euler_axisym_source<<<grid_blocks((long long)p->d.mx * p->d.my), 256, 0, p->st>>>(
        p->q[p->cur], p->aux + (size_t)radius_aux * p->L.plane, p->L, gamma, dt);
    CUDA_TRY(cudaGetLastError());
    return CLAW2_OK;
}

int claw2_patch_wait_output(claw2_patch* p) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    if (!p->writer) return CLAW2_OK;
    p->writer->join();
    delete p->writer;
    p->writer = nullptr;
    const int rc = p->writer_rc;
    p->writer_rc = 0;
    return rc;
}

int claw2_patch_write_ascii_async(claw2_patch* p, const char* path, int append, const char* header,
                                  int nthreads) {
    if (!p || !path || !header) return fail(CLAW2_EINVAL, "null pointer argument");
    int rc = claw2_patch_wait_output(p);  // one frame in flight at a time
    if (rc) return rc;
    DeviceGuard g(p->device);
    const int me = p->d.num_eqn, mx = p->d.mx, my = p->d.my;
    const size_t n = (size_t)me * mx * my;
    if (!p->out_host) {
        if (cudaMallocHost(&p->out_host, n * 8) != cudaSuccess ||
            cudaEventCreateWithFlags(&p->out_ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            cudaFreeHost(p->out_host);
            p->out_host = nullptr;
            return fail(CLAW2_ENOMEM, "pinned frame buffer of %zu bytes could not be allocated", n * 8);
        }
    }
    // the current state, in stream order: later steps cannot overwrite it first
    k_planes_to_aos<<<grid_blocks((long long)mx * my), 256, 0, p->st>>>(p->q[p->cur], p->stage, p->L, me, 0);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(p->out_host, p->stage, n * 8, cudaMemcpyDeviceToHost, p->st));
    CUDA_TRY(cudaEventRecord(p->out_ev, p->st));
    std::string spath(path), shead(header);
    const int dev = p->device;
    p->writer = new std::thread([p, spath, shead, append, me, mx, my, nthreads, dev]() {
        cudaSetDevice(dev);
        if (cudaEventSynchronize(p->out_ev) != cudaSuccess) {
            p->writer_rc = CLAW2_ECUDA;
            return;
        }
        p->writer_rc = claw2_internal_write_ascii(spath.c_str(), append, shead.c_str(), p->out_host, me, mx, my,
                                                  nthreads);
    });
    return CLAW2_OK;
}

int claw2_patch_download_q(claw2_patch* p, double* q) {
    if (!p || !q) return fail(CLAW2_EINVAL, "null pointer argument");
    DeviceGuard g(p->device);
    const size_t n = (size_t)p->d.num_eqn * p->d.mx * p->d.my;
    k_planes_to_aos<<<grid_blocks((long long)p->d.mx * p->d.my), 256, 0, p->st>>>(p->q[p->cur], p->stage, p->L,
                                                                                   p->d.num_eqn, 0);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(q, p->stage, n * 8, cudaMemcpyDeviceToHost, p->st));
    CUDA_TRY(cudaStreamSynchronize(p->st));
    return CLAW2_OK;
}

}  // extern "C"

namespace {

// Ghost fill + step (+ learned guess pre-pass, + tile schedule) of a patch on
// its stream; the result goes to the pending buffer.  part 0: the whole step.
// part 1 / part 2 (claw2_patch_step_part): a plain unsplit step split around a
// halo exchange -- part 1 fills every ghost cell but the ghost rows of
// internal sides and steps the row blocks that read no ghost row; part 2
// fills those rows' ghost columns and steps the first and last row blocks.
// Any other step (split, exact solver, custom BCs, no row block clear of the
// ghost rows) runs whole in part 2.
int patch_enqueue_step(claw2_patch* p, double dt, int part = 0) {
    double* qc = p->q[p->cur];
    int ns = 0, H = 0, nb = 0;
    unsplit_tiling(p->d.riemann, p->L.mx, p->L.my, ns, H, nb);
    // row block b reads padded rows H b .. H b + min(H, my - H b) + 3: blocks
    // 1 .. b_hi read no ghost row (H (b+1) + 3 <= my + 1 for a full block;
    // a ragged last block of one row pushes its neighbour into the edge set)
    const int b_hi = std::min(nb - 2, (p->L.my - 2) / std::max(H, 1) - 1);
    if (part != 0) {
        const bool simple = !p->d.dimensional_split && !p->ghosts_supplied &&
                            p->d.riemann != CLAW2_RP_EULER_EXACT && b_hi >= 1;
        if (!simple) {
            if (part == 1) return CLAW2_OK;  // nothing runs before the exchange
            part = 0;                        // part 2: the whole step
        }
    }
    if (p->ghosts_supplied) {  // the host filled every ghost cell (custom BCs)
        CUDA_TRY(cudaMemsetAsync(p->cfl, 0, sizeof(unsigned long long), p->st));
        p->ghosts_supplied = false;
    } else {
        launch_bc(qc, p->L, p->d.num_eqn, p->d.bc_lower, p->d.bc_upper, p->cfl, p->st, 1, part);
        ++p->step_launches;
    }
    StepArgs a = patch_args(p, dt);
    if (part != 0) {
        a.H = H;
        a.nstrips = ns;
        if (part == 1) {  // row blocks 1 .. b_hi
            a.tile_offset = ns;
            a.tile_count = ns * b_hi;
        } else {          // row block 0 and b_hi+1 .. nb-1
            a.tile_jump_at = ns;
            a.tile_jump = ns * b_hi;
            a.tile_count = ns * (nb - b_hi);
        }
        if (part == 1 && p->timing) CUDA_TRY(cudaEventRecord(p->ev0, p->st));
        dispatch<UnsplitF>(p->d.riemann, a, p->st, p->has_tmap ? &p->tmap[p->cur] : nullptr);
        ++p->step_launches;
        if (part == 2 && p->timing) CUDA_TRY(cudaEventRecord(p->ev1, p->st));
        CUDA_TRY(cudaGetLastError());
        if (part == 2) p->pending = true;
        return CLAW2_OK;
    }
    const bool exact_unsplit = p->d.riemann == CLAW2_RP_EULER_EXACT && !p->d.dimensional_split;
    if (exact_unsplit && p->exact_guess == 1) {
        // converged pressures as guesses, outside the timed region: the step
        // kernel's time with them is the floor for any guess
        dim3 grid((p->L.mx + 4 + 31) / 32, (p->L.my + 4 + 3) / 4);
        k_exact_pstar_guess<<<grid, 128, 0, p->st>>>(qc, p->L, p->rp.c[0], p->rp.c[1], p->exact_guess_err,
                                                     p->guess);
        a.guess = p->guess;
        ++p->step_launches;
    }
    if (p->timing) CUDA_TRY(cudaEventRecord(p->ev0, p->st));
    if (exact_unsplit && p->mlp && p->exact_guess == 0) {
        mlp_guess_launch(p->mlp, qc, p->L, p->rp.c[0], p->guess, p->status, p->st);
        a.guess = p->guess;
        ++p->step_launches;
    }
    int lpt_n = 0;
    if (p->d.dimensional_split) {
        StepArgs ax = a, ay = a;
        ax.qnew = p->tmp;
        ay.qold = p->tmp;
        dispatch<SplitF>(p->d.riemann, ax, ay, p->st, 3);
        p->step_launches += 2;
    } else {
        // a schedule only matters when the tiles outnumber the CTA slots (2 per SM)
        if (ns * nb > 2 * p->nsm && lpt_prepare(p, ns * nb, H) == CLAW2_OK) {
            lpt_n = ns * nb;
            a.H = H;
            a.nstrips = ns;
            a.tile_order = p->tile_order;
            a.tile_cost = p->tile_cost;
        }
        dispatch<UnsplitF>(p->d.riemann, a, p->st, p->has_tmap ? &p->tmap[p->cur] : nullptr);
        ++p->step_launches;
    }
    if (p->timing) CUDA_TRY(cudaEventRecord(p->ev1, p->st));
    if (lpt_n > 0 && (p->tile_steps++ % LPT_EVERY) == 0) {
        launch_lpt(p->tile_cost, p->tile_order, lpt_n, p->st);
        ++p->step_launches;
    }
    CUDA_TRY(cudaGetLastError());
    p->pending = true;
    return CLAW2_OK;
}

// ---------------------------------------------------------------------------
// Device-resident time loop (claw2_patch_evolve)
// ---------------------------------------------------------------------------
// get_dt of the reference's loop (src/pyclaw/solver.py:524-552) on the loop
// state, with Python's min/max tie rules (same values), then dt/dx, dt/dy.
__host__ __device__ inline void evolve_get_dt(EvolveDev& e) {
    if (e.dt_variable && e.dt_old_set) {
        if (e.cfl > 0.0) {
            const double x = e.dt * e.cfl_desired / e.cfl;
            e.dt = (x < e.dt_max) ? x : e.dt_max;             // min(dt_max, x)
            e.dtmin = (e.dtmin < e.dt) ? e.dtmin : e.dt;      // min(dt, dtmin)
            e.dtmax = (e.dtmax > e.dt) ? e.dtmax : e.dt;      // max(dt, dtmax)
        } else {
            e.dt = e.dt_max;
        }
    } else {
        e.dt_old_set = 1;
    }
    if (e.t + e.dt > e.tend && e.tstart < e.tend) e.dt = e.tend - e.t;
    if (e.tend - e.t - e.dt < 1.e-14 * e.t) e.dt = e.tend - e.t;
    e.dtdx = e.dt / e.dx;
    e.dtdy = e.dt / e.dy;
}

// After one step of the loop (one thread): the reference's accept/reject
// (solver.py:554-666): accept when cfl <= cfl_max (t += dt, or t = tstart +
// (n + 1) dt with a fixed dt); a rejected step keeps t and is restored by
// k_evolve_restore (a fixed dt ends the loop with cfl_error); the loop is
// done when t >= tend, after max_steps attempts, or when the step produced a
// non-finite value (fault, the step restored); otherwise the next dt.
static __global__ void k_evolve_finalize(EvolveDev* e, const unsigned long long* cfl_bits, const int* status) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || e->done) return;
    const double cfl = __longlong_as_double((long long)*cfl_bits);
    const int n = e->attempts;
    e->attempts = n + 1;
    e->cfl = cfl;
    const int st = *status & 3;
    if (st) {
        e->fault = st;
        e->reject = 1;
        e->done = 1;
        return;
    }
    if (!(cfl > e->cfl_max)) {
        e->cflmax = (e->cflmax > cfl) ? e->cflmax : cfl;  // max(cfl, cflmax)
        e->t = e->dt_variable ? __dadd_rn(e->t, e->dt) : __dadd_rn(e->tstart, __dmul_rn((double)(n + 1), e->dt));
        e->num_steps += 1;
        e->reject = 0;
    } else {
        e->reject = 1;
        if (!e->dt_variable) {
            e->cflmax = (e->cflmax > cfl) ? e->cflmax : cfl;
            e->cfl_error = 1;
            e->done = 1;
            return;
        }
    }
    if (e->t >= e->tend || e->attempts >= e->max_steps) {
        e->done = 1;
        return;
    }
    evolve_get_dt(*e);
}

// A rejected step: the state it started from continues in the other buffer.
static __global__ void k_evolve_restore(const EvolveDev* e, const double* __restrict__ from, double* __restrict__ to,
                                        long long n) {
    if (!e->reject) return;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        to[k] = from[k];
}

// One attempt of the loop from buffer c: ghost fill, step into buffer 1-c
// with the loop's dt, finalize, restore on reject.
int evolve_enqueue_attempt(claw2_patch* p, int c) {
    double* qc = p->q[c];
    launch_bc(qc, p->L, p->d.num_eqn, p->d.bc_lower, p->d.bc_upper, p->cfl, p->st);
    StepArgs a = patch_args(p, 0.0);
    a.qold = p->q[c];
    a.qnew = p->q[c ^ 1];
    a.evo = p->evo;
    if (p->d.riemann == CLAW2_RP_EULER_EXACT && p->mlp && !p->d.dimensional_split) {
        mlp_guess_launch(p->mlp, qc, p->L, p->rp.c[0], p->guess, p->status, p->st);
        a.guess = p->guess;
    }
    int lpt_n = 0;
    if (p->d.dimensional_split) {
        StepArgs ax = a, ay = a;
        ax.qnew = p->tmp;
        ay.qold = p->tmp;
        dispatch<SplitF>(p->d.riemann, ax, ay, p->st, 3);
    } else {
        int ns, H, nb;
        unsplit_tiling(p->d.riemann, p->L.mx, p->L.my, ns, H, nb);
        if (ns * nb > 2 * p->nsm && lpt_prepare(p, ns * nb, H) == CLAW2_OK) {
            lpt_n = ns * nb;
            a.H = H;
            a.nstrips = ns;
            a.tile_order = p->tile_order;
            a.tile_cost = p->tile_cost;
        }
        dispatch<UnsplitF>(p->d.riemann, a, p->st, p->has_tmap ? &p->tmap[c] : nullptr);
    }
    if (lpt_n > 0 && (p->tile_steps++ % LPT_EVERY) == 0) launch_lpt(p->tile_cost, p->tile_order, lpt_n, p->st);
    k_evolve_finalize<<<1, 32, 0, p->st>>>(p->evo, p->cfl, p->status);
    const long long n = (long long)p->d.num_eqn * p->L.plane;
    // grid-stride copy on a few blocks per SM: accepted attempts (almost all)
    // leave it at once, so its launch stays short
    const int rb = (int)std::max<long long>(1, std::min<long long>(grid_blocks(n), 4LL * p->nsm));
    k_evolve_restore<<<rb, 256, 0, p->st>>>(p->evo, p->q[c], p->q[c ^ 1], n);
    CUDA_TRY(cudaGetLastError());
    return CLAW2_OK;
}

// Buffers of claw2_patch_run_host: a copy stream, two input and two output
// staging buffers, their events and the per-step CFL words.
int host_pipe_reserve(claw2_patch* p, int nsteps) {
    const size_t n = (size_t)p->d.num_eqn * p->d.mx * p->d.my;
    if (!p->cst) {
        bool ok = cudaStreamCreateWithFlags(&p->cst, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&p->dst, cudaStreamNonBlocking) == cudaSuccess;
        for (int i = 0; i < 2 && ok; ++i)
            ok = cudaMalloc(&p->stage_in[i], n * 8) == cudaSuccess &&
                 cudaEventCreateWithFlags(&p->h2d_done[i], cudaEventDisableTiming) == cudaSuccess &&
                 cudaEventCreateWithFlags(&p->in_free[i], cudaEventDisableTiming) == cudaSuccess &&
                 cudaEventCreateWithFlags(&p->out_ready[i], cudaEventDisableTiming) == cudaSuccess &&
                 cudaEventCreateWithFlags(&p->out_free[i], cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaMalloc(&p->stage_out1, n * 8) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            return fail(CLAW2_ENOMEM, "staging buffers for the host pipeline could not be allocated");
        }
    }
    if (nsteps > p->cfl_hist_cap) {
        cudaFree(p->cfl_hist);
        cudaFreeHost(p->h_cfl_hist);
        p->cfl_hist = nullptr;
        p->h_cfl_hist = nullptr;
        p->cfl_hist_cap = 0;
        if (cudaMalloc(&p->cfl_hist, sizeof(unsigned long long) * nsteps) != cudaSuccess ||
            cudaMallocHost(&p->h_cfl_hist, sizeof(unsigned long long) * nsteps) != cudaSuccess) {
            cudaGetLastError();
            return fail(CLAW2_ENOMEM, "CFL history of %d steps could not be allocated", nsteps);
        }
        p->cfl_hist_cap = nsteps;
    }
    return CLAW2_OK;
}

}  // namespace

extern "C" {

int claw2_patch_step(claw2_patch* p, double dt, double* cfl) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    if (p->split_part == 1) return fail(CLAW2_EINVAL, "part 1 of a split step is enqueued: finish it with part 2");
    if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(CLAW2_EINVAL, "dt must be finite and >= 0");
    DeviceGuard g(p->device);
    const int rc = patch_enqueue_step(p, dt);
    if (rc) return rc;
    if (cfl) return claw2_patch_cfl(p, cfl);
    return CLAW2_OK;
}

int claw2_patch_step_part(claw2_patch* p, double dt, int part, double* cfl) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    if (part != 1 && part != 2) return fail(CLAW2_EINVAL, "part must be 1 or 2 (got %d)", part);
    if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(CLAW2_EINVAL, "dt must be finite and >= 0");
    if (p->pending) return fail(CLAW2_EINVAL, "a step is pending: accept or reject it first");
    if (part == 2 && p->split_part != 1) return fail(CLAW2_EINVAL, "part 2 must follow part 1 of the same step");
    if (part == 1 && p->split_part == 1) return fail(CLAW2_EINVAL, "part 1 of this step is already enqueued");
    DeviceGuard g(p->device);
    const int rc = patch_enqueue_step(p, dt, part);
    if (rc) {
        p->split_part = 0;
        return rc;
    }
    p->split_part = part == 1 ? 1 : 0;
    if (part == 2 && cfl) return claw2_patch_cfl(p, cfl);
    return CLAW2_OK;
}

int claw2_patch_evolve(claw2_patch* p, claw2_evolve_state* s) {
    if (!p || !s) return fail(CLAW2_EINVAL, "null pointer argument");
    if (p->pending) return fail(CLAW2_EINVAL, "a step is pending: accept or reject it first");
    if (p->ghosts_supplied)
        return fail(CLAW2_EINVAL, "host-filled ghost cells (custom BCs) need the host at every step");
    if (s->max_steps < 0) return fail(CLAW2_EINVAL, "max_steps must be >= 0");
    if (!std::isfinite(s->t) || !std::isfinite(s->tend) || !std::isfinite(s->dt) || !(s->dt >= 0.0))
        return fail(CLAW2_EINVAL, "t, tend and dt must be finite, dt >= 0");
    s->num_steps = 0;
    s->attempts = 0;
    s->cfl_error = 0;
    if (s->max_steps == 0) return CLAW2_OK;
    DeviceGuard g(p->device);
    if (!p->evo) {
        if (cudaMalloc(&p->evo, sizeof(EvolveDev)) != cudaSuccess ||
            cudaMallocHost(&p->h_evo, sizeof(EvolveDev)) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(p->evo);
            p->evo = nullptr;
            return fail(CLAW2_ENOMEM, "time-loop state could not be allocated");
        }
    }
    EvolveDev& e = *p->h_evo;
    std::memset(&e, 0, sizeof e);
    e.t = s->t;
    e.tstart = s->tstart;
    e.tend = s->tend;
    e.dt = s->dt;
    e.cfl = s->cfl;
    e.cfl_desired = s->cfl_desired;
    e.cfl_max = s->cfl_max;
    e.dt_max = s->dt_max;
    e.dtmin = s->dtmin;
    e.dtmax = s->dtmax;
    e.cflmax = s->cflmax;
    e.dx = p->d.dx;
    e.dy = p->d.dy;
    e.dt_variable = s->dt_variable ? 1 : 0;
    e.dt_old_set = s->dt_old_set ? 1 : 0;
    e.max_steps = s->max_steps;
    evolve_get_dt(e);  // the first attempt's dt
    CUDA_TRY(cudaMemcpyAsync(p->evo, p->h_evo, sizeof(EvolveDev), cudaMemcpyHostToDevice, p->st));
    CUDA_TRY(cudaMemsetAsync(p->status, 0, sizeof(int), p->st));
    const int cur0 = p->cur;
    long long issued = 0;
    int chunk = 4;
    // After the first chunk (issued directly: it also sets up launch attributes
    // and schedule buffers) four attempts are captured as one CUDA graph and
    // replayed: four attempts return to the same buffer parity, so the same
    // graph serves every later chunk, and the host no longer pays one launch
    // per kernel.  The graph is kept for the next call from the same parity
    // while nothing it captured has changed.  Any capture failure falls back
    // to direct launches.
    cudaGraphExec_t exec = nullptr;
    constexpr int GRAPH_ATTEMPTS = 4;
    bool try_graph = true;
    int rc = CLAW2_OK;
    for (;;) {
        if (issued > 0 && try_graph && !exec) {
            try_graph = false;
            const int c = (int)((cur0 + issued) & 1);
            const unsigned long long stamp =
                ((unsigned long long)p->graph_gen << 32) | (unsigned long long)g_tune_gen.load();
            if (p->evo_exec[c] && p->evo_stamp[c] == stamp) {
                exec = p->evo_exec[c];
            } else if (cudaStreamBeginCapture(p->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                cudaGraph_t graph = nullptr;
                int crc = CLAW2_OK;
                for (int j = 0; j < GRAPH_ATTEMPTS && crc == CLAW2_OK; ++j) crc = evolve_enqueue_attempt(p, (c + j) & 1);
                const cudaError_t ec = cudaStreamEndCapture(p->st, &graph);
                if (crc != CLAW2_OK || ec != cudaSuccess || !graph ||
                    cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
                    cudaGetLastError();
                    exec = nullptr;
                }
                if (graph) cudaGraphDestroy(graph);
                if (exec) {
                    if (p->evo_exec[c]) cudaGraphExecDestroy(p->evo_exec[c]);
                    p->evo_exec[c] = exec;
                    p->evo_stamp[c] = stamp;
                }
            } else {
                cudaGetLastError();
            }
        }
        if (exec) {
            for (int j = 0; j < chunk; j += GRAPH_ATTEMPTS, issued += GRAPH_ATTEMPTS)
                if (cudaGraphLaunch(exec, p->st) != cudaSuccess) {
                    rc = fail(CLAW2_ECUDA, "graph launch of the time loop failed");
                    break;
                }
        } else {
            for (int j = 0; j < chunk && rc == CLAW2_OK; ++j, ++issued)
                rc = evolve_enqueue_attempt(p, (int)((cur0 + issued) & 1));
        }
        if (rc == CLAW2_OK) {
            if (cudaMemcpyAsync(p->h_evo, p->evo, sizeof(EvolveDev), cudaMemcpyDeviceToHost, p->st) != cudaSuccess ||
                cudaStreamSynchronize(p->st) != cudaSuccess)
                rc = fail(CLAW2_ECUDA, "reading the time loop's state failed");
        }
        if (rc != CLAW2_OK || e.done) break;
        if (issued > (long long)s->max_steps + 128) {  // the loop marks itself done after max_steps attempts
            rc = fail(CLAW2_ECUDA, "the device time loop did not finish");
            break;
        }
        chunk = std::min(chunk * 2, 64);
    }
    if (rc != CLAW2_OK) return rc;
    p->cur = (cur0 + e.attempts) & 1;
    s->t = e.t;
    s->dt = e.dt;
    s->cfl = e.cfl;
    s->dtmin = e.dtmin;
    s->dtmax = e.dtmax;
    s->cflmax = e.cflmax;
    s->dt_old_set = e.dt_old_set;
    s->num_steps = e.num_steps;
    s->attempts = e.attempts;
    s->cfl_error = e.cfl_error;
    if (e.fault) {
        cudaMemsetAsync(p->status, 0, sizeof(int), p->st);
        if (e.fault & 2) return fail(CLAW2_ETIMEOUT, "a TMA row copy did not complete within the kernel's wait bound");
        return fail(CLAW2_ENONFINITE, "the step produced a non-finite value");
    }
    return CLAW2_OK;
}

int claw2_patch_run_host(claw2_patch* p, int nsteps, const double* const* q_in, double* const* q_out,
                         const double* dt, double* cfl_out) {
    if (!p || !q_in || !q_out || !dt || !cfl_out || nsteps < 1) return fail(CLAW2_EINVAL, "bad arguments");
    for (int k = 0; k < nsteps; ++k) {
        if (!q_in[k] || !q_out[k]) return fail(CLAW2_EINVAL, "null buffer for step %d", k);
        if (!(dt[k] >= 0.0) || !std::isfinite(dt[k])) return fail(CLAW2_EINVAL, "dt[%d] must be finite and >= 0", k);
    }
    DeviceGuard g(p->device);
    int rc = host_pipe_reserve(p, nsteps);
    if (rc) return rc;
    const size_t n = (size_t)p->d.num_eqn * p->d.mx * p->d.my;
    const long long cells = (long long)p->d.mx * p->d.my;
    double* stage_out[2] = {p->stage, p->stage_out1};
    // all staging buffers start free; the first input goes up at once
    for (int i = 0; i < 2; ++i) {
        CUDA_TRY(cudaEventRecord(p->in_free[i], p->st));
        CUDA_TRY(cudaEventRecord(p->out_free[i], p->st));
    }
    CUDA_TRY(cudaStreamWaitEvent(p->cst, p->in_free[0], 0));
    CUDA_TRY(cudaMemcpyAsync(p->stage_in[0], q_in[0], n * 8, cudaMemcpyHostToDevice, p->cst));
    CUDA_TRY(cudaEventRecord(p->h2d_done[0], p->cst));
    for (int k = 0; k < nsteps; ++k) {
        const int s = k & 1;
        if (k + 1 < nsteps) {  // next input on the copy stream while this step computes
            const int s1 = (k + 1) & 1;
            CUDA_TRY(cudaStreamWaitEvent(p->cst, p->in_free[s1], 0));
            CUDA_TRY(cudaMemcpyAsync(p->stage_in[s1], q_in[k + 1], n * 8, cudaMemcpyHostToDevice, p->cst));
            CUDA_TRY(cudaEventRecord(p->h2d_done[s1], p->cst));
        }
        CUDA_TRY(cudaStreamWaitEvent(p->st, p->h2d_done[s], 0));
        k_aos_to_planes<<<grid_blocks(cells), 256, 0, p->st>>>(p->stage_in[s], p->q[p->cur], p->L, p->d.num_eqn, 0);
        CUDA_TRY(cudaEventRecord(p->in_free[s], p->st));
        rc = patch_enqueue_step(p, dt[k]);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(p->cfl_hist + k, p->cfl, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                 p->st));
        p->cur ^= 1;  // accepted
        p->pending = false;
        // the result goes down on the download stream while the next step computes
        CUDA_TRY(cudaStreamWaitEvent(p->st, p->out_free[s], 0));
        k_planes_to_aos<<<grid_blocks(cells), 256, 0, p->st>>>(p->q[p->cur], stage_out[s], p->L, p->d.num_eqn, 0);
        CUDA_TRY(cudaEventRecord(p->out_ready[s], p->st));
        CUDA_TRY(cudaStreamWaitEvent(p->dst, p->out_ready[s], 0));
        CUDA_TRY(cudaMemcpyAsync(q_out[k], stage_out[s], n * 8, cudaMemcpyDeviceToHost, p->dst));
        CUDA_TRY(cudaEventRecord(p->out_free[s], p->dst));
    }
    CUDA_TRY(cudaMemcpyAsync(p->h_cfl_hist, p->cfl_hist, sizeof(unsigned long long) * nsteps,
                             cudaMemcpyDeviceToHost, p->st));
    CUDA_TRY(cudaMemcpyAsync(p->h_status, p->status, sizeof(int), cudaMemcpyDeviceToHost, p->st));
    CUDA_TRY(cudaStreamSynchronize(p->st));
    CUDA_TRY(cudaStreamSynchronize(p->cst));
    CUDA_TRY(cudaStreamSynchronize(p->dst));
    // later work on the patch's stream must not overtake the last download
    CUDA_TRY(cudaStreamWaitEvent(p->st, p->out_free[(nsteps - 1) & 1], 0));
    for (int k = 0; k < nsteps; ++k) std::memcpy(&cfl_out[k], &p->h_cfl_hist[k], sizeof(double));
    if (*p->h_status & 2) {
        cudaMemsetAsync(p->status, 0, sizeof(int), p->st);
        return fail(CLAW2_ETIMEOUT, "a TMA row copy did not complete within the kernel's wait bound");
    }
    if (*p->h_status & 1) {
        cudaMemsetAsync(p->status, 0, sizeof(int), p->st);
        return fail(CLAW2_ENONFINITE, "a step produced a non-finite value");
    }
    return CLAW2_OK;
}

int claw2_patch_accept(claw2_patch* p, int accept) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    if (!p->pending) return fail(CLAW2_EINVAL, "no pending step to accept or reject");
    if (accept) p->cur ^= 1;
    p->pending = false;
    return CLAW2_OK;
}

int claw2_patch_cfl(claw2_patch* p, double* cfl) {
    if (!p || !cfl) return fail(CLAW2_EINVAL, "null pointer argument");
    DeviceGuard g(p->device);
    CUDA_TRY(cudaMemcpyAsync(p->h_cfl, p->cfl, sizeof(unsigned long long), cudaMemcpyDeviceToHost, p->st));
    CUDA_TRY(cudaMemcpyAsync(p->h_status, p->status, sizeof(int), cudaMemcpyDeviceToHost, p->st));
    CUDA_TRY(cudaStreamSynchronize(p->st));
    double c;
    std::memcpy(&c, p->h_cfl, sizeof c);
    *cfl = c;
    if (*p->h_status & 2) {
        cudaMemsetAsync(p->status, 0, sizeof(int), p->st);
        return fail(CLAW2_ETIMEOUT, "a TMA row copy did not complete within the kernel's wait bound");
    }
    if (*p->h_status & 1) {
        cudaMemsetAsync(p->status, 0, sizeof(int), p->st);
        return fail(CLAW2_ENONFINITE, "the step produced a non-finite value");
    }
    return CLAW2_OK;
}

int claw2_patch_sync(claw2_patch* p) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    DeviceGuard g(p->device);
    CUDA_TRY(cudaMemcpyAsync(p->h_status, p->status, sizeof(int), cudaMemcpyDeviceToHost, p->st));
    CUDA_TRY(cudaStreamSynchronize(p->st));
    if (*p->h_status & 2) {
        cudaMemsetAsync(p->status, 0, sizeof(int), p->st);
        return fail(CLAW2_ETIMEOUT, "a TMA row copy did not complete within the kernel's wait bound");
    }
    if (*p->h_status & 1) {
        cudaMemsetAsync(p->status, 0, sizeof(int), p->st);
        return fail(CLAW2_ENONFINITE, "a step produced a non-finite value");
    }
    return CLAW2_OK;
}

int claw2_patch_set_stream(claw2_patch* p, void* stream) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    DeviceGuard g(p->device);
    CUDA_TRY(cudaStreamSynchronize(p->st));
    p->st = stream ? (cudaStream_t)stream : p->own_st;
    return CLAW2_OK;
}

int claw2_patch_set_timing(claw2_patch* p, int on) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    DeviceGuard g(p->device);
    if (on && !p->ev0) {
        CUDA_TRY(cudaEventCreate(&p->ev0));
        CUDA_TRY(cudaEventCreate(&p->ev1));
    }
    p->timing = on != 0;
    return CLAW2_OK;
}

int claw2_patch_kernel_ms(claw2_patch* p, float* ms) {
    if (!p || !ms) return fail(CLAW2_EINVAL, "null pointer argument");
    if (!p->timing) return fail(CLAW2_EINVAL, "timing is off (claw2_patch_set_timing)");
    DeviceGuard g(p->device);
    CUDA_TRY(cudaEventSynchronize(p->ev1));
    CUDA_TRY(cudaEventElapsedTime(ms, p->ev0, p->ev1));
    return CLAW2_OK;
}

int claw2_probe_fp64(int device, double* tflops) {
    if (!tflops) return fail(CLAW2_EINVAL, "null pointer argument");
    DeviceGuard g(device);
    int nsm = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    const int blocks = nsm * 8, threads = 256, iters = 4096;
    double* out = nullptr;
    CUDA_TRY(cudaMalloc(&out, sizeof(double) * blocks * threads));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fp64_fma<<<blocks, threads>>>(out, iters, 1.0000001);  // warm-up
    cudaEventRecord(e0);
    k_fp64_fma<<<blocks, threads>>>(out, iters, 1.0000001);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return fail(CLAW2_ECUDA, "fp64 probe failed: %s", cudaGetErrorString(e));
    const double flops = 2.0 * 16.0 * iters * (double)blocks * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return CLAW2_OK;
}

int claw2_selftest_rcp(int device, int n, unsigned long long seed, double* max_ulp) {
    if (!max_ulp) return fail(CLAW2_EINVAL, "null pointer argument");
    if (n < 1) return fail(CLAW2_EINVAL, "n must be positive (got %d)", n);
    DeviceGuard g(device);
    unsigned long long* worst = nullptr;
    CUDA_TRY(cudaMalloc(&worst, sizeof(unsigned long long)));
    cudaMemset(worst, 0, sizeof(unsigned long long));
    k_selftest_rcp<<<(n + 255) / 256, 256>>>(n, seed, worst);
    unsigned long long h = 0;
    cudaError_t e = cudaMemcpy(&h, worst, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(worst);
    if (e != cudaSuccess) return fail(CLAW2_ECUDA, "reciprocal self-test failed: %s", cudaGetErrorString(e));
    *max_ulp = (double)h;
    return CLAW2_OK;
}

}  // extern "C"

namespace {
// one seeded self-test kernel over n values; *max_ulp = its largest distance
int run_selftest(void (*kernel)(int, unsigned long long, unsigned long long*), const char* what, int device, int n,
                 unsigned long long seed, double* max_ulp) {
    if (!max_ulp) return fail(CLAW2_EINVAL, "null pointer argument");
    if (n < 1) return fail(CLAW2_EINVAL, "n must be positive (got %d)", n);
    DeviceGuard g(device);
    unsigned long long* worst = nullptr;
    CUDA_TRY(cudaMalloc(&worst, sizeof(unsigned long long)));
    cudaMemset(worst, 0, sizeof(unsigned long long));
    kernel<<<(n + 255) / 256, 256>>>(n, seed, worst);
    unsigned long long h = 0;
    cudaError_t e = cudaMemcpy(&h, worst, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(worst);
    if (e != cudaSuccess) return fail(CLAW2_ECUDA, "%s self-test failed: %s", what, cudaGetErrorString(e));
    *max_ulp = (double)h;
    return CLAW2_OK;
}
}  // namespace

extern "C" {

int claw2_selftest_sqrt(int device, int n, unsigned long long seed, double* max_ulp) {
    return run_selftest(k_selftest_sqrt, "square-root", device, n, seed, max_ulp);
}

int claw2_selftest_rsqrt(int device, int n, unsigned long long seed, double* max_ulp) {
    return run_selftest(k_selftest_rsqrt, "reciprocal square-root", device, n, seed, max_ulp);
}

int claw2_selftest_lpt(int device, int n, unsigned long long seed, int* mismatches) {
    if (!mismatches) return fail(CLAW2_EINVAL, "null pointer argument");
    if (n < 1 || n > LPT_MAX_TILES) return fail(CLAW2_EINVAL, "n must be 1..%d (got %d)", LPT_MAX_TILES, n);
    DeviceGuard g(device);
    // costs with many ties (a few dozen distinct values) from a 64-bit LCG
    std::vector<unsigned int> cost(n);
    unsigned long long z = seed * 2862933555777941757ull + 3037000493ull;
    for (int i = 0; i < n; ++i) {
        z = z * 6364136223846793005ull + 1442695040888963407ull;
        cost[i] = (unsigned int)((z >> 33) % 37u) * 100000u + (unsigned int)((z >> 20) & 1u);
    }
    std::vector<int> want(n), got(n);
    for (int i = 0; i < n; ++i) want[i] = i;
    std::stable_sort(want.begin(), want.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    unsigned int* dc = nullptr;
    int* dord = nullptr;
    if (cudaMalloc(&dc, sizeof(unsigned int) * n) != cudaSuccess || cudaMalloc(&dord, sizeof(int) * n) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(dc);
        return fail(CLAW2_ENOMEM, "self-test buffers");
    }
    cudaError_t e = cudaMemcpy(dc, cost.data(), sizeof(unsigned int) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        launch_lpt(dc, dord, n, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(got.data(), dord, sizeof(int) * n, cudaMemcpyDeviceToHost);
    cudaFree(dc);
    cudaFree(dord);
    if (e != cudaSuccess) return fail(CLAW2_ECUDA, "schedule sort self-test failed: %s", cudaGetErrorString(e));
    int bad = 0;
    for (int i = 0; i < n; ++i) bad += got[i] != want[i];
    *mismatches = bad;
    return CLAW2_OK;
}

int claw2_tune_set(int riemann, int variant, int rows) {
    int me = 0, mw = 0;
    if (rp_shape(riemann, &me, &mw) != 0) return fail(CLAW2_EINVAL, "unknown Riemann solver id %d", riemann);
    if (variant < 0 || (variant > 4 && variant != 8))
        return fail(CLAW2_EINVAL, "variant must be 0..4 or 8 (got %d)", variant);
    if (rows < 0 || rows > 4096) return fail(CLAW2_EINVAL, "rows must be 0..4096 (got %d)", rows);
    g_tune[riemann & (TUNE_SLOTS - 1)].variant = variant;
    g_tune[riemann & (TUNE_SLOTS - 1)].rows = rows;
    ++g_tune_gen;
    return CLAW2_OK;
}

int claw2_tune_get(int riemann, int* variant, int* rows) {
    int me = 0, mw = 0;
    if (rp_shape(riemann, &me, &mw) != 0 || !variant || !rows) return fail(CLAW2_EINVAL, "bad arguments");
    *variant = g_tune[riemann & (TUNE_SLOTS - 1)].variant;
    *rows = g_tune[riemann & (TUNE_SLOTS - 1)].rows;
    return CLAW2_OK;
}

int claw2_patch_launch_count(claw2_patch* p, long long* n) {
    if (!p || !n) return fail(CLAW2_EINVAL, "null pointer argument");
    *n = p->step_launches;
    return CLAW2_OK;
}

int claw2_patch_set_mlp(claw2_patch* p, claw2_mlp* m) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    if (m && p->d.riemann != CLAW2_RP_EULER_EXACT)
        return fail(CLAW2_EINVAL, "learned guesses apply to the exact Euler solver only");
    if (m && m->device != p->device) return fail(CLAW2_EINVAL, "network and patch are on different devices");
    p->mlp = m;
    ++p->graph_gen;
    return CLAW2_OK;
}

int claw2_patch_counters(claw2_patch* p, unsigned long long* out, int reset) {
    if (!p || !out) return fail(CLAW2_EINVAL, "null pointer argument");
    unsigned long long c[3];
    const int rc = claw2_patch_newton_counts(p, c, reset);
    out[0] = c[0];
    out[1] = c[2];
    return rc;
}

int claw2_patch_newton_counts(claw2_patch* p, unsigned long long* out, int reset) {
    if (!p || !out) return fail(CLAW2_EINVAL, "null pointer argument");
    out[0] = out[1] = out[2] = 0;
    if (!p->counters) return CLAW2_OK;
    DeviceGuard g(p->device);
    unsigned long long c[3];
    CUDA_TRY(cudaMemcpyAsync(c, p->counters, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, p->st));
    CUDA_TRY(cudaStreamSynchronize(p->st));
    if (reset) CUDA_TRY(cudaMemsetAsync(p->counters, 0, 3 * sizeof(unsigned long long), p->st));
    out[0] = c[0];  // needed
    out[1] = c[2];  // applied
    out[2] = c[1];  // solves
    return CLAW2_OK;
}

int claw2_patch_set_exact_guess(claw2_patch* p, int mode) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    if (mode != 0 && mode != 1) return fail(CLAW2_EINVAL, "mode must be 0 or 1 (got %d)", mode);
    if (mode && p->d.riemann != CLAW2_RP_EULER_EXACT)
        return fail(CLAW2_EINVAL, "converged guesses apply to the exact Euler solver only");
    if (mode && !p->guess) return fail(CLAW2_EUNSUPPORTED, "this patch has no guess planes");
    p->exact_guess = mode;
    ++p->graph_gen;
    return CLAW2_OK;
}

int claw2_patch_set_exact_guess_error(claw2_patch* p, double rel) {
    if (!p) return fail(CLAW2_EINVAL, "null patch");
    if (!(rel >= 0.0 && rel < 0.5)) return fail(CLAW2_EINVAL, "relative error must be in [0, 0.5) (got %g)", rel);
    p->exact_guess_err = rel;
    ++p->graph_gen;
    return CLAW2_OK;
}

int claw2_patch_device_q(claw2_patch* p, double** q, long long* layout) {
    if (!p || !q || !layout) return fail(CLAW2_EINVAL, "null pointer argument");
    *q = p->q[p->cur];
    layout[0] = p->d.mx + 4;
    layout[1] = p->d.my + 4;
    layout[2] = p->L.pitch;
    layout[3] = p->L.plane;
    return CLAW2_OK;
}

}  // extern "C"

// ===========================================================================
// Batches of independent problems
// ===========================================================================
struct claw2_batch {
    int device = 0;
    int n = 0;
    claw2_desc d0;                   // shared solver / method / BC settings
    std::vector<claw2_desc> descs;
    std::vector<BatchInst> h_inst;
    std::vector<int> order;          // instances by decreasing size
    std::vector<int> tile_first, tile_count;
    std::vector<int2> h_tiles;
    BatchInst* d_inst = nullptr;
    BatchState* d_st = nullptr;
    int2* d_tiles = nullptr;
    double* arena = nullptr;
    double* stage = nullptr;
    size_t stage_doubles = 0;
    RPParams rp;
    Method meth;
    BatchCtl ctl;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    int persistent_grid = 0;
};

namespace {

int batch_build_tiles(claw2_batch* b, const int* rows) {
    constexpr int W = NT_UNSPLIT - 4;
    b->h_tiles.clear();
    b->tile_first.assign(b->n, 0);
    b->tile_count.assign(b->n, 0);
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess || nsm <= 0) nsm = 148;
    for (int i : b->order) {
        BatchInst& in = b->h_inst[i];
        in.nstrips = (in.L.mx + W - 1) / W;
        in.H = (rows && rows[i] > 0) ? rows[i] : pick_rows(in.nstrips, in.L.my, nsm);
        const int nblk = (in.L.my + in.H - 1) / in.H;
        b->tile_first[i] = (int)b->h_tiles.size();
        b->tile_count[i] = in.nstrips * nblk;
        for (int k = 0; k < in.nstrips * nblk; ++k) b->h_tiles.push_back(make_int2(i, k));
    }
    DeviceGuard g(b->device);
    cudaFree(b->d_tiles);
    b->d_tiles = nullptr;
    CUDA_TRY(cudaMalloc(&b->d_tiles, sizeof(int2) * b->h_tiles.size()));
    CUDA_TRY(cudaMemcpy(b->d_tiles, b->h_tiles.data(), sizeof(int2) * b->h_tiles.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(b->d_inst, b->h_inst.data(), sizeof(BatchInst) * b->n, cudaMemcpyHostToDevice));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        b->graph_steps = 0;
    }
    return CLAW2_OK;
}

BatchArgs batch_args(claw2_batch* b) {
    BatchArgs a;
    a.inst = b->d_inst;
    a.st = b->d_st;
    a.tiles = b->d_tiles;
    a.ntiles = (int)b->h_tiles.size();
    a.ninst = b->n;
    a.rp = b->rp;
    a.meth = b->meth;
    a.ctl = b->ctl;
    return a;
}

// Shared-memory opt-in of the batched step kernel; done at batch creation,
// before any graph capture.
template <class RP>
int batch_smem_attr() {
    constexpr int smem = (int)sizeof(UnsplitSmem<RP, NT_UNSPLIT>);
    static unsigned long long attr = 0, attr2 = 0;
    smem_attr(k_batch_step<RP, NT_UNSPLIT, 2, SPEC_ANY>, smem, attr);
    smem_attr(k_batch_step<RP, NT_UNSPLIT, 2, SPEC_MC2>, smem, attr2);
    return smem;
}

template <class RP>
struct BatchStepF {
    static void run(const BatchArgs& a, int first, int count, int grid, cudaStream_t st) {
        constexpr int smem = (int)sizeof(UnsplitSmem<RP, NT_UNSPLIT>);
        if (is_mc2(a.meth, RP::MWAVES))
            k_batch_step<RP, NT_UNSPLIT, 2, SPEC_MC2><<<grid, NT_UNSPLIT, smem, st>>>(a, first, count);
        else
            k_batch_step<RP, NT_UNSPLIT, 2, SPEC_ANY><<<grid, NT_UNSPLIT, smem, st>>>(a, first, count);
    }
};

template <class RP>
struct BatchOccF {
    static void run(int* nb) {
        const int smem = batch_smem_attr<RP>();
        // sized from the generic kernel: both are compiled for 2 blocks per SM,
        // and no CTA of the persistent kernel waits on another
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(nb, k_batch_step<RP, NT_UNSPLIT, 2, SPEC_ANY>, NT_UNSPLIT,
                                                      smem);
    }
};

// One batched step: ghost fill of every instance, the persistent step, finalize.
void batch_step_all(claw2_batch* b) {
    const BatchArgs a = batch_args(b);
    int maxg = 0;
    for (const auto& in : b->h_inst) maxg = std::max(maxg, 4 * (in.L.mx + 4) + 4 * in.L.my);
    dim3 gbc((maxg + 255) / 256, b->n);
    k_batch_bc<<<gbc, 256, 0, b->st>>>(a, 0, b->d0.bc_lower[0], b->d0.bc_lower[1], b->d0.bc_upper[0],
                                      b->d0.bc_upper[1], b->d0.num_eqn);
    dispatch<BatchStepF>(b->d0.riemann, a, 0, a.ntiles, b->persistent_grid, b->st);
    k_batch_finalize<<<(b->n + 127) / 128, 128, 0, b->st>>>(a, 0, b->n);
}

// The same step as one independent launch sequence per instance.
void batch_step_each(claw2_batch* b) {
    const BatchArgs a = batch_args(b);
    for (int i = 0; i < b->n; ++i) {
        const BatchInst& in = b->h_inst[i];
        const int ng = 4 * (in.L.mx + 4) + 4 * in.L.my;
        k_batch_bc<<<dim3((ng + 255) / 256, 1), 256, 0, b->st>>>(a, i, b->d0.bc_lower[0], b->d0.bc_lower[1],
                                                                 b->d0.bc_upper[0], b->d0.bc_upper[1],
                                                                 b->d0.num_eqn);
        dispatch<BatchStepF>(b->d0.riemann, a, b->tile_first[i], b->tile_count[i], b->tile_count[i], b->st);
        k_batch_finalize<<<1, 32, 0, b->st>>>(a, i, 1);
    }
}

}  // namespace

extern "C" {

int claw2_batch_create(const claw2_desc* descs, int n, claw2_batch** out) {
    if (!descs || !out || n < 1) return fail(CLAW2_EINVAL, "bad arguments");
    *out = nullptr;
    const claw2_desc& d0 = descs[0];
    int me = 0, mw = 0;
    if (rp_shape(d0.riemann, &me, &mw) != 0) return fail(CLAW2_EINVAL, "unknown Riemann solver id %d", d0.riemann);
    for (int i = 0; i < n; ++i) {
        const claw2_desc& d = descs[i];
        if (d.riemann != d0.riemann || d.order != d0.order || d.transverse != d0.transverse || d.fwave != d0.fwave ||
            d.dimensional_split || d.num_eqn != me || d.num_waves != mw || d.num_ghost != 2 || d.num_aux != 0 ||
            d.mcapa != 0 ||
            d.device != d0.device || std::memcmp(d.mthlim, d0.mthlim, sizeof d.mthlim) ||
            std::memcmp(d.bc_lower, d0.bc_lower, sizeof d.bc_lower) ||
            std::memcmp(d.bc_upper, d0.bc_upper, sizeof d.bc_upper) || d.ncparam != d0.ncparam ||
            std::memcmp(d.cparam, d0.cparam, sizeof d.cparam))
            return fail(CLAW2_EINVAL, "instance %d: batched instances share solver, method, BCs and parameters "
                                      "(unsplit step only)", i);
        if (d.mx < 2 || d.my < 2 || !(d.dx > 0.0) || !(d.dy > 0.0))
            return fail(CLAW2_EINVAL, "instance %d: bad sizes", i);
    }
    int rc = check_method(d0.riemann, d0.order, d0.transverse, d0.mthlim, mw, d0.fwave);
    if (rc) return rc;
    rc = check_bc(d0.bc_lower, d0.bc_upper, 2, 2);
    if (rc) return rc;

    claw2_batch* b = new claw2_batch();
    b->device = d0.device;
    b->n = n;
    b->d0 = d0;
    b->descs.assign(descs, descs + n);
    b->rp = make_params(d0.riemann, d0.cparam, d0.ncparam);
    b->meth.order = d0.order;
    b->meth.transverse = d0.transverse;
    b->meth.fwave = d0.fwave;
    for (int k = 0; k < CLAW2_MAX_WAVES; ++k) b->meth.mthlim[k] = k < mw ? d0.mthlim[k] : 0;
    b->ctl.cfl_desired = 0.9;
    b->ctl.cfl_max = 1.0;
    b->ctl.dt_max = 1e99;
    b->ctl.tend = 1e99;
    DeviceGuard g(b->device);
    size_t total = 0;
    b->h_inst.resize(n);
    for (int i = 0; i < n; ++i) {
        BatchInst& in = b->h_inst[i];
        in.L = make_layout(descs[i].mx, descs[i].my);
        in.dx = descs[i].dx;
        in.dy = descs[i].dy;
        total += 2 * (size_t)me * in.L.plane;
        b->stage_doubles = std::max(b->stage_doubles, (size_t)me * descs[i].mx * descs[i].my);
    }
    b->order.resize(n);
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
        return (long long)descs[x].mx * descs[x].my > (long long)descs[y].mx * descs[y].my;
    });
    bool ok = cudaMalloc(&b->arena, total * 8) == cudaSuccess &&
              cudaMalloc(&b->stage, b->stage_doubles * 8) == cudaSuccess &&
              cudaMalloc(&b->d_inst, sizeof(BatchInst) * n) == cudaSuccess &&
              cudaMalloc(&b->d_st, sizeof(BatchState) * n) == cudaSuccess &&
              cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreate(&b->e0) == cudaSuccess && cudaEventCreate(&b->e1) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        claw2_batch_destroy(b);
        return fail(CLAW2_ENOMEM, "device allocation for a batch of %d instances failed", n);
    }
    cudaMemset(b->arena, 0, total * 8);
    cudaMemset(b->d_st, 0, sizeof(BatchState) * n);
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        BatchInst& in = b->h_inst[i];
        in.q[0] = b->arena + off;
        off += (size_t)me * in.L.plane;
        in.q[1] = b->arena + off;
        off += (size_t)me * in.L.plane;
    }
    rc = batch_build_tiles(b, nullptr);
    if (rc) {
        claw2_batch_destroy(b);
        return rc;
    }
    int nb = 0, nsm = 0;
    dispatch<BatchOccF>(d0.riemann, &nb);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
    b->persistent_grid = std::max(1, nb) * std::max(1, nsm);
    *out = b;
    return CLAW2_OK;
}

int claw2_batch_destroy(claw2_batch* b) {
    if (!b) return CLAW2_OK;
    {
        DeviceGuard g(b->device);
        if (b->st) cudaStreamSynchronize(b->st);
        if (b->graph) cudaGraphExecDestroy(b->graph);
        cudaFree(b->arena);
        cudaFree(b->stage);
        cudaFree(b->d_inst);
        cudaFree(b->d_st);
        cudaFree(b->d_tiles);
        if (b->e0) cudaEventDestroy(b->e0);
        if (b->e1) cudaEventDestroy(b->e1);
        if (b->st) cudaStreamDestroy(b->st);
    }
    delete b;
    return CLAW2_OK;
}

int claw2_batch_set_rows(claw2_batch* b, const int* rows) {
    if (!b) return fail(CLAW2_EINVAL, "null batch");
    return batch_build_tiles(b, rows);
}

int claw2_batch_upload_q(claw2_batch* b, int i, const double* q) {
    if (!b || !q || i < 0 || i >= b->n) return fail(CLAW2_EINVAL, "bad arguments");
    DeviceGuard g(b->device);
    BatchState s;
    CUDA_TRY(cudaMemcpy(&s, b->d_st + i, sizeof s, cudaMemcpyDeviceToHost));
    const BatchInst& in = b->h_inst[i];
    const size_t n = (size_t)b->d0.num_eqn * in.L.mx * in.L.my;
    CUDA_TRY(cudaMemcpyAsync(b->stage, q, n * 8, cudaMemcpyHostToDevice, b->st));
    k_aos_to_planes<<<grid_blocks((long long)in.L.mx * in.L.my), 256, 0, b->st>>>(b->stage, in.q[s.cur], in.L,
                                                                                  b->d0.num_eqn, 0);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(b->st));
    return CLAW2_OK;
}

int claw2_batch_download_q(claw2_batch* b, int i, double* q) {
    if (!b || !q || i < 0 || i >= b->n) return fail(CLAW2_EINVAL, "bad arguments");
    DeviceGuard g(b->device);
    BatchState s;
    CUDA_TRY(cudaMemcpy(&s, b->d_st + i, sizeof s, cudaMemcpyDeviceToHost));
    const BatchInst& in = b->h_inst[i];
    const size_t n = (size_t)b->d0.num_eqn * in.L.mx * in.L.my;
    k_planes_to_aos<<<grid_blocks((long long)in.L.mx * in.L.my), 256, 0, b->st>>>(in.q[s.cur], b->stage, in.L,
                                                                                  b->d0.num_eqn, 0);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(q, b->stage, n * 8, cudaMemcpyDeviceToHost, b->st));
    CUDA_TRY(cudaStreamSynchronize(b->st));
    return CLAW2_OK;
}

int claw2_batch_set_time(claw2_batch* b, const double* dt0, double t0, double tend, double cfl_desired,
                         double cfl_max, double dt_max) {
    if (!b || !dt0) return fail(CLAW2_EINVAL, "bad arguments");
    if (!(cfl_desired > 0.0) || cfl_desired > cfl_max) return fail(CLAW2_EINVAL, "need 0 < cfl_desired <= cfl_max");
    DeviceGuard g(b->device);
    std::vector<BatchState> s(b->n);
    for (int i = 0; i < b->n; ++i) {
        std::memset(&s[i], 0, sizeof(BatchState));
        s[i].dt = dt0[i];
        s[i].t = t0;
        s[i].done = t0 >= tend;
    }
    CUDA_TRY(cudaStreamSynchronize(b->st));
    // keep the current buffer index of each instance
    std::vector<BatchState> old(b->n);
    CUDA_TRY(cudaMemcpy(old.data(), b->d_st, sizeof(BatchState) * b->n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < b->n; ++i) s[i].cur = old[i].cur;
    CUDA_TRY(cudaMemcpy(b->d_st, s.data(), sizeof(BatchState) * b->n, cudaMemcpyHostToDevice));
    b->ctl.cfl_desired = cfl_desired;
    b->ctl.cfl_max = cfl_max;
    b->ctl.dt_max = dt_max;
    b->ctl.tend = tend;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        b->graph_steps = 0;
    }
    return CLAW2_OK;
}

int claw2_batch_run(claw2_batch* b, int nsteps, int mode, float* ms) {
    if (!b || nsteps < 0 || mode < 0 || mode > 2) return fail(CLAW2_EINVAL, "bad arguments");
    DeviceGuard g(b->device);
    if (mode == 0 && b->graph_steps != nsteps) {
        if (b->graph) cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        cudaGraph_t graph = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < nsteps; ++k) batch_step_all(b);
        CUDA_TRY(cudaStreamEndCapture(b->st, &graph));
        cudaError_t e = cudaGraphInstantiate(&b->graph, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(CLAW2_ECUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
        b->graph_steps = nsteps;
    }
    CUDA_TRY(cudaEventRecord(b->e0, b->st));
    if (mode == 0) {
        CUDA_TRY(cudaGraphLaunch(b->graph, b->st));
    } else if (mode == 1) {
        for (int k = 0; k < nsteps; ++k) batch_step_all(b);
    } else {
        for (int k = 0; k < nsteps; ++k) batch_step_each(b);
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(b->e1, b->st));
    CUDA_TRY(cudaEventSynchronize(b->e1));
    float t = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&t, b->e0, b->e1));
    if (ms) *ms = t;
    return CLAW2_OK;
}

int claw2_batch_get_state(claw2_batch* b, double* t, double* dt, int* nsteps, int* nreject, double* cfl_last,
                          int* status) {
    if (!b) return fail(CLAW2_EINVAL, "null batch");
    DeviceGuard g(b->device);
    std::vector<BatchState> s(b->n);
    CUDA_TRY(cudaStreamSynchronize(b->st));
    CUDA_TRY(cudaMemcpy(s.data(), b->d_st, sizeof(BatchState) * b->n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < b->n; ++i) {
        if (t) t[i] = s[i].t;
        if (dt) dt[i] = s[i].dt;
        if (nsteps) nsteps[i] = s[i].nsteps;
        if (nreject) nreject[i] = s[i].nreject;
        if (cfl_last) cfl_last[i] = s[i].cfl_last;
        if (status) status[i] = s[i].status;
    }
    return CLAW2_OK;
}

int claw2_batch_tiles(claw2_batch* b, int* ntiles, int* persistent_grid) {
    if (!b || !ntiles || !persistent_grid) return fail(CLAW2_EINVAL, "bad arguments");
    *ntiles = (int)b->h_tiles.size();
    *persistent_grid = b->persistent_grid;
    return CLAW2_OK;
}

}  // extern "C"
