// relax_b200.cu -- context API, RK2 driver and operator entry points of the
// B200 relaxation-loop library (C ABI in include/relax_b200.h).
//
// The driver restates the reference's time loop (src/relax.f90:555-890,
// GPU variant src/curelax.f90:447-927) over fused device kernels:
//
//   predictor  [m, Maxwell minima already computed by the previous step's
//               tail kernel]  friction planes -> k_dt (integrationstep on
//               device) -> Green(-div m) with v = u + Dt/2 w fused in the
//               last pass
//   corrector  k_stress<CORR>: sig = -Dt/2 m - tau + C:E(v), m = eigen(sig),
//               gamma += Dt gd -> friction planes, patch monitor ->
//               Green(-div m) with u += Dt w fused in the last pass
//   tail       k_stress<END>: tau += Dt m, sig = -tau + C:E(u), next
//               predictor m = eigen(sig), Maxwell minima, log amplitudes
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "okada.cuh"
#include "zspec_tc.cuh"

using namespace relax;

static thread_local std::string g_err;

static int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

// error reporting for the allocation-free operator of noalloc.cu (not exported)
extern "C" __attribute__((visibility("hidden"))) int relax_noalloc_fail(int code, const char *msg)
{
    g_err = msg;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(RELAX_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,       \
                        cudaGetErrorString(e_));                                          \
    } while (0)

#define CKL()                                                                             \
    do {                                                                                  \
        cudaError_t e_ = cudaGetLastError();                                              \
        if (e_ != cudaSuccess)                                                            \
            return fail(RELAX_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__,          \
                        cudaGetErrorString(e_));                                          \
    } while (0)

// Device memory of the contexts and batches comes from a memory pool of the
// library's own per device (not the device's default pool, which other code
// in the process may tune), which keeps freed memory for the next context:
// creating and destroying a context costs no cudaMalloc / cudaFree once the
// pool is warm.  Allocations and frees are ordered on the legacy default
// stream and made synchronous for the caller (allocations wait for the
// allocation, frees happen only after the owner's streams were synchronized),
// so the buffers behave like cudaMalloc'd ones on every stream.
// The pool keeps freed memory until relax_release_cached_memory trims it.
// Whether a device has a pool is decided once, at its first allocation: if
// the pool cannot be created the device takes plain cudaMalloc / cudaFree
// from then on, so that every buffer is freed the way it was allocated.
static cudaMemPool_t dpool(int device)
{
    static std::mutex mu;
    static std::vector<int> state;             // 0 undecided, 1 pool, -1 plain
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)pools.size() <= device) {
        pools.resize(device + 1, nullptr);
        state.resize(device + 1, 0);
    }
    if (state[device] == 0) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;   // no release to the device between contexts
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            pools[device] = pool;
            state[device] = 1;
        } else {
            cudaGetLastError();
            state[device] = -1;
        }
    }
    return pools[device];
}

template <typename T>
static int dalloc(T **p, size_t n)
{
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    cudaMemPool_t pool = e == cudaSuccess ? dpool(device) : nullptr;
    if (pool) {
        e = cudaMallocFromPoolAsync((void **)p, bytes, pool, 0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    } else {
        e = cudaMalloc((void **)p, bytes);
    }
    if (e != cudaSuccess) return fail(RELAX_ERR_NOMEM, "device allocation of %zu bytes: %s", bytes, cudaGetErrorString(e));
    return RELAX_OK;
}

// Small page-locked host blocks of a context (its step state and time-step
// inputs) from one page-locked slab per process, so that creating a context
// makes no cudaMallocHost call; larger requests, or a full slab, fall back to
// cudaMallocHost.
namespace hpin {
constexpr size_t kBlock = 1024, kBlocks = 512;
std::mutex mu;
char *slab = nullptr;
std::vector<int> free_list;

int alloc(void **p, size_t bytes)
{
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!slab && cudaMallocHost((void **)&slab, kBlock * kBlocks) == cudaSuccess)
            for (int k = (int)kBlocks - 1; k >= 0; k--) free_list.push_back(k);
        if (slab && bytes <= kBlock && !free_list.empty()) {
            *p = slab + kBlock * (size_t)free_list.back();
            free_list.pop_back();
            memset(*p, 0, kBlock);
            return RELAX_OK;
        }
    }
    CK(cudaMallocHost(p, bytes));
    return RELAX_OK;
}

void release(void *p)
{
    if (!p) return;
    std::lock_guard<std::mutex> lock(mu);
    if (slab && (char *)p >= slab && (char *)p < slab + kBlock * kBlocks) {
        free_list.push_back((int)(((char *)p - slab) / kBlock));
        return;
    }
    cudaFreeHost(p);
}
}  // namespace hpin

// frees a dalloc'd buffer once the device is idle (as cudaFree would wait),
// back into the pool; `idle`: the caller has synchronized the device already
static void dfree(void *p, bool idle = false)
{
    if (!p) return;
    int device = 0;
    cudaGetDevice(&device);
    if (!idle) cudaDeviceSynchronize();
    if (dpool(device)) cudaFreeAsync(p, 0);
    else cudaFree(p);
}

extern "C" int relax_release_cached_memory(int device)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return fail(RELAX_ERR_ARG, "relax_release_cached_memory: no device %d", device);
    }
    int cur = 0;
    CK(cudaGetDevice(&cur));
    CK(cudaSetDevice(device));
    cudaError_t e = cudaDeviceSynchronize();
    cudaMemPool_t pool = dpool(device);
    if (e == cudaSuccess && pool) e = cudaMemPoolTrimTo(pool, 0);
    cudaSetDevice(cur);
    if (e != cudaSuccess) return fail(RELAX_ERR_CUDA, "relax_release_cached_memory: %s", cudaGetErrorString(e));
    return RELAX_OK;
}

#define TRY(call)                  \
    do {                               \
        int r_ = (call);               \
        if (r_ != RELAX_OK) return r_; \
    } while (0)

static unsigned nblocks(size_t n, int t = RELAX_NTHREADS) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// FFT plans and twiddle tables
// ---------------------------------------------------------------------------
static bool factor(int n, int *r, int *nr)
{
    int k = 0;
    while (n % 8 == 0 && n > 8) { r[k++] = 8; n /= 8; }
    if (n == 8) { r[k++] = 8; n = 1; }
    while (n % 4 == 0) { r[k++] = 4; n /= 4; }
    while (n % 2 == 0) { r[k++] = 2; n /= 2; }
    while (n % 3 == 0) { r[k++] = 3; n /= 3; }
    *nr = k;
    return n == 1 && k <= 12;
}

static bool fft_size_ok(int n)
{
    int r[16], k;
    return n >= 2 && factor(n, r, &k);
}

// Per-stage device timing: CUDA events recorded around every launch of the
// context's stream while enabled; launches are counted always.
enum Stage {
    ST_STRESS_END = 0, ST_STRESS_CORR, ST_STRESS_INIT, ST_XFWD, ST_YFWD, ST_ZSPEC, ST_YINV, ST_XINV,
    ST_FRICTION, ST_MONITOR, ST_DT, ST_REDUCE, ST_SOURCE, ST_OTHER, ST_COUNT
};
static const char *kStageNames[ST_COUNT] = {
    "k_stress<END>", "k_stress<CORR>", "k_stress<INIT>", "k_xfwd", "k_ypass<fwd>", "k_zspec",
    "k_ypass<inv>", "k_xinv", "k_friction", "k_monitor", "k_dt", "k_reduce_amp", "k_source", "other"};

struct Prof {
    bool on = false;
    long long launches = 0;
    std::vector<cudaEvent_t> pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> recs;
    size_t used = 0;
    cudaEvent_t get()
    {
        if (used == pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            pool.push_back(e);
        }
        return pool[used++];
    }
    void begin(int stage, cudaStream_t st, cudaEvent_t *e0)
    {
        launches++;
        if (!on) return;
        *e0 = get();
        cudaEventRecord(*e0, st);
        recs.push_back({stage, {*e0, nullptr}});
    }
    void end(cudaStream_t st)
    {
        if (!on) return;
        cudaEvent_t e1 = get();
        cudaEventRecord(e1, st);
        recs.back().second.second = e1;
    }
    void reset()
    {
        recs.clear();
        used = 0;
    }
    ~Prof()
    {
        for (auto e : pool) cudaEventDestroy(e);
    }
};

#define TIMED(prof, stage, st, launch)                     \
    do {                                                    \
        cudaEvent_t e0_ = nullptr;                          \
        if (prof) (prof)->begin((stage), (st), &e0_);       \
        launch;                                             \
        CKL();                                              \
        if (prof) (prof)->end(st);                          \
    } while (0)

// register-resident column passes for the lengths they are instantiated for
constexpr int kCW = 16;

// Launch helpers of the register-resident passes.  `nm` members: with
// nm > 1 the argument struct carries a device table (`tab`) with one entry
// per member and the batched instantiation runs all members in one launch
// (the member index is a spare grid dimension).
template <typename K>
static void set_smem(K kern, size_t sm)
{
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
}

// A launch with programmatic dependent launch allowed: the kernel (one that
// enters through pdl_enter) may be scheduled while the previous kernel in the
// stream finishes its last wave, and waits for it before touching memory.
// Errors are left for cudaGetLastError, as with <<< >>>.
template <typename... P, typename... A>
static void launch_pdl(void (*kern)(P...), dim3 grid, dim3 block, size_t sm, cudaStream_t st, const A &...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    (void)cudaLaunchKernelEx(&cfg, kern, args...);
}

template <int N1, int N2, int SIGN>
static void launch_ypass_sign(const YArgs &ya, dim3 grid, size_t sm, int nm, cudaStream_t st)
{
    if (nm > 1) {
        set_smem(k_ypass_reg<N1, N2, kCW, SIGN, true>, sm);
        launch_pdl(k_ypass_reg<N1, N2, kCW, SIGN, true>, dim3(grid.x, nm), kCW * N2, sm, st, ya);
    } else {
        set_smem(k_ypass_reg<N1, N2, kCW, SIGN>, sm);
        launch_pdl(k_ypass_reg<N1, N2, kCW, SIGN>, grid, kCW * N2, sm, st, ya);
    }
}

template <int N1, int N2>
static cudaError_t launch_ypass_reg(const YArgs &ya, int sign, dim3 grid, int nm, cudaStream_t st)
{
    const size_t sm = (size_t)N1 * N2 * kCW * sizeof(float2);
    if (sign < 0) launch_ypass_sign<N1, N2, -1>(ya, grid, sm, nm, st);
    else launch_ypass_sign<N1, N2, +1>(ya, grid, sm, nm, st);
    return cudaGetLastError();
}

static bool ypass_reg(const YArgs &ya, int sign, cudaStream_t st, cudaError_t *e, int nm = 1)
{
    // CW columns per block over the flattened (component, plane, k1) columns
    const size_t ncol = (size_t)3 * (ya.nbody + ya.traction) * ya.g.K1;
    const dim3 grid((unsigned)((ncol + kCW - 1) / kCW));
    switch (ya.g.sx2) {
    case 32: *e = launch_ypass_reg<8, 4>(ya, sign, grid, nm, st); return true;
    case 96: *e = launch_ypass_reg<24, 4>(ya, sign, grid, nm, st); return true;
    case 192: *e = launch_ypass_reg<24, 8>(ya, sign, grid, nm, st); return true;
    case 64: *e = launch_ypass_reg<8, 8>(ya, sign, grid, nm, st); return true;
    case 128: *e = launch_ypass_reg<16, 8>(ya, sign, grid, nm, st); return true;
    case 256: *e = launch_ypass_reg<16, 16>(ya, sign, grid, nm, st); return true;
    case 512: *e = launch_ypass_reg<32, 16>(ya, sign, grid, nm, st); return true;
    default: return false;
    }
}

template <int N1, int N2, bool PRUNED>
static void launch_zspec_pr(const ZArgs &za, dim3 grid, size_t sm, int nm, cudaStream_t st)
{
    if (nm > 1) {
        set_smem(k_zspec_sm<N1, N2, kCW, PRUNED, true>, sm);
        launch_pdl(k_zspec_sm<N1, N2, kCW, PRUNED, true>, dim3(grid.x, nm), kCW * N2, sm, st, za);
    } else {
        set_smem(k_zspec_sm<N1, N2, kCW, PRUNED>, sm);
        launch_pdl(k_zspec_sm<N1, N2, kCW, PRUNED>, grid, kCW * N2, sm, st, za);
    }
}

template <int N1, int N2>
static cudaError_t launch_zspec_reg(const ZArgs &za, dim3 grid, int nm, cudaStream_t st)
{
    const size_t sm = 3 * (size_t)N1 * N2 * kCW * sizeof(float2) + (size_t)N2 * 12 * kCW * sizeof(float) +
                      (size_t)kCW * ZCOL * sizeof(float);
    const bool pruned = 2 * za.nin == za.g.sx3 && 2 * za.nout == za.g.sx3;
    if (pruned) launch_zspec_pr<N1, N2, true>(za, grid, sm, nm, st);
    else launch_zspec_pr<N1, N2, false>(za, grid, sm, nm, st);
    return cudaGetLastError();
}

static bool zspec_reg(const ZArgs &za, dim3 grid, cudaStream_t st, cudaError_t *e, int nm = 1)
{
    switch (za.g.sx3) {
    case 96: *e = launch_zspec_reg<24, 4>(za, grid, nm, st); return true;
    case 64: *e = launch_zspec_reg<8, 8>(za, grid, nm, st); return true;
    case 128: *e = launch_zspec_reg<16, 8>(za, grid, nm, st); return true;
    case 256: *e = launch_zspec_reg<16, 16>(za, grid, nm, st); return true;
    default: return false;
    }
}

template <int N1, int N2, int V>
static void launch_xinv_v(const XiArgs &xi, int nout, size_t sm, int nm, cudaStream_t st)
{
    constexpr int RW = 32;
    if (nm > 1) {
        set_smem(k_xinv_reg<N1, N2, RW, V, true>, sm);
        launch_pdl(k_xinv_reg<N1, N2, RW, V, true>, dim3(xi.g.sx2 / RW, nout, 3 * nm), RW * N2, sm, st, xi);
    } else {
        set_smem(k_xinv_reg<N1, N2, RW, V>, sm);
        launch_pdl(k_xinv_reg<N1, N2, RW, V>, dim3(xi.g.sx2 / RW, nout, 3), RW * N2, sm, st, xi);
    }
}

template <int N1, int N2>
static cudaError_t launch_xinv_reg(const XiArgs &xi, int nout, int nm, cudaStream_t st)
{
    constexpr int RW = 32, N2P = N2 + 1, K1 = N1 * N2 + 1;
    constexpr int RS0 = (N1 * N2P > K1 ? N1 * N2P : K1), RS = RS0 + ((8 - RS0 % 16) + 16) % 16;
    const size_t sm = (size_t)RW * RS * sizeof(float2);
    // 16-byte output rows: float4 epilogue (the members of a batch share the layout)
    bool v4 = xi.rp % 4 == 0 && xi.pp % 4 == 0;
    for (int k = 0; k < 3; k++) {
        v4 = v4 && ((uintptr_t)xi.out[k] % 16 == 0);
        if (xi.base[k]) v4 = v4 && ((uintptr_t)xi.base[k] % 16 == 0);
    }
    if (v4) launch_xinv_v<N1, N2, 4>(xi, nout, sm, nm, st);
    else launch_xinv_v<N1, N2, 2>(xi, nout, sm, nm, st);
    return cudaGetLastError();
}

static bool xinv_reg(const XiArgs &xi, int nout, cudaStream_t st, cudaError_t *e, int nm = 1)
{
    if (xi.g.sx2 % 32) return false;
    // the epilogue moves at least float2: even pitches, 8-byte aligned rows
    if (xi.rp % 2 || xi.pp % 2) return false;
    for (int k = 0; k < 3; k++)
        if ((uintptr_t)xi.out[k] % 8 || (uintptr_t)xi.base[k] % 8) return false;
    switch (xi.g.M) {
    case 32: *e = launch_xinv_reg<8, 4>(xi, nout, nm, st); return true;
    case 96: *e = launch_xinv_reg<24, 4>(xi, nout, nm, st); return true;
    case 64: *e = launch_xinv_reg<8, 8>(xi, nout, nm, st); return true;
    case 128: *e = launch_xinv_reg<16, 8>(xi, nout, nm, st); return true;
    case 256: *e = launch_xinv_reg<16, 16>(xi, nout, nm, st); return true;
    default: return false;
    }
}

template <int XIN, int N1, int N2>
static void launch_xfwd_in(const XfArgs &xa, dim3 grid, size_t sm, int nm, cudaStream_t st)
{
    constexpr int RW = 16;
    if (nm > 1) {
        set_smem(k_xfwd_reg<XIN, N1, N2, RW, true>, sm);
        launch_pdl(k_xfwd_reg<XIN, N1, N2, RW, true>, dim3(grid.x, grid.y, nm), RW * N2, sm, st, xa);
    } else {
        set_smem(k_xfwd_reg<XIN, N1, N2, RW>, sm);
        launch_pdl(k_xfwd_reg<XIN, N1, N2, RW>, grid, RW * N2, sm, st, xa);
    }
}

template <int N1, int N2>
static cudaError_t launch_xfwd_reg(const XfArgs &xa, bool div, dim3 grid, int nm, cudaStream_t st)
{
    constexpr int RW = 16, N2P = N2 + 1, M = N1 * N2;
    constexpr int RS0 = (N1 * N2P > M + 1 ? N1 * N2P : M + 1), RS = RS0 + ((8 - RS0 % 16) + 16) % 16;
    const size_t sm = (size_t)RW * RS * sizeof(float2);
    if (div) launch_xfwd_in<XIN_DIV, N1, N2>(xa, grid, sm, nm, st);
    else launch_xfwd_in<XIN_REAL, N1, N2>(xa, grid, sm, nm, st);
    return cudaGetLastError();
}

static bool xfwd_reg(const XfArgs &xa, bool div, int nplanes, cudaStream_t st, cudaError_t *e, int nm = 1)
{
    // the 7-point filters are applied by k_xfwd alone (grids of the x2
    // filter have no rows of 16 anyway, nor those of the x1 filter a register
    // x pass)
    if (xa.g.sx2 % 16 || (div && (xa.fx.n || xa.fy.n))) return false;
    const dim3 grid(xa.g.sx2 / 16, nplanes);
    switch (xa.g.M) {
    case 32: *e = launch_xfwd_reg<8, 4>(xa, div, grid, nm, st); return true;
    case 96: *e = launch_xfwd_reg<24, 4>(xa, div, grid, nm, st); return true;
    case 64: *e = launch_xfwd_reg<8, 8>(xa, div, grid, nm, st); return true;
    case 128: *e = launch_xfwd_reg<16, 8>(xa, div, grid, nm, st); return true;
    case 256: *e = launch_xfwd_reg<16, 16>(xa, div, grid, nm, st); return true;
    default: return false;
    }
}

// the lengths the register passes are instantiated for
static bool reg_shape(const Grid &g)
{
    return (g.M == 32 || g.M == 64 || g.M == 96 || g.M == 128 || g.M == 256) && g.sx2 % 32 == 0 &&
           (g.sx2 == 32 || g.sx2 == 64 || g.sx2 == 96 || g.sx2 == 128 || g.sx2 == 192 || g.sx2 == 256 ||
            g.sx2 == 512) &&
           (g.sx3 == 64 || g.sx3 == 96 || g.sx3 == 128 || g.sx3 == 256);
}

// the x3 pass with its DFT-64 sub-transforms on the tensor cores: 128-deep
// boxes, pruned transform (the time step's Green's functions)
static bool zspec_tc_ok(const ZArgs &za) { return za.g.sx3 == 128 && za.nin == 64 && za.nout == 64; }

static cudaError_t launch_zspec_tc(const ZArgs &za, int nsm, int *err, const uint4 *tab, cudaStream_t st)
{
    ZtcArgs t{};
    t.z = za;
    t.ncol = za.g.sx2 * za.g.K1;
    t.ntiles = (t.ncol + ZT_COLS - 1) / ZT_COLS;
    t.err = err;
    t.tab = tab;
    set_smem(k_zspec_tc, ZT_SMEM);
    k_zspec_tc<<<std::min(t.ntiles, std::max(1, nsm)), ZT_THREADS, ZT_SMEM, st>>>(t);
    return cudaGetLastError();
}

struct Spectral {
    Prof *prof = nullptr;
    bool use_reg = true;   // register-resident y/z passes where instantiated
    int mixed = 0;         // 1: the x3 pass on the tensor cores where zspec_tc_ok
    int *tc_err = nullptr; // device flag of k_zspec_tc (the context's error word)
    uint4 *ztab = nullptr; // constant operands of k_zspec_tc (set_mixed)
    int nsm = 0;           // SMs of the device (persistent x3 pass)

    // switches the tensor-core x3 pass on (its constant table built once) or off
    int set_mixed(int on, int *err, cudaStream_t st)
    {
        if (on && !ztab) {
            TRY(dalloc(&ztab, ZT_TAB_BYTES / 16));
            k_ztc_tables<<<8, 256, 0, st>>>(ztab);
            CKL();
        }
        mixed = on;
        tc_err = err;
        return RELAX_OK;
    }
    bool yreg = false;
    Grid g{};
    float2 *S = nullptr;
    float2 *tw = nullptr;          // tables for M, sx1, sx2, sx3
    FftPlan pm{}, py{}, pz{};
    const float2 *tw1 = nullptr;
    int rows = 1, twy = 16, twz = 16;
    size_t smx = 0, smy = 0, smz = 0;

    int init(const Grid &gg, cudaStream_t st)
    {
        g = gg;
        {
            int dev = 0;
            CK(cudaGetDevice(&dev));
            CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        }
        int nr;
        if (!factor(g.M, pm.r, &pm.nr) || !factor(g.sx2, py.r, &py.nr) || !factor(g.sx3, pz.r, &pz.nr))
            return fail(RELAX_ERR_UNSUPPORTED, "FFT sizes must be products of 2 and 3 (sx1/2=%d sx2=%d sx3=%d)",
                        g.M, g.sx2, g.sx3);
        (void)nr;
        pm.n = g.M; py.n = g.sx2; pz.n = g.sx3;
        const int ns[4] = {g.M, g.sx1, g.sx2, g.sx3};
        size_t tot = 0;
        for (int i = 0; i < 4; i++) tot += ns[i];
        std::vector<float2> h(tot);
        size_t off[4], o = 0;
        for (int i = 0; i < 4; i++) {
            off[i] = o;
            for (int j = 0; j < ns[i]; j++) {
                const double a = -2.0 * M_PI * (double)j / (double)ns[i];
                h[o + j] = make_float2((float)cos(a), (float)sin(a));
            }
            o += ns[i];
        }
        TRY(dalloc(&tw, tot));
        CK(cudaMemcpyAsync(tw, h.data(), tot * sizeof(float2), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        pm.tw = tw + off[0];
        tw1 = tw + off[1];
        py.tw = tw + off[2];
        pz.tw = tw + off[3];
        TRY(dalloc(&S, 3 * (size_t)(g.sx3 + 1) * g.sx2 * g.K1));
        // tile choices
        rows = 1;
        while (rows * 2 <= std::max(1, 1024 / g.M) && g.sx2 % (rows * 2) == 0) rows *= 2;
        twy = 16;
        while (twy > 1 && 2 * (size_t)g.sx2 * twy * 8 > 96 * 1024) twy /= 2;
        twz = 16;
        while (twz > 1 && 2 * (size_t)g.sx3 * 3 * twz * 8 > 100 * 1024) twz /= 2;
        smx = 2 * (size_t)3 * rows * (g.M + 1) * sizeof(float2);
        smy = 2 * (size_t)g.sx2 * twy * sizeof(float2);
        const int P = RELAX_NTHREADS / twz;
        smz = 2 * (size_t)g.sx3 * 3 * twz * sizeof(float2) + (size_t)P * twz * 6 * sizeof(double) +
              (size_t)twz * 12 * sizeof(float);
        CK(cudaFuncSetAttribute(k_xfwd<XIN_DIV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
        CK(cudaFuncSetAttribute(k_xfwd<XIN_REAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
        CK(cudaFuncSetAttribute(k_xinv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
        CK(cudaFuncSetAttribute(k_ypass<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy));
        CK(cudaFuncSetAttribute(k_ypass<+1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy));
        CK(cudaFuncSetAttribute(k_zspec, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz));
        return RELAX_OK;
    }

    void release(bool idle = false)
    {
        if (S) dfree(S, idle);
        if (tw) dfree(tw, idle);
        if (ztab) dfree(ztab, idle);
        S = nullptr;
        tw = nullptr;
        ztab = nullptr;
    }

    // arguments of the five passes (the caller's parts of `xa` and `xi`
    // kept: the input / epilogue fields)
    XfArgs xargs(XfArgs xa, int nin) const
    {
        xa.g = g; xa.S = S; xa.pm = pm; xa.tw1 = tw1; xa.nin = nin; xa.rows = rows; xa.has_trac = 1;
        xa.scale3 = (float)(g.dx1 * g.dx2 * g.dx3);
        xa.scale2 = (float)(g.dx1 * g.dx2);
        return xa;
    }
    YArgs yargs(int nplanes, int traction, int tile) const { return YArgs{g, S, py, tile, nplanes, traction}; }
    ZArgs zargs(int nin, int nout, double lambda, double mu, double gam, int tile) const
    {
        ZArgs za{};
        za.g = g; za.S = S; za.pz = pz; za.tw = tile; za.nin = nin; za.nout = nout;
        za.ratio1 = (float)((lambda + mu) / (lambda + 2.0 * mu) / mu / (4.0 * M_PI * M_PI));
        za.ratio2 = (float)(mu / (lambda + mu));
        za.lambda = lambda; za.mu = mu; za.gam = gam;
        return za;
    }
    XiArgs xiargs(XiArgs xi) const
    {
        xi.g = g; xi.S = S; xi.pm = pm; xi.tw1 = tw1; xi.rows = rows;
        xi.scale = (float)(2.0 / ((double)g.sx1 * g.dx1 * g.sx2 * g.dx2 * g.sx3 * g.dx3));
        return xi;
    }

    // Green's function: forward (x pass from `xa`), y, z spectral, y inverse,
    // x inverse with the epilogue in `xi`.
    int green(XfArgs xa, bool div, int nin, int nout, XiArgs xi, double lambda, double mu, double gam,
              cudaStream_t st, cudaEvent_t join_before_xinv = nullptr)
    {
        xa = xargs(xa, nin);
        dim3 gx(g.sx2 / rows, nin + 1);
        bool xr0 = false;
        cudaError_t re0 = cudaSuccess;
        if (use_reg) {
            TIMED(prof, ST_XFWD, st, (xr0 = xfwd_reg(xa, div, nin + 1, st, &re0)));
            if (re0 != cudaSuccess) return fail(RELAX_ERR_CUDA, "k_xfwd_reg: %s", cudaGetErrorString(re0));
        }
        if (!xr0) {
            if (div) TIMED(prof, ST_XFWD, st, (k_xfwd<XIN_DIV><<<gx, RELAX_NTHREADS, smx, st>>>(xa)));
            else TIMED(prof, ST_XFWD, st, (k_xfwd<XIN_REAL><<<gx, RELAX_NTHREADS, smx, st>>>(xa)));
        }
        YArgs ya = yargs(nin, 1, twy);
        cudaError_t re = cudaSuccess;
        if (use_reg) {
            TIMED(prof, ST_YFWD, st, (ya.tw = kCW, yreg = ypass_reg(ya, -1, st, &re)));
            if (re != cudaSuccess) return fail(RELAX_ERR_CUDA, "k_ypass_reg: %s", cudaGetErrorString(re));
        }
        if (!use_reg || !yreg) {
            ya.tw = twy;
            TIMED(prof, ST_YFWD, st,
                  (k_ypass<-1><<<dim3((g.K1 + twy - 1) / twy, nin + 1, 3), RELAX_NTHREADS, smy, st>>>(ya)));
        }
        ZArgs za = zargs(nin, nout, lambda, mu, gam, twz);
        bool zr = false;
        if (mixed && tc_err && ztab && zspec_tc_ok(za)) {
            TIMED(prof, ST_ZSPEC, st, (re = launch_zspec_tc(za, nsm, tc_err, ztab, st)));
            if (re != cudaSuccess) return fail(RELAX_ERR_CUDA, "k_zspec_tc: %s", cudaGetErrorString(re));
            zr = true;
        }
        if (use_reg && !zr) {
            TIMED(prof, ST_ZSPEC, st, (zr = zspec_reg(za, dim3((g.sx2 * g.K1 + kCW - 1) / kCW), st, &re)));
            if (re != cudaSuccess) return fail(RELAX_ERR_CUDA, "k_zspec_reg: %s", cudaGetErrorString(re));
        }
        if (!zr) {
            za.tw = twz;
            TIMED(prof, ST_ZSPEC, st, (k_zspec<<<dim3((g.K1 + twz - 1) / twz, g.sx2), RELAX_NTHREADS, smz, st>>>(za)));
        }
        YArgs yb = yargs(nout, 0, twy);
        bool yr2 = false;
        if (use_reg) {
            yb.tw = kCW;
            TIMED(prof, ST_YINV, st, (yr2 = ypass_reg(yb, +1, st, &re)));
            if (re != cudaSuccess) return fail(RELAX_ERR_CUDA, "k_ypass_reg: %s", cudaGetErrorString(re));
        }
        if (!yr2) {
            yb.tw = twy;
            TIMED(prof, ST_YINV, st,
                  (k_ypass<+1><<<dim3((g.K1 + twy - 1) / twy, nout, 3), RELAX_NTHREADS, smy, st>>>(yb)));
        }
        xi = xiargs(xi);
        if (join_before_xinv) CK(cudaStreamWaitEvent(st, join_before_xinv, 0));
        bool xr = false;
        if (use_reg) {
            TIMED(prof, ST_XINV, st, (xr = xinv_reg(xi, nout, st, &re)));
            if (re != cudaSuccess) return fail(RELAX_ERR_CUDA, "k_xinv_reg: %s", cudaGetErrorString(re));
        }
        if (!xr) TIMED(prof, ST_XINV, st, (k_xinv<<<dim3(g.sx2 / rows, nout), RELAX_NTHREADS, smx, st>>>(xi)));
        return RELAX_OK;
    }
};

static int make_grid(Grid &g, int sx1, int sx2, int sx3, double dx1, double dx2, double dx3)
{
    if (sx1 < 8 || sx2 < 2 || sx3 < 4 || (sx1 % 4) || (sx3 % 2))
        return fail(RELAX_ERR_UNSUPPORTED, "grid %dx%dx%d: need sx1 >= 8 and a multiple of 4, even sx3",
                    sx1, sx2, sx3);
    // optimalfilter (src/elastic3d.f90:846-907) has no differentiator for a
    // depth sx3/2 below 5
    if (sx3 / 2 < 5)
        return fail(RELAX_ERR_UNSUPPORTED, "grid %dx%dx%d: the depth sx3/2 must be at least 5", sx1, sx2, sx3);
    if (!fft_size_ok(sx1 / 2) || !fft_size_ok(sx2) || !fft_size_ok(sx3))
        return fail(RELAX_ERR_UNSUPPORTED, "grid %dx%dx%d: FFT lengths must be products of 2 and 3", sx1, sx2, sx3);
    if (!(dx1 > 0 && dx2 > 0 && dx3 > 0)) return fail(RELAX_ERR_ARG, "non-positive sampling");
    g.sx1 = sx1; g.sx2 = sx2; g.sx3 = sx3; g.sx3h = sx3 / 2;
    g.M = sx1 / 2; g.K1 = sx1 / 2 + 1;
    g.dx1 = dx1; g.dx2 = dx2; g.dx3 = dx3;
    g.plane = (size_t)sx1 * sx2;
    g.nh = g.plane * g.sx3h;
    return RELAX_OK;
}

// The differentiator of optimalfilter (src/elastic3d.f90:846-907) along a
// periodic axis of n samples: the 7-point FIR fir7 of src/kernel7.inc scaled
// by 1/dx for 5 <= n <= 14 (the REAL*8 literals of kernel7.inc are
// single-precision constants), else the central difference (n = 0, the
// kernels' k = 0.5/dx).
static Fir7 fir7_of(int n, double dx)
{
    static const float fir7[7] = {8.77856e-01f, -2.81913e-01f, +6.22696e-02f, +2.82441e-02f,
                                  -5.09029e-02f, +4.20471e-02f, -1.59409e-02f};
    Fir7 f{};
    if (n >= 5 && n <= 14) {
        f.n = 7;
        for (int l = 0; l < 7; l++) f.c[l] = (float)((double)fir7[l] / dx);
    }
    return f;
}
static Fir7 fir_x(const Grid &g) { return fir7_of(g.sx1, g.dx1); }
static Fir7 fir_y(const Grid &g) { return fir7_of(g.sx2, g.dx2); }
static bool has_fir(const Grid &g) { return fir_x(g).n || fir_y(g).n; }

// ---------------------------------------------------------------------------
// host helpers: depth structures (src/elastic3d.f90:630-829)
// ---------------------------------------------------------------------------
static int fixr(double v)
{
    double f = floor(v), c = ceil(v);
    return (int)((v - f) > 0.5 ? c : f);
}

extern "C" int relax_viscoelastic_structure(const relax_layer *layers, int nv, double dx3, int sx3,
                                            relax_layer *vs)
{
    if (nv <= 0 || !layers || !vs || sx3 <= 0) return fail(RELAX_ERR_ARG, "invalid structure arguments");
    for (int k = 0; k < sx3; k++) {
        vs[k].z = 0; vs[k].gammadot0 = 0; vs[k].friction = 0.6; vs[k].cohesion = 0;
        vs[k].stressexponent = layers[0].stressexponent; vs[k].Gk = 0;
    }
    double z0 = fixr(layers[0].z / dx3) * dx3, z1 = z0;
    double g0 = 0, p0 = 0, f0 = 0, c0 = 0, k0 = 0, g1 = 0, p1 = 0, f1 = 0, c1 = 0, k1 = 0;
    int i3e = 1;
    for (int k = 0; k < nv; k++) {
        z1 = fixr(layers[k].z / dx3) * dx3;
        if (z1 < z0) return fail(RELAX_ERR_ARG, "invalid mechanical structure: depths must be increasing");
        g1 = layers[k].gammadot0; p1 = layers[k].stressexponent; f1 = layers[k].friction;
        c1 = layers[k].cohesion; k1 = layers[k].Gk;
        if (z1 == z0) {
            i3e = fixr(z1 / dx3 + 1);
        } else {
            const int i3s = fixr(z0 / dx3) + 1;
            i3e = std::min(fixr(z1 / dx3 + 1), sx3);
            for (int i3 = std::max(i3s, 1); i3 <= i3e; i3++) {
                const double z = (i3 - 1.0) * dx3;
                vs[i3 - 1].gammadot0 = ((z - z0) * g1 + (z1 - z) * g0) / (z1 - z0);
                vs[i3 - 1].stressexponent = ((z - z0) * p1 + (z1 - z) * p0) / (z1 - z0);
                vs[i3 - 1].friction = ((z - z0) * f1 + (z1 - z) * f0) / (z1 - z0);
                vs[i3 - 1].cohesion = ((z - z0) * c1 + (z1 - z) * c0) / (z1 - z0);
                vs[i3 - 1].Gk = ((z - z0) * k1 + (z1 - z) * k0) / (z1 - z0);
            }
        }
        z0 = z1; g0 = g1; p0 = p1; f0 = f1; c0 = c1; k0 = k1;
    }
    if (fixr(z1 / dx3) < sx3 - 1)
        for (int i3 = std::max(i3e, 1); i3 <= sx3; i3++) {
            vs[i3 - 1].gammadot0 = (float)g1;   // REAL(...), src/elastic3d.f90:821-825
            vs[i3 - 1].stressexponent = (float)p1;
            vs[i3 - 1].friction = (float)f1;
            vs[i3 - 1].cohesion = (float)c1;
            vs[i3 - 1].Gk = (float)k1;
        }
    return RELAX_OK;
}

extern "C" int relax_tensor_structure(const relax_tensor_layer *layers, int nv, double dx3, int sx3,
                                      relax_tensor_layer *vs)
{
    if (nv <= 0 || !layers || !vs || sx3 <= 0) return fail(RELAX_ERR_ARG, "invalid tensor structure");
    memset(vs, 0, sizeof(relax_tensor_layer) * (size_t)sx3);
    double z0 = fixr(layers[0].z / dx3) * dx3, z1 = z0;
    relax_tensor t0{}, t1{};
    int i3e = 1;
    for (int k = 0; k < nv; k++) {
        z1 = fixr(layers[k].z / dx3) * dx3;
        if (z1 < z0) return fail(RELAX_ERR_ARG, "invalid tensor structure: depths must be increasing");
        t1 = layers[k].t;
        if (z1 == z0) {
            i3e = fixr(z1 / dx3 + 1);
        } else {
            const int i3s = fixr(z0 / dx3) + 1;
            i3e = std::min(fixr(z1 / dx3 + 1), sx3);
            for (int i3 = std::max(i3s, 1); i3 <= i3e; i3++) {
                const double z = (i3 - 1.0) * dx3;
                const float a = (float)(z - z0), b = (float)(z1 - z), s = (float)(1.0 / (z1 - z0));
                relax_tensor t;
                t.s11 = s * (a * t1.s11 + b * t0.s11); t.s12 = s * (a * t1.s12 + b * t0.s12);
                t.s13 = s * (a * t1.s13 + b * t0.s13); t.s22 = s * (a * t1.s22 + b * t0.s22);
                t.s23 = s * (a * t1.s23 + b * t0.s23); t.s33 = s * (a * t1.s33 + b * t0.s33);
                vs[i3 - 1].t = t;
            }
        }
        z0 = z1; t0 = t1;
    }
    if (fixr(z1 / dx3) < sx3 - 1)
        for (int i3 = std::max(i3e, 1); i3 <= sx3; i3++) vs[i3 - 1].t = t1;
    return RELAX_OK;
}

extern "C" void relax_wang_convention(double *slip, double *x, double *y, double *z, double length,
                                      double width, double *strike, double *dip, double *rake, double x0,
                                      double y0, double rot)
{
    const double D2R = 0.01745329251994329547437168059786927;
    *slip = -*slip;
    *strike = -90.0 - *strike;
    *dip = 90.0 - *dip;
    *strike *= D2R; *dip *= D2R; *rake *= D2R;
    *x = *x - x0 - length / 2.0 * sin(*strike) + width / 2.0 * sin(*dip) * cos(*strike);
    *y = *y - y0 - length / 2.0 * cos(*strike) - width / 2.0 * sin(*dip) * sin(*strike);
    *z = *z + width / 2.0 * cos(*dip);
    const double a = rot * D2R, xx = *x, yy = *y;
    *x = +xx * cos(a) + yy * sin(a);
    *y = -xx * sin(a) + yy * cos(a);
    *strike += rot * D2R;
}

// deviatoric prestress and (taup/mu)^(n-1) per depth, as
// src/viscoelastic3d.f90:254-258 computes them (REAL*4 deviatoric part)
static void prestress_terms(const relax_tensor_layer *pre, int nz, double mu, const relax_layer *vs,
                            std::vector<float> *spdev, std::vector<DepthVisc> *dv)
{
    if (spdev) spdev->assign(6 * (size_t)nz, 0.f);
    dv->resize(nz);
    for (int i3 = 0; i3 < nz; i3++) {
        float s[6] = {0, 0, 0, 0, 0, 0};
        if (pre) {
            const relax_tensor &t = pre[i3].t;
            const float diag = (float)((double)(t.s11 + t.s22 + t.s33) / 3.0);
            s[0] = t.s11 - diag; s[1] = t.s12; s[2] = t.s13;
            s[3] = t.s22 - diag; s[4] = t.s23; s[5] = t.s33 - diag;
        }
        if (spdev)
            for (int c = 0; c < 6; c++) (*spdev)[(size_t)c * nz + i3] = s[c];
        const double taup = sqrt(((double)(s[0] * s[0]) + 2.0 * (double)(s[1] * s[1]) + 2.0 * (double)(s[2] * s[2]) +
                                  (double)(s[3] * s[3]) + 2.0 * (double)(s[4] * s[4]) + (double)(s[5] * s[5])) / 2.0);
        DepthVisc d;
        d.g0 = (float)vs[i3].gammadot0;
        d.power = (float)vs[i3].stressexponent;
        d.cohesion = (float)vs[i3].cohesion;
        d.tpow = (float)pow(taup / mu, vs[i3].stressexponent - 1);
        (*dv)[i3] = d;
    }
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct EventCopy {
    double time;
    std::vector<relax_source> s, ts, m, l;
    std::vector<relax_weakzone> cub;       // cuboid eigenstrain sources
    std::vector<relax_tetrahedron> tet;    // tetrahedral ones, over `vert`
    std::vector<double> vert;
};

struct relax_ctx {
    int device = 0;
    cudaStream_t st = nullptr;
    Grid g{};
    Spectral sp;
    relax_config cfg{};
    std::vector<relax_layer> lin, non, fc;
    std::vector<relax_tensor_layer> pre;
    std::vector<relax_plane> planes;
    std::vector<EventCopy> events;
    EventCopy inter;
    std::vector<float> hdg0[2];

    // device fields
    float *tau = nullptr, *m = nullptr, *sig = nullptr, *u = nullptr, *vp = nullptr, *gamma = nullptr;
    float *work = nullptr, *twork = nullptr, *tload = nullptr;
    float *wxy = nullptr;    // x1 and x2 derivatives of the strain source (grids where x1 or x2 takes fir7)
    DepthVisc *visc[2] = {nullptr, nullptr};
    // transient (Burgers) rheology: structures, weak zones, epsilonik, epsilonikdot
    std::vector<relax_layer> lt, nlt;
    TransLayer *tvisc[2] = {nullptr, nullptr};
    float *tdg0[2] = {nullptr, nullptr};
    float *eps = nullptr, *epsdot = nullptr;
    bool trans = false;
    float *spdev = nullptr, *dg0[2] = {nullptr, nullptr};
    double *fcd = nullptr;
    relax_slippatch *patch = nullptr;
    std::vector<int> patch_off;
    // per afterslip plane: band points and their impulse (fixed geometry)
    std::vector<unsigned *> band_idx;
    std::vector<double *> band_imp;
    std::vector<int> band_n;
    // groups of 4 points whose stress friction or monitoring reads; the
    // stress kernels store sig only there
    unsigned char *sig_mask = nullptr;
    unsigned *ticket = nullptr;                 // last-block counter of the stress kernels
    // a side stream for the step's two kernels off the critical path: the
    // time-step choice runs beside the predictor's FFT passes (joined before
    // the x-inverse pass, the first to read Dt) and the patch monitor beside
    // the corrector's (joined before the END pass, which rewrites sig)
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_dt = nullptr, ev_fork2 = nullptr, ev_mon = nullptr;
    StepState *dst = nullptr, *hst = nullptr;   // device state, pinned host mirror
    bool own_dst = true;                         // false: dst lives in a batch's array
    float *tm_part = nullptr, *fr_part = nullptr;
    double *amp_part = nullptr, *amp_alt = nullptr;
    int *err = nullptr;
    int nblk = 0, nfr = 0;
    // optional outputs of the corrector: velocity v (planes < vel_planes),
    // postseismic displacement sum Dt v (planes < ur_planes, and in urs
    // plane inter_i3 alone)
    float *vel = nullptr, *ur = nullptr, *urs = nullptr;
    int vel_planes = 0, ur_planes = 0, inter_i3 = -1;
    // the step's time-step inputs (pinned host copy, device copy) and the
    // captured graph of a step's kernels (steps without surface loads)
    DtParams *dtp_h = nullptr, *dtp_d = nullptr;
    cudaGraphExec_t gexec = nullptr;
    long long glaunches = 0;
    bool graph_off = false;
    int plain_steps = 0;

    // host time-loop state
    double t = 0.0;
    int i = 0, e = 0, oi = 1;
    bool cos_done = false, m_valid = false, sig_valid = false;
    bool store_sig = false;
    relax_step_log pending{};
    Prof prof;
};

static void free_ctx(relax_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    // one wait for the device, then every buffer goes back to the pool
    cudaDeviceSynchronize();
    const bool idle = true;
    float *fs[] = {c->tau, c->m, c->sig, c->u, c->vp, c->wxy, c->gamma, c->work, c->twork, c->tload, c->spdev,
                   c->dg0[0], c->dg0[1], c->tm_part, c->fr_part, c->vel, c->ur, c->urs};
    for (float *p : fs)
        if (p) dfree(p, idle);
    if (c->visc[0]) dfree(c->visc[0], idle);
    if (c->visc[1]) dfree(c->visc[1], idle);
    if (c->fcd) dfree(c->fcd, idle);
    if (c->patch) dfree(c->patch, idle);
    for (auto p : c->band_idx) if (p) dfree(p, idle);
    for (auto p : c->band_imp) if (p) dfree(p, idle);
    if (c->sig_mask) dfree(c->sig_mask, idle);
    for (int k = 0; k < 2; k++) {
        if (c->tvisc[k]) dfree(c->tvisc[k], idle);
        if (c->tdg0[k]) dfree(c->tdg0[k], idle);
    }
    if (c->eps) dfree(c->eps, idle);
    if (c->epsdot) dfree(c->epsdot, idle);
    if (c->ticket) dfree(c->ticket, idle);
    if (c->dst && c->own_dst) dfree(c->dst, idle);
    hpin::release(c->hst);
    hpin::release(c->dtp_h);
    if (c->dtp_d) dfree(c->dtp_d, idle);
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->amp_part) dfree(c->amp_part, idle);
    if (c->amp_alt) dfree(c->amp_alt, idle);
    c->sp.release(idle);
    for (cudaEvent_t e : {c->ev_fork, c->ev_dt, c->ev_fork2, c->ev_mon})
        if (e) cudaEventDestroy(e);
    if (c->st2) cudaStreamDestroy(c->st2);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

extern "C" const char *relax_version(void) { return "relax_b200 1.0 (sm_100a)"; }
extern "C" const char *relax_last_error(void) { return g_err.c_str(); }


static int build_bands(relax_ctx *c);

// dst[c][i] = v[c][depth of i] for the 6 components of a tensor field
__global__ void k_fill_depth(float *dst, const float *v, int nz, size_t plane, size_t nh)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 6 * nh) return;
    const size_t cc = q / nh, i3 = (q % nh) / plane;
    dst[q] = v[cc * nz + i3];
}

static int create(const relax_config *cfg, int device, relax_ctx *c)
{
    c->device = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&c->ev_fork, &c->ev_dt, &c->ev_fork2, &c->ev_mon})
        CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    TRY(make_grid(c->g, cfg->sx1, cfg->sx2, cfg->sx3, cfg->dx1, cfg->dx2, cfg->dx3));
    const Grid &g = c->g;
    const int nz = g.sx3h;
    c->cfg = *cfg;
    if (cfg->ne <= 0 || !cfg->events) return fail(RELAX_ERR_ARG, "at least one event is required");
    if (cfg->np > 0 && (!cfg->planes || !cfg->faultcreepstruc))
        return fail(RELAX_ERR_ARG, "afterslip planes need a fault-creep structure");
    auto copyv = [&](const relax_layer *p, std::vector<relax_layer> &v) {
        if (p) v.assign(p, p + nz);
    };
    copyv(cfg->linearstruc, c->lin);
    copyv(cfg->nonlinearstruc, c->non);
    copyv(cfg->faultcreepstruc, c->fc);
    copyv(cfg->ltransientstruc, c->lt);
    copyv(cfg->nltransientstruc, c->nlt);
    c->trans = !c->lt.empty() || !c->nlt.empty();
    if (cfg->stressstruc) c->pre.assign(cfg->stressstruc, cfg->stressstruc + nz);
    if (cfg->np > 0) c->planes.assign(cfg->planes, cfg->planes + cfg->np);
    auto copye = [](const relax_event &e, EventCopy &o) {
        o.time = e.time;
        if (e.ns > 0 && e.s) o.s.assign(e.s, e.s + e.ns);
        if (e.nt > 0 && e.ts) o.ts.assign(e.ts, e.ts + e.nt);
        if (e.nm > 0 && e.m) o.m.assign(e.m, e.m + e.nm);
        if (e.nl > 0 && e.l) o.l.assign(e.l, e.l + e.nl);
        if (e.nc > 0 && e.c) o.cub.assign(e.c, e.c + e.nc);
        if (e.ntet > 0 && e.tet) o.tet.assign(e.tet, e.tet + e.ntet);
        if (e.nvert > 0 && e.vert) o.vert.assign(e.vert, e.vert + 3 * (size_t)e.nvert);
    };
    c->events.resize(cfg->ne);
    for (int k = 0; k < cfg->ne; k++) copye(cfg->events[k], c->events[k]);
    copye(cfg->inter, c->inter);
    for (size_t k = 0; k < c->events.size(); k++)
        for (const auto &q : c->events[k].tet)
            for (int v : {q.i1, q.i2, q.i3, q.i4})
                if (v < 1 || (size_t)v > c->events[k].vert.size() / 3)
                    return fail(RELAX_ERR_ARG, "event %zu: tetrahedron vertex %d out of range", k, v);
    for (const auto *v : {&c->lin, &c->non, &c->lt, &c->nlt})
        for (const auto &l : *v)
            if (l.stressexponent < 0.999999)
                return fail(RELAX_ERR_POWER, "invalid power exponent %g", l.stressexponent);
    c->cfg.stressstruc = nullptr; c->cfg.linearstruc = nullptr; c->cfg.nonlinearstruc = nullptr;
    c->cfg.faultcreepstruc = nullptr; c->cfg.planes = nullptr; c->cfg.events = nullptr;
    c->cfg.lineardgammadot0 = nullptr; c->cfg.nonlineardgammadot0 = nullptr;
    c->cfg.ltransientstruc = nullptr; c->cfg.nltransientstruc = nullptr;
    c->cfg.ltransientdgammadot0 = nullptr; c->cfg.nltransientdgammadot0 = nullptr;

    const size_t nh = g.nh;
    TRY(dalloc(&c->tau, 6 * nh));
    TRY(dalloc(&c->m, 6 * nh));
    TRY(dalloc(&c->sig, 6 * nh));
    TRY(dalloc(&c->u, 3 * nh));
    TRY(dalloc(&c->vp, 3 * nh));
    TRY(dalloc(&c->gamma, nh));
    TRY(dalloc(&c->work, 6 * nh));   // coseismic body force over the whole box (3 x sx3 layers)
    TRY(dalloc(&c->twork, 3 * g.plane));
    TRY(dalloc(&c->tload, g.plane));
    if (has_fir(g)) TRY(dalloc(&c->wxy, 6 * nh));
    CK(cudaMemsetAsync(c->m, 0, 6 * nh * sizeof(float), c->st));
    CK(cudaMemsetAsync(c->sig, 0, 6 * nh * sizeof(float), c->st));
    CK(cudaMemsetAsync(c->u, 0, 3 * nh * sizeof(float), c->st));
    CK(cudaMemsetAsync(c->vp, 0, 3 * nh * sizeof(float), c->st));
    CK(cudaMemsetAsync(c->gamma, 0, nh * sizeof(float), c->st));
    TRY(c->sp.init(g, c->st));
    c->sp.prof = &c->prof;

    // tau = -prestress (src/relax.f90:287-297)
    // tau = -prestress(depth) (src/relax.f90:290-296), filled on the device
    if (c->pre.empty()) {
        CK(cudaMemsetAsync(c->tau, 0, 6 * nh * sizeof(float), c->st));
    } else {
        std::vector<float> h(6 * (size_t)nz);
        for (int i3 = 0; i3 < nz; i3++) {
            const relax_tensor &t = c->pre[i3].t;
            const float v[6] = {-t.s11, -t.s12, -t.s13, -t.s22, -t.s23, -t.s33};
            for (int cc = 0; cc < 6; cc++) h[(size_t)cc * nz + i3] = v[cc];
        }
        float *d = nullptr;
        TRY(dalloc(&d, h.size()));
        cudaError_t e = cudaMemcpyAsync(d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, c->st);
        if (e == cudaSuccess) {
            k_fill_depth<<<nblocks(6 * nh), RELAX_NTHREADS, 0, c->st>>>(c->tau, d, nz, g.plane, nh);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
        dfree(d);
        if (e != cudaSuccess) return fail(RELAX_ERR_CUDA, "prestress: %s", cudaGetErrorString(e));
    }
    // rheology tables
    std::vector<float> spdev;
    const relax_tensor_layer *pre = c->pre.empty() ? nullptr : c->pre.data();
    const std::vector<relax_layer> *vs[2] = {&c->lin, &c->non};
    const float *dgs[2] = {cfg->lineardgammadot0, cfg->nonlineardgammadot0};
    for (int k = 0; k < 2; k++) {
        if (vs[k]->empty()) continue;
        std::vector<DepthVisc> dv;
        prestress_terms(pre, nz, cfg->mu, vs[k]->data(), &spdev, &dv);
        TRY(dalloc(&c->visc[k], nz));
        CK(cudaMemcpy(c->visc[k], dv.data(), nz * sizeof(DepthVisc), cudaMemcpyHostToDevice));
        if (dgs[k]) {
            TRY(dalloc(&c->dg0[k], nh));
            CK(cudaMemcpy(c->dg0[k], dgs[k], nh * sizeof(float), cudaMemcpyHostToDevice));
        }
    }
    // transient structures (gammadot0, exponent, REAL(2 Gk) per layer), weak
    // zones, and epsilonik = epsilonikdot = 0 (allocated, src/relax.f90:299-302)
    if (c->trans) {
        const std::vector<relax_layer> *ts[2] = {&c->lt, &c->nlt};
        const float *tdg[2] = {cfg->ltransientdgammadot0, cfg->nltransientdgammadot0};
        for (int k = 0; k < 2; k++) {
            if (ts[k]->empty()) continue;
            std::vector<TransLayer> tl(nz);
            for (int i3 = 0; i3 < nz; i3++) {
                const relax_layer &l = (*ts[k])[i3];
                tl[i3] = TransLayer{(float)l.gammadot0, (float)l.stressexponent, (float)(2.0 * l.Gk), 0.f};
            }
            TRY(dalloc(&c->tvisc[k], nz));
            CK(cudaMemcpy(c->tvisc[k], tl.data(), nz * sizeof(TransLayer), cudaMemcpyHostToDevice));
            if (tdg[k]) {
                TRY(dalloc(&c->tdg0[k], nh));
                CK(cudaMemcpy(c->tdg0[k], tdg[k], nh * sizeof(float), cudaMemcpyHostToDevice));
            }
        }
        TRY(dalloc(&c->eps, 6 * nh));
        TRY(dalloc(&c->epsdot, 6 * nh));
        CK(cudaMemsetAsync(c->eps, 0, 6 * nh * sizeof(float), c->st));
        CK(cudaMemsetAsync(c->epsdot, 0, 6 * nh * sizeof(float), c->st));
    }
    if (pre) {
        if (spdev.empty()) {
            std::vector<DepthVisc> dv;
            std::vector<relax_layer> dummy(nz);
            for (auto &l : dummy) l.stressexponent = 1.0;
            prestress_terms(pre, nz, cfg->mu, dummy.data(), &spdev, &dv);
        }
        TRY(dalloc(&c->spdev, 6 * (size_t)nz));
        CK(cudaMemcpy(c->spdev, spdev.data(), 6 * nz * sizeof(float), cudaMemcpyHostToDevice));
    }
    if (!c->fc.empty()) {
        std::vector<double> h(4 * (size_t)nz);
        for (int i3 = 0; i3 < nz; i3++) {
            h[i3] = c->fc[i3].gammadot0;
            h[nz + i3] = c->fc[i3].stressexponent;
            h[2 * nz + i3] = c->fc[i3].friction;
            h[3 * nz + i3] = c->fc[i3].cohesion;
        }
        TRY(dalloc(&c->fcd, 4 * (size_t)nz));
        CK(cudaMemcpy(c->fcd, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    // afterslip patches
    int np_tot = 0;
    for (auto &p : c->planes) {
        c->patch_off.push_back(np_tot);
        np_tot += std::max(0, p.px2) * std::max(0, p.px3);
    }
    if (np_tot > 0) {
        TRY(dalloc(&c->patch, np_tot));
        CK(cudaMemset(c->patch, 0, np_tot * sizeof(relax_slippatch)));
    }
    // reductions
    c->nblk = (int)nblocks(nh / 4);
    TRY(dalloc(&c->tm_part, 4 * (size_t)c->nblk));
    TRY(dalloc(&c->amp_part, 2 * (size_t)c->nblk));
    TRY(dalloc(&c->amp_alt, 2 * (size_t)c->nblk));
    c->nfr = 1;
    TRY(dalloc(&c->fr_part, 1));
    TRY(dalloc(&c->dst, 1));
    CK(cudaMemset(c->dst, 0, sizeof(StepState)));
    TRY(hpin::alloc((void **)&c->hst, sizeof(StepState)));
    TRY(hpin::alloc((void **)&c->dtp_h, sizeof(DtParams)));
    TRY(dalloc(&c->dtp_d, 1));
    memset(c->hst, 0, sizeof(StepState));
    c->err = &c->dst->error;   // read back with the step state
    TRY(dalloc(&c->ticket, 1));
    CK(cudaMemset(c->ticket, 0, sizeof(unsigned)));
    c->store_sig = !c->planes.empty();
    TRY(build_bands(c));
    CK(cudaStreamSynchronize(c->st));
    return RELAX_OK;
}

extern "C" int relax_create(const relax_config *cfg, int device, relax_ctx **out)
{
    if (!cfg || !out) return fail(RELAX_ERR_ARG, "null argument");
    *out = nullptr;
    relax_ctx *c = new relax_ctx();
    int rc = create(cfg, device, c);
    if (rc != RELAX_OK) {
        free_ctx(c);
        return rc;
    }
    *out = c;
    return RELAX_OK;
}

extern "C" int relax_destroy(relax_ctx *c)
{
    free_ctx(c);
    return RELAX_OK;
}

extern "C" int relax_get_stream(relax_ctx *c, void **s)
{
    if (!c || !s) return fail(RELAX_ERR_ARG, "null argument");
    *s = (void *)c->st;
    return RELAX_OK;
}

extern "C" int relax_synchronize(relax_ctx *c)
{
    if (!c) return fail(RELAX_ERR_ARG, "null context");
    CK(cudaStreamSynchronize(c->st));
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// step pieces
// ---------------------------------------------------------------------------
static StressArgs stress_args(relax_ctx *c, const float *w)
{
    const Grid &g = c->g;
    StressArgs a{};
    a.g = g;
    a.w = w;
    a.tau = c->tau; a.m = c->m; a.sig = c->sig; a.gamma = c->gamma;
    a.dg0[0] = c->dg0[0]; a.dg0[1] = c->dg0[1];
    a.visc[0] = c->visc[0]; a.visc[1] = c->visc[1];
    a.spdev = c->spdev;
    a.st = c->dst;
    a.k1 = (float)(0.5 / g.dx1); a.k2 = (float)(0.5 / g.dx2);
    a.k3 = (float)(0.5 / g.dx3); a.k3b = (float)(1.0 / g.dx3);
    a.lam = (float)c->cfg.lambda; a.mu2 = (float)(2.0 * c->cfg.mu); a.muinv = (float)(1.0 / c->cfg.mu);
    a.store_sig = c->store_sig;
    a.sig_mask = c->sig_mask;
    a.ticket = c->ticket;
    a.fin = c->dst;
    a.dv = g.dx1 * g.dx2 * g.dx3;
    for (int k = 0; k < 2; k++) { a.trans[k] = c->tvisc[k]; a.tdg0[k] = c->tdg0[k]; }
    a.eps = c->eps; a.epsdot = c->epsdot;
    a.tm_part = c->tm_part;
    a.amp_part = c->amp_part;
    return a;
}

template <int MODE>
static int launch_stress(relax_ctx *c, StressArgs a)
{
    const int stage = MODE == MODE_END ? ST_STRESS_END : MODE == MODE_CORR ? ST_STRESS_CORR
                      : MODE == MODE_INIT ? ST_STRESS_INIT : ST_OTHER;
    const bool trans = c->trans && MODE != MODE_OP && MODE != MODE_EIGEN;
    if (c->wxy && MODE != MODE_EIGEN) {
        // grids of the 7-point filter along x1 or x2: the derivatives first,
        // then the stress instantiation that reads them
        const Grid &g = c->g;
        TIMED(&c->prof, stage, c->st,
              (k_fir_xy<<<nblocks(3 * (g.nh / 4)), RELAX_NTHREADS, 0, c->st>>>(
                  g, a.w, c->wxy, c->wxy + 3 * g.nh, fir_x(g), fir_y(g), a.k1, a.k2)));
        a.wx = c->wxy;
        a.wy = c->wxy + 3 * g.nh;
        if constexpr (MODE != MODE_OP && MODE != MODE_EIGEN) {
            if (trans) {
                TIMED(&c->prof, stage, c->st,
                      (launch_pdl(k_stress<MODE, false, true, true>, c->nblk, RELAX_NTHREADS, 0, c->st, a)));
                return RELAX_OK;
            }
        }
        TIMED(&c->prof, stage, c->st, (launch_pdl(k_stress<MODE, false, false, true>, c->nblk, RELAX_NTHREADS, 0, c->st, a)));
        return RELAX_OK;
    }
    if (trans)
        TIMED(&c->prof, stage, c->st, (launch_pdl(k_stress<MODE, false, true>, c->nblk, RELAX_NTHREADS, 0, c->st, a)));
    else
        TIMED(&c->prof, stage, c->st, (launch_pdl(k_stress<MODE>, c->nblk, RELAX_NTHREADS, 0, c->st, a)));
    return RELAX_OK;
}

static XfArgs xf_div(relax_ctx *c)
{
    XfArgs x{};
    const Grid &g = c->g;
    x.m = c->m;
    x.k1 = (float)(0.5 / g.dx1); x.k2 = (float)(0.5 / g.dx2);
    x.k3 = (float)(0.5 / g.dx3); x.k3b = (float)(1.0 / g.dx3);
    x.fx = fir_x(g);
    x.fy = fir_y(g);
    x.tload = nullptr;
    return x;
}

static XiArgs xi_update(relax_ctx *c, float *out, const float *base, float cmul, bool use_dt)
{
    XiArgs x{};
    const Grid &g = c->g;
    for (int k = 0; k < 3; k++) {
        x.out[k] = out + k * g.nh;
        x.base[k] = base ? base + k * g.nh : nullptr;
    }
    x.rp = g.sx1; x.pp = g.plane;
    x.st = use_dt ? c->dst : nullptr;
    x.cmul = cmul;
    return x;
}

// surface loads (traction, src/elastic3d.f90:2517-2590) into tload
static int upload_loads(relax_ctx *c, const EventCopy &ev, double t, double Dt, bool rate, bool *any)
{
    *any = false;
    if (ev.l.empty()) return RELAX_OK;
    const Grid &g = c->g;
    std::vector<float> h(g.plane, 0.f);
    for (const auto &l : ev.l) {
        const double L = l.length, W = l.width, beta = l.beta;
        const double Lp = L * (1.0 + 2.0 * beta) / 2.0, Wp = W * (1.0 + 2.0 * beta) / 2.0;
        if (Lp == 0 || Wp == 0) continue;
        const double mm = std::max(Lp, Wp);
        for (int i2 = 0; i2 < g.sx2; i2++)
            for (int i1 = 0; i1 < g.sx1; i1++) {
                const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
                const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
                if (fabs(x1 - l.x) > mm || fabs(x2 - l.y) > mm) continue;
                auto om = [beta](double x) {
                    const double ax = fabs(x);
                    if (ax <= (1.0 - 2.0 * beta) / (1.0 - beta) / 2.0) return 1.0;
                    if (ax < 1.0 / (1.0 - beta) / 2.0) {
                        const double cc = cos(M_PI * ((1.0 - beta) * ax - 0.5 + beta) / 2.0 / beta);
                        return cc * cc;
                    }
                    return 0.0;
                };
                const double amp = om((x1 - l.x) / L) * om((x2 - l.y) / W) * l.slip;
                float &v = h[(size_t)i2 * g.sx1 + i1];
                if (rate) {
                    if (l.period != 0)
                        v = (float)(v - amp * (sin(2 * M_PI * (t + Dt) / l.period + l.phase) -
                                               sin(2 * M_PI * t / l.period + l.phase)) / Dt);
                } else {
                    v = (float)(l.period == 0 ? v - amp : v - amp * sin(2 * M_PI * t / l.period + l.phase));
                }
            }
    }
    CK(cudaMemcpyAsync(c->tload, h.data(), g.plane * sizeof(float), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    *any = true;
    return RELAX_OK;
}

// shear sources of one event: body force + traction into work/twork, and
// the relaxed moment density into tau (dislocations, src/relax.f90:1116-1289)
// dislocations, src/relax.f90:1116-1289: body forces of the event's
// shear, tensile and point sources into c->work (3 components of the whole
// box, sx1 sx2 sx3 each; shear sources only touch the physical layers,
// tensile and point sources also their images below the surface), the
// surface traction into c->twork, and the moment densities into tau.
// *full: the lower half of the box is non-zero.
// the arguments of the eigenstrain kernels for one cuboid or tetrahedron
static EigArgs eig_args(relax_ctx *c, const relax_tensor &e)
{
    EigArgs a{};
    a.g = c->g; a.lambda = c->cfg.lambda; a.mu = c->cfg.mu; a.beta = c->cfg.beta;
    const float ev[6] = {e.s11, e.s12, e.s13, e.s22, e.s23, e.s33};
    for (int k = 0; k < 6; k++) a.e[k] = ev[k];
    const size_t nb = 2 * c->g.nh;
    for (int k = 0; k < 3; k++) a.f[k] = c->work + k * nb;
    a.tau = c->tau;
    return a;
}

// tensorsymmetricdyadprod (src/elastic3d.f90:206-218) in the reference's
// REAL*4 result
static void sdyad6(const double u[3], const double v[3], float out[6])
{
    out[0] = (float)(u[0] * v[0]);
    out[1] = (float)((u[0] * v[1] + u[1] * v[0]) / 2.0);
    out[2] = (float)((u[0] * v[2] + u[2] * v[0]) / 2.0);
    out[3] = (float)(u[1] * v[1]);
    out[4] = (float)((u[1] * v[2] + u[2] * v[1]) / 2.0);
    out[5] = (float)(u[2] * v[2]);
}

// outward unit normals, centroids and tractions (c : e) n of the faces BCD,
// CDA, DAB, ABC (src/elastic3d.f90:1946-1985); false without volume
static bool tet_setup(EigArgs &a, const double *A, const double *B, const double *C, const double *D)
{
    const double *P[4] = {A, B, C, D};
    const int tri[4][3] = {{1, 2, 3}, {2, 3, 0}, {3, 0, 1}, {0, 1, 2}};
    double nrm[4];
    for (int f = 0; f < 4; f++) {
        const double *p = P[tri[f][0]], *q = P[tri[f][1]], *r = P[tri[f][2]];
        const double u[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]}, v[3] = {r[0] - p[0], r[1] - p[1], r[2] - p[2]};
        a.n[f][0] = u[1] * v[2] - u[2] * v[1];
        a.n[f][1] = u[2] * v[0] - u[0] * v[2];
        a.n[f][2] = u[0] * v[1] - u[1] * v[0];
        nrm[f] = sqrt(a.n[f][0] * a.n[f][0] + a.n[f][1] * a.n[f][1] + a.n[f][2] * a.n[f][2]);
    }
    for (int f = 0; f < 4; f++)
        if (nrm[f] == 0.0) return false;
    // isotropicstressstrain (src/elastic3d.f90:129-142) of the eigenstrain
    float m[6];
    const double epskk = (double)(a.e[0] + a.e[3] + a.e[5]);
    const float mu2 = (float)(2.0 * a.mu);
    for (int k = 0; k < 6; k++) m[k] = mu2 * a.e[k];
    m[0] = (float)(m[0] + a.lambda * epskk);
    m[3] = (float)(m[3] + a.lambda * epskk);
    m[5] = (float)(m[5] + a.lambda * epskk);
    for (int f = 0; f < 4; f++) {
        for (int k = 0; k < 3; k++) a.n[f][k] = a.n[f][k] / nrm[f];
        const double *p = P[tri[f][0]], *q = P[tri[f][1]], *r = P[tri[f][2]];
        for (int k = 0; k < 3; k++) a.cen[f][k] = (p[k] + q[k] + r[k]) / 3;
        const double *o = P[f];
        const double dd = a.n[f][0] * (o[0] - a.cen[f][0]) + a.n[f][1] * (o[1] - a.cen[f][1]) +
                          a.n[f][2] * (o[2] - a.cen[f][2]);
        if (dd > 0)
            for (int k = 0; k < 3; k++) a.n[f][k] = -a.n[f][k];
        const double *n = a.n[f];
        a.tr[f][0] = m[0] * n[0] + m[1] * n[1] + m[2] * n[2];
        a.tr[f][1] = m[1] * n[0] + m[3] * n[1] + m[4] * n[2];
        a.tr[f][2] = m[2] * n[0] + m[4] * n[1] + m[5] * n[2];
    }
    return true;
}

static int event_sources(relax_ctx *c, const EventCopy &ev, bool *any, bool *full)
{
    const Grid &g = c->g;
    const size_t nb = 2 * g.nh;            // one component of the whole box
    CK(cudaMemsetAsync(c->work, 0, 3 * nb * sizeof(float), c->st));
    CK(cudaMemsetAsync(c->twork, 0, 3 * g.plane * sizeof(float), c->st));
    const double mind = std::min(std::min(g.dx1, g.dx2), g.dx3);
    auto args = [&](const relax_source &s) {
        SrcArgs a{};
        a.g = g; a.mu = c->cfg.mu; a.lambda = c->cfg.lambda; a.s = s.slip; a.x = s.x; a.y = s.y; a.z = s.z;
        a.L = s.width; a.W = s.length; a.strike = s.strike; a.dip = s.dip; a.rake = s.rake; a.beta = s.beta;
        for (int k = 0; k < 3; k++) { a.f[k] = c->work + k * nb; a.t[k] = c->twork + k * g.plane; }
        a.tau = c->tau;
        return a;
    };
    for (const auto &s : ev.s) {
        SrcArgs a = args(s);
        if (c->cfg.nyquist * mind < s.length || c->cfg.nyquist * mind < s.width) {
            k_source_traction<<<nblocks(g.plane), RELAX_NTHREADS, 0, c->st>>>(a);
            CKL();
            k_source_force<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
            CKL();
        }
    }
    // cuboid and tetrahedral eigenstrain (src/relax.f90:1154-1181): the
    // cuboid's L = width, W = length, T = thickness, the global beta
    for (const auto &q : ev.cub) {
        EigArgs a = eig_args(c, q.e);
        a.x = q.x; a.y = q.y; a.z = q.z; a.L = q.width; a.W = q.length; a.T = q.thickness;
        a.strike = q.strike; a.dip = q.dip;
        k_source_cuboid<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
        CKL();
    }
    for (const auto &q : ev.tet) {
        EigArgs a = eig_args(c, q.e);
        const double *V = ev.vert.data();
        if (!tet_setup(a, V + 3 * (q.i1 - 1), V + 3 * (q.i2 - 1), V + 3 * (q.i3 - 1), V + 3 * (q.i4 - 1))) continue;
        k_source_tetra<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
        CKL();
    }
    for (const auto &s : ev.s) {
        SrcArgs a = args(s);
        k_moment_shear<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
        CKL();
    }
    // their moment densities into tau (src/relax.f90:1208-1224)
    for (const auto &q : ev.cub) {
        EigArgs a = eig_args(c, q.e);
        a.x = q.x; a.y = q.y; a.z = q.z; a.L = q.width; a.W = q.length; a.T = q.thickness;
        a.strike = q.strike; a.dip = q.dip;
        const double cs = cos(q.strike), ss = sin(q.strike), cd = cos(q.dip), sd = sin(q.dip);
        const double n[3] = {+cd * cs, -cd * ss, -sd}, sv[3] = {-ss, -cs, 0}, d[3] = {+cs * sd, -ss * sd, +cd};
        sdyad6(sv, sv, a.sdy[0]);
        sdyad6(n, sv, a.sdy[1]);
        sdyad6(sv, d, a.sdy[2]);
        sdyad6(n, n, a.sdy[3]);
        sdyad6(n, d, a.sdy[4]);
        sdyad6(d, d, a.sdy[5]);
        k_moment_cuboid<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
        CKL();
    }
    for (const auto &q : ev.tet) {
        EigArgs a = eig_args(c, q.e);
        const double *V = ev.vert.data();
        if (!tet_setup(a, V + 3 * (q.i1 - 1), V + 3 * (q.i2 - 1), V + 3 * (q.i3 - 1), V + 3 * (q.i4 - 1))) continue;
        k_moment_tetra<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
        CKL();
    }
    // tensile cracks: the opening, the global beta (src/relax.f90:1226-1260)
    for (const auto &s : ev.ts) {
        SrcArgs a = args(s);
        a.s = s.opening; a.beta = c->cfg.beta;
        if (c->cfg.nyquist * mind < s.length || c->cfg.nyquist * mind < s.width) {
            k_source_tensile<<<nblocks(nb), RELAX_NTHREADS, 0, c->st>>>(a);
            CKL();
        }
    }
    for (const auto &s : ev.ts) {
        SrcArgs a = args(s);
        a.s = s.opening; a.beta = c->cfg.beta;
        k_moment_tensile<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
        CKL();
    }
    // dilatation point sources (src/relax.f90:1262-1287)
    for (const auto &s : ev.m) {
        SrcArgs a = args(s);
        k_source_mogi<<<nblocks(nb), RELAX_NTHREADS, 0, c->st>>>(a);
        CKL();
    }
    for (const auto &s : ev.m) {
        SrcArgs a = args(s);
        k_moment_mogi<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
        CKL();
    }
    *any = !ev.s.empty() || !ev.ts.empty() || !ev.m.empty() || !ev.l.empty() || !ev.cub.empty() ||
           !ev.tet.empty();
    *full = !ev.ts.empty() || !ev.m.empty();
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// space-domain solution of the small coseismic sources (dislocations_disp,
// src/relax.f90:1298-1349; grnfct_okada, src/okada/green_space.f90:114-144)
// ---------------------------------------------------------------------------
// one thread per physical grid point, all sources in turn; u in rows of
// pitch rp and planes of pitch pp
__global__ void k_okada(Grid g, const relax_source *src, int n, double lambda, double mu, float *u1, float *u2,
                        float *u3, size_t rp, size_t pp)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1);
    const size_t r = q / g.sx1;
    const int i2 = (int)(r % g.sx2), i3 = (int)(r / g.sx2);
    // shiftedcoordinates, src/elastic3d.f90:4027-4048
    const double x1 = (double)(i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (double)(i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = (double)i3 * g.dx3;
    const size_t o = (size_t)i3 * pp + (size_t)i2 * rp + i1;
    float a0 = u1[o], a1 = u2[o], a2 = u3[o];
    for (int k = 0; k < n; k++) {
        const relax_source &s = src[k];
        double d[3];
        okada_relax(lambda, mu, s.slip, s.opening, s.x, s.y, s.z, s.width, s.length, s.strike, s.dip, s.rake, x1,
                    x2, x3, d);
        a0 += (float)d[0];
        a1 += (float)d[1];
        a2 += (float)d[2];
    }
    u1[o] = a0;
    u2[o] = a1;
    u3[o] = a2;
}

// A source of the configuration (after wangconvention and the rotation,
// src/input.f90:1780-1822) back in the input-file convention that the
// space-domain solution is evaluated in.
static relax_source input_convention(const relax_source &s, const relax_config &cfg, bool tensile)
{
    const double deg = 0.01745329251994329547437168059786927;
    const double strike = s.strike - cfg.rot * deg, dip = s.dip;
    const double a = -cfg.rot * deg;
    const double xx = +s.x * cos(a) + s.y * sin(a), yy = -s.x * sin(a) + s.y * cos(a);
    relax_source o{};
    o.x = xx + cfg.x0 + s.length / 2.0 * sin(strike) - s.width / 2.0 * sin(dip) * cos(strike);
    o.y = yy + cfg.y0 + s.length / 2.0 * cos(strike) + s.width / 2.0 * sin(dip) * sin(strike);
    o.z = s.z - s.width / 2.0 * cos(dip);
    o.width = s.width;
    o.length = s.length;
    o.strike = -90.0 - strike / deg;
    o.dip = 90.0 - dip / deg;
    o.rake = tensile ? 0.0 : s.rake / deg;
    o.slip = tensile ? 0.0 : -s.slip;
    o.opening = tensile ? s.opening : 0.0;
    return o;
}

// u += the space-domain solution of event 0's sources no longer than
// nyquist * min(dx) along strike or dip (src/relax.f90:1320-1347)
static int event_okada(relax_ctx *c, const EventCopy &ev)
{
    const Grid &g = c->g;
    const double small = c->cfg.nyquist * std::min(std::min(g.dx1, g.dx2), g.dx3);
    std::vector<relax_source> h;
    for (const auto &s : ev.s)
        if (small >= s.length || small >= s.width) h.push_back(input_convention(s, c->cfg, false));
    for (const auto &s : ev.ts)
        if (small >= s.length || small >= s.width) h.push_back(input_convention(s, c->cfg, true));
    if (h.empty()) return RELAX_OK;
    relax_source *d = nullptr;
    TRY(dalloc(&d, h.size()));
    cudaError_t e = cudaMemcpyAsync(d, h.data(), h.size() * sizeof(relax_source), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) {
        k_okada<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(g, d, (int)h.size(), c->cfg.lambda, c->cfg.mu, c->u,
                                                             c->u + g.nh, c->u + 2 * g.nh, g.sx1, g.plane);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    dfree(d);
    if (e != cudaSuccess) return fail(RELAX_ERR_CUDA, "okada: %s", cudaGetErrorString(e));
    return RELAX_OK;
}

// the coseismic Green's function of c->work (the whole box when `full`,
// else its physical half), u += the displacement
static int event_green(relax_ctx *c, bool loads, bool full)
{
    const Grid &g = c->g;
    XfArgs xa{};
    for (int k = 0; k < 3; k++) {
        xa.in[k] = c->work + k * 2 * g.nh;
        xa.tin[k] = c->twork + k * g.plane;
    }
    xa.rp = g.sx1; xa.pp = g.plane; xa.trp = g.sx1;
    xa.tload = loads ? c->tload : nullptr;
    XiArgs xi = xi_update(c, c->u, c->u, 1.0f, false);
    return c->sp.green(xa, false, full ? g.sx3 : g.sx3h, g.sx3h, xi, c->cfg.lambda, c->cfg.mu, c->cfg.gam, c->st);
}

// strike/dip/rake trigonometry and the rotated plane centre of
// src/friction3d.f90:128-152, once per plane on the host
static void set_plane_geometry(FrictionArgs &a)
{
    a.cs = cos(a.strike); a.ss = sin(a.strike); a.cd = cos(a.dip); a.sd = sin(a.dip);
    a.cr = cos(a.rake); a.sr = sin(a.rake);
    const double x2r0 = a.cs * a.x - a.ss * a.y;
    a.xr = a.cd * x2r0 - a.sd * a.z;
    a.yr = a.ss * a.x + a.cs * a.y;
    a.zr = a.sd * x2r0 + a.cd * a.z;
    a.Wp = a.W * (1.0 + 2.0 * a.beta) / 2.0;
    a.Lp = a.L * (1.0 + 2.0 * a.beta) / 2.0;
}

// index box of a plane's band: x1, x2 as shifted-coordinate indices in
// [-sx/2, sx/2-1], x3 in the physical layers
static bool plane_box(const Grid &g, const FrictionArgs &a, int *j1lo, int *n1, int *j2lo, int *n2, int *i3lo, int *n3)
{
    const double mw = std::max(a.Wp, a.Lp);
    int a1 = (int)ceil((a.x - mw) / g.dx1) - 1, b1 = (int)floor((a.x + mw) / g.dx1) + 1;
    a1 = std::max(a1, -g.sx1 / 2); b1 = std::min(b1, g.sx1 / 2 - 1);
    int a2 = (int)ceil((a.y - mw) / g.dx2) - 1, b2 = (int)floor((a.y + mw) / g.dx2) + 1;
    a2 = std::max(a2, -g.sx2 / 2); b2 = std::min(b2, g.sx2 / 2 - 1);
    const double zlo = std::min(a.z, -a.z) - a.Lp, zhi = std::max(a.z, -a.z) + a.Lp;
    const int a3 = std::max(0, (int)floor(zlo / g.dx3) - 1), b3 = std::min(g.sx3h - 1, (int)ceil(zhi / g.dx3) + 1);
    if (b1 < a1 || b2 < a2 || b3 < a3) return false;
    *j1lo = a1; *n1 = b1 - a1 + 1; *j2lo = a2; *n2 = b2 - a2 + 1; *i3lo = a3; *n3 = b3 - a3 + 1;
    return true;
}

static FrictionArgs plane_args(relax_ctx *c, const relax_plane &p)
{
    FrictionArgs a{};
    a.g = c->g;
    a.x = p.x; a.y = p.y; a.z = p.z; a.L = p.width; a.W = p.length;
    a.strike = p.strike; a.dip = p.dip; a.rake = p.rake; a.beta = c->cfg.beta; a.mu = c->cfg.mu;
    a.fc = c->fcd; a.sig = c->sig; a.m = c->m; a.err = c->err;
    set_plane_geometry(a);
    return a;
}

// band point lists of every plane, once per context
// Band compaction on the device, in the order of the plane's box: the points
// whose impulse is defined (>= 0) go to consecutive slots.
__global__ void k_band_count(const double *imp, size_t n, unsigned *cnt)
{
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int v = __syncthreads_count(t < n && imp[t] >= 0.0);
    if (threadIdx.x == 0) cnt[blockIdx.x] = (unsigned)v;
}

// exclusive scan of the per-block counts, one block; total in cnt[nb]
__global__ void k_band_scan(unsigned *cnt, int nb)
{
    __shared__ unsigned carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const unsigned v = i < nb ? cnt[i] : 0u;
        // inclusive warp scan, then across warps
        unsigned x = v;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        __shared__ unsigned ws[32];
        if (lane == 31) ws[w] = x;
        __syncthreads();
        if (w == 0) {
            unsigned s = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0u;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            ws[lane] = s;
        }
        __syncthreads();
        const unsigned incl = x + (w ? ws[w - 1] : 0u) + carry;
        if (i < nb) cnt[i] = incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) cnt[nb] = carry;
}

__global__ void k_band_write(FrictionArgs a, const double *imp, const unsigned *off, unsigned *idx, double *out)
{
    const Grid &g = a.g;
    const size_t n = (size_t)a.n1 * a.n2 * a.n3;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < n && imp[t] >= 0.0;
    const unsigned ball = __ballot_sync(0xffffffffu, in);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __shared__ unsigned wc[32];
    if (lane == 0) wc[w] = __popc(ball);
    __syncthreads();
    unsigned before = 0;
    for (int k = 0; k < w; k++) before += wc[k];
    if (!in) return;
    const unsigned slot = off[blockIdx.x] + before + __popc(ball & ((1u << lane) - 1u));
    const int j1 = a.j1lo + (int)(t % a.n1);
    const int j2 = a.j2lo + (int)((t / a.n1) % a.n2);
    const int i3 = a.i3lo + (int)(t / ((size_t)a.n1 * a.n2));
    const int i1 = (j1 + g.sx1) % g.sx1, i2 = (j2 + g.sx2) % g.sx2;
    idx[slot] = (unsigned)(((size_t)i3 * g.sx2 + i2) * g.sx1 + i1);
    out[slot] = imp[t];
}

static int build_bands(relax_ctx *c)
{
    const Grid &g = c->g;
    for (size_t k = 0; k < c->planes.size(); k++) {
        FrictionArgs a = plane_args(c, c->planes[k]);
        c->band_idx.push_back(nullptr);
        c->band_imp.push_back(nullptr);
        c->band_n.push_back(0);
        if (!plane_box(g, a, &a.j1lo, &a.n1, &a.j2lo, &a.n2, &a.i3lo, &a.n3)) continue;
        const size_t n = (size_t)a.n1 * a.n2 * a.n3;
        const int nb = (int)nblocks(n);
        double *dimp = nullptr;
        unsigned *cnt = nullptr;
        TRY(dalloc(&dimp, n));
        if (dalloc(&cnt, (size_t)nb + 1) != RELAX_OK) {
            dfree(dimp);
            return RELAX_ERR_NOMEM;
        }
        unsigned total = 0;
        k_friction_mark<<<nb, RELAX_NTHREADS, 0, c->st>>>(a, dimp);
        k_band_count<<<nb, RELAX_NTHREADS, 0, c->st>>>(dimp, n, cnt);
        k_band_scan<<<1, 1024, 0, c->st>>>(cnt, nb);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&total, cnt + nb, sizeof total, cudaMemcpyDeviceToHost, c->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
        if (e == cudaSuccess && total > 0) {
            if (dalloc(&c->band_idx[k], total) != RELAX_OK || dalloc(&c->band_imp[k], total) != RELAX_OK) {
                dfree(dimp);
                dfree(cnt);
                return RELAX_ERR_NOMEM;
            }
            k_band_write<<<nb, RELAX_NTHREADS, 0, c->st>>>(a, dimp, cnt, c->band_idx[k], c->band_imp[k]);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
        }
        dfree(dimp);
        dfree(cnt);
        if (e != cudaSuccess) return fail(RELAX_ERR_CUDA, "band of plane %zu: %s", k, cudaGetErrorString(e));
        c->band_n[k] = (int)total;
    }
    if (c->planes.empty()) return RELAX_OK;
    TRY(dalloc(&c->sig_mask, g.nh / 4));
    CK(cudaMemsetAsync(c->sig_mask, 0, g.nh / 4, c->st));
    for (size_t k = 0; k < c->planes.size(); k++) {
        if (c->band_n[k] > 0) {
            k_mark_points<<<nblocks(c->band_n[k]), RELAX_NTHREADS, 0, c->st>>>(c->band_idx[k], c->band_n[k],
                                                                               c->sig_mask);
            CKL();
        }
        const relax_plane &p = c->planes[k];
        const int n = std::max(0, p.px2) * std::max(0, p.px3);
        if (n == 0) continue;
        MonitorArgs a{};
        a.g = g;
        a.x = p.x; a.y = p.y; a.z = p.z; a.strike = p.strike; a.dip = p.dip; a.rake = p.rake;
        a.px2 = p.px2; a.px3 = p.px3;
        k_mark_monitor<<<nblocks(n, 128), 128, 0, c->st>>>(a, c->sig_mask);
        CKL();
    }
    return RELAX_OK;
}

// arguments of frictioneigenstress on the band points of plane k
static FrictionPtsArgs friction_pts_args(relax_ctx *c, size_t k, bool want_tm)
{
    const relax_plane &p = c->planes[k];
    FrictionArgs fa = plane_args(c, p);
    FrictionPtsArgs a{};
    a.g = c->g; a.mu = c->cfg.mu; a.rake = p.rake; a.L = p.width; a.W = p.length;
    a.n0 = fa.cd * fa.cs; a.n1 = -fa.cd * fa.ss; a.n2 = -fa.sd;
    a.r0 = fa.ss * fa.cr + fa.cs * fa.sd * fa.sr;
    a.r1 = fa.cs * fa.cr - fa.ss * fa.sd * fa.sr;
    a.r2 = fa.cd * fa.sr;
    a.fc = c->fcd; a.sig = c->sig; a.m = c->m; a.err = c->err;
    a.idx = c->band_idx[k]; a.imp = c->band_imp[k]; a.npts = c->band_n[k];
    a.want_tm = want_tm;
    return a;
}

// arguments of monitorfriction on the patches of plane k
static MonitorArgs monitor_args(relax_ctx *c, size_t k, bool with_dt)
{
    const relax_plane &p = c->planes[k];
    MonitorArgs a{};
    a.g = c->g;
    a.x = p.x; a.y = p.y; a.z = p.z; a.strike = p.strike; a.dip = p.dip; a.rake = p.rake;
    a.fc = c->fcd; a.sig = c->sig; a.patch = c->patch + c->patch_off[k];
    a.px2 = p.px2; a.px3 = p.px3;
    a.st = with_dt ? c->dst : nullptr;
    return a;
}

// Maxwell-time partial slots of the friction kernels: the blocks of each
// plane in turn.  Grows the partial array when needed.
static int friction_slots(relax_ctx *c, int *total)
{
    int blk = 0;
    for (size_t k = 0; k < c->planes.size(); k++) blk += (int)nblocks(c->band_n[k]);
    if (blk > c->nfr) {
        CK(cudaStreamSynchronize(c->st));
        float *np = nullptr;
        TRY(dalloc(&np, (size_t)blk));
        if (c->fr_part) dfree(c->fr_part);
        c->fr_part = np;
        c->nfr = blk;
    }
    *total = blk;
    return RELAX_OK;
}

static int friction_planes(relax_ctx *c, bool want_tm, int *nblk_out)
{
    int blk_total = 0;
    *nblk_out = 0;
    if (want_tm) TRY(friction_slots(c, &blk_total));
    blk_total = 0;
    for (size_t k = 0; k < c->planes.size(); k++) {
        if (c->band_n[k] == 0) continue;
        FrictionPtsArgs a = friction_pts_args(c, k, want_tm);
        const int nb = (int)nblocks(a.npts);
        if (want_tm) a.tm_part = c->fr_part + blk_total;
        TIMED(&c->prof, ST_FRICTION, c->st, (launch_pdl(k_friction_pts<false>, nb, RELAX_NTHREADS, 0, c->st, a)));
        blk_total += nb;
    }
    *nblk_out = blk_total;
    return RELAX_OK;
}

static int monitor_planes(relax_ctx *c, bool with_dt, cudaStream_t st = nullptr)
{
    if (!st) st = c->st;
    for (size_t k = 0; k < c->planes.size(); k++) {
        const relax_plane &p = c->planes[k];
        const int n = std::max(0, p.px2) * std::max(0, p.px3);
        if (n == 0) continue;
        MonitorArgs a = monitor_args(c, k, with_dt);
        TIMED(&c->prof, ST_MONITOR, st, (k_monitor<<<nblocks(n, 128), 128, 0, st>>>(a)));
    }
    return RELAX_OK;
}

// device error flags, from the step state last copied to the host
static int check_err(relax_ctx *c)
{
    if (c->hst->error & (1 << RELAX_ERR_FRICTION))
        return fail(RELAX_ERR_FRICTION, "wrong value of (a-b)sigma: tau/((a-b)sigma) > 20");
    if (c->hst->error & (1 << RELAX_ERR_CUDA))
        return fail(RELAX_ERR_CUDA, "tensor-core x3 pass: a wait on the tensor cores timed out");
    return RELAX_OK;
}

static int pull_state(relax_ctx *c)
{
    CK(cudaMemcpyAsync(c->hst, c->dst, sizeof(StepState), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return RELAX_OK;
}

// sig = -tau + C:E(u), next predictor moment, log amplitude of tau
static int tail_init(relax_ctx *c)
{
    TRY(launch_stress<MODE_INIT>(c, stress_args(c, c->u)));
    k_reduce_amp<<<1, RELAX_NTHREADS, 0, c->st>>>(c->dst, c->amp_part, c->nblk, nullptr,
                                                    c->g.dx1 * c->g.dx2 * c->g.dx3);
    CKL();
    c->m_valid = true;
    c->sig_valid = c->store_sig && !c->sig_mask;
    return RELAX_OK;
}

extern "C" int relax_coseismic(relax_ctx *c, int e, relax_step_log *log0)
{
    if (!c) return fail(RELAX_ERR_ARG, "null context");
    if (e < 0 || e >= (int)c->events.size()) return fail(RELAX_ERR_ARG, "event %d out of range", e);
    CK(cudaSetDevice(c->device));
    bool any = false, loads = false, full = false;
    TRY(event_sources(c, c->events[e], &any, &full));
    TRY(upload_loads(c, c->events[e], c->t, 0.0, false, &loads));
    if (any) TRY(event_green(c, loads, full));
    if (e == 0) TRY(event_okada(c, c->events[0]));
    TRY(tail_init(c));
    CK(cudaMemcpyAsync(c->hst, c->dst, sizeof(StepState), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (e == 0) { c->t = 0.0; c->i = 0; c->oi = 1; }
    c->e = e;
    c->cos_done = true;
    if (log0) {
        memset(log0, 0, sizeof *log0);
        log0->i = 0;
        log0->cei = c->hst->cei;
        log0->output = 1;   // format 1101, src/relax.f90:469-472
    }
    return RELAX_OK;
}

static DtPolicy policy(relax_ctx *c)
{
    DtPolicy p{};
    p.interval = c->cfg.interval; p.odt = c->cfg.odt; p.tscale = c->cfg.tscale; p.skip = c->cfg.skip;
    p.has_next_event = c->e < (int)c->events.size() - 1;
    p.next_event_time = p.has_next_event ? c->events[c->e + 1].time : 0.0;
    p.has_inter = !c->inter.s.empty() || !c->inter.ts.empty();
    p.mech[0] = !c->lin.empty();
    p.mech[1] = !c->non.empty();
    p.mech[2] = !c->fc.empty();
    p.mech[3] = !c->lt.empty();
    p.mech[4] = !c->nlt.empty();
    return p;
}

// The host part of the end of a step, from the step state in c->hst: time,
// counters, the event branch when k_dt found that t + Dt reaches the next
// event, isoutput, the error flags and the log line.
static int finish_step(relax_ctx *c, relax_step_log *log)
{
    const Grid &g = c->g;
    double Dt = 0.0;
    if (!(c->hst->dt_raw > 0.0) || !std::isfinite(c->hst->dt_raw))
        return fail(RELAX_ERR_ARG, "invalid time step %g", c->hst->dt_raw);
    Dt = c->hst->Dt;
    const double mw[5] = {c->hst->maxwell[0], c->hst->maxwell[1], c->hst->maxwell[2], c->hst->maxwell[3],
                          c->hst->maxwell[4]};
    c->t = c->t + Dt;
    c->i++;
    const int fired = c->hst->fire;
    if (fired) {
        // tau += Dt m, then the coseismic event, then the stress
        k_tau_update<<<c->nblk, RELAX_NTHREADS, 0, c->st>>>(g, c->tau, c->m, c->dst, c->amp_alt);
        CKL();
        c->e++;
        bool any = false, ld = false, full = false;
        TRY(event_sources(c, c->events[c->e], &any, &full));
        TRY(upload_loads(c, c->events[c->e], c->t, 0.0, false, &ld));
        TRY(event_green(c, ld, full));
        TRY(launch_stress<MODE_INIT>(c, stress_args(c, c->u)));
        k_reduce_amp<<<1, RELAX_NTHREADS, 0, c->st>>>(c->dst, c->amp_part, c->nblk, c->amp_alt,
                                                        g.dx1 * g.dx2 * g.dx3);
        CKL();
        TRY(pull_state(c));
    }
    c->m_valid = true;
    c->sig_valid = c->store_sig && !c->sig_mask;
    // isoutput, src/relax.f90:1364-1376
    int output = 0;
    {
        const double odt = c->cfg.odt, etime = c->events[c->e].time;
        if ((0 == c->cfg.skip && fabs(c->t - c->oi * odt) < 1e-6 * odt) ||
            (0 < c->cfg.skip && ((c->i - 1) % c->cfg.skip) == 0) || fabs(c->t - etime) < 1e-6) {
            c->oi++;
            output = 1;
        }
    }
    if (!c->fc.empty()) TRY(check_err(c));
    log->i = c->i;
    log->event = fired;
    log->dt = Dt;
    log->tm_ve = mw[0]; log->tm_pl = mw[1]; log->tm_as = mw[2];
    log->tm_tl = mw[3]; log->tm_tnl = mw[4];
    log->t = c->t;
    log->power = c->hst->power;
    log->cei = c->hst->cei;
    log->output = output;
    return RELAX_OK;
}

// The kernels of one RK2 step, after the step's time-step inputs are in
// c->dtp_d.  Without surface loads on the current event the sequence does
// not depend on the host between its launches, and do_step captures it once
// in a CUDA graph and replays it.
static int step_kernels(relax_ctx *c)
{
    const Grid &g = c->g;
    // ---- predictor -------------------------------------------------------
    int nfr = 0;
    if (!c->fc.empty()) TRY(friction_planes(c, true, &nfr));
    // the Maxwell-time minima come reduced from the last INIT/END stress
    // pass; the policy and the step's inputs are in c->dtp_d.  The choice
    // runs on the side stream: nothing before the predictor's x-inverse pass
    // reads Dt (surface loads join at once, below).
    CK(cudaEventRecord(c->ev_fork, c->st));
    CK(cudaStreamWaitEvent(c->st2, c->ev_fork, 0));
    TIMED(&c->prof, ST_DT, c->st2, (k_dt_dev<<<1, RELAX_NTHREADS, 0, c->st2>>>(c->dst, c->dtp_d, c->fr_part, nfr)));
    CK(cudaEventRecord(c->ev_dt, c->st2));
    // The kernels take Dt from the device state.  The host needs it before
    // the end of the step only for surface loads (evaluated on the host at
    // t + Dt); otherwise the step runs with one synchronisation, at its end.
    // An invalid Dt is replaced by 0 on the device, so that the step leaves
    // the state unchanged, and reported here.
    const EventCopy &ev = c->events[c->e];
    double Dt = 0.0;
    if (!ev.l.empty()) {
        CK(cudaStreamWaitEvent(c->st, c->ev_dt, 0));
        TRY(pull_state(c));
        Dt = c->hst->Dt;
        if (!(c->hst->dt_raw > 0.0) || !std::isfinite(c->hst->dt_raw))
            return fail(RELAX_ERR_ARG, "invalid time step %g", c->hst->dt_raw);
    }
    bool loads = false;
    // note: the reference passes Dt/2.d8 here (src/relax.f90:685)
    TRY(upload_loads(c, ev, c->t, Dt / 2.0e8, true, &loads));
    {
        XfArgs xa = xf_div(c);
        xa.tload = loads ? c->tload : nullptr;
        XiArgs xi = xi_update(c, c->vp, c->u, 0.5f, true);
        TRY(c->sp.green(xa, true, g.sx3h, g.sx3h, xi, c->cfg.lambda, c->cfg.mu, c->cfg.gam, c->st, c->ev_dt));
    }
    // ---- corrector -------------------------------------------------------
    bool mon_forked = false;
    TRY(launch_stress<MODE_CORR>(c, stress_args(c, c->vp)));
    if (!c->fc.empty()) {
        int unused = 0;
        TRY(friction_planes(c, false, &unused));
        // the patches read sig and Dt only; joined before the END pass
        CK(cudaEventRecord(c->ev_fork2, c->st));
        CK(cudaStreamWaitEvent(c->st2, c->ev_fork2, 0));
        TRY(monitor_planes(c, true, c->st2));
        CK(cudaEventRecord(c->ev_mon, c->st2));
        mon_forked = true;
    }
    if (!c->inter.s.empty()) {
        for (const auto &s : c->inter.s) {
            SrcArgs a{};
            a.g = g; a.mu = c->cfg.mu; a.s = s.slip; a.x = s.x; a.y = s.y; a.z = s.z;
            a.L = s.width; a.W = s.length; a.strike = s.strike; a.dip = s.dip; a.rake = s.rake; a.beta = s.beta;
            a.tau = c->m;
            k_moment_shear<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
            CKL();
            a.tau = c->tau;   // src/relax.f90:1199-1206 also adds it to tau
            k_moment_shear<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
            CKL();
        }
    }
    // interseismic tensile segments (src/relax.f90:1242-1260), opening rates
    for (const auto &s : c->inter.ts) {
        SrcArgs a{};
        a.g = g; a.mu = c->cfg.mu; a.lambda = c->cfg.lambda; a.s = s.opening; a.x = s.x; a.y = s.y; a.z = s.z;
        a.L = s.width; a.W = s.length; a.strike = s.strike; a.dip = s.dip; a.beta = c->cfg.beta;
        a.tau = c->m;
        k_moment_tensile<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
        a.tau = c->tau;
        k_moment_tensile<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(a);
        CKL();
    }
    TRY(upload_loads(c, ev, c->t, Dt, true, &loads));
    {
        XfArgs xa = xf_div(c);
        xa.tload = loads ? c->tload : nullptr;
        XiArgs xi = xi_update(c, c->u, c->u, 1.0f, true);
        if (c->vel) {
            const size_t vs = (size_t)c->vel_planes * g.plane;
            for (int k = 0; k < 3; k++) xi.vout[k] = c->vel + k * vs;
            xi.vplanes = c->vel_planes;
        }
        TRY(c->sp.green(xa, true, g.sx3h, g.sx3h, xi, c->cfg.lambda, c->cfg.mu, c->cfg.gam, c->st));
    }
    if (c->ur || c->urs) {
        const size_t n = 3 * (size_t)c->ur_planes * g.plane + (c->urs ? 3 * g.plane : 0);
        k_relax_accum<<<nblocks(n), RELAX_NTHREADS, 0, c->st>>>(c->vel, (size_t)c->vel_planes * g.plane, c->ur,
                                                                c->ur_planes, c->urs, c->inter_i3, g.plane,
                                                                c->dst);
        CKL();
    }
    // tau += Dt m, sig, next predictor moment; tmin, power and cei reduced by
    // the kernel's last block.  When t + Dt reaches the next event (the test
    // of src/relax.f90:859, made by k_dt) the kernel does nothing and
    // finish_step runs the event branch instead.
    if (mon_forked) CK(cudaStreamWaitEvent(c->st, c->ev_mon, 0));
    TRY(launch_stress<MODE_END>(c, stress_args(c, c->u)));
    return RELAX_OK;
}

static void drop_graph(relax_ctx *c)
{
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
}

// captures step_kernels into c->gexec; on any failure the context steps
// without a graph from then on
static int capture_step(relax_ctx *c)
{
    cudaGraph_t graph = nullptr;
    const long long l0 = c->prof.launches;
    if (cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaGetLastError();
        c->graph_off = true;
        return RELAX_OK;
    }
    const int rc = step_kernels(c);
    const cudaError_t e = cudaStreamEndCapture(c->st, &graph);
    c->glaunches = c->prof.launches - l0;
    c->prof.launches = l0;
    if (rc != RELAX_OK || e != cudaSuccess || !graph ||
        cudaGraphInstantiate(&c->gexec, graph, 0) != cudaSuccess) {
        cudaGetLastError();
        if (graph) cudaGraphDestroy(graph);
        c->gexec = nullptr;
        c->graph_off = true;
        return rc;
    }
    cudaGraphDestroy(graph);
    return RELAX_OK;
}

static int do_step(relax_ctx *c, const double *dt_override, relax_step_log *log)
{
    if (!c->cos_done) TRY(relax_coseismic(c, 0, nullptr));
    if (!c->m_valid) TRY(tail_init(c));
    memset(log, 0, sizeof *log);
    if (c->t >= c->cfg.interval) return RELAX_OK;
    // the step's time-step inputs; the pinned copy is free again once the
    // previous step's state came back
    c->dtp_h->pol = policy(c);
    c->dtp_h->in = DtIn{};
    c->dtp_h->in.t = c->t;
    c->dtp_h->in.dt_override = dt_override ? *dt_override : 0.0;
    c->dtp_h->in.oi = c->oi;
    c->dtp_h->in.use_override = dt_override ? 1 : 0;
    CK(cudaMemcpyAsync(c->dtp_d, c->dtp_h, sizeof(DtParams), cudaMemcpyHostToDevice, c->st));
    // a graph replays the step where the host has no part in it: no surface
    // loads, no per-launch profiling, after one plain step (which sizes the
    // friction partials)
    const bool graphable = c->events[c->e].l.empty() && !c->prof.on && !c->graph_off && c->plain_steps > 0;
    if (graphable && !c->gexec) TRY(capture_step(c));
    if (graphable && c->gexec) {
        CK(cudaGraphLaunch(c->gexec, c->st));
        c->prof.launches += c->glaunches;
    } else {
        TRY(step_kernels(c));
        c->plain_steps++;
    }
    TRY(pull_state(c));
    return finish_step(c, log);
}

extern "C" int relax_step(relax_ctx *c, const double *dt_override, relax_step_log *log)
{
    if (!c || !log) return fail(RELAX_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->device));
    return do_step(c, dt_override, log);
}

extern "C" int relax_run(relax_ctx *c, int max_steps, const double *dt_schedule, relax_step_log *logs,
                         int *nsteps_done)
{
    if (!c || !logs) return fail(RELAX_ERR_ARG, "null argument");
    if (c->cos_done) return fail(RELAX_ERR_STATE, "relax_run needs a context that has not been stepped");
    CK(cudaSetDevice(c->device));
    if (nsteps_done) *nsteps_done = 0;
    TRY(relax_coseismic(c, 0, &logs[0]));
    for (int k = 0; k < max_steps; k++) {
        relax_step_log lg;
        TRY(do_step(c, dt_schedule ? &dt_schedule[k] : nullptr, &lg));
        if (lg.i == 0) break;
        logs[k + 1] = lg;
        if (nsteps_done) *nsteps_done = k + 1;
    }
    return RELAX_OK;
}

extern "C" int relax_get_time(relax_ctx *c, double *t, int *i, int *e)
{
    if (!c) return fail(RELAX_ERR_ARG, "null context");
    if (t) *t = c->t;
    if (i) *i = c->i;
    if (e) *e = c->e;
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// field access in the reference layout
// ---------------------------------------------------------------------------
__global__ void k_scale(float *p, size_t n, float s)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) p[q] *= s;
}

static const float *tensor_field(relax_ctx *c, int which)
{
    switch (which) {
    case RELAX_FIELD_SIG: return c->sig;
    case RELAX_FIELD_TAU: return c->tau;
    case RELAX_FIELD_MOMENT: return c->m;
    case RELAX_FIELD_EPS: return c->eps;
    default: return nullptr;
    }
}

static int field_sig(relax_ctx *c)
{
    const Grid &g = c->g;
    if (c->sig_valid) return RELAX_OK;
    CK(cudaMemcpyAsync(c->sig, c->tau, 6 * g.nh * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
    k_scale<<<nblocks(6 * g.nh), RELAX_NTHREADS, 0, c->st>>>(c->sig, 6 * g.nh, -1.f);
    CKL();
    StressArgs a = stress_args(c, c->u);
    TRY(launch_stress<MODE_OP>(c, a));
    c->sig_valid = true;
    return RELAX_OK;
}

extern "C" int relax_get_field(relax_ctx *c, int which, void *host, size_t bytes)
{
    if (!c || !host) return fail(RELAX_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->device));
    const Grid &g = c->g;
    const size_t nvec = (size_t)(g.sx1 + 2) * g.sx2 * g.sx3h;
    float *tmp = nullptr;
    switch (which) {
    case RELAX_FIELD_U:
    case RELAX_FIELD_GAMMA: {
        const int nc = which == RELAX_FIELD_U ? 3 : 1;
        if (bytes != nc * nvec * sizeof(float)) return fail(RELAX_ERR_ARG, "field size %zu != %zu", bytes, nc * nvec * sizeof(float));
        tmp = c->work;   // free between steps; holds 6 nh >= 3 nvec floats
        const float *src = which == RELAX_FIELD_U ? c->u : c->gamma;
        for (int k = 0; k < nc; k++) {
            k_pad<<<nblocks(nvec), RELAX_NTHREADS, 0, c->st>>>(src + k * g.nh, tmp + k * nvec, g.sx1,
                                                                  (size_t)g.sx2 * g.sx3h);
        }
        break;
    }
    case RELAX_FIELD_SIG:
    case RELAX_FIELD_TAU:
    case RELAX_FIELD_MOMENT:
    case RELAX_FIELD_EPS: {
        if (bytes != g.nh * sizeof(relax_tensor)) return fail(RELAX_ERR_ARG, "field size %zu != %zu", bytes, g.nh * sizeof(relax_tensor));
        if (which == RELAX_FIELD_EPS && !c->eps) return fail(RELAX_ERR_STATE, "no transient rheology");
        if (which == RELAX_FIELD_SIG) TRY(field_sig(c));
        const float *src = tensor_field(c, which);
        tmp = c->work;
        k_soa_to_aos<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(src, (relax_tensor *)tmp, g.nh);
        break;
    }
    default:
        return fail(RELAX_ERR_ARG, "unknown field %d", which);
    }
    CKL();
    // one copy: a DMA straight into page-locked host memory, else the
    // driver's staged copy of pageable memory
    CK(cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return RELAX_OK;
}

extern "C" int relax_set_field(relax_ctx *c, int which, const void *host, size_t bytes)
{
    if (!c || !host) return fail(RELAX_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->device));
    const Grid &g = c->g;
    const size_t nvec = (size_t)(g.sx1 + 2) * g.sx2 * g.sx3h;
    float *tmp = nullptr;
    switch (which) {
    case RELAX_FIELD_U:
    case RELAX_FIELD_GAMMA: {
        const int nc = which == RELAX_FIELD_U ? 3 : 1;
        if (bytes != nc * nvec * sizeof(float)) return fail(RELAX_ERR_ARG, "field size mismatch");
        TRY(dalloc(&tmp, nc * nvec));
        CK(cudaMemcpyAsync(tmp, host, bytes, cudaMemcpyHostToDevice, c->st));
        float *dst = which == RELAX_FIELD_U ? c->u : c->gamma;
        for (int k = 0; k < nc; k++)
            k_unpad<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>(tmp + k * nvec, dst + k * g.nh, g.sx1,
                                                                 (size_t)g.sx2 * g.sx3h);
        break;
    }
    case RELAX_FIELD_SIG:
    case RELAX_FIELD_TAU:
    case RELAX_FIELD_MOMENT:
    case RELAX_FIELD_EPS: {
        if (bytes != g.nh * sizeof(relax_tensor)) return fail(RELAX_ERR_ARG, "field size mismatch");
        if (which == RELAX_FIELD_EPS && !c->eps) return fail(RELAX_ERR_STATE, "no transient rheology");
        TRY(dalloc(&tmp, 6 * g.nh));
        CK(cudaMemcpyAsync(tmp, host, bytes, cudaMemcpyHostToDevice, c->st));
        float *dst = const_cast<float *>(tensor_field(c, which));
        k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, c->st>>>((const relax_tensor *)tmp, dst, g.nh);
        break;
    }
    default:
        return fail(RELAX_ERR_ARG, "unknown field %d", which);
    }
    CKL();
    CK(cudaStreamSynchronize(c->st));
    dfree(tmp);
    if (which == RELAX_FIELD_SIG) c->sig_valid = true;
    else c->m_valid = false, c->sig_valid = false;
    if (which == RELAX_FIELD_MOMENT) c->m_valid = true;
    return RELAX_OK;
}

// One horizontal plane of a field, the slice cuexportspatial_ reads for
// exportgrd (src/export.f90:952-955): components one after the other, each
// sx1 x sx2 floats with x1 fastest and no padding.
extern "C" int relax_get_plane(relax_ctx *c, int which, int i3, float *host, size_t bytes)
{
    if (!c || !host) return fail(RELAX_ERR_ARG, "null argument");
    const Grid &g = c->g;
    if (i3 < 0 || i3 >= g.sx3h) return fail(RELAX_ERR_ARG, "plane %d outside [0, %d)", i3, g.sx3h);
    CK(cudaSetDevice(c->device));
    const size_t np = (size_t)g.sx1 * g.sx2;
    const float *src = nullptr;
    int nc = 0;
    size_t cs = g.nh, off = (size_t)i3 * np;    // component stride, plane offset
    switch (which) {
    case RELAX_FIELD_U: src = c->u; nc = 3; break;
    case RELAX_FIELD_GAMMA: src = c->gamma; nc = 1; break;
    case RELAX_FIELD_V:
        if (i3 >= c->vel_planes) return fail(RELAX_ERR_STATE, "velocity of plane %d not kept", i3);
        src = c->vel; nc = 3; cs = (size_t)c->vel_planes * g.plane;
        break;
    case RELAX_FIELD_UR:
        nc = 3;
        if (i3 < c->ur_planes) {
            src = c->ur; cs = (size_t)c->ur_planes * g.plane;
        } else if (i3 == c->inter_i3) {
            src = c->urs; cs = g.plane; off = 0;   // the slice buffer holds this plane alone
        } else {
            return fail(RELAX_ERR_STATE, "postseismic displacement of plane %d not kept", i3);
        }
        break;
    case RELAX_FIELD_SIG:
    case RELAX_FIELD_TAU:
    case RELAX_FIELD_MOMENT:
    case RELAX_FIELD_EPS:
        if (which == RELAX_FIELD_EPS && !c->eps) return fail(RELAX_ERR_STATE, "no transient rheology");
        if (which == RELAX_FIELD_SIG) TRY(field_sig(c));
        src = tensor_field(c, which);
        nc = 6;
        break;
    default:
        return fail(RELAX_ERR_ARG, "unknown field %d", which);
    }
    if (bytes != nc * np * sizeof(float)) return fail(RELAX_ERR_ARG, "plane size %zu != %zu", bytes, nc * np * sizeof(float));
    for (int k = 0; k < nc; k++)
        CK(cudaMemcpyAsync(host + k * np, src + k * cs + off, np * sizeof(float),
                           cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return RELAX_OK;
}

__global__ void k_gather_points(const float *u, const float *sig, size_t nh, const int *idx, int n, float *out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const size_t q = (size_t)idx[p];
    for (int k = 0; k < 3; k++) out[9 * p + k] = u[k * nh + q];
    for (int k = 0; k < 6; k++) out[9 * p + 3 + k] = sig[k * nh + q];
}

// Displacement and stress at grid points, the read-back of cuexportpoints_
// (src/util.f90:104-105) for n points at once.  index: n triples
// (i1, i2, i3), 0-based; u: 3n doubles; sig: n tensors.
extern "C" int relax_get_points(relax_ctx *c, int n, const int *index, double *u, relax_tensor *sig)
{
    if (!c || n < 0 || (n > 0 && (!index || !u || !sig))) return fail(RELAX_ERR_ARG, "null argument");
    if (n == 0) return RELAX_OK;
    const Grid &g = c->g;
    std::vector<int> q(n);
    for (int p = 0; p < n; p++) {
        const int i1 = index[3 * p], i2 = index[3 * p + 1], i3 = index[3 * p + 2];
        if (i1 < 0 || i1 >= g.sx1 || i2 < 0 || i2 >= g.sx2 || i3 < 0 || i3 >= g.sx3h)
            return fail(RELAX_ERR_ARG, "point %d (%d, %d, %d) outside the grid", p, i1, i2, i3);
        q[p] = i1 + g.sx1 * (i2 + g.sx2 * i3);
    }
    CK(cudaSetDevice(c->device));
    TRY(field_sig(c));
    float *buf = nullptr;
    TRY(dalloc(&buf, 10 * (size_t)n));
    int *didx = (int *)(buf + 9 * (size_t)n);
    std::vector<float> out(9 * (size_t)n);
    cudaError_t e = cudaMemcpyAsync(didx, q.data(), n * sizeof(int), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) {
        k_gather_points<<<(n + 127) / 128, 128, 0, c->st>>>(c->u, c->sig, g.nh, didx, n, buf);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), buf, out.size() * sizeof(float), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    dfree(buf);
    if (e != cudaSuccess) return fail(RELAX_ERR_CUDA, "point read-back: %s", cudaGetErrorString(e));
    for (int p = 0; p < n; p++) {
        const float *o = &out[9 * (size_t)p];
        u[3 * p] = o[0]; u[3 * p + 1] = o[1]; u[3 * p + 2] = o[2];
        sig[p].s11 = o[3]; sig[p].s12 = o[4]; sig[p].s13 = o[5];
        sig[p].s22 = o[6]; sig[p].s23 = o[7]; sig[p].s33 = o[8];
    }
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// observation planes: monitorstressfield / monitorfield,
// src/elastic3d.f90:3404-3762
// ---------------------------------------------------------------------------
struct MonitorGeom {
    double x, y, z, cs, ss, cd, sd;   // plane centre, cos / sin of strike and dip
    int px2, px3;
};

// fix, src/elastic3d.f90:70-83: the nearest integer, halves rounded down
__device__ __forceinline__ int fix_d(double v)
{
    const double f = floor(v), c = ceil(v);
    return (int)(__dsub_rn(v, f) > 0.5 ? c : f);
}

// sinc, src/elastic3d.f90:498-506 (pi in double precision)
__device__ __forceinline__ double sinc_d(double x)
{
    const double pi = 3.141592653589793115997963468544185161;
    return x != 0.0 ? sin(__dmul_rn(pi, x)) / __dmul_rn(pi, x) : 1.0;
}

// One thread per sample point j2 + (px2 + 1) j3 of the plane.  NC = 6
// samples the stress (sampletensor: a single-precision weighted sum, then
// the single-precision factor 1/sum), NC = 1 the scalar field (sample:
// double-precision sum).  The arithmetic keeps the reference's order and
// precisions, with no contraction into fused multiply-adds.  out: 5 + NC
// doubles per point -- x1, x2, x3, yr, zr and the sampled values.
template <int NC>
__global__ void k_monitor_plane(Grid g, const float *f, MonitorGeom p, double *out)
{
    const int n2 = p.px2 + 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n2 * (p.px3 + 1)) return;
    const int j2 = q % n2 + 1, j3 = q / n2 + 1;
    // ref2local
    const double xa = __dsub_rn(__dmul_rn(p.cs, p.x), __dmul_rn(p.ss, p.y));
    const double xr = __dsub_rn(__dmul_rn(p.cd, xa), __dmul_rn(p.sd, p.z));
    double yr = __dadd_rn(__dmul_rn(p.ss, p.x), __dmul_rn(p.cs, p.y));
    double zr = __dadd_rn(__dmul_rn(p.sd, xa), __dmul_rn(p.cd, p.z));
    // single-precision offsets along strike and down dip
    yr = (double)__fadd_rn((float)yr, (float)(((double)j2 - (double)p.px2 / 2.0 - 1.0) * g.dx2));
    zr = (double)__fadd_rn((float)zr, (float)(((double)j3 - (double)p.px3 / 2.0 - 1.0) * g.dx3));
    // local2ref
    const double x2p = __dadd_rn(__dmul_rn(p.cd, xr), __dmul_rn(p.sd, zr));
    const double x1 = __dadd_rn(__dmul_rn(p.cs, x2p), __dmul_rn(p.ss, yr));
    const double x2 = __dadd_rn(-__dmul_rn(p.ss, x2p), __dmul_rn(p.cs, yr));
    const double x3 = __dadd_rn(-__dmul_rn(p.sd, xr), __dmul_rn(p.cd, zr));
    double *o = out + (size_t)q * (5 + NC);
    o[0] = x1; o[1] = x2; o[2] = x3; o[3] = yr; o[4] = zr;
    float acc[NC];
    for (int m = 0; m < NC; m++) acc[m] = 0.f;
    double value = 0.0;
    const int sx1 = g.sx1, sx2 = g.sx2, sx3 = g.sx3h;
    const double dx1 = g.dx1, dx2 = g.dx2, dx3 = g.dx3;
    const bool inside = !(x1 > (double)(sx1 / 2 - 1) * dx1 || x1 < -(double)(sx1 / 2) * dx1 ||
                          x2 > (double)(sx2 / 2 - 1) * dx2 || x2 < -(double)(sx2 / 2) * dx2 ||
                          x3 > (double)(sx3 - 1) * dx3 || x3 < 0.0);
    if (inside) {
        // shiftedindex (1-based) and shiftedcoordinates of the closest node
        const int i = (sx1 + fix_d(x1 / dx1)) % sx1 + 1;
        const int j = (sx2 + fix_d(x2 / dx2)) % sx2 + 1;
        const int k = fix_d(x3 / dx3) + 1;
        const double x = (double)(i <= sx1 / 2 ? i - 1 : i - sx1 - 1) * dx1;
        const double y = (double)(j <= sx2 / 2 ? j - 1 : j - sx2 - 1) * dx2;
        const double z = (double)(k <= sx3 ? k - 1 : k - 2 * sx3 - 1) * dx3;
        const double eps = (double)1e-2f;   // a single-precision literal in the reference
        const size_t nh = g.nh;
        if (fabs(x - x1) < eps * dx1 && fabs(y - x2) < eps * dx2 && fabs(z - x3) < eps * dx3) {
            const size_t c = (size_t)(i - 1) + (size_t)sx1 * ((size_t)(j - 1) + (size_t)sx2 * (k - 1));
            if (NC == 1) value = (double)f[c];
            else for (int m = 0; m < NC; m++) acc[m] = f[m * nh + c];
        } else {
            double sum = 0.0;
            for (int l3 = -2; l3 <= 2; l3++) {
                if (k + l3 <= 0 || k + l3 > sx3) continue;
                const int i3p = k + l3;
                const double w3 = sinc_d(__dsub_rn(__dadd_rn(z, __dmul_rn((double)l3, dx3)), x3) / dx3);
                for (int l2 = -2; l2 <= 2; l2++) {
                    const int i2p = (sx2 + j - 1 + l2) % sx2 + 1;
                    const double w2 = sinc_d(__dsub_rn(__dadd_rn(y, __dmul_rn((double)l2, dx2)), x2) / dx2);
                    for (int l1 = -2; l1 <= 2; l1++) {
                        const int i1p = (sx1 + i - 1 + l1) % sx1 + 1;
                        const double w1 = sinc_d(__dsub_rn(__dadd_rn(x, __dmul_rn((double)l1, dx1)), x1) / dx1);
                        // sinc(.)*dx1*sinc(.)*dx2*sinc(.)*dx3, left to right
                        double w = __dmul_rn(w1, dx1);
                        w = __dmul_rn(w, w2);
                        w = __dmul_rn(w, dx2);
                        w = __dmul_rn(w, w3);
                        w = __dmul_rn(w, dx3);
                        const size_t c = (size_t)(i1p - 1) + (size_t)sx1 * ((size_t)(i2p - 1) + (size_t)sx2 * (i3p - 1));
                        if (NC == 1) {
                            value = __dadd_rn(value, __dmul_rn(w, (double)f[c]));
                        } else {
                            const float wf = (float)w;
                            for (int m = 0; m < NC; m++) acc[m] = __fadd_rn(acc[m], __fmul_rn(wf, f[m * nh + c]));
                        }
                        sum = __dadd_rn(sum, w);
                    }
                }
            }
            if (sum > (double)1e-6f) {
                if (NC == 1) {
                    value = value / sum;
                } else {
                    const float r = (float)(1.0 / sum);
                    for (int m = 0; m < NC; m++) acc[m] = __fmul_rn(r, acc[m]);
                }
            }
        }
    }
    if (NC == 1) o[5] = value;
    else for (int m = 0; m < NC; m++) o[5 + m] = (double)acc[m];
}

extern "C" int relax_monitor_plane(relax_ctx *c, int which, const relax_obsplane *op, double beta,
                                   relax_slippatch *out, size_t n, int *px2, int *px3)
{
    if (!c || !op) return fail(RELAX_ERR_ARG, "null argument");
    if (which != RELAX_FIELD_SIG && which != RELAX_FIELD_GAMMA)
        return fail(RELAX_ERR_ARG, "planes sample the stress or gamma, not field %d", which);
    const Grid &g = c->g;
    // called as monitorstressfield(x, y, z, width, length, ...): its L is the
    // plane's width (down dip), its W the length (along strike)
    const double Wp = op->length * (1.0 + 2.0 * beta), Lp = op->width * (1.0 + 2.0 * beta);
    const int p2 = fixr(Wp / g.dx2), p3 = fixr(Lp / g.dx3);
    if (p2 < 0 || p3 < 0 || p2 > (1 << 15) || p3 > (1 << 15))
        return fail(RELAX_ERR_ARG, "observation plane of %d x %d samples", p2 + 1, p3 + 1);
    if (px2) *px2 = p2;
    if (px3) *px3 = p3;
    if (!out) return RELAX_OK;
    const size_t np = (size_t)(p2 + 1) * (p3 + 1);
    if (n < np) return fail(RELAX_ERR_ARG, "%zu patches for a plane of %zu samples", n, np);
    const int nc = which == RELAX_FIELD_SIG ? 6 : 1;
    CK(cudaSetDevice(c->device));
    if (which == RELAX_FIELD_SIG) TRY(field_sig(c));
    double *buf = nullptr;
    TRY(dalloc(&buf, (5 + nc) * np));
    const MonitorGeom geo{op->x, op->y, op->z, cos(op->strike), sin(op->strike), cos(op->dip), sin(op->dip), p2, p3};
    const unsigned nb = (unsigned)((np + 127) / 128);
    if (nc == 6) k_monitor_plane<6><<<nb, 128, 0, c->st>>>(g, c->sig, geo, buf);
    else k_monitor_plane<1><<<nb, 128, 0, c->st>>>(g, c->gamma, geo, buf);
    cudaError_t e = cudaGetLastError();
    std::vector<double> h((5 + nc) * np);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), buf, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    dfree(buf);
    if (e != cudaSuccess) return fail(RELAX_ERR_CUDA, "plane sampling: %s", cudaGetErrorString(e));
    for (size_t q = 0; q < np; q++) {
        const double *v = &h[(5 + nc) * q];
        relax_slippatch &s = out[q];
        memset(&s, 0, sizeof s);
        s.x1 = v[0]; s.x2 = v[1]; s.x3 = v[2]; s.lx = v[3]; s.lz = v[4];
        if (nc == 1) {
            s.slip = v[5];
        } else {
            s.sig.s11 = (float)v[5]; s.sig.s12 = (float)v[6]; s.sig.s13 = (float)v[7];
            s.sig.s22 = (float)v[8]; s.sig.s23 = (float)v[9]; s.sig.s33 = (float)v[10];
        }
    }
    return RELAX_OK;
}

extern "C" int relax_segment_stress(relax_ctx *c, int n, const relax_segment *sop, relax_tensor *sig)
{
    if (!c || n < 0 || (n > 0 && (!sop || !sig))) return fail(RELAX_ERR_ARG, "null argument");
    if (n == 0) return RELAX_OK;
    const Grid &g = c->g;
    std::vector<int> idx(3 * (size_t)n);
    for (int k = 0; k < n; k++) {
        // shiftedindex with the full sx3, as the segment exports call it
        TRY(relax_shifted_index(sop[k].x, sop[k].y, sop[k].z, g.sx1, g.sx2, 2 * g.sx3h, g.dx1, g.dx2, g.dx3,
                                &idx[3 * k], &idx[3 * k + 1], &idx[3 * k + 2]));
        if (idx[3 * k + 2] >= g.sx3h)
            return fail(RELAX_ERR_ARG, "segment %d at depth %g lies below the stored half of the grid", k + 1,
                        sop[k].z);
    }
    std::vector<double> u(3 * (size_t)n);
    return relax_get_points(c, n, idx.data(), u.data(), sig);
}

// Keeps the corrector's velocity field v (src/relax.f90:829, the v1..v3
// of the output block :959-975) for planes i3 < vel_planes, and accumulates
// the postseismic displacement sum Dt v over planes i3 < ur_planes (u1r..u3r,
// :846-850) and in plane inter_i3 alone (inter1..inter3, :839-843; -1: off).
// Every later step writes them; relax_get_plane reads them as RELAX_FIELD_V
// and RELAX_FIELD_UR.
extern "C" int relax_set_precision(relax_ctx *c, int mode)
{
    if (!c) return fail(RELAX_ERR_ARG, "null context");
    if (mode != RELAX_PRECISION_FP32 && mode != RELAX_PRECISION_MIXED)
        return fail(RELAX_ERR_ARG, "precision mode %d", mode);
    if (mode == RELAX_PRECISION_MIXED && c->g.sx3 != 128)
        return fail(RELAX_ERR_UNSUPPORTED, "the mixed-precision x3 pass needs a 128-deep box (sx3 = %d)", c->g.sx3);
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->st));
    TRY(c->sp.set_mixed(mode, c->err, c->st));
    CK(cudaStreamSynchronize(c->st));
    drop_graph(c);
    return RELAX_OK;
}

extern "C" int relax_track_relaxation(relax_ctx *c, int vel_planes, int ur_planes, int inter_i3)
{
    if (!c) return fail(RELAX_ERR_ARG, "null context");
    const Grid &g = c->g;
    if (!c->own_dst) return fail(RELAX_ERR_UNSUPPORTED, "batch members do not track the relaxation");
    if (vel_planes < 0 || vel_planes > g.sx3h || ur_planes < 0 || ur_planes > g.sx3h || inter_i3 < -1 ||
        inter_i3 >= g.sx3h)
        return fail(RELAX_ERR_ARG, "planes outside [0, %d]", g.sx3h);
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->st));
    drop_graph(c);   // the corrector's epilogue arguments change
    for (float **p : {&c->vel, &c->ur, &c->urs})
        if (*p) { dfree(*p); *p = nullptr; }
    const int nv = std::max(std::max(vel_planes, ur_planes), inter_i3 + 1);
    c->vel_planes = nv;
    c->ur_planes = ur_planes;
    c->inter_i3 = inter_i3;
    if (nv > 0) {
        TRY(dalloc(&c->vel, 3 * (size_t)nv * g.plane));
        CK(cudaMemsetAsync(c->vel, 0, 3 * (size_t)nv * g.plane * sizeof(float), c->st));
    }
    if (ur_planes > 0) {
        TRY(dalloc(&c->ur, 3 * (size_t)ur_planes * g.plane));
        CK(cudaMemsetAsync(c->ur, 0, 3 * (size_t)ur_planes * g.plane * sizeof(float), c->st));
    }
    if (inter_i3 >= 0) {
        TRY(dalloc(&c->urs, 3 * g.plane));
        CK(cudaMemsetAsync(c->urs, 0, 3 * g.plane * sizeof(float), c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return RELAX_OK;
}

extern "C" int relax_get_grid(relax_ctx *c, int *sx, double *dx)
{
    if (!c) return fail(RELAX_ERR_ARG, "null context");
    if (sx) { sx[0] = c->g.sx1; sx[1] = c->g.sx2; sx[2] = c->g.sx3; }
    if (dx) { dx[0] = c->g.dx1; dx[1] = c->g.dx2; dx[2] = c->g.dx3; }
    return RELAX_OK;
}

extern "C" int relax_get_plane_shape(relax_ctx *c, int k, int *px2, int *px3)
{
    if (!c) return fail(RELAX_ERR_ARG, "null context");
    if (k < 0 || k >= (int)c->planes.size()) return fail(RELAX_ERR_ARG, "plane %d out of range", k);
    if (px2) *px2 = std::max(0, c->planes[k].px2);
    if (px3) *px3 = std::max(0, c->planes[k].px3);
    return RELAX_OK;
}

extern "C" int relax_num_planes(relax_ctx *c, int *np)
{
    if (!c || !np) return fail(RELAX_ERR_ARG, "null argument");
    *np = (int)c->planes.size();
    return RELAX_OK;
}

extern "C" int relax_get_patches(relax_ctx *c, int k, relax_slippatch *host, size_t n)
{
    if (!c || !host) return fail(RELAX_ERR_ARG, "null argument");
    if (k < 0 || k >= (int)c->planes.size()) return fail(RELAX_ERR_ARG, "plane %d out of range", k);
    const size_t np = (size_t)std::max(0, c->planes[k].px2) * std::max(0, c->planes[k].px3);
    if (n != np) return fail(RELAX_ERR_ARG, "plane %d has %zu patches", k, np);
    CK(cudaMemcpyAsync(host, c->patch + c->patch_off[k], np * sizeof(relax_slippatch), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// checkpoint: the state a step reads, to a raw file and back
// ---------------------------------------------------------------------------
namespace ckpt {

const char MAGIC[8] = {'R', 'L', 'X', 'C', 'K', 'P', 'T', '1'};

struct Header {
    char magic[8];
    int sx1, sx2, sx3, npatch;
    int has_eps, vel_planes, ur_planes, inter_i3;
    double t;
    int i, e, oi, cos_done, m_valid, sig_valid;
    StepState st;
    unsigned long long payload_bytes, checksum;
};

struct Block {
    void *d;
    size_t bytes;
};

// FNV-1a over the payload, in the order written
inline void fnv(unsigned long long &h, const unsigned char *p, size_t n)
{
    for (size_t k = 0; k < n; k++) {
        h ^= p[k];
        h *= 1099511628211ull;
    }
}

std::vector<Block> blocks(relax_ctx *c, int npatch)
{
    const Grid &g = c->g;
    std::vector<Block> b = {{c->u, 3 * g.nh * sizeof(float)},   {c->tau, 6 * g.nh * sizeof(float)},
                            {c->m, 6 * g.nh * sizeof(float)},   {c->sig, 6 * g.nh * sizeof(float)},
                            {c->gamma, g.nh * sizeof(float)}};
    if (c->eps) b.push_back({c->eps, 6 * g.nh * sizeof(float)});
    if (c->epsdot) b.push_back({c->epsdot, 6 * g.nh * sizeof(float)});
    if (npatch > 0) b.push_back({c->patch, (size_t)npatch * sizeof(relax_slippatch)});
    if (c->vel) b.push_back({c->vel, 3 * (size_t)c->vel_planes * g.plane * sizeof(float)});
    if (c->ur) b.push_back({c->ur, 3 * (size_t)c->ur_planes * g.plane * sizeof(float)});
    if (c->urs) b.push_back({c->urs, 3 * g.plane * sizeof(float)});
    return b;
}

int npatch(const relax_ctx *c)
{
    int n = 0;
    for (const auto &p : c->planes) n += std::max(0, p.px2) * std::max(0, p.px3);
    return n;
}

}  // namespace ckpt

// Writes the state of a context between steps (displacement, stress,
// moment, prestress, afterslip history, transient strain, slip patches,
// the tracked relaxation fields, time, counters and the step state) to a
// raw file.  RELAX has no restart (its output files cannot restart a run);
// a context created from the same configuration and given the file with
// relax_checkpoint_load continues bit for bit.
extern "C" int relax_checkpoint_save(relax_ctx *c, const char *path)
{
    if (!c || !path) return fail(RELAX_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->device));
    if (c->cos_done && !c->m_valid) TRY(tail_init(c));
    CK(cudaMemcpyAsync(c->hst, c->dst, sizeof(StepState), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    ckpt::Header h{};
    memcpy(h.magic, ckpt::MAGIC, 8);
    h.sx1 = c->g.sx1; h.sx2 = c->g.sx2; h.sx3 = c->g.sx3;
    h.npatch = ckpt::npatch(c);
    h.has_eps = c->eps ? 1 : 0;
    h.vel_planes = c->vel ? c->vel_planes : 0;
    h.ur_planes = c->ur ? c->ur_planes : 0;
    h.inter_i3 = c->urs ? c->inter_i3 : -1;
    h.t = c->t; h.i = c->i; h.e = c->e; h.oi = c->oi;
    h.cos_done = c->cos_done; h.m_valid = c->m_valid; h.sig_valid = c->sig_valid;
    h.st = *c->hst;
    const std::vector<ckpt::Block> bl = ckpt::blocks(c, h.npatch);
    FILE *fp = fopen(path, "wb");
    if (!fp) return fail(RELAX_ERR_ARG, "cannot open %s for writing", path);
    // header first (rewritten with the checksum at the end)
    bool ok = fwrite(&h, sizeof h, 1, fp) == 1;
    unsigned long long sum = 1469598103934665603ull, total = 0;
    std::vector<unsigned char> buf;
    for (const auto &b : bl) {
        if (!ok) break;
        buf.resize(b.bytes);
        if (cudaMemcpy(buf.data(), b.d, b.bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
            fclose(fp);
            return fail(RELAX_ERR_CUDA, "checkpoint: device copy failed");
        }
        ckpt::fnv(sum, buf.data(), b.bytes);
        total += b.bytes;
        ok = fwrite(buf.data(), 1, b.bytes, fp) == b.bytes;
    }
    h.payload_bytes = total;
    h.checksum = sum;
    if (ok) ok = fseek(fp, 0, SEEK_SET) == 0 && fwrite(&h, sizeof h, 1, fp) == 1;
    if (fclose(fp) != 0) ok = false;
    if (!ok) return fail(RELAX_ERR_ARG, "writing %s failed", path);
    return RELAX_OK;
}

// Restores a checkpoint into a context created from the same configuration
// (grid, mechanisms, afterslip planes) and with the same tracking of the
// relaxation fields.  The file's checksum is verified before the state is
// replaced.
extern "C" int relax_checkpoint_load(relax_ctx *c, const char *path)
{
    if (!c || !path) return fail(RELAX_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->device));
    FILE *fp = fopen(path, "rb");
    if (!fp) return fail(RELAX_ERR_ARG, "cannot open %s", path);
    ckpt::Header h{};
    if (fread(&h, sizeof h, 1, fp) != 1 || memcmp(h.magic, ckpt::MAGIC, 8) != 0) {
        fclose(fp);
        return fail(RELAX_ERR_ARG, "%s is not a checkpoint", path);
    }
    const int npatch = ckpt::npatch(c);
    if (h.sx1 != c->g.sx1 || h.sx2 != c->g.sx2 || h.sx3 != c->g.sx3 || h.npatch != npatch ||
        h.has_eps != (c->eps ? 1 : 0) || h.vel_planes != (c->vel ? c->vel_planes : 0) ||
        h.ur_planes != (c->ur ? c->ur_planes : 0) || h.inter_i3 != (c->urs ? c->inter_i3 : -1)) {
        fclose(fp);
        return fail(RELAX_ERR_STATE, "checkpoint %s does not match this context (grid %dx%dx%d, %d patches)", path,
                    h.sx1, h.sx2, h.sx3, h.npatch);
    }
    const std::vector<ckpt::Block> bl = ckpt::blocks(c, npatch);
    std::vector<std::vector<unsigned char>> data(bl.size());
    unsigned long long sum = 1469598103934665603ull, total = 0;
    bool ok = true;
    for (size_t k = 0; k < bl.size() && ok; k++) {
        data[k].resize(bl[k].bytes);
        ok = fread(data[k].data(), 1, bl[k].bytes, fp) == bl[k].bytes;
        if (ok) ckpt::fnv(sum, data[k].data(), bl[k].bytes);
        total += bl[k].bytes;
    }
    unsigned char extra;
    if (ok && fread(&extra, 1, 1, fp) == 1) ok = false;
    fclose(fp);
    if (!ok || total != h.payload_bytes || sum != h.checksum)
        return fail(RELAX_ERR_ARG, "checkpoint %s is truncated or corrupt", path);
    CK(cudaStreamSynchronize(c->st));
    for (size_t k = 0; k < bl.size(); k++)
        CK(cudaMemcpy(bl[k].d, data[k].data(), bl[k].bytes, cudaMemcpyHostToDevice));
    *c->hst = h.st;
    CK(cudaMemcpy(c->dst, c->hst, sizeof(StepState), cudaMemcpyHostToDevice));
    c->t = h.t; c->i = h.i; c->e = h.e; c->oi = h.oi;
    c->cos_done = h.cos_done != 0;
    c->m_valid = h.m_valid != 0;
    c->sig_valid = h.sig_valid != 0;
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// stateless operators on device buffers in the reference layout
// ---------------------------------------------------------------------------
struct Scratch {
    std::vector<void *> p;
    cudaStream_t st;
    explicit Scratch(cudaStream_t s) : st(s) {}
    template <typename T>
    int get(T **out, size_t n)
    {
        void *q = nullptr;
        cudaError_t e = cudaMallocAsync(&q, std::max<size_t>(n, 1) * sizeof(T), st);
        if (e != cudaSuccess) return fail(RELAX_ERR_NOMEM, "cudaMallocAsync: %s", cudaGetErrorString(e));
        p.push_back(q);
        *out = (T *)q;
        return RELAX_OK;
    }
    ~Scratch()
    {
        for (void *q : p) cudaFreeAsync(q, st);
    }
};

static StressArgs op_args(const Grid &g, double lambda, double mu)
{
    StressArgs a{};
    a.g = g;
    a.k1 = (float)(0.5 / g.dx1); a.k2 = (float)(0.5 / g.dx2);
    a.k3 = (float)(0.5 / g.dx3); a.k3b = (float)(1.0 / g.dx3);
    a.lam = (float)lambda; a.mu2 = (float)(2.0 * mu); a.muinv = (float)(1.0 / mu);
    return a;
}

extern "C" int relax_op_stressupdate(const float *u1, const float *u2, const float *u3, double lambda,
                                     double mu, double dx1, double dx2, double dx3, int sx1, int sx2,
                                     int sx3h, relax_tensor *sig, void *stream)
{
    Grid g;
    TRY(make_grid(g, sx1, sx2, 2 * sx3h, dx1, dx2, dx3));
    cudaStream_t st = (cudaStream_t)stream;
    Scratch sc(st);
    float *w, *s;
    TRY(sc.get(&w, 3 * g.nh));
    TRY(sc.get(&s, 6 * g.nh));
    const float *us[3] = {u1, u2, u3};
    for (int k = 0; k < 3; k++)
        k_unpad<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(us[k], w + k * g.nh, sx1, (size_t)sx2 * sx3h);
    k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(sig, s, g.nh);
    StressArgs a = op_args(g, lambda, mu);
    a.w = w;
    a.sig = s;
    if (has_fir(g)) {
        float *wxy;
        TRY(sc.get(&wxy, 6 * g.nh));
        k_fir_xy<<<nblocks(3 * (g.nh / 4)), RELAX_NTHREADS, 0, st>>>(g, w, wxy, wxy + 3 * g.nh, fir_x(g),
                                                                     fir_y(g), a.k1, a.k2);
        a.wx = wxy;
        a.wy = wxy + 3 * g.nh;
        k_stress<MODE_OP, false, false, true><<<nblocks(g.nh / 4), RELAX_NTHREADS, 0, st>>>(a);
    } else {
        k_stress<MODE_OP><<<nblocks(g.nh / 4), RELAX_NTHREADS, 0, st>>>(a);
    }
    k_soa_to_aos<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(s, sig, g.nh);
    CKL();
    return RELAX_OK;
}

extern "C" int relax_op_bodyforce(const relax_tensor *sig, double dx1, double dx2, double dx3, int sx1,
                                  int sx2, int sx3h, float *c1, float *c2, float *c3, float *t1, float *t2,
                                  float *t3, void *stream)
{
    Grid g;
    TRY(make_grid(g, sx1, sx2, 2 * sx3h, dx1, dx2, dx3));
    cudaStream_t st = (cudaStream_t)stream;
    Scratch sc(st);
    float *s;
    TRY(sc.get(&s, 6 * g.nh));
    k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(sig, s, g.nh);
    k_bodyforce<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(g, s, c1, c2, c3, t1, t2, t3, (float)(0.5 / dx1),
                                                          (float)(0.5 / dx2), (float)(0.5 / dx3), (float)(1.0 / dx3),
                                                          fir_x(g), fir_y(g));
    CKL();
    return RELAX_OK;
}

extern "C" int relax_op_viscouseigenstress(double mu, const relax_layer *structure,
                                           const relax_tensor_layer *prestress, const relax_tensor *sig,
                                           int sx1, int sx2, int sx3h, relax_tensor *moment,
                                           double *maxwelltime, float *gamma, const float *dgammadot0,
                                           void *stream)
{
    Grid g;
    TRY(make_grid(g, sx1, sx2, 2 * sx3h, 1.0, 1.0, 1.0));
    if (!structure) return fail(RELAX_ERR_ARG, "null structure");
    for (int i = 0; i < sx3h; i++)
        if (structure[i].stressexponent < 0.999999) return fail(RELAX_ERR_POWER, "invalid power exponent");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch sc(st);
    std::vector<float> spdev;
    std::vector<DepthVisc> dv;
    prestress_terms(prestress, sx3h, mu, structure, &spdev, &dv);
    float *s, *mo, *gm = nullptr, *spd = nullptr, *tmp;
    DepthVisc *dvd;
    double *amp;
    const int nb = (int)nblocks(g.nh / 4);
    TRY(sc.get(&s, 6 * g.nh));
    TRY(sc.get(&mo, 6 * g.nh));
    TRY(sc.get(&dvd, sx3h));
    TRY(sc.get(&tmp, 2 * (size_t)nb));
    TRY(sc.get(&amp, 2 * (size_t)nb));
    CK(cudaMemcpyAsync(dvd, dv.data(), sx3h * sizeof(DepthVisc), cudaMemcpyHostToDevice, st));
    if (prestress) {
        TRY(sc.get(&spd, 6 * (size_t)sx3h));
        CK(cudaMemcpyAsync(spd, spdev.data(), 6 * sx3h * sizeof(float), cudaMemcpyHostToDevice, st));
    }
    if (gamma) {
        TRY(sc.get(&gm, g.nh));
        k_unpad<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(gamma, gm, sx1, (size_t)sx2 * sx3h);
    }
    k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(sig, s, g.nh);
    k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(moment, mo, g.nh);
    StressArgs a = op_args(g, 1.0, mu);
    a.sig = s; a.m = mo; a.gamma = gm; a.visc[0] = dvd; a.spdev = spd;
    a.dg0[0] = dgammadot0;
    a.tm_part = tmp; a.amp_part = amp;
    k_stress<MODE_EIGEN><<<nb, RELAX_NTHREADS, 0, st>>>(a);
    k_soa_to_aos<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(mo, moment, g.nh);
    if (gamma)   // back into the first sx1 entries of each padded row
        k_repad<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(gm, gamma, sx1, (size_t)sx2 * sx3h);
    CKL();
    if (maxwelltime) {
        std::vector<float> h(nb);
        CK(cudaMemcpyAsync(h.data(), tmp, nb * sizeof(float), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        float tm = (float)*maxwelltime;
        for (float v : h) tm = std::min(tm, v);
        *maxwelltime = std::min((double)tm, *maxwelltime);
    }
    return RELAX_OK;
}

extern "C" int relax_op_transienteigenstress(double mu, const relax_layer *structure, const relax_tensor *sig,
                                             const relax_tensor *epsilonik, int sx1, int sx2, int sx3h,
                                             relax_tensor *moment, relax_tensor *epsilonikdot,
                                             double *maxwelltime, const float *dgammadot0, void *stream)
{
    Grid g;
    TRY(make_grid(g, sx1, sx2, 2 * sx3h, 1.0, 1.0, 1.0));
    if (!structure || !sig || !epsilonik || !moment || !epsilonikdot) return fail(RELAX_ERR_ARG, "null argument");
    for (int i = 0; i < sx3h; i++)
        if (structure[i].stressexponent < 0.999999) return fail(RELAX_ERR_POWER, "invalid power exponent");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch sc(st);
    std::vector<TransLayer> tl(sx3h);
    for (int i = 0; i < sx3h; i++)
        tl[i] = TransLayer{(float)structure[i].gammadot0, (float)structure[i].stressexponent,
                           (float)(2.0 * structure[i].Gk), 0.f};
    float *s, *e, *mo, *ed, *tmp;
    TransLayer *tld;
    const int nb = (int)nblocks(g.nh);
    TRY(sc.get(&s, 6 * g.nh));
    TRY(sc.get(&e, 6 * g.nh));
    TRY(sc.get(&mo, 6 * g.nh));
    TRY(sc.get(&ed, 6 * g.nh));
    TRY(sc.get(&tld, sx3h));
    TRY(sc.get(&tmp, (size_t)nb));
    CK(cudaMemcpyAsync(tld, tl.data(), sx3h * sizeof(TransLayer), cudaMemcpyHostToDevice, st));
    k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(sig, s, g.nh);
    k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(epsilonik, e, g.nh);
    k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(moment, mo, g.nh);
    TransArgs a{};
    a.g = g; a.L = tld; a.dg0 = dgammadot0; a.sig = s; a.eps = e; a.m = mo; a.epsdot = ed;
    a.muinv = (float)(1.0 / mu); a.tm_part = tmp;
    k_transient<<<nb, RELAX_NTHREADS, 0, st>>>(a);
    k_soa_to_aos<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(mo, moment, g.nh);
    k_soa_to_aos<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(ed, epsilonikdot, g.nh);
    CKL();
    if (maxwelltime) {
        std::vector<float> h(nb);
        CK(cudaMemcpyAsync(h.data(), tmp, nb * sizeof(float), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        float tm = (float)*maxwelltime;
        for (float v : h) tm = std::min(tm, v);
        *maxwelltime = std::min((double)tm, *maxwelltime);
    }
    return RELAX_OK;
}

extern "C" int relax_op_dgammadot0(const relax_weakzone *zones, int nz, int sx1, int sx2, int sx3h, double dx1,
                                   double dx2, double dx3, double beta, float *out, void *stream)
{
    if (!out || (nz > 0 && !zones) || nz < 0) return fail(RELAX_ERR_ARG, "null argument");
    if (sx1 < 1 || sx2 < 1 || sx3h < 1) return fail(RELAX_ERR_ARG, "grid");
    Grid g{};
    g.sx1 = sx1; g.sx2 = sx2; g.sx3 = 2 * sx3h; g.sx3h = sx3h; g.dx1 = dx1; g.dx2 = dx2; g.dx3 = dx3;
    g.plane = (size_t)sx1 * sx2; g.nh = g.plane * sx3h;
    cudaStream_t st = (cudaStream_t)stream;
    Scratch sc(st);
    relax_weakzone *zd = nullptr;
    TRY(sc.get(&zd, (size_t)std::max(nz, 1)));
    if (nz > 0) CK(cudaMemcpyAsync(zd, zones, nz * sizeof(relax_weakzone), cudaMemcpyHostToDevice, st));
    k_dgammadot0<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(g, zd, nz, beta, out);
    CKL();
    return RELAX_OK;
}

extern "C" int relax_op_okada(const relax_source *sources, int n, double lambda, double mu, int sx1, int sx2,
                              int sx3h, double dx1, double dx2, double dx3, float *u1, float *u2, float *u3,
                              void *stream)
{
    if (n < 0 || (n > 0 && !sources) || !u1 || !u2 || !u3) return fail(RELAX_ERR_ARG, "null argument");
    if (sx1 < 2 || sx2 < 2 || sx3h < 1) return fail(RELAX_ERR_ARG, "grid");
    if (n == 0) return RELAX_OK;
    Grid g{};
    g.sx1 = sx1; g.sx2 = sx2; g.sx3 = 2 * sx3h; g.sx3h = sx3h; g.dx1 = dx1; g.dx2 = dx2; g.dx3 = dx3;
    g.plane = (size_t)sx1 * sx2; g.nh = g.plane * sx3h;
    cudaStream_t st = (cudaStream_t)stream;
    Scratch sc(st);
    relax_source *d = nullptr;
    TRY(sc.get(&d, (size_t)n));
    CK(cudaMemcpyAsync(d, sources, n * sizeof(relax_source), cudaMemcpyHostToDevice, st));
    const size_t rp = (size_t)sx1 + 2;
    k_okada<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(g, d, n, lambda, mu, u1, u2, u3, rp, rp * sx2);
    CKL();
    return RELAX_OK;
}

extern "C" int relax_okada_point(const relax_source *s, double lambda, double mu, double x1, double x2, double x3,
                                 double *disp)
{
    if (!s || !disp) return fail(RELAX_ERR_ARG, "null argument");
    okada_relax(lambda, mu, s->slip, s->opening, s->x, s->y, s->z, s->width, s->length, s->strike, s->dip, s->rake,
                x1, x2, x3, disp);
    return RELAX_OK;
}

extern "C" int relax_op_frictioneigenstress(double x, double y, double z, double L, double W, double strike,
                                            double dip, double rake, double beta, const relax_tensor *sig,
                                            double mu, const relax_layer *structure, int sx1, int sx2,
                                            int sx3h, double dx1, double dx2, double dx3,
                                            relax_tensor *moment, double *maxwelltime, void *stream)
{
    // a private context-free run of the plane kernel
    Grid g;
    TRY(make_grid(g, sx1, sx2, 2 * sx3h, dx1, dx2, dx3));
    if (!structure) return fail(RELAX_ERR_ARG, "null structure");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch sc(st);
    float *s, *mo;
    double *fcd;
    int *err;
    TRY(sc.get(&s, 6 * g.nh));
    TRY(sc.get(&mo, 6 * g.nh));
    TRY(sc.get(&fcd, 4 * (size_t)sx3h));
    TRY(sc.get(&err, 1));
    std::vector<double> h(4 * (size_t)sx3h);
    for (int i3 = 0; i3 < sx3h; i3++) {
        h[i3] = structure[i3].gammadot0; h[sx3h + i3] = structure[i3].stressexponent;
        h[2 * sx3h + i3] = structure[i3].friction; h[3 * sx3h + i3] = structure[i3].cohesion;
    }
    CK(cudaMemcpyAsync(fcd, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(err, 0, sizeof(int), st));
    k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(sig, s, g.nh);
    k_aos_to_soa<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(moment, mo, g.nh);
    FrictionArgs a{};
    a.g = g; a.x = x; a.y = y; a.z = z; a.L = L; a.W = W; a.strike = strike; a.dip = dip; a.rake = rake;
    a.beta = beta; a.mu = mu; a.fc = fcd; a.sig = s; a.m = mo; a.err = err; a.want_tm = maxwelltime != nullptr;
    set_plane_geometry(a);
    a.j1lo = -sx1 / 2; a.n1 = sx1; a.j2lo = -sx2 / 2; a.n2 = sx2; a.i3lo = 0; a.n3 = sx3h;
    const int nb = (int)nblocks(g.nh);
    float *tmp;
    TRY(sc.get(&tmp, nb));
    a.tm_part = tmp;
    k_friction<<<nb, RELAX_NTHREADS, 0, st>>>(a);
    k_soa_to_aos<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(mo, moment, g.nh);
    CKL();
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    std::vector<float> ht(nb);
    if (maxwelltime) CK(cudaMemcpyAsync(ht.data(), tmp, nb * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (maxwelltime) {
        float tm = (float)*maxwelltime;
        for (float v : ht) tm = std::min(tm, v);
        *maxwelltime = std::min((double)tm, *maxwelltime);
    }
    if (herr) return fail(RELAX_ERR_FRICTION, "wrong value of (a-b)sigma: tau/((a-b)sigma) > 20");
    return RELAX_OK;
}

extern "C" int relax_op_green(float *c1, float *c2, float *c3, float *t1, float *t2, float *t3, int sx1,
                              int sx2, int sx3, double dx1, double dx2, double dx3, double lambda, double mu,
                              double gam, void *stream)
{
    Grid g;
    TRY(make_grid(g, sx1, sx2, sx3, dx1, dx2, dx3));
    cudaStream_t st = (cudaStream_t)stream;
    Spectral sp;
    int rc = sp.init(g, st);
    if (rc != RELAX_OK) {
        sp.release();
        return rc;
    }
    XfArgs xa{};
    float *cs[3] = {c1, c2, c3}, *ts[3] = {t1, t2, t3};
    for (int k = 0; k < 3; k++) { xa.in[k] = cs[k]; xa.tin[k] = ts[k]; }
    xa.rp = sx1 + 2; xa.pp = (size_t)(sx1 + 2) * sx2; xa.trp = sx1 + 2;
    XiArgs xi{};
    for (int k = 0; k < 3; k++) { xi.out[k] = cs[k]; xi.base[k] = nullptr; }
    xi.rp = sx1 + 2; xi.pp = (size_t)(sx1 + 2) * sx2; xi.st = nullptr; xi.cmul = 1.f;
    rc = sp.green(xa, false, sx3, sx3, xi, lambda, mu, gam, st);
    cudaStreamSynchronize(st);
    sp.release();
    return rc;
}

extern "C" int relax_op_green_mixed(float *c1, float *c2, float *c3, float *t1, float *t2, float *t3, int sx1,
                                    int sx2, int sx3, double dx1, double dx2, double dx3, double lambda,
                                    double mu, double gam, void *stream)
{
    Grid g;
    TRY(make_grid(g, sx1, sx2, sx3, dx1, dx2, dx3));
    if (sx3 != 128) return fail(RELAX_ERR_UNSUPPORTED, "relax_op_green_mixed: the box must be 128 deep (sx3 = %d)", sx3);
    cudaStream_t st = (cudaStream_t)stream;
    Spectral sp;
    int *err = nullptr;
    int rc = sp.init(g, st);
    if (rc == RELAX_OK) rc = dalloc(&err, 1);
    if (rc != RELAX_OK) {
        sp.release();
        dfree(err);
        return rc;
    }
    cudaMemsetAsync(err, 0, sizeof(int), st);
    rc = sp.set_mixed(1, err, st);
    if (rc != RELAX_OK) {
        sp.release();
        dfree(err);
        return rc;
    }
    XfArgs xa{};
    float *cs[3] = {c1, c2, c3}, *ts[3] = {t1, t2, t3};
    for (int k = 0; k < 3; k++) { xa.in[k] = cs[k]; xa.tin[k] = ts[k]; }
    xa.rp = sx1 + 2; xa.pp = (size_t)(sx1 + 2) * sx2; xa.trp = sx1 + 2;
    XiArgs xi{};
    for (int k = 0; k < 3; k++) { xi.out[k] = cs[k]; xi.base[k] = nullptr; }
    xi.rp = sx1 + 2; xi.pp = (size_t)(sx1 + 2) * sx2; xi.st = nullptr; xi.cmul = 1.f;
    rc = sp.green(xa, false, sx3 / 2, sx3 / 2, xi, lambda, mu, gam, st);
    int herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        if (rc == RELAX_OK) rc = fail(RELAX_ERR_CUDA, "relax_op_green_mixed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    if (rc == RELAX_OK && herr) rc = fail(RELAX_ERR_CUDA, "tensor-core x3 pass: a wait on the tensor cores timed out");
    sp.release();
    dfree(err);
    return rc;
}

extern "C" int relax_op_dft64_tc(const float *in, float *out, int inverse, void *stream)
{
    if (!in || !out) return fail(RELAX_ERR_ARG, "null buffer");
    cudaStream_t st = (cudaStream_t)stream;
    int *err = nullptr;
    TRY(dalloc(&err, 1));
    cudaMemsetAsync(err, 0, sizeof(int), st);
    set_smem(k_dft64_tc, DP_SMEM);
    k_dft64_tc<<<1, 128, DP_SMEM, st>>>((const float2 *)in, (float2 *)out, inverse ? 1 : 0, err);
    cudaError_t e = cudaGetLastError();
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    dfree(err);
    if (e != cudaSuccess) return fail(RELAX_ERR_CUDA, "relax_op_dft64_tc: %s", cudaGetErrorString(e));
    if (herr) return fail(RELAX_ERR_CUDA, "relax_op_dft64_tc: a wait on the tensor cores timed out");
    return RELAX_OK;
}

__global__ void k_amp_aos(const relax_tensor *t, size_t n, double *part)
{
    __shared__ double shd[32];
    double a = 0.0;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const relax_tensor v = t[q];
        a += (double)tnorm6(v.s11, v.s12, v.s13, v.s22, v.s23, v.s33);
    }
    a = block_sum(a, shd);
    if (threadIdx.x == 0) part[blockIdx.x] = a;
}

extern "C" int relax_op_tensoramplitude(const relax_tensor *t, int sx1, int sx2, int sx3h, double dx1,
                                        double dx2, double dx3, double *amp, void *stream)
{
    if (!t || !amp || sx1 <= 0 || sx2 <= 0 || sx3h <= 0) return fail(RELAX_ERR_ARG, "invalid arguments");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch sc(st);
    const int nb = 296;
    double *part;
    TRY(sc.get(&part, nb));
    k_amp_aos<<<nb, RELAX_NTHREADS, 0, st>>>(t, (size_t)sx1 * sx2 * sx3h, part);
    CKL();
    std::vector<double> h(nb);
    CK(cudaMemcpyAsync(h.data(), part, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double s = 0;
    for (double v : h) s += v;
    *amp = s * (dx1 * dx2 * dx3);
    return RELAX_OK;
}

// fft3 (src/fourier.f90:177-201) on a padded (sx1+2, sx2, sx3) array
__global__ void k_zfft_plain(Grid g, float2 *S, FftPlan pz, int tw, int sign)
{
    extern __shared__ float2 sm[];
    const int n = g.sx3;
    const int k1t = blockIdx.x * tw, ncol = min(tw, g.K1 - k1t), k2 = blockIdx.y;
    float2 *A = sm, *B = sm + (size_t)n * tw;
    for (int t = threadIdx.x; t < n * tw; t += blockDim.x) {
        const int j = t / tw, col = t % tw;
        A[t] = col < ncol ? S[sidx(g, 0, j, k2, k1t + col)] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2 *R = sign < 0 ? fft_smem<-1>(A, B, pz, tw, tw, 1) : fft_smem<+1>(A, B, pz, tw, tw, 1);
    for (int t = threadIdx.x; t < n * tw; t += blockDim.x) {
        const int j = t / tw, col = t % tw;
        if (col < ncol) S[sidx(g, 0, j, k2, k1t + col)] = R[t];
    }
}

__global__ void k_spec_copy(Grid g, float2 *S, float *data, int to_data)
{
    const size_t n = (size_t)g.K1 * g.sx2 * g.sx3;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int k1 = (int)(q % g.K1), i2 = (int)((q / g.K1) % g.sx2), i3 = (int)(q / ((size_t)g.K1 * g.sx2));
    float2 *d = reinterpret_cast<float2 *>(data + ((size_t)i3 * g.sx2 + i2) * (g.sx1 + 2)) + k1;
    if (to_data) *d = S[sidx(g, 0, i3, i2, k1)];
    else S[sidx(g, 0, i3, i2, k1)] = *d;
}

extern "C" int relax_op_fft3(float *data, int sx1, int sx2, int sx3, double dx1, double dx2, double dx3,
                             int direction, void *stream)
{
    Grid g;
    if (!data) return fail(RELAX_ERR_ARG, "null data");
    if (sx1 < 4 || sx1 % 4 || !fft_size_ok(sx1 / 2) || !fft_size_ok(sx2) || !fft_size_ok(sx3))
        return fail(RELAX_ERR_UNSUPPORTED, "FFT sizes %dx%dx%d", sx1, sx2, sx3);
    g.sx1 = sx1; g.sx2 = sx2; g.sx3 = sx3; g.sx3h = sx3 / 2; g.M = sx1 / 2; g.K1 = sx1 / 2 + 1;
    g.dx1 = dx1; g.dx2 = dx2; g.dx3 = dx3; g.plane = (size_t)sx1 * sx2; g.nh = g.plane * g.sx3h;
    cudaStream_t st = (cudaStream_t)stream;
    Spectral sp;
    int rc = sp.init(g, st);
    if (rc != RELAX_OK) {
        sp.release();
        return rc;
    }
    const int twz = std::max(1, std::min(16, (int)(96 * 1024 / (2 * (size_t)sx3 * 8))));
    int tw = 1;
    while (tw * 2 <= twz) tw *= 2;
    const size_t smz = 2 * (size_t)sx3 * tw * sizeof(float2);
    cudaFuncSetAttribute(k_zfft_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz);
    if (direction < 0) {
        XfArgs xa{};
        xa.g = g; xa.S = sp.S; xa.pm = sp.pm; xa.tw1 = sp.tw1; xa.nin = sx3; xa.rows = sp.rows; xa.has_trac = 0;
        xa.in[0] = data; xa.rp = sx1 + 2; xa.pp = (size_t)(sx1 + 2) * sx2;
        xa.scale3 = (float)(dx1 * dx2 * dx3);
        // only component 0 is meaningful: point the others at the same data
        xa.in[1] = data; xa.in[2] = data;
        k_xfwd<XIN_REAL><<<dim3(sx2 / sp.rows, sx3), RELAX_NTHREADS, sp.smx, st>>>(xa);
        YArgs ya{g, sp.S, sp.py, sp.twy, sx3, 0};
        k_ypass<-1><<<dim3((g.K1 + sp.twy - 1) / sp.twy, sx3, 1), RELAX_NTHREADS, sp.smy, st>>>(ya);
        k_zfft_plain<<<dim3((g.K1 + tw - 1) / tw, sx2), RELAX_NTHREADS, smz, st>>>(g, sp.S, sp.pz, tw, -1);
        k_spec_copy<<<nblocks((size_t)g.K1 * sx2 * sx3), RELAX_NTHREADS, 0, st>>>(g, sp.S, data, 1);
    } else {
        k_spec_copy<<<nblocks((size_t)g.K1 * sx2 * sx3), RELAX_NTHREADS, 0, st>>>(g, sp.S, data, 0);
        k_zfft_plain<<<dim3((g.K1 + tw - 1) / tw, sx2), RELAX_NTHREADS, smz, st>>>(g, sp.S, sp.pz, tw, +1);
        YArgs yb{g, sp.S, sp.py, sp.twy, sx3, 0};
        k_ypass<+1><<<dim3((g.K1 + sp.twy - 1) / sp.twy, sx3, 1), RELAX_NTHREADS, sp.smy, st>>>(yb);
        // component 0 only: k_xinv handles 3 components; use a 1-row-per-line
        // variant through the same kernel with out/base of components 1,2
        // pointed at a scratch buffer
        Scratch sc(st);
        float *junk;
        rc = sc.get(&junk, (size_t)(sx1 + 2) * sx2 * sx3);
        if (rc == RELAX_OK) {
            XiArgs xi{};
            xi.g = g; xi.S = sp.S; xi.pm = sp.pm; xi.tw1 = sp.tw1; xi.rows = sp.rows;
            xi.out[0] = data; xi.out[1] = junk; xi.out[2] = junk;
            xi.base[0] = xi.base[1] = xi.base[2] = nullptr;
            xi.rp = sx1 + 2; xi.pp = (size_t)(sx1 + 2) * sx2; xi.st = nullptr; xi.cmul = 1.f;
            xi.scale = (float)(2.0 / ((double)sx1 * dx1 * sx2 * dx2 * sx3 * dx3));
            k_xinv<<<dim3(sx2 / sp.rows, sx3), RELAX_NTHREADS, sp.smx, st>>>(xi);
        }
    }
    cudaError_t e = cudaGetLastError();
    cudaStreamSynchronize(st);
    sp.release();
    if (rc != RELAX_OK) return rc;
    if (e != cudaSuccess) return fail(RELAX_ERR_CUDA, "relax_op_fft3: %s", cudaGetErrorString(e));
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// per-stage device timing
// ---------------------------------------------------------------------------
extern "C" int relax_profile(relax_ctx *c, int enable)
{
    if (!c) return fail(RELAX_ERR_ARG, "null context");
    CK(cudaStreamSynchronize(c->st));
    c->prof.reset();
    c->prof.on = enable != 0;
    return RELAX_OK;
}

extern "C" int relax_profile_stages(void) { return ST_COUNT; }

extern "C" int relax_profile_read(relax_ctx *c, int stage, double *total_ms, int *launches, const char **name)
{
    if (!c || stage < 0 || stage >= ST_COUNT) return fail(RELAX_ERR_ARG, "invalid stage");
    CK(cudaStreamSynchronize(c->st));
    double tot = 0.0;
    int n = 0;
    for (auto &rec : c->prof.recs) {
        if (rec.first != stage || !rec.second.second) continue;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, rec.second.first, rec.second.second));
        tot += ms;
        n++;
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = n;
    if (name) *name = kStageNames[stage];
    return RELAX_OK;
}

extern "C" int relax_launch_count(relax_ctx *c, long long *n)
{
    if (!c || !n) return fail(RELAX_ERR_ARG, "null argument");
    *n = c->prof.launches;
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// batches: members that share the grid and the elastic constants, stepped
// together.  Each stage of the RK2 step is one launch for all members (the
// member is a spare grid dimension, its arguments an entry of a device
// table); the host synchronises once per batch step.  Members differ in
// their events, rheology, prestress, weak zones and afterslip planes (the
// same number of planes).
// ---------------------------------------------------------------------------
struct BatchTables {
    unsigned char *dev = nullptr;
    StressArgs *corr = nullptr, *end = nullptr;
    XfArgs *xf = nullptr;
    YArgs *yf = nullptr, *yi = nullptr;
    ZArgs *z = nullptr;
    XiArgs *xip = nullptr, *xic = nullptr;
    std::vector<FrictionPtsArgs *> frp, frc;
    std::vector<MonitorArgs *> mon;
    std::vector<int> frblk, monblk;       // grid.x of plane k's launches
    DtArgs *dt = nullptr;
    // member 0's host copies: shapes and kernel choices of the launches
    StressArgs corr0{}, end0{};
    XfArgs xf0{};
    YArgs yf0{}, yi0{};
    ZArgs z0{};
    XiArgs xip0{}, xic0{};
    std::vector<FrictionPtsArgs> frp0, frc0;
    std::vector<MonitorArgs> mon0;
};

struct relax_batch {
    std::vector<relax_ctx *> m;
    int device = 0;
    cudaStream_t st = nullptr;
    bool batched = false;          // register passes instantiated for the grid
    bool trans = false;            // a member has the transient rheology
    bool tables_valid = false;
    BatchTables tab;
    StepState *dst = nullptr;      // the members' device states, contiguous
    StepState *hst = nullptr;      // pinned mirror
    DtArgs *hdt = nullptr;         // pinned: this step's k_dt inputs
    std::vector<int> nfr;          // friction partial slots per member
    long long launches = 0;
    // the captured graph of a batched step's kernels (dropped when the
    // argument tables are rebuilt)
    cudaGraphExec_t gexec = nullptr;
    long long glaunches = 0;
    bool graph_off = false;
    int plain_steps = 0;
    // autotuning: whether one launch per stage for all members beats the
    // members stepped in turn (each with its own captured step) is decided
    // from the batch's own steps.  Steps 1-3 run batched (plain, capture,
    // replay: the third is timed with CUDA events), steps 4-6 in turn (the
    // sixth is timed on the host clock, the members' host tails included);
    // the faster form runs from then on.  Both forms give the same
    // results, bit for bit.
    int mode = 0;                  // 0 measuring, 1 batched, 2 members in turn
    int tune_steps = 0;
    double tb_ms = -1.0, tt_ms = -1.0;
    cudaEvent_t tev[2] = {nullptr, nullptr};
    bool tev_pending = false;
};

static void free_batch(relax_batch *b)
{
    if (!b) return;
    for (auto *c : b->m) free_ctx(c);
    cudaDeviceSynchronize();
    for (cudaEvent_t ev : b->tev)
        if (ev) cudaEventDestroy(ev);
    if (b->tab.dev) dfree(b->tab.dev, true);
    if (b->dst) dfree(b->dst, true);
    if (b->hst) cudaFreeHost(b->hst);
    if (b->hdt) cudaFreeHost(b->hdt);
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

static int same_shape(const relax_config &a, const relax_config &b)
{
    return a.sx1 == b.sx1 && a.sx2 == b.sx2 && a.sx3 == b.sx3 && a.dx1 == b.dx1 && a.dx2 == b.dx2 &&
           a.dx3 == b.dx3 && a.lambda == b.lambda && a.mu == b.mu && a.gam == b.gam && a.np == b.np;
}

extern "C" int relax_batch_create(const relax_config *members, int n, int device, relax_batch **out)
{
    if (!members || !out || n < 1) return fail(RELAX_ERR_ARG, "null argument or empty batch");
    *out = nullptr;
    for (int k = 1; k < n; k++)
        if (!same_shape(members[0], members[k]))
            return fail(RELAX_ERR_ARG, "batch member %d: grid, spacing, elastic constants and the number of "
                                       "afterslip planes must match member 0", k);
    relax_batch *b = new relax_batch();
    b->device = device;
    auto bail = [&](int rc) { free_batch(b); return rc; };
    if (cudaSetDevice(device) != cudaSuccess) return bail(fail(RELAX_ERR_CUDA, "cudaSetDevice(%d)", device));
    for (int k = 0; k < n; k++) {
        relax_ctx *c = new relax_ctx();
        const int rc = create(&members[k], device, c);
        if (rc != RELAX_OK) {
            free_ctx(c);
            return bail(rc);
        }
        b->m.push_back(c);
        for (const auto &ev : c->events)
            if (!ev.l.empty())
                return bail(fail(RELAX_ERR_UNSUPPORTED, "batch member %d: surface loads are evaluated on the host "
                                                        "at t + Dt; step such members alone", k));
    }
    if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->tev[0]) != cudaSuccess || cudaEventCreate(&b->tev[1]) != cudaSuccess)
        return bail(fail(RELAX_ERR_CUDA, "stream"));
    // member states in one array (one read-back per step)
    if (dalloc(&b->dst, (size_t)n) != RELAX_OK) return bail(RELAX_ERR_NOMEM);
    if (cudaMemset(b->dst, 0, n * sizeof(StepState)) != cudaSuccess ||
        cudaMallocHost(&b->hst, n * sizeof(StepState)) != cudaSuccess ||
        cudaMallocHost(&b->hdt, n * sizeof(DtArgs)) != cudaSuccess)
        return bail(fail(RELAX_ERR_NOMEM, "batch state"));
    for (int k = 0; k < n; k++) {
        relax_ctx *c = b->m[k];
        dfree(c->dst);
        c->dst = b->dst + k;
        c->own_dst = false;
        c->err = &c->dst->error;
    }
    b->batched = reg_shape(b->m[0]->g);
    for (auto *c : b->m) b->trans = b->trans || c->trans;
    b->nfr.assign(n, 0);
    *out = b;
    return RELAX_OK;
}

extern "C" int relax_batch_destroy(relax_batch *b)
{
    free_batch(b);
    return RELAX_OK;
}

extern "C" int relax_batch_size(relax_batch *b, int *n)
{
    if (!b || !n) return fail(RELAX_ERR_ARG, "null argument");
    *n = (int)b->m.size();
    return RELAX_OK;
}

extern "C" int relax_batch_member(relax_batch *b, int k, relax_ctx **c)
{
    if (!b || !c) return fail(RELAX_ERR_ARG, "null argument");
    if (k < 0 || k >= (int)b->m.size()) return fail(RELAX_ERR_ARG, "member %d out of range", k);
    *c = b->m[k];
    return RELAX_OK;
}

extern "C" int relax_batch_coseismic(relax_batch *b, relax_step_log *logs)
{
    if (!b) return fail(RELAX_ERR_ARG, "null batch");
    for (size_t k = 0; k < b->m.size(); k++) TRY(relax_coseismic(b->m[k], 0, logs ? &logs[k] : nullptr));
    b->tables_valid = false;
    return RELAX_OK;
}

template <typename T>
static T *carve(unsigned char *base, size_t *off, size_t n)
{
    *off = (*off + 255) & ~(size_t)255;
    T *p = reinterpret_cast<T *>(base + *off);
    *off += n * sizeof(T);
    return p;
}

// the argument tables of every member (pointers, geometry and constants);
// rebuilt after an event or a change of plane geometry
static int build_tables(relax_batch *b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);   // its arguments live in the old tables
    b->gexec = nullptr;
    const int n = (int)b->m.size();
    relax_ctx *c0 = b->m[0];
    const Grid &g = c0->g;
    const size_t np = c0->planes.size();
    std::vector<StressArgs> corr(n), end(n);
    std::vector<XfArgs> xf(n);
    std::vector<YArgs> yf(n), yi(n);
    std::vector<ZArgs> z(n);
    std::vector<XiArgs> xip(n), xic(n);
    std::vector<std::vector<FrictionPtsArgs>> frp(np, std::vector<FrictionPtsArgs>(n)),
        frc(np, std::vector<FrictionPtsArgs>(n));
    std::vector<std::vector<MonitorArgs>> mon(np, std::vector<MonitorArgs>(n));
    BatchTables &t = b->tab;
    t.frblk.assign(np, 0);
    t.monblk.assign(np, 0);
    for (int k = 0; k < n; k++) {
        relax_ctx *c = b->m[k];
        if (!c->m_valid) TRY(tail_init(c));
        // batched shapes have sx2 % 32 == 0 and sx1 >= 64: no 7-point filter (c->wxy is null)
        corr[k] = stress_args(c, c->vp);
        end[k] = stress_args(c, c->u);
        xf[k] = c->sp.xargs(xf_div(c), g.sx3h);
        yf[k] = c->sp.yargs(g.sx3h, 1, kCW);
        yi[k] = c->sp.yargs(g.sx3h, 0, kCW);
        z[k] = c->sp.zargs(g.sx3h, g.sx3h, c->cfg.lambda, c->cfg.mu, c->cfg.gam, kCW);
        xip[k] = c->sp.xiargs(xi_update(c, c->vp, c->u, 0.5f, true));
        xic[k] = c->sp.xiargs(xi_update(c, c->u, c->u, 1.0f, true));
        int tot = 0;
        TRY(friction_slots(c, &tot));
        b->nfr[k] = tot;
        int off = 0;
        for (size_t q = 0; q < np; q++) {
            frp[q][k] = friction_pts_args(c, q, true);
            frp[q][k].tm_part = c->fr_part + off;
            frc[q][k] = friction_pts_args(c, q, false);
            mon[q][k] = monitor_args(c, q, true);
            const int nb = (int)nblocks(c->band_n[q]);
            off += nb;
            t.frblk[q] = std::max(t.frblk[q], nb);
            const int npch = std::max(0, c->planes[q].px2) * std::max(0, c->planes[q].px3);
            t.monblk[q] = std::max(t.monblk[q], (int)nblocks(npch, 128));
        }
    }
    size_t off = 0;
    unsigned char *nul = nullptr;
    // sizes first (offsets from a null base), then one allocation
    auto layout = [&](unsigned char *base) {
        off = 0;
        t.corr = carve<StressArgs>(base, &off, n); t.end = carve<StressArgs>(base, &off, n);
        t.xf = carve<XfArgs>(base, &off, n);
        t.yf = carve<YArgs>(base, &off, n); t.yi = carve<YArgs>(base, &off, n);
        t.z = carve<ZArgs>(base, &off, n);
        t.xip = carve<XiArgs>(base, &off, n); t.xic = carve<XiArgs>(base, &off, n);
        t.frp.assign(np, nullptr); t.frc.assign(np, nullptr); t.mon.assign(np, nullptr);
        for (size_t q = 0; q < np; q++) {
            t.frp[q] = carve<FrictionPtsArgs>(base, &off, n);
            t.frc[q] = carve<FrictionPtsArgs>(base, &off, n);
            t.mon[q] = carve<MonitorArgs>(base, &off, n);
        }
        t.dt = carve<DtArgs>(base, &off, n);
    };
    layout(nul);
    if (t.dev) dfree(t.dev);
    t.dev = nullptr;
    TRY(dalloc(&t.dev, off));
    layout(t.dev);
    auto up = [&](void *dst, const void *src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, b->st);
    };
    cudaError_t e = up(t.corr, corr.data(), n * sizeof(StressArgs));
    if (e == cudaSuccess) e = up(t.end, end.data(), n * sizeof(StressArgs));
    if (e == cudaSuccess) e = up(t.xf, xf.data(), n * sizeof(XfArgs));
    if (e == cudaSuccess) e = up(t.yf, yf.data(), n * sizeof(YArgs));
    if (e == cudaSuccess) e = up(t.yi, yi.data(), n * sizeof(YArgs));
    if (e == cudaSuccess) e = up(t.z, z.data(), n * sizeof(ZArgs));
    if (e == cudaSuccess) e = up(t.xip, xip.data(), n * sizeof(XiArgs));
    if (e == cudaSuccess) e = up(t.xic, xic.data(), n * sizeof(XiArgs));
    for (size_t q = 0; q < np && e == cudaSuccess; q++) {
        e = up(t.frp[q], frp[q].data(), n * sizeof(FrictionPtsArgs));
        if (e == cudaSuccess) e = up(t.frc[q], frc[q].data(), n * sizeof(FrictionPtsArgs));
        if (e == cudaSuccess) e = up(t.mon[q], mon[q].data(), n * sizeof(MonitorArgs));
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
    if (e != cudaSuccess) return fail(RELAX_ERR_CUDA, "batch tables: %s", cudaGetErrorString(e));
    t.corr0 = corr[0]; t.corr0.tab = t.corr;
    t.end0 = end[0]; t.end0.tab = t.end;
    t.xf0 = xf[0]; t.xf0.tab = t.xf;
    t.yf0 = yf[0]; t.yf0.tab = t.yf;
    t.yi0 = yi[0]; t.yi0.tab = t.yi;
    t.z0 = z[0]; t.z0.tab = t.z;
    t.xip0 = xip[0]; t.xip0.tab = t.xip;
    t.xic0 = xic[0]; t.xic0.tab = t.xic;
    t.frp0.resize(np); t.frc0.resize(np); t.mon0.resize(np);
    for (size_t q = 0; q < np; q++) {
        t.frp0[q] = frp[q][0]; t.frp0[q].tab = t.frp[q];
        t.frc0[q] = frc[q][0]; t.frc0[q].tab = t.frc[q];
        t.mon0[q] = mon[q][0]; t.mon0[q].tab = t.mon[q];
    }
    b->tables_valid = true;
    return RELAX_OK;
}

// the batched Green's function: five launches for all members
static int batch_green(relax_batch *b, const XiArgs &xi0)
{
    BatchTables &t = b->tab;
    const int n = (int)b->m.size();
    const Grid &g = b->m[0]->g;
    cudaError_t e = cudaSuccess;
    if (!xfwd_reg(t.xf0, true, g.sx3h + 1, b->st, &e, n) || e != cudaSuccess)
        return fail(RELAX_ERR_CUDA, "batched x pass: %s", cudaGetErrorString(e));
    if (!ypass_reg(t.yf0, -1, b->st, &e, n) || e != cudaSuccess)
        return fail(RELAX_ERR_CUDA, "batched y pass: %s", cudaGetErrorString(e));
    if (!zspec_reg(t.z0, dim3((g.sx2 * g.K1 + kCW - 1) / kCW), b->st, &e, n) || e != cudaSuccess)
        return fail(RELAX_ERR_CUDA, "batched z pass: %s", cudaGetErrorString(e));
    if (!ypass_reg(t.yi0, +1, b->st, &e, n) || e != cudaSuccess)
        return fail(RELAX_ERR_CUDA, "batched y pass: %s", cudaGetErrorString(e));
    if (!xinv_reg(xi0, g.sx3h, b->st, &e, n) || e != cudaSuccess)
        return fail(RELAX_ERR_CUDA, "batched x inverse: %s", cudaGetErrorString(e));
    b->launches += 5;
    return RELAX_OK;
}

// One RK2 step of every member (the steps of src/relax.f90:555-890 as in
// relax_step).  Members whose time reached the interval take Dt = 0 on the
// device and report i = 0.
// the kernels of a batched step, after the members' time-step inputs are in
// the k_dt table
static int batch_kernels(relax_batch *b)
{
    const int n = (int)b->m.size();
    BatchTables &t = b->tab;
    relax_ctx *c0 = b->m[0];
    const Grid &g = c0->g;
    const size_t np = c0->planes.size();
    cudaStream_t st = b->st;
    if (!c0->fc.empty())
        for (size_t q = 0; q < np; q++)
            if (t.frblk[q] > 0) {
                launch_pdl(k_friction_pts<true>, dim3(t.frblk[q], n), RELAX_NTHREADS, 0, st, t.frp0[q]);
                b->launches++;
            }
    k_dt_batch<<<n, RELAX_NTHREADS, 0, st>>>(t.dt);
    b->launches++;
    CKL();
    TRY(batch_green(b, t.xip0));
    // ---- corrector
    if (b->trans) launch_pdl(k_stress<MODE_CORR, true, true>, dim3(c0->nblk, n), RELAX_NTHREADS, 0, st, t.corr0);
    else launch_pdl(k_stress<MODE_CORR, true>, dim3(c0->nblk, n), RELAX_NTHREADS, 0, st, t.corr0);
    b->launches++;
    if (!c0->fc.empty())
        for (size_t q = 0; q < np; q++) {
            if (t.frblk[q] > 0) {
                launch_pdl(k_friction_pts<true>, dim3(t.frblk[q], n), RELAX_NTHREADS, 0, st, t.frc0[q]);
                b->launches++;
            }
            if (t.monblk[q] > 0) {
                k_monitor<true><<<dim3(t.monblk[q], n), 128, 0, st>>>(t.mon0[q]);
                b->launches++;
            }
        }
    for (int k = 0; k < n; k++) {
        relax_ctx *c = b->m[k];
        for (const auto &s : c->inter.s) {
            SrcArgs a{};
            a.g = g; a.mu = c->cfg.mu; a.s = s.slip; a.x = s.x; a.y = s.y; a.z = s.z;
            a.L = s.width; a.W = s.length; a.strike = s.strike; a.dip = s.dip; a.rake = s.rake; a.beta = s.beta;
            a.tau = c->m;
            k_moment_shear<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(a);
            a.tau = c->tau;   // src/relax.f90:1199-1206 also adds it to tau
            k_moment_shear<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(a);
            b->launches += 2;
        }
        for (const auto &s : c->inter.ts) {
            SrcArgs a{};
            a.g = g; a.mu = c->cfg.mu; a.lambda = c->cfg.lambda; a.s = s.opening; a.x = s.x; a.y = s.y;
            a.z = s.z; a.L = s.width; a.W = s.length; a.strike = s.strike; a.dip = s.dip; a.beta = c->cfg.beta;
            a.tau = c->m;
            k_moment_tensile<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(a);
            a.tau = c->tau;
            k_moment_tensile<<<nblocks(g.nh), RELAX_NTHREADS, 0, st>>>(a);
            b->launches += 2;
        }
    }
    CKL();
    TRY(batch_green(b, t.xic0));
    if (b->trans) launch_pdl(k_stress<MODE_END, true, true>, dim3(c0->nblk, n), RELAX_NTHREADS, 0, st, t.end0);
    else launch_pdl(k_stress<MODE_END, true>, dim3(c0->nblk, n), RELAX_NTHREADS, 0, st, t.end0);
    b->launches++;
    CKL();
    return RELAX_OK;
}

// The launch half of a batch step: every member's time-step inputs, the
// step's kernels (a captured graph after one plain step) and the read-back
// of the members' states, all queued on the batch's stream.  *queued is
// false when the members were stepped in turn (no batched instantiation)
// or none is live; batch_step_finish then has nothing to collect.
static int batch_step_begin(relax_batch *b, relax_step_log *logs, std::vector<char> &live, bool *queued,
                            cudaEvent_t after = nullptr)
{
    *queued = false;
    CK(cudaSetDevice(b->device));
    const int n = (int)b->m.size();
    live.assign(n, 0);
    int nlive = 0;
    for (int k = 0; k < n; k++) {
        relax_ctx *c = b->m[k];
        if (!c->cos_done) TRY(relax_coseismic(c, 0, nullptr));
        memset(&logs[k], 0, sizeof(relax_step_log));
        live[k] = c->t < c->cfg.interval;
        nlive += live[k];
    }
    if (!nlive) return RELAX_OK;
    // no batched instantiation for this grid: the members in turn
    if (!b->batched || n == 1) b->mode = 2;
    bool turn = b->mode == 2, time_turn = false, time_batched = false;
    if (b->mode == 0) {
        turn = b->tune_steps >= 3;
        time_turn = b->tune_steps == 5;
        time_batched = b->tune_steps == 2;
        b->tune_steps++;
    }
    if (turn) {
        const auto t0 = std::chrono::steady_clock::now();
        for (int k = 0; k < n; k++) {
            if (!live[k]) continue;
            relax_ctx *c = b->m[k];
            if (after) CK(cudaStreamWaitEvent(c->st, after, 0));
            const int e0 = c->e;
            TRY(do_step(c, nullptr, &logs[k]));
            if (c->e != e0) b->tables_valid = false;   // as after a batched step's event branch
        }
        if (time_turn) {
            b->tt_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            b->mode = (b->tb_ms > 0.0 && b->tb_ms <= b->tt_ms) ? 1 : 2;
        }
        return RELAX_OK;
    }
    if (!b->tables_valid) TRY(build_tables(b));
    // the members' own streams carry their set-up and event work
    for (auto *c : b->m) CK(cudaStreamSynchronize(c->st));
    BatchTables &t = b->tab;
    cudaStream_t st = b->st;
    if (after) CK(cudaStreamWaitEvent(st, after, 0));
    // ---- predictor
    for (int k = 0; k < n; k++) {
        relax_ctx *c = b->m[k];
        DtArgs &d = b->hdt[k];
        d.st = c->dst;
        d.pol = policy(c);
        d.in = DtIn{};
        d.in.t = c->t;
        d.in.oi = c->oi;
        d.in.use_override = live[k] ? 0 : 1;   // finished members: Dt = 0
        d.in.dt_override = 0.0;
        d.fr_part = c->fr_part;
        d.nfr = c->fc.empty() ? 0 : b->nfr[k];
    }
    CK(cudaMemcpyAsync(t.dt, b->hdt, n * sizeof(DtArgs), cudaMemcpyHostToDevice, st));
    // the kernels, replayed from a captured graph after one plain step
    if (!b->graph_off && b->plain_steps > 0 && !b->gexec) {
        cudaGraph_t graph = nullptr;
        const long long l0 = b->launches;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
            const int rc = batch_kernels(b);
            const cudaError_t e = cudaStreamEndCapture(st, &graph);
            b->glaunches = b->launches - l0;
            if (rc != RELAX_OK || e != cudaSuccess || !graph ||
                cudaGraphInstantiate(&b->gexec, graph, 0) != cudaSuccess) {
                b->gexec = nullptr;
                b->graph_off = true;
            }
            if (graph) cudaGraphDestroy(graph);
        } else {
            b->graph_off = true;
        }
        cudaGetLastError();
        b->launches = l0;
    }
    if (time_batched) CK(cudaEventRecord(b->tev[0], st));
    if (b->gexec) {
        CK(cudaGraphLaunch(b->gexec, st));
        b->launches += b->glaunches;
    } else {
        TRY(batch_kernels(b));
        b->plain_steps++;
    }
    if (time_batched) {
        CK(cudaEventRecord(b->tev[1], st));
        b->tev_pending = true;
    }
    CK(cudaMemcpyAsync(b->hst, b->dst, n * sizeof(StepState), cudaMemcpyDeviceToHost, st));
    *queued = true;
    return RELAX_OK;
}

// The host half: waits for the batch's stream and runs each live member's
// step end (counters, event branch, log).
static int batch_step_finish(relax_batch *b, relax_step_log *logs, const std::vector<char> &live)
{
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->st));
    if (b->tev_pending) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, b->tev[0], b->tev[1]));
        b->tb_ms = ms;
        b->tev_pending = false;
    }
    for (int k = 0; k < (int)b->m.size(); k++) {
        if (!live[k]) continue;
        relax_ctx *c = b->m[k];
        *c->hst = b->hst[k];
        const int e0 = c->e;
        TRY(finish_step(c, &logs[k]));
        if (c->e != e0) b->tables_valid = false;   // the event branch ran on the member's stream
    }
    return RELAX_OK;
}

extern "C" int relax_batch_step(relax_batch *b, relax_step_log *logs)
{
    if (!b || !logs) return fail(RELAX_ERR_ARG, "null argument");
    std::vector<char> live;
    bool queued = false;
    TRY(batch_step_begin(b, logs, live, &queued));
    if (queued) TRY(batch_step_finish(b, logs, live));
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// ensembles of uneven grids: one batch per grid shape, each on its own
// stream, stepped with one host synchronisation per step.  The groups' steps
// run one after the other (each stream waits for the previous group's step):
// run concurrently they competed for L2 and took longer than in sequence.
// ---------------------------------------------------------------------------
struct relax_ensemble {
    std::vector<relax_batch *> groups;
    std::vector<std::vector<int>> index;   // member numbers of each group
    std::vector<std::pair<int, int>> where;   // group and slot of each member
    std::vector<std::vector<relax_step_log>> glog;
    std::vector<cudaEvent_t> done;          // end of each group's queued step
    int device = 0;
};

static void free_ensemble(relax_ensemble *e)
{
    if (!e) return;
    for (cudaEvent_t ev : e->done)
        if (ev) cudaEventDestroy(ev);
    for (auto *b : e->groups) free_batch(b);
    delete e;
}

extern "C" int relax_ensemble_create(const relax_config *members, int n, int device, relax_ensemble **out)
{
    if (!members || !out || n < 1) return fail(RELAX_ERR_ARG, "null argument or empty ensemble");
    *out = nullptr;
    relax_ensemble *e = new relax_ensemble();
    e->device = device;
    e->where.resize(n);
    for (int k = 0; k < n; k++) {
        int gidx = -1;
        for (size_t q = 0; q < e->index.size(); q++)
            if (same_shape(members[e->index[q][0]], members[k])) { gidx = (int)q; break; }
        if (gidx < 0) {
            gidx = (int)e->index.size();
            e->index.emplace_back();
        }
        e->where[k] = {gidx, (int)e->index[gidx].size()};
        e->index[gidx].push_back(k);
    }
    for (auto &idx : e->index) {
        std::vector<relax_config> cfgs;
        for (int k : idx) cfgs.push_back(members[k]);
        relax_batch *b = nullptr;
        const int rc = relax_batch_create(cfgs.data(), (int)cfgs.size(), device, &b);
        if (rc != RELAX_OK) {
            free_ensemble(e);
            return rc;
        }
        e->groups.push_back(b);
        e->glog.emplace_back(idx.size());
        cudaEvent_t ev = nullptr;
        const cudaError_t ce = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (ce != cudaSuccess) {
            free_ensemble(e);
            return fail(RELAX_ERR_CUDA, "cudaEventCreate: %s", cudaGetErrorString(ce));
        }
        e->done.push_back(ev);
    }
    *out = e;
    return RELAX_OK;
}

extern "C" int relax_ensemble_destroy(relax_ensemble *e)
{
    free_ensemble(e);
    return RELAX_OK;
}

extern "C" int relax_ensemble_size(relax_ensemble *e, int *n, int *ngroups)
{
    if (!e) return fail(RELAX_ERR_ARG, "null ensemble");
    if (n) *n = (int)e->where.size();
    if (ngroups) *ngroups = (int)e->groups.size();
    return RELAX_OK;
}

extern "C" int relax_ensemble_member(relax_ensemble *e, int k, relax_ctx **c)
{
    if (!e || !c) return fail(RELAX_ERR_ARG, "null argument");
    if (k < 0 || k >= (int)e->where.size()) return fail(RELAX_ERR_ARG, "member %d out of range", k);
    *c = e->groups[e->where[k].first]->m[e->where[k].second];
    return RELAX_OK;
}

extern "C" int relax_ensemble_coseismic(relax_ensemble *e, relax_step_log *logs)
{
    if (!e) return fail(RELAX_ERR_ARG, "null ensemble");
    for (size_t q = 0; q < e->groups.size(); q++) {
        TRY(relax_batch_coseismic(e->groups[q], e->glog[q].data()));
        if (logs)
            for (size_t j = 0; j < e->index[q].size(); j++) logs[e->index[q][j]] = e->glog[q][j];
    }
    return RELAX_OK;
}

extern "C" int relax_ensemble_step(relax_ensemble *e, relax_step_log *logs)
{
    if (!e || !logs) return fail(RELAX_ERR_ARG, "null argument");
    const size_t ng = e->groups.size();
    std::vector<std::vector<char>> live(ng);
    std::vector<char> queued(ng, 0);
    // every group's step queued on its own stream behind the previous
    // group's, then one wait per group
    cudaEvent_t prev = nullptr;
    for (size_t q = 0; q < ng; q++) {
        bool qd = false;
        TRY(batch_step_begin(e->groups[q], e->glog[q].data(), live[q], &qd, prev));
        queued[q] = qd;
        if (qd) {
            CK(cudaEventRecord(e->done[q], e->groups[q]->st));
            prev = e->done[q];
        }
    }
    for (size_t q = 0; q < ng; q++)
        if (queued[q]) TRY(batch_step_finish(e->groups[q], e->glog[q].data(), live[q]));
    for (size_t q = 0; q < ng; q++)
        for (size_t j = 0; j < e->index[q].size(); j++) logs[e->index[q][j]] = e->glog[q][j];
    return RELAX_OK;
}

extern "C" int relax_ensemble_launch_count(relax_ensemble *e, long long *n)
{
    if (!e || !n) return fail(RELAX_ERR_ARG, "null argument");
    *n = 0;
    for (auto *b : e->groups) {
        long long m = 0;
        TRY(relax_batch_launch_count(b, &m));
        *n += m;
    }
    return RELAX_OK;
}

extern "C" int relax_batch_launch_count(relax_batch *b, long long *n)
{
    if (!b || !n) return fail(RELAX_ERR_ARG, "null argument");
    *n = b->launches;
    for (auto *c : b->m) *n += c->prof.launches;
    return RELAX_OK;
}

extern "C" int relax_batch_tuning(relax_batch *b, int *mode, double *batched_ms, double *in_turn_ms)
{
    if (!b) return fail(RELAX_ERR_ARG, "null batch");
    if (mode) *mode = b->mode;
    if (batched_ms) *batched_ms = b->tb_ms;
    if (in_turn_ms) *in_turn_ms = b->tt_ms;
    return RELAX_OK;
}

extern "C" int relax_ensemble_tuning(relax_ensemble *e, int group, int *sx, int *nmembers, int *mode,
                                     double *batched_ms, double *in_turn_ms)
{
    if (!e) return fail(RELAX_ERR_ARG, "null ensemble");
    if (group < 0 || group >= (int)e->groups.size()) return fail(RELAX_ERR_ARG, "group %d out of range", group);
    relax_batch *b = e->groups[group];
    if (sx) {
        sx[0] = b->m[0]->g.sx1; sx[1] = b->m[0]->g.sx2; sx[2] = b->m[0]->g.sx3;
    }
    if (nmembers) *nmembers = (int)b->m.size();
    return relax_batch_tuning(b, mode, batched_ms, in_turn_ms);
}

extern "C" int relax_batch_get_stream(relax_batch *b, void **s)
{
    if (!b || !s) return fail(RELAX_ERR_ARG, "null argument");
    *s = (void *)b->st;
    return RELAX_OK;
}
