// noalloc.cu -- the Green's function operator without any allocation.
//
// relax_op_green (relax_b200.cu) takes its spectrum buffer and twiddle
// tables from the library's own device memory pool on every call.  Some
// callers cannot allow that: a host that hands all device memory to its own
// pool allocator (and forbids other allocations, which also synchronise the
// device), or code running where allocation is not allowed at all.  relax_op_green_noalloc
// does the same transform with its scratch in a fixed device array defined
// in this file, so the only memory it touches is the caller's buffers and
// that array.
//
// The array is per device and lives for as long as the library is loaded on
// that device.  All calls share it and it keeps the previous call's
// contents; every word a call reads is written earlier in the same call, so
// nothing has to be cleared.  Calls whose work overlaps on the GPU (two
// streams, or two host threads on one device) race on the array: order them
// on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

using namespace relax;

namespace relax_noalloc {

// 16 MiB: a 3-component spectrum of (sx1/2+1) x sx2 x (sx3+1) complex
// values plus the twiddle tables, e.g. up to a 128 x 128 x 64 box.
constexpr size_t kScratchBytes = 16u << 20;
static __device__ __align__(256) unsigned char g_green_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// exp(-2 pi i j / n) for the four tables of one grid
__global__ void k_twiddles(float2 *tw, int n0, int n1, int n2, int n3)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int ns[4] = {n0, n1, n2, n3};
    int off = 0;
    for (int t = 0; t < 4; t++) {
        if (j < ns[t]) {
            double s, c;
            sincospi(-2.0 * (double)j / (double)ns[t], &s, &c);
            tw[off + j] = make_float2((float)c, (float)s);
        }
        off += ns[t];
    }
}

bool factor(int n, int *r, int *nr)
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

// Set-up of the current device, once: the device address of the scratch
// array (host code cannot use the symbol itself) and the shared-memory
// limits of the kernels.  Returns the address or null with *err set.
void *device_scratch(cudaError_t *err)
{
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) return nullptr;
    if (dev < 0 || dev >= kMaxDevices) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_addr[dev]) return g_addr[dev];
    void *p = nullptr;
    *err = cudaGetSymbolAddress(&p, g_green_scratch);
    if (*err != cudaSuccess) return nullptr;
    const int big = 200 * 1024;
    cudaError_t e = cudaFuncSetAttribute(k_xfwd<XIN_REAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xinv, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ypass<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ypass<+1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_zspec, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e != cudaSuccess) {
        *err = e;
        return nullptr;
    }
    g_addr[dev] = p;
    return p;
}

}  // namespace relax_noalloc

extern "C" __attribute__((visibility("hidden"))) int relax_noalloc_fail(int code, const char *msg);

using namespace relax_noalloc;

extern "C" int relax_op_green_noalloc(float *c1, float *c2, float *c3, float *t1, float *t2, float *t3,
                                      int sx1, int sx2, int sx3, double dx1, double dx2, double dx3,
                                      double lambda, double mu, double gam, void *stream)
{
    char msg[256];
    if (!c1 || !c2 || !c3 || !t1 || !t2 || !t3) return relax_noalloc_fail(RELAX_ERR_ARG, "null buffer");
    if (sx1 < 8 || sx1 % 4 || sx2 < 2 || sx3 < 4 || sx3 % 2 || !(dx1 > 0 && dx2 > 0 && dx3 > 0))
        return relax_noalloc_fail(RELAX_ERR_UNSUPPORTED, "grid: need sx1 >= 8, a multiple of 4, and even sx3");
    Grid g{};
    g.sx1 = sx1; g.sx2 = sx2; g.sx3 = sx3; g.sx3h = sx3 / 2; g.M = sx1 / 2; g.K1 = sx1 / 2 + 1;
    g.dx1 = dx1; g.dx2 = dx2; g.dx3 = dx3; g.plane = (size_t)sx1 * sx2; g.nh = g.plane * g.sx3h;
    FftPlan pm{}, py{}, pz{};
    if (!factor(g.M, pm.r, &pm.nr) || !factor(sx2, py.r, &py.nr) || !factor(sx3, pz.r, &pz.nr))
        return relax_noalloc_fail(RELAX_ERR_UNSUPPORTED, "FFT lengths must be products of 2 and 3");
    pm.n = g.M; py.n = sx2; pz.n = sx3;
    const size_t spec = 3 * (size_t)(sx3 + 1) * sx2 * g.K1 * sizeof(float2);
    const size_t ntw = (size_t)g.M + sx1 + sx2 + sx3;
    const size_t need = spec + ntw * sizeof(float2);
    if (need > kScratchBytes) {
        snprintf(msg, sizeof msg,
                 "grid %dx%dx%d needs %zu bytes of scratch; relax_op_green_noalloc holds %zu "
                 "(use relax_op_green)", sx1, sx2, sx3, need, kScratchBytes);
        return relax_noalloc_fail(RELAX_ERR_ARG, msg);
    }
    cudaError_t e = cudaSuccess;
    unsigned char *base = (unsigned char *)device_scratch(&e);
    if (!base) {
        snprintf(msg, sizeof msg, "scratch set-up: %s", cudaGetErrorString(e));
        return relax_noalloc_fail(RELAX_ERR_CUDA, msg);
    }
    cudaStream_t st = (cudaStream_t)stream;
    float2 *S = (float2 *)base;
    float2 *tw = (float2 *)(base + spec);
    pm.tw = tw;
    const float2 *tw1 = tw + g.M;
    py.tw = tw + g.M + sx1;
    pz.tw = tw + g.M + sx1 + sx2;
    k_twiddles<<<(unsigned)((std::max(std::max(g.M, sx1), std::max(sx2, sx3)) + 255) / 256), 256, 0, st>>>(
        tw, g.M, sx1, sx2, sx3);

    // tile choices as relax_op_green
    int rows = 1;
    while (rows * 2 <= std::max(1, 1024 / g.M) && sx2 % (rows * 2) == 0) rows *= 2;
    int twy = 16;
    while (twy > 1 && 2 * (size_t)sx2 * twy * 8 > 96 * 1024) twy /= 2;
    int twz = 16;
    while (twz > 1 && 2 * (size_t)sx3 * 3 * twz * 8 > 100 * 1024) twz /= 2;
    const size_t smx = 2 * (size_t)3 * rows * (g.M + 1) * sizeof(float2);
    const size_t smy = 2 * (size_t)sx2 * twy * sizeof(float2);
    const int P = RELAX_NTHREADS / twz;
    const size_t smz = 2 * (size_t)sx3 * 3 * twz * sizeof(float2) + (size_t)P * twz * 6 * sizeof(double) +
                       (size_t)twz * 12 * sizeof(float);

    XfArgs xa{};
    float *cs[3] = {c1, c2, c3}, *ts[3] = {t1, t2, t3};
    for (int k = 0; k < 3; k++) { xa.in[k] = cs[k]; xa.tin[k] = ts[k]; }
    xa.g = g; xa.S = S; xa.pm = pm; xa.tw1 = tw1; xa.nin = sx3; xa.rows = rows; xa.has_trac = 1;
    xa.rp = sx1 + 2; xa.pp = (size_t)(sx1 + 2) * sx2; xa.trp = sx1 + 2;
    xa.scale3 = (float)(dx1 * dx2 * dx3);
    xa.scale2 = (float)(dx1 * dx2);
    k_xfwd<XIN_REAL><<<dim3(sx2 / rows, sx3 + 1), RELAX_NTHREADS, smx, st>>>(xa);
    YArgs ya{g, S, py, twy, sx3, 1};
    k_ypass<-1><<<dim3((g.K1 + twy - 1) / twy, sx3 + 1, 3), RELAX_NTHREADS, smy, st>>>(ya);
    ZArgs za{};
    za.g = g; za.S = S; za.pz = pz; za.tw = twz; za.nin = sx3; za.nout = sx3;
    za.ratio1 = (float)((lambda + mu) / (lambda + 2.0 * mu) / mu / (4.0 * M_PI * M_PI));
    za.ratio2 = (float)(mu / (lambda + mu));
    za.lambda = lambda; za.mu = mu; za.gam = gam;
    k_zspec<<<dim3((g.K1 + twz - 1) / twz, sx2), RELAX_NTHREADS, smz, st>>>(za);
    YArgs yb{g, S, py, twy, sx3, 0};
    k_ypass<+1><<<dim3((g.K1 + twy - 1) / twy, sx3, 3), RELAX_NTHREADS, smy, st>>>(yb);
    XiArgs xi{};
    for (int k = 0; k < 3; k++) { xi.out[k] = cs[k]; xi.base[k] = nullptr; }
    xi.g = g; xi.S = S; xi.pm = pm; xi.tw1 = tw1; xi.rows = rows;
    xi.rp = sx1 + 2; xi.pp = (size_t)(sx1 + 2) * sx2; xi.st = nullptr; xi.cmul = 1.f;
    xi.scale = (float)(2.0 / ((double)sx1 * dx1 * sx2 * dx2 * sx3 * dx3));
    k_xinv<<<dim3(sx2 / rows, sx3), RELAX_NTHREADS, smx, st>>>(xi);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(msg, sizeof msg, "relax_op_green_noalloc launch: %s", cudaGetErrorString(e));
        return relax_noalloc_fail(RELAX_ERR_CUDA, msg);
    }
    return RELAX_OK;
}
