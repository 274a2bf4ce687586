// kernels.cuh -- sm_100a kernels of RELAX's relaxation step.
//
// Field layout on the device: structure of arrays, i1 fastest, physical
// half-space only (sx3h layers); a tensor field is 6 planes
// {s11,s12,s13,s22,s23,s33} of nh floats, a vector field 3 planes.
#pragma once

#include "common.cuh"
#include "rfft.cuh"

namespace relax {
// kernels and their argument types have internal linkage: each translation
// unit that launches them carries its own copy
namespace {

// ------------------------------------------------------------------------
// small helpers
// ------------------------------------------------------------------------
__device__ __forceinline__ float warp_min(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide min / sum in a fixed order (deterministic).  All threads of
// the block must call; the result is valid in thread 0.
__device__ __forceinline__ float block_min(float v, float *sh)
{
    v = warp_min(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < nw ? sh[l] : 3.0e38f;
        v = warp_min(v);
    }
    return v;
}
__device__ __forceinline__ double block_sum(double v, double *sh)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < nw ? sh[l] : 0.0;
        v = warp_sum(v);
    }
    return v;
}

// tensornorm, src/elastic3d.f90:311-319
__device__ __forceinline__ float tnorm6(float a, float b, float c, float d, float e, float f)
{
    return sqrtf((a * a + 2.f * b * b + 2.f * c * c + d * d + 2.f * e * e + f * f) * 0.5f);
}

// Programmatic dependent launch.  A kernel launched with the
// programmatic-serialization attribute may be scheduled while the kernel
// before it in the stream still runs; pdl_wait (griddepcontrol.wait) blocks
// until that kernel has completed and its memory operations are visible, and
// returns at once in a launch without the attribute.  pdl_trigger
// (griddepcontrol.launch_dependents) lets the next kernel be scheduled once
// every block of this one has issued it.  The step's streaming kernels call
// both first thing, wait before trigger, so that at most the next kernel's
// blocks are placed during a kernel's last wave, and none reads memory
// before its wait.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_enter() { pdl_wait(); }

__device__ __forceinline__ float4 ld4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ float4 ldc4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float geti(const float4 &v, int j) { return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w; }

// 1/x by the hardware's approximate reciprocal (PTX rcp.approx.ftz.f32,
// relative error about 2^-23; a subnormal x flushes to zero).  The x3
// passes use it for the elastic response 1/|k|^2 and the Cerruti kernel
// 1/((2 pi k3)^2 + beta^2), whose operands are positive and normal; it
// takes the z pass from 69.6 to 66.5 us on the 256 x 256 x 128 box, with
// a relative L2 difference of 4.5e-8 to the divided form.
__device__ __forceinline__ float rcp_fast(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Derivatives along the periodic axes x1 and x2.  optimalfilter
// (src/elastic3d.f90:846-907) takes the central difference
// (w[i+1] - w[i-1]) / (2 dx) for sx <= 4 and sx >= 15, and the 7-point FIR
// differentiator fir7 of src/kernel7.inc for 5 <= sx <= 14: sum over
// l = 1..7 of (w[i+l] - w[i-l]) fir7(l) / dx, indexes periodic
// (localstrain_ani, src/elastic3d.f90:1140-1178, and localdivergence_ani,
// :1431-1470).  A Fir7 with n = 7 selects the filter, c[l-1] = fir7(l) / dx;
// n = 0 the central difference.  Along x3, fir7 is selected for
// 5 <= sx3/2 <= 14, but then every layer is a boundary layer of the filter
// ((i3 > 7) and (i3 < sx3/2 - 6) is never true, stressupdate :975-976), so
// the finite differences of localstrain_ani apply throughout.
struct Fir7 {
    int n;
    float c[7];
};

// sum_l (w[(i2+l) % sx2] - w[(i2-l) % sx2]) c[l-1] at 4 consecutive points
// of rows of pitch sx1 (w points at x1 of the row i2 = 0 of the plane)
__device__ __forceinline__ float4 fir_y4(const float *w, int i2, int sx2, int sx1, const Fir7 &f)
{
    float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int l = 1; l <= 7; l++) {
        const float4 p = ld4(w + (size_t)((i2 + l) % sx2) * sx1);
        const float4 m = ld4(w + (size_t)((i2 + 2 * sx2 - l) % sx2) * sx1);   // sx2 >= 5 > l / 2
        d.x += (p.x - m.x) * f.c[l - 1];
        d.y += (p.y - m.y) * f.c[l - 1];
        d.z += (p.z - m.z) * f.c[l - 1];
        d.w += (p.w - m.w) * f.c[l - 1];
    }
    return d;
}

// the same along x1 for the point i1 of a row (sx1 >= 5)
__device__ __forceinline__ float fir_x1(const float *row, int i1, int sx1, const Fir7 &f)
{
    float d = 0.f;
#pragma unroll
    for (int l = 1; l <= 7; l++)
        d += (__ldg(row + (i1 + l) % sx1) - __ldg(row + (i1 + 2 * sx1 - l) % sx1)) * f.c[l - 1];
    return d;
}

// The x1 and x2 derivatives of the 3 components of w (3 x nh each) for
// k_stress on grids where either axis takes fir7 (kept out of the stress
// kernel's registers): by the filter where its Fir7 says so, else by the
// central difference exactly as k_stress forms it ((right - left) * k).
__global__ void __launch_bounds__(RELAX_NTHREADS) k_fir_xy(Grid g, const float *w, float *wx, float *wy, Fir7 fx,
                                                           Fir7 fy, float k1, float k2)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 3 * (g.nh >> 2)) return;
    const int c = (int)(q / (g.nh >> 2));
    const size_t p = 4 * (q % (g.nh >> 2));
    const int i1 = (int)(p % g.sx1), i2 = (int)((p / g.sx1) % g.sx2), i3 = (int)(p / g.plane);
    const float *wc = w + c * g.nh;
    const float *row = wc + p - i1;
    float4 dx;
    if (fx.n == 7) {
        dx = make_float4(fir_x1(row, i1, g.sx1, fx), fir_x1(row, i1 + 1, g.sx1, fx),
                         fir_x1(row, i1 + 2, g.sx1, fx), fir_x1(row, i1 + 3, g.sx1, fx));
    } else {
        const float4 cv = ld4(wc + p);
        const float lft = __ldg(row + (i1 + g.sx1 - 1) % g.sx1), rgt = __ldg(row + (i1 + 4) % g.sx1);
        dx = make_float4((cv.y - lft) * k1, (cv.z - cv.x) * k1, (cv.w - cv.y) * k1, (rgt - cv.z) * k1);
    }
    float4 dy;
    if (fy.n == 7) {
        dy = fir_y4(wc + (size_t)i3 * g.plane + i1, i2, g.sx2, g.sx1, fy);
    } else {
        const float4 ym = ld4(wc + (size_t)i3 * g.plane + (size_t)((i2 + g.sx2 - 1) % g.sx2) * g.sx1 + i1);
        const float4 yp = ld4(wc + (size_t)i3 * g.plane + (size_t)((i2 + 1) % g.sx2) * g.sx1 + i1);
        dy = make_float4((yp.x - ym.x) * k2, (yp.y - ym.y) * k2, (yp.z - ym.z) * k2, (yp.w - ym.w) * k2);
    }
    *reinterpret_cast<float4 *>(wx + c * g.nh + p) = dx;
    *reinterpret_cast<float4 *>(wy + c * g.nh + p) = dy;
}

__device__ __forceinline__ float fir_y1(const float *w, int i2, int sx2, int sx1, const Fir7 &f)
{
    float d = 0.f;
#pragma unroll
    for (int l = 1; l <= 7; l++)
        d += (__ldg(w + (size_t)((i2 + l) % sx2) * sx1) - __ldg(w + (size_t)((i2 + 2 * sx2 - l) % sx2) * sx1)) *
             f.c[l - 1];
    return d;
}

// ------------------------------------------------------------------------
// Fused stress / eigenstress kernel.
//
//   MODE_OP   sig += C:E(w)                                (stressupdate)
//   MODE_INIT sig = -tau + C:E(w);         m = eigen(sig)  (coseismic end)
//   MODE_END  tau += Dt m; sig = -tau + C:E(w); m = eigen(sig)
//             (corrector tail + stressupdate + next predictor eigenstress,
//              src/relax.f90:836,888-890 then :569-600)
//   MODE_CORR sig = -Dt/2 m - tau + C:E(w); m = eigen(sig); gamma += Dt gd
//             (src/relax.f90:696-738)
//   MODE_EIGEN m += eigen(sig), gamma = gd tauc/mu where active
//             (viscouseigenstress as called, for the operator API)
// C:E is Hooke's law on the FIR/finite-difference strain of
// src/elastic3d.f90:956-1180 (central differences for sx >= 15, one-sided
// at the top and bottom layers); eigen is viscouseigenstress,
// src/viscoelastic3d.f90:217-314, for the linear and the power-law
// mechanisms.  Per-block Maxwell-time minima and tensor-amplitude sums
// (src/elastic3d.f90:446-466) go to partial arrays reduced in a fixed order.
// Each thread handles 4 consecutive points along x1 (float4 I/O).
// ------------------------------------------------------------------------
enum { MODE_OP = 0, MODE_INIT = 1, MODE_END = 2, MODE_CORR = 3, MODE_EIGEN = 4 };

struct StressArgs {
    Grid g;
    const float *w;          // strain source (3 x nh)
    float *tau;              // 6 x nh
    float *m;                // 6 x nh
    float *sig;              // 6 x nh (MODE_OP: in/out)
    float *gamma;            // nh (MODE_CORR)
    const float *dg0[2];     // weak-zone fluidity perturbations or null
    const DepthVisc *visc[2];// per-depth rheology (null = mechanism absent)
    const float *spdev;      // 6 x sx3h deviatoric prestress (or null)
    const StepState *st;
    float k1, k2, k3, k3b;   // 0.5/dx1, 0.5/dx2, 0.5/dx3, 1/dx3
    const float *wx, *wy;    // FIR: the x1 and x2 derivatives of w (3 x nh each, k_fir_xy)
    float lam, mu2, muinv;   // lambda, 2 mu, 1/mu
    int store_sig;
    const unsigned char *sig_mask;   // store_sig: only groups of 4 points flagged here (null = all)
    float *tm_part;          // [2][gridDim.x]
    double *amp_part;        // [2][gridDim.x] (power, cei)
    unsigned *ticket;        // INIT/END: blocks done (zero between launches), or null
    StepState *fin;          // with ticket: receives tmin, power, cei
    double dv;               // cell volume dx1 dx2 dx3 (amplitude scale)
    const struct StressArgs *tab;   // batched launch: one entry per member (blockIdx.y)
    // transient (Burgers) rheology, TRANS instantiations only
    const TransLayer *trans[2];      // linear / nonlinear transient structures or null
    const float *tdg0[2];            // their weak-zone perturbations or null
    float *eps, *epsdot;             // epsilonik, epsilonikdot (6 x nh each)
};

// BATCH: blockIdx.y selects a member of a batch, whose arguments are a0.tab[blockIdx.y].
// TRANS: also the transient rheology (transienteigenstress,
// src/viscoelastic3d.f90:123-202): in INIT/END the predictor's calls
// (src/relax.f90:614-645: epsilonikdot from epsilonik, two more Maxwell-time
// minima), in CORR the predicted strain epsilonikdot = Dt/2 epsilonikdot +
// epsilonik (:693-695), the corrector's calls on it (:764-787) and
// epsilonik += Dt epsilonikdot (:789).
// FIR: the x1 and x2 derivatives of w come from a.wx, a.wy (k_fir_xy, grids
// where x1 or x2 takes the 7-point filter) instead of the central differences.
template <int MODE, bool BATCH = false, bool TRANS = false, bool FIR = false>
__global__ void __launch_bounds__(RELAX_NTHREADS, TRANS ? 2 : 3) k_stress(const __grid_constant__ StressArgs a0)
{
    pdl_enter();
    const StressArgs &a = BATCH ? a0.tab[blockIdx.y] : a0;
    __shared__ float shf[32];
    __shared__ double shd[32];
    if (MODE == MODE_END && a.st->fire) return;   // the event branch of the step runs instead
    const Grid &g = a.g;
    const int q4 = g.sx1 >> 2;
    const size_t nq = g.nh >> 2;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = q < nq;
    constexpr int NTM = TRANS ? 4 : 2;        // Maxwell-time minima: viscous 2 (+ transient 2)
    float tmin[4] = {3.0e38f, 3.0e38f, 3.0e38f, 3.0e38f};
    double amp_m = 0.0, amp_t = 0.0;

    if (live) {
        // point indexes by 32-bit division (nh / 4 < 2^32) and the periodic
        // neighbours by selects: no 64-bit division on the device
        const unsigned qq = (unsigned)q, q4u = (unsigned)q4, sx2u = (unsigned)g.sx2;
        const unsigned r = qq / q4u, r3 = r / sx2u;
        const int i1 = (int)(qq - r * q4u) * 4;
        const int i2 = (int)(r - r3 * sx2u), i3 = (int)r3;
        const size_t nh = g.nh;
        const size_t row = ((size_t)i3 * g.sx2 + i2) * g.sx1;
        const size_t idx = row + i1;
        const int i1m = i1 == 0 ? g.sx1 - 1 : i1 - 1, i1p = i1 + 4 == g.sx1 ? 0 : i1 + 4;
        const int i2m = i2 == 0 ? g.sx2 - 1 : i2 - 1, i2p = i2 + 1 == g.sx2 ? 0 : i2 + 1;
        const size_t rym = ((size_t)i3 * g.sx2 + i2m) * g.sx1 + i1;
        const size_t ryp = ((size_t)i3 * g.sx2 + i2p) * g.sx1 + i1;
        size_t rzm, rzp;
        float kz;
        if (i3 == 0) { rzm = idx; rzp = idx + g.plane; kz = a.k3b; }
        else if (i3 == g.sx3h - 1) { rzm = idx - g.plane; rzp = idx; kz = a.k3b; }
        else { rzm = idx - g.plane; rzp = idx + g.plane; kz = a.k3; }

        // END: tau += Dt m first, with every load of tau and m issued before
        // the stores of tau (which could alias them), so that the kernel waits
        // for memory once here and once for the strain source below
        float tn[6][4];
        if (MODE == MODE_END) {
            const float dt = (float)a.st->Dt;
            float4 tv[6], mv[6];
#pragma unroll
            for (int c = 0; c < 6; c++) {
                tv[c] = ldc4(a.tau + c * nh + idx);
                mv[c] = ldc4(a.m + c * nh + idx);
            }
            constexpr float wn[6] = {1.f, 2.f, 2.f, 1.f, 2.f, 1.f};
            float qm[4], qt[4];
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const float m4[4] = {mv[c].x, mv[c].y, mv[c].z, mv[c].w};
                const float t4[4] = {tv[c].x, tv[c].y, tv[c].z, tv[c].w};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    tn[c][j] = t4[j] + dt * m4[j];
                    qm[j] = c == 0 ? m4[j] * m4[j] : qm[j] + wn[c] * m4[j] * m4[j];
                    qt[j] = c == 0 ? tn[c][j] * tn[c][j] : qt[j] + wn[c] * tn[c][j] * tn[c][j];
                }
            }
#pragma unroll
            for (int c = 0; c < 6; c++)
                st4(a.tau + c * nh + idx, make_float4(tn[c][0], tn[c][1], tn[c][2], tn[c][3]));
#pragma unroll
            for (int j = 0; j < 4; j++) {
                amp_m += (double)sqrtf(qm[j] * 0.5f);
                amp_t += (double)sqrtf(qt[j] * 0.5f);
            }
        }

        // Hooke's law (src/elastic3d.f90:129-142) on the strain of w at 4
        // points; h = C:E is added to the base stress below
        float h[6][4];
        if (MODE != MODE_EIGEN) {
            float dxw[3][4], dyw[3][4], dzw[3][4];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float *wc = a.w + c * nh;
                if (FIR) {
                    const float4 d = ld4(a.wx + c * nh + idx);
                    dxw[c][0] = d.x; dxw[c][1] = d.y; dxw[c][2] = d.z; dxw[c][3] = d.w;
                } else {
                    const float4 cv = ld4(wc + idx);
                    const float lft = __ldg(wc + row + i1m), rgt = __ldg(wc + row + i1p);
                    dxw[c][0] = (cv.y - lft) * a.k1;
                    dxw[c][1] = (cv.z - cv.x) * a.k1;
                    dxw[c][2] = (cv.w - cv.y) * a.k1;
                    dxw[c][3] = (rgt - cv.z) * a.k1;
                }
                if (FIR) {
                    const float4 d = ld4(a.wy + c * nh + idx);
                    dyw[c][0] = d.x; dyw[c][1] = d.y; dyw[c][2] = d.z; dyw[c][3] = d.w;
                } else {
                    const float4 ym = ld4(wc + rym), yp = ld4(wc + ryp);
                    dyw[c][0] = (yp.x - ym.x) * a.k2;
                    dyw[c][1] = (yp.y - ym.y) * a.k2;
                    dyw[c][2] = (yp.z - ym.z) * a.k2;
                    dyw[c][3] = (yp.w - ym.w) * a.k2;
                }
                const float4 zm = ld4(wc + rzm), zp = ld4(wc + rzp);
                dzw[c][0] = (zp.x - zm.x) * kz;
                dzw[c][1] = (zp.y - zm.y) * kz;
                dzw[c][2] = (zp.z - zm.z) * kz;
                dzw[c][3] = (zp.w - zm.w) * kz;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float e11 = dxw[0][j];
                const float e12 = (dxw[1][j] + dyw[0][j]) * 0.5f;
                const float e13 = (dxw[2][j] + dzw[0][j]) * 0.5f;
                const float e22 = dyw[1][j];
                const float e23 = (dyw[2][j] + dzw[1][j]) * 0.5f;
                const float e33 = dzw[2][j];
                const float tr = e11 + e22 + e33;
                h[0][j] = a.mu2 * e11 + a.lam * tr;
                h[1][j] = a.mu2 * e12;
                h[2][j] = a.mu2 * e13;
                h[3][j] = a.mu2 * e22 + a.lam * tr;
                h[4][j] = a.mu2 * e23;
                h[5][j] = a.mu2 * e33 + a.lam * tr;
            }
        }

        // base stress + h.  Tensor amplitudes (tensornorm, weights 1 2 2 1 2 1
        // over the components) accumulate one component at a time.
        float s[6][4];
        constexpr float wnorm[6] = {1.f, 2.f, 2.f, 1.f, 2.f, 1.f};
        if (MODE == MODE_OP) {
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const float4 v = ldc4(a.sig + c * nh + idx);
                s[c][0] = v.x + h[c][0]; s[c][1] = v.y + h[c][1]; s[c][2] = v.z + h[c][2]; s[c][3] = v.w + h[c][3];
            }
        } else if (MODE == MODE_EIGEN) {
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const float4 v = ldc4(a.sig + c * nh + idx);
                s[c][0] = v.x; s[c][1] = v.y; s[c][2] = v.z; s[c][3] = v.w;
            }
        } else if (MODE == MODE_INIT) {
            float qt[4];
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const float4 t = ldc4(a.tau + c * nh + idx);
                const float tv[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    qt[j] = c == 0 ? tv[j] * tv[j] : qt[j] + wnorm[c] * tv[j] * tv[j];
                    s[c][j] = -tv[j] + h[c][j];
                }
            }
#pragma unroll
            for (int j = 0; j < 4; j++) amp_t += (double)sqrtf(qt[j] * 0.5f);
        } else if (MODE == MODE_END) {
#pragma unroll
            for (int c = 0; c < 6; c++)
#pragma unroll
                for (int j = 0; j < 4; j++) s[c][j] = -tn[c][j] + h[c][j];
        } else {  // MODE_CORR
            const float c1 = -(float)(a.st->Dt / 2);
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const float4 t = ldc4(a.tau + c * nh + idx);
                const float4 m = ldc4(a.m + c * nh + idx);
                s[c][0] = (c1 * m.x - t.x) + h[c][0]; s[c][1] = (c1 * m.y - t.y) + h[c][1];
                s[c][2] = (c1 * m.z - t.z) + h[c][2]; s[c][3] = (c1 * m.w - t.w) + h[c][3];
            }
        }
        if (MODE == MODE_OP || (MODE != MODE_EIGEN && a.store_sig && (!a.sig_mask || a.sig_mask[q]))) {
#pragma unroll
            for (int c = 0; c < 6; c++)
                st4(a.sig + c * nh + idx, make_float4(s[c][0], s[c][1], s[c][2], s[c][3]));
        }

        if (MODE != MODE_OP) {
            // viscouseigenstress for the linear and power-law mechanisms
            float mo[6][4];
#pragma unroll
            for (int c = 0; c < 6; c++) {
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (MODE == MODE_EIGEN) v = ldc4(a.m + c * nh + idx);
                mo[c][0] = v.x; mo[c][1] = v.y; mo[c][2] = v.z; mo[c][3] = v.w;
            }
            float sp[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (a.spdev) {
#pragma unroll
                for (int c = 0; c < 6; c++) sp[c] = __ldg(a.spdev + c * g.sx3h + i3);
            }
            float gsum[4] = {0.f, 0.f, 0.f, 0.f};
            const float dtf = MODE == MODE_CORR ? (float)a.st->Dt : 0.f;
            float4 gold = make_float4(0.f, 0.f, 0.f, 0.f);
            if ((MODE == MODE_CORR || MODE == MODE_EIGEN) && a.gamma) gold = ldc4(a.gamma + idx);
            float gacc[4] = {gold.x, gold.y, gold.z, gold.w};
            // the largest gammadot per mechanism: its reciprocal is the
            // minimum of the points' 1/gammadot (a correctly rounded
            // reciprocal is monotonic), one division instead of four
            float gmx[2] = {0.f, 0.f};
#pragma unroll
            for (int mech = 0; mech < 2; mech++) {
                if (!a.visc[mech]) continue;
                const DepthVisc dv = a.visc[mech][i3];
                float g0v[4] = {dv.g0, dv.g0, dv.g0, dv.g0};
                if (a.dg0[mech]) {
                    const float4 d = ld4(a.dg0[mech] + idx);
                    g0v[0] += d.x; g0v[1] += d.y; g0v[2] += d.z; g0v[3] += d.w;
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    gsum[j] = 0.f;
                    if (!(g0v[j] >= 1.0e-20f)) continue;
                    const float tr3 = (s[0][j] + s[3][j] + s[5][j]) * (1.f / 3.f);
                    const float d11 = s[0][j] - tr3, d22 = s[3][j] - tr3, d33 = s[5][j] - tr3;
                    const float tau = tnorm6(d11 + sp[0], s[1][j] + sp[1], s[2][j] + sp[2],
                                             d22 + sp[3], s[4][j] + sp[4], d33 + sp[5]);
                    const float tauc = fmaxf(0.f, tau - dv.cohesion);
                    if (!(tauc > 1.0e-20f)) continue;
                    const float x = tauc * a.muinv;
                    const float pe = dv.power - 1.f;
                    float gd;
                    if (pe == 0.f) gd = g0v[j];
                    else if (pe == 1.f) gd = g0v[j] * x;
                    else if (pe == 2.f) gd = g0v[j] * x * x;
                    else gd = g0v[j] * powf(x, pe);
                    const float gd2 = 2.f * gd, gp2 = 2.f * g0v[j] * dv.tpow;
                    mo[0][j] += gd2 * d11 - gp2 * sp[0];
                    mo[1][j] += gd2 * s[1][j] - gp2 * sp[1];
                    mo[2][j] += gd2 * s[2][j] - gp2 * sp[2];
                    mo[3][j] += gd2 * d22 - gp2 * sp[3];
                    mo[4][j] += gd2 * s[4][j] - gp2 * sp[4];
                    mo[5][j] += gd2 * d33 - gp2 * sp[5];
                    gmx[mech] = fmaxf(gmx[mech], gd);
                    gsum[j] = gd * x;
                    if (MODE == MODE_EIGEN) gacc[j] = gsum[j];
                }
                if (MODE == MODE_CORR) {
#pragma unroll
                    for (int j = 0; j < 4; j++) gacc[j] = gacc[j] + dtf * gsum[j];
                }
            }
#pragma unroll
            for (int mech = 0; mech < 2; mech++) tmin[mech] = fminf(tmin[mech], 1.f / gmx[mech]);
            if (TRANS && (MODE == MODE_INIT || MODE == MODE_END || MODE == MODE_CORR) && a.eps) {
                float ep[6][4], in[6][4], rate[6][4];
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    const float4 e = ldc4(a.eps + c * nh + idx);
                    ep[c][0] = e.x; ep[c][1] = e.y; ep[c][2] = e.z; ep[c][3] = e.w;
                }
                if (MODE == MODE_CORR) {
                    const float h = (float)(a.st->Dt / 2);
#pragma unroll
                    for (int c = 0; c < 6; c++) {
                        const float4 r = ldc4(a.epsdot + c * nh + idx);
                        in[c][0] = h * r.x + ep[c][0]; in[c][1] = h * r.y + ep[c][1];
                        in[c][2] = h * r.z + ep[c][2]; in[c][3] = h * r.w + ep[c][3];
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < 6; c++)
#pragma unroll
                        for (int j = 0; j < 4; j++) in[c][j] = ep[c][j];
                }
#pragma unroll
                for (int c = 0; c < 6; c++)
#pragma unroll
                    for (int j = 0; j < 4; j++) rate[c][j] = 0.f;
#pragma unroll
                for (int tm = 0; tm < 2; tm++) {
                    if (!a.trans[tm]) continue;
                    const TransLayer L = a.trans[tm][i3];
                    float g0v[4] = {L.g0, L.g0, L.g0, L.g0};
                    if (a.tdg0[tm]) {
                        const float4 d = ld4(a.tdg0[tm] + idx);
                        g0v[0] += d.x; g0v[1] += d.y; g0v[2] += d.z; g0v[3] += d.w;
                    }
#pragma unroll
                    for (int j = 0; j < 4; j++) {
#pragma unroll
                        for (int c = 0; c < 6; c++) rate[c][j] = 0.f;
                        if (1.0e-20f > g0v[j]) continue;
                        const float tr3 = (s[0][j] + s[3][j] + s[5][j]) * (1.f / 3.f);
                        // Q = s' - 2 Gk epsilonik
                        const float Q[6] = {(s[0][j] - tr3) - L.gk2 * in[0][j], s[1][j] - L.gk2 * in[1][j],
                                            s[2][j] - L.gk2 * in[2][j], (s[3][j] - tr3) - L.gk2 * in[3][j],
                                            s[4][j] - L.gk2 * in[4][j], (s[5][j] - tr3) - L.gk2 * in[5][j]};
                        const float x = tnorm6(Q[0], Q[1], Q[2], Q[3], Q[4], Q[5]) * a.muinv;
                        const float pe = L.power - 1.f;
                        float gd;
                        if (pe == 0.f) gd = g0v[j];
                        else if (pe == 1.f) gd = g0v[j] * x;
                        else if (pe == 2.f) gd = g0v[j] * x * x;
                        else gd = g0v[j] * powf(x, pe);
                        const float rq = gd * a.muinv, gd2 = 2.f * gd;
#pragma unroll
                        for (int c = 0; c < 6; c++) {
                            rate[c][j] = rq * Q[c];
                            mo[c][j] += gd2 * Q[c];
                        }
                        if (MODE != MODE_CORR) tmin[2 + tm] = fminf(tmin[2 + tm], 1.f / gd);
                    }
                    if (MODE == MODE_CORR) {
                        // the corrector's next call reads epsilonikdot, i.e. this rate
#pragma unroll
                        for (int c = 0; c < 6; c++)
#pragma unroll
                            for (int j = 0; j < 4; j++) in[c][j] = rate[c][j];
                    }
                }
                if (MODE == MODE_CORR) {
#pragma unroll
                    for (int c = 0; c < 6; c++)
                        st4(a.eps + c * nh + idx,
                            make_float4(ep[c][0] + dtf * rate[c][0], ep[c][1] + dtf * rate[c][1],
                                        ep[c][2] + dtf * rate[c][2], ep[c][3] + dtf * rate[c][3]));
                } else {
#pragma unroll
                    for (int c = 0; c < 6; c++)
                        st4(a.epsdot + c * nh + idx, make_float4(rate[c][0], rate[c][1], rate[c][2], rate[c][3]));
                }
            }
#pragma unroll
            for (int c = 0; c < 6; c++)
                st4(a.m + c * nh + idx, make_float4(mo[c][0], mo[c][1], mo[c][2], mo[c][3]));
            if ((MODE == MODE_CORR || MODE == MODE_EIGEN) && a.gamma)
                st4(a.gamma + idx, make_float4(gacc[0], gacc[1], gacc[2], gacc[3]));
        }
    }

    if (MODE == MODE_INIT || MODE == MODE_END || MODE == MODE_EIGEN) {
        // the block reductions in one pass (fixed order, one barrier); 8 warps
        float tq[4];
#pragma unroll
        for (int q = 0; q < NTM; q++) tq[q] = warp_min(tmin[q]);
        double am = warp_sum(amp_m), at = warp_sum(amp_t);
        {
            const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
            if (l == 0) {
#pragma unroll
                for (int q = 0; q < NTM; q++) shf[8 * q + w] = tq[q];
                shd[w] = am; shd[16 + w] = at;
            }
            __syncthreads();
            if (w == 0) {
#pragma unroll
                for (int q = 0; q < NTM; q++) tq[q] = warp_min(l < nw ? shf[8 * q + l] : 3.0e38f);
                am = warp_sum(l < nw ? shd[l] : 0.0);
                at = warp_sum(l < nw ? shd[16 + l] : 0.0);
            }
        }
        __shared__ unsigned last;
        if (threadIdx.x == 0) {
#pragma unroll
            for (int q = 0; q < NTM; q++) a.tm_part[q * gridDim.x + blockIdx.x] = tq[q];
            a.amp_part[blockIdx.x] = am;
            a.amp_part[gridDim.x + blockIdx.x] = at;
            if (a.ticket) {
                __threadfence();
                last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
            }
        }
        if (MODE != MODE_EIGEN && a.ticket) {
            // the last block to finish reduces the partials of all blocks in
            // a fixed order: Maxwell-time minima and the log amplitudes
            __syncthreads();
            if (last) {
                __threadfence();
                const int n = gridDim.x, nt = blockDim.x;
                float mq[4] = {3.0e38f, 3.0e38f, 3.0e38f, 3.0e38f};
                double s0 = 0.0, s1 = 0.0;
                for (int b = 0; b < n; b += 8 * nt) {
                    float v[4][8];
                    double w0[8], w1[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        const int i = b + u * nt + threadIdx.x;
                        const bool in = i < n;
#pragma unroll
                        for (int q = 0; q < NTM; q++) v[q][u] = in ? __ldcg(a.tm_part + q * n + i) : 3.0e38f;
                        w0[u] = in ? __ldcg(a.amp_part + i) : 0.0;
                        w1[u] = in ? __ldcg(a.amp_part + n + i) : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) {
#pragma unroll
                        for (int q = 0; q < NTM; q++) mq[q] = fminf(mq[q], v[q][u]);
                        s0 += w0[u];
                        s1 += w1[u];
                    }
                }
#pragma unroll
                for (int q = 0; q < NTM; q++) {
                    mq[q] = block_min(mq[q], shf);
                    __syncthreads();
                }
                s0 = block_sum(s0, shd);
                __syncthreads();
                s1 = block_sum(s1, shd);
                if (threadIdx.x == 0) {
#pragma unroll
                    for (int q = 0; q < 4; q++) a.fin->tmin[q] = q < NTM ? mq[q] : 3.0e38f;
                    a.fin->power = s0 * a.dv;
                    a.fin->cei = s1 * a.dv;
                    *a.ticket = 0u;
                }
            }
        }
    }
}

// tau += Dt m with the amplitude of m (coseismic-event path of the step,
// src/relax.f90:836 followed by :858-886)
__global__ void __launch_bounds__(RELAX_NTHREADS) k_tau_update(Grid g, float *tau, const float *m,
                                                               const StepState *st, double *amp_part)
{
    __shared__ double shd[32];
    const size_t nq = g.nh >> 2;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double am = 0.0;
    if (q < nq) {
        const float dt = (float)st->Dt;
        float mm[6][4];
#pragma unroll
        for (int c = 0; c < 6; c++) {
            const float4 t = ldc4(tau + c * g.nh + 4 * q), v = ldc4(m + c * g.nh + 4 * q);
            mm[c][0] = v.x; mm[c][1] = v.y; mm[c][2] = v.z; mm[c][3] = v.w;
            st4(tau + c * g.nh + 4 * q, make_float4(t.x + dt * v.x, t.y + dt * v.y, t.z + dt * v.z, t.w + dt * v.w));
        }
#pragma unroll
        for (int j = 0; j < 4; j++) am += (double)tnorm6(mm[0][j], mm[1][j], mm[2][j], mm[3][j], mm[4][j], mm[5][j]);
    }
    am = block_sum(am, shd);
    if (threadIdx.x == 0) amp_part[blockIdx.x] = am;
}

// ------------------------------------------------------------------------
// frictioneigenstress, src/friction3d.f90:82-241, for one afterslip plane,
// launched over the index box that bounds the plane's band.
// ------------------------------------------------------------------------
struct FrictionArgs {
    Grid g;
    double x, y, z, L, W, strike, dip, rake, beta, mu;
    // plane geometry, precomputed on the host (src/friction3d.f90:128-152)
    double cs, ss, cd, sd, cr, sr, xr, yr, zr, Wp, Lp;
    const double *fc;        // 4 x sx3h: V0, (a-b)sigma, friction, cohesion
    const float *sig;        // 6 x nh
    float *m;                // 6 x nh
    int j1lo, n1, j2lo, n2, i3lo, n3;
    int want_tm;
    float *tm_part;          // one per block
    int *err;
};

__device__ __forceinline__ double d_gauss(double x, double s)
{
    return exp(-0.5 * (x / s) * (x / s)) / sqrt(6.28318530717958623199592693708837032318) / s;
}
__device__ __forceinline__ double d_omega(double x, double beta)
{
    const double ax = fabs(x);
    if (ax <= (1.0 - 2.0 * beta) / (1.0 - beta) / 2.0) return 1.0;
    if (ax < 1.0 / (1.0 - beta) / 2.0) {
        const double c = cos(3.141592653589793115997963468544185161 * ((1.0 - beta) * ax - 0.5 + beta) / 2.0 / beta);
        return c * c;
    }
    return 0.0;
}
__device__ __forceinline__ double d_omegap(double x, double beta)
{
    const double ax = fabs(x);
    if (ax > (1.0 - 2.0 * beta) / (1.0 - beta) / 2.0 && ax < 1.0 / (1.0 - beta) / 2.0)
        return -copysign(1.0, x) * 3.141592653589793115997963468544185161 * (1.0 - beta) / 2.0 / beta *
               sin(3.141592653589793115997963468544185161 * ((1.0 - beta) * ax - 0.5 + beta) / beta);
    return 0.0;
}
__device__ __forceinline__ double d_gaussp(double x, double s)
{
    return -x * exp(-0.5 * (x / s) * (x / s)) / sqrt(6.28318530717958623199592693708837032318) / (s * s * s);
}
__device__ __forceinline__ double my_sinh(double x)
{
    return fabs(x) > 11.0 ? copysign(1.0, x) * sinh(11.0) : sinh(x);
}

__global__ void __launch_bounds__(RELAX_NTHREADS) k_friction(FrictionArgs a)
{
    __shared__ float shf[32];
    const Grid &g = a.g;
    const size_t n = (size_t)a.n1 * a.n2 * a.n3;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    float tm = 3.0e38f;
    if (t < n) {
        const int j1 = a.j1lo + (int)(t % a.n1);
        const int j2 = a.j2lo + (int)((t / a.n1) % a.n2);
        const int i3 = a.i3lo + (int)(t / ((size_t)a.n1 * a.n2));
        const double dx1 = g.dx1, dx2 = g.dx2, dx3 = g.dx3;
        const double x3 = (double)i3 * dx3;
        const double Wp = a.Wp, Lp = a.Lp;
        const double mwp = Wp > Lp ? Wp : Lp;
        // shifted coordinates: index j (may be negative) -> x = j dx
        const double x1 = (double)j1 * dx1, x2 = (double)j2 * dx2;
        bool ok = !(fabs(x3 - a.z) > Lp && fabs(x3 + a.z) > Lp);
        ok = ok && !(fabs(x1 - a.x) > mwp || fabs(x2 - a.y) > mwp);
        const double cs = a.cs, ss = a.ss, cd = a.cd, sd = a.sd, cr = a.cr, sr = a.sr;
        const double xr = a.xr, yr = a.yr, zr = a.zr;
        double x2r = cs * x1 - ss * x2;
        const double x1s = cd * x2r - sd * x3, x1i = cd * x2r + sd * x3;
        ok = ok && !(fabs(x1s - xr) > 7.01 * dx1 && fabs(x1i - xr) > 7.01 * dx1);
        if (ok) {
            const double x2s = ss * x1 + cs * x2;
            const double x3s = sd * x2r + cd * x3, x3i = -sd * x2r + cd * x3;
            double temp1 = d_gauss(x1s - xr, dx1), temp2 = d_omega((x2s - yr) / a.W, a.beta);
            double temp3 = d_omega((x3s - zr) / a.L, a.beta);
            const double sourc = temp1 * temp2 * temp3;
            temp1 = d_gauss(x1i - xr, dx1);
            temp3 = d_omega((x3i + zr) / a.L, a.beta);
            const double impulse = sourc + temp1 * temp2 * temp3;
            const int i1 = (j1 + g.sx1) % g.sx1, i2 = (j2 + g.sx2) % g.sx2;
            const size_t o = ((size_t)i3 * g.sx2 + i2) * g.sx1 + i1;
            double sv[6];
#pragma unroll
            for (int c = 0; c < 6; c++) sv[c] = (double)a.sig[c * g.nh + o];
            const double n0 = cd * cs, n1 = -cd * ss, n2 = -sd;
            const double r0 = ss * cr + cs * sd * sr, r1 = cs * cr - ss * sd * sr, r2 = cd * sr;
            const double t0 = sv[0] * n0 + sv[1] * n1 + sv[2] * n2;
            const double t1 = sv[1] * n0 + sv[3] * n1 + sv[4] * n2;
            const double t2 = sv[2] * n0 + sv[4] * n1 + sv[5] * n2;
            const double taun = t0 * n0 + t1 * n1 + t2 * n2;
            double ts0 = t0 - taun * n0, ts1 = t1 - taun * n1, ts2 = t2 - taun * n2;
            const double taus = sqrt(ts0 * ts0 + ts1 * ts1 + ts2 * ts2);
            const double vo = a.fc[i3], tauc = a.fc[g.sx3h + i3];
            const double fr = a.fc[2 * g.sx3h + i3], coh = a.fc[3 * g.sx3h + i3];
            double tau = taus + fr * taun - coh;
            if (tau < 0.0) tau = 0.0;
            const bool back = (ts0 * r0 + ts1 * r1 + ts2 * r2) < 0.0 &&
                              fabs(a.rake) < 6.28318530717958623199592693708837032318 * 1.5;
            if (!back) {
                if ((tau / tauc) > 20) atomicOr(a.err, 1 << RELAX_ERR_FRICTION);
                ts0 /= taus; ts1 /= taus; ts2 /= taus;
                const double gd = vo * 2.0 * my_sinh(tau / tauc);
                if (a.want_tm) {
                    const float cand = (float)(tau / a.mu / gd * ((a.L < a.W ? a.L : a.W) / sqrt(dx1 * dx3)));
                    if (cand < tm) tm = cand;
                }
                const double b = 2.0 * a.mu * impulse * gd;
                const double b0 = b * n0, b1 = b * n1, b2 = b * n2;
                float *mp = a.m + o;
                mp[0 * g.nh] += (float)(ts0 * b0);
                mp[1 * g.nh] += (float)((ts0 * b1 + ts1 * b0) / 2.0);
                mp[2 * g.nh] += (float)((ts0 * b2 + ts2 * b0) / 2.0);
                mp[3 * g.nh] += (float)(ts1 * b1);
                mp[4 * g.nh] += (float)((ts1 * b2 + ts2 * b1) / 2.0);
                mp[5 * g.nh] += (float)(ts2 * b2);
            }
        }
    }
    if (a.want_tm) {
        tm = block_min(tm, shf);
        if (threadIdx.x == 0) a.tm_part[blockIdx.x] = tm;
    }
}


// The band of an afterslip plane and the geometric impulse of each band
// point (src/friction3d.f90:143-183) do not change during a run: k_friction_mark
// evaluates them once over the plane's index box (impulse, or -1 outside the
// band); the host compacts the box into a point list for k_friction_pts.
__global__ void k_friction_mark(FrictionArgs a, double *imp)
{
    const Grid &g = a.g;
    const size_t n = (size_t)a.n1 * a.n2 * a.n3;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int j1 = a.j1lo + (int)(t % a.n1);
    const int j2 = a.j2lo + (int)((t / a.n1) % a.n2);
    const int i3 = a.i3lo + (int)(t / ((size_t)a.n1 * a.n2));
    const double dx1 = g.dx1, dx2 = g.dx2, dx3 = g.dx3;
    const double x3 = (double)i3 * dx3, x1 = (double)j1 * dx1, x2 = (double)j2 * dx2;
    const double mwp = a.Wp > a.Lp ? a.Wp : a.Lp;
    double out = -1.0;
    bool ok = !(fabs(x3 - a.z) > a.Lp && fabs(x3 + a.z) > a.Lp);
    ok = ok && !(fabs(x1 - a.x) > mwp || fabs(x2 - a.y) > mwp);
    const double x2r = a.cs * x1 - a.ss * x2;
    const double x1s = a.cd * x2r - a.sd * x3, x1i = a.cd * x2r + a.sd * x3;
    ok = ok && !(fabs(x1s - a.xr) > 7.01 * dx1 && fabs(x1i - a.xr) > 7.01 * dx1);
    if (ok) {
        const double x2s = a.ss * x1 + a.cs * x2;
        const double x3s = a.sd * x2r + a.cd * x3, x3i = -a.sd * x2r + a.cd * x3;
        double temp1 = d_gauss(x1s - a.xr, dx1), temp2 = d_omega((x2s - a.yr) / a.W, a.beta);
        double temp3 = d_omega((x3s - a.zr) / a.L, a.beta);
        const double sourc = temp1 * temp2 * temp3;
        temp1 = d_gauss(x1i - a.xr, dx1);
        temp3 = d_omega((x3i + a.zr) / a.L, a.beta);
        out = sourc + temp1 * temp2 * temp3;
    }
    imp[t] = out;
}

struct FrictionPtsArgs {
    Grid g;
    double mu, rake, L, W;
    double n0, n1, n2, r0, r1, r2;     // plane normal and rake vectors
    const double *fc;
    const float *sig;
    float *m;
    const unsigned *idx;               // band points (flat physical index)
    const double *imp;                 // their impulse
    int npts;
    int want_tm;
    float *tm_part;
    int *err;
    const struct FrictionPtsArgs *tab;   // batched launch: one entry per member (blockIdx.y)
};

// frictioneigenstress on the band points of one plane (the per-step part of
// src/friction3d.f90:185-235)
template <bool BATCH = false>
__global__ void __launch_bounds__(RELAX_NTHREADS) k_friction_pts(const __grid_constant__ FrictionPtsArgs a0)
{
    pdl_enter();
    const FrictionPtsArgs &a = BATCH ? a0.tab[blockIdx.y] : a0;
    __shared__ float shf[32];
    const Grid &g = a.g;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float tm = 3.0e38f;
    if (t < a.npts) {
        const size_t o = a.idx[t];
        const int i3 = (int)(o / g.plane);
        const double impulse = a.imp[t];
        double sv[6];
#pragma unroll
        for (int c = 0; c < 6; c++) sv[c] = (double)a.sig[c * g.nh + o];
        const double n0 = a.n0, n1 = a.n1, n2 = a.n2;
        const double t0 = sv[0] * n0 + sv[1] * n1 + sv[2] * n2;
        const double t1 = sv[1] * n0 + sv[3] * n1 + sv[4] * n2;
        const double t2 = sv[2] * n0 + sv[4] * n1 + sv[5] * n2;
        const double taun = t0 * n0 + t1 * n1 + t2 * n2;
        double ts0 = t0 - taun * n0, ts1 = t1 - taun * n1, ts2 = t2 - taun * n2;
        const double taus = sqrt(ts0 * ts0 + ts1 * ts1 + ts2 * ts2);
        const double vo = a.fc[i3], tauc = a.fc[g.sx3h + i3];
        const double fr = a.fc[2 * g.sx3h + i3], coh = a.fc[3 * g.sx3h + i3];
        double tau = taus + fr * taun - coh;
        if (tau < 0.0) tau = 0.0;
        const bool back = (ts0 * a.r0 + ts1 * a.r1 + ts2 * a.r2) < 0.0 &&
                          fabs(a.rake) < 6.28318530717958623199592693708837032318 * 1.5;
        if (!back) {
            if ((tau / tauc) > 20) atomicOr(a.err, 1 << RELAX_ERR_FRICTION);
            ts0 /= taus; ts1 /= taus; ts2 /= taus;
            const double gd = vo * 2.0 * my_sinh(tau / tauc);
            if (a.want_tm) {
                const float cand = (float)(tau / a.mu / gd * ((a.L < a.W ? a.L : a.W) / sqrt(g.dx1 * g.dx3)));
                if (cand < tm) tm = cand;
            }
            const double b = 2.0 * a.mu * impulse * gd;
            const double b0 = b * n0, b1 = b * n1, b2 = b * n2;
            float *mp = a.m + o;
            mp[0 * g.nh] += (float)(ts0 * b0);
            mp[1 * g.nh] += (float)((ts0 * b1 + ts1 * b0) / 2.0);
            mp[2 * g.nh] += (float)((ts0 * b2 + ts2 * b0) / 2.0);
            mp[3 * g.nh] += (float)(ts1 * b1);
            mp[4 * g.nh] += (float)((ts1 * b2 + ts2 * b1) / 2.0);
            mp[5 * g.nh] += (float)(ts2 * b2);
        }
    }
    if (a.want_tm) {
        tm = block_min(tm, shf);
        if (threadIdx.x == 0) a.tm_part[blockIdx.x] = tm;
    }
}

// monitorfriction + frictionadd, src/friction3d.f90:263-453, one thread
// per patch.  dt = 0 leaves the cumulative slip unchanged.
struct MonitorArgs {
    Grid g;
    double x, y, z, strike, dip, rake;
    const double *fc;
    const float *sig;
    relax_slippatch *patch;
    int px2, px3;
    const StepState *st;
    const struct MonitorArgs *tab;   // batched launch: one entry per member (blockIdx.y)
};

// Position of patch t of a plane and the grid cell it samples (the nearest
// point, src/friction3d.f90:311-335); false when it falls outside the box.
__device__ __forceinline__ bool monitor_cell(const MonitorArgs &a, int t, double X[3], double *yr_out,
                                             double *zr_out, size_t *o, int *i3_out)
{
    const Grid &g = a.g;
    const int j2 = t % a.px2 + 1, j3 = t / a.px2 + 1;
    const double cs = cos(a.strike), ss = sin(a.strike), cd = cos(a.dip), sd = sin(a.dip);
    const double x2 = cs * a.x - ss * a.y;
    const double xr = cd * x2 - sd * a.z;
    double yr = ss * a.x + cs * a.y, zr = sd * x2 + cd * a.z;
    yr = (double)((float)yr + (float)(((double)j2 - (double)a.px2 / 2.0 - 1.0) * g.dx2));
    zr = (double)((float)zr + (float)(((double)j3 - (double)a.px3 / 2.0 - 1.0) * g.dx3));
    const double x2p = cd * xr + sd * zr;
    X[0] = cs * x2p + ss * yr; X[1] = -ss * x2p + cs * yr; X[2] = -sd * xr + cd * zr;
    *yr_out = yr; *zr_out = zr;
    const bool ok = !(X[0] > (double)(g.sx1 / 2 - 1) * g.dx1 || X[0] < -(double)(g.sx1 / 2) * g.dx1 ||
                      X[1] > (double)(g.sx2 / 2 - 1) * g.dx2 || X[1] < -(double)(g.sx2 / 2) * g.dx2 ||
                      X[2] > (double)(g.sx3h - 1) * g.dx3 || X[2] < 0.0);
    if (!ok) return false;
    auto fix = [](double v) { double f = floor(v), c = ceil(v); return (int)((v - f) > 0.5 ? c : f); };
    const int i1 = ((g.sx1 + fix(X[0] / g.dx1)) % g.sx1 + g.sx1) % g.sx1;
    const int i2 = ((g.sx2 + fix(X[1] / g.dx2)) % g.sx2 + g.sx2) % g.sx2;
    const int i3 = fix(X[2] / g.dx3);
    if (i3 < 0 || i3 >= g.sx3h) return false;
    *o = ((size_t)i3 * g.sx2 + i2) * g.sx1 + i1;
    *i3_out = i3;
    return true;
}

// cells whose stress the friction and monitor kernels read: one flag per
// group of 4 points along x1 (the stress kernels' float4 groups)
__global__ void k_mark_points(const unsigned *idx, int n, unsigned char *mask)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) mask[idx[t] >> 2] = 1;
}

__global__ void k_mark_monitor(MonitorArgs a, unsigned char *mask)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.px2 * a.px3) return;
    double X[3], yr, zr;
    size_t o;
    int i3;
    if (monitor_cell(a, t, X, &yr, &zr, &o, &i3)) mask[o >> 2] = 1;
}

template <bool BATCH = false>
__global__ void k_monitor(const __grid_constant__ MonitorArgs a0)
{
    const MonitorArgs &a = BATCH ? a0.tab[blockIdx.y] : a0;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.px2 * a.px3) return;
    const Grid &g = a.g;
    relax_slippatch *p = a.patch + t;
    const double cs = cos(a.strike), ss = sin(a.strike), cd = cos(a.dip), sd = sin(a.dip);
    const double cr = cos(a.rake), sr = sin(a.rake);
    const double svv[3] = {ss, cs, 0.0}, dvv[3] = {-cs * sd, ss * sd, -cd};
    const double n[3] = {cd * cs, -cd * ss, -sd};
    const double r[3] = {ss * cr + cs * sd * sr, cs * cr - ss * sd * sr, cd * sr};
    double X[3], yr, zr;
    size_t o;
    int i3;
    const bool in = monitor_cell(a, t, X, &yr, &zr, &o, &i3);
    p->x1 = X[0]; p->x2 = X[1]; p->x3 = X[2]; p->lx = yr; p->lz = zr;
    if (in) {
        {
            float s6[6];
            for (int c = 0; c < 6; c++) s6[c] = a.sig[c * g.nh + o];
            p->sig.s11 = s6[0]; p->sig.s12 = s6[1]; p->sig.s13 = s6[2];
            p->sig.s22 = s6[3]; p->sig.s23 = s6[4]; p->sig.s33 = s6[5];
            const double t0 = s6[0] * n[0] + s6[1] * n[1] + s6[2] * n[2];
            const double t1 = s6[1] * n[0] + s6[3] * n[1] + s6[4] * n[2];
            const double t2 = s6[2] * n[0] + s6[4] * n[1] + s6[5] * n[2];
            const double taun = t0 * n[0] + t1 * n[1] + t2 * n[2];
            double ts[3] = {t0 - taun * n[0], t1 - taun * n[1], t2 - taun * n[2]};
            const double taus = sqrt(ts[0] * ts[0] + ts[1] * ts[1] + ts[2] * ts[2]);
            const double vo = a.fc[i3], tauc = a.fc[g.sx3h + i3];
            const double fr = a.fc[2 * g.sx3h + i3], coh = a.fc[3 * g.sx3h + i3];
            double tau = taus + fr * taun - coh;
            if (tau < 0.0) tau = 0.0;
            const bool back = (ts[0] * r[0] + ts[1] * r[1] + ts[2] * r[2]) < 0.0 &&
                              fabs(a.rake) < 6.28318530717958623199592693708837032318 * 1.5;
            if (!back) {
                p->taus = taus;
                p->v = vo * 2.0 * my_sinh(tau / tauc);
                for (int k = 0; k < 3; k++) ts[k] /= taus;
                p->vss = p->v * (ts[0] * svv[0] + ts[1] * svv[1] + ts[2] * svv[2]);
                p->vds = p->v * (ts[0] * dvv[0] + ts[1] * dvv[1] + ts[2] * dvv[2]);
            }
        }
    }
    const double dt = a.st ? a.st->Dt : 0.0;
    p->ss = p->ss + dt * p->vss;
    p->ds = p->ds + dt * p->vds;
    p->slip = sqrt(p->ds * p->ds + p->ss * p->ss);
}

// transienteigenstress (src/viscoelastic3d.f90:123-202) on SoA tensors, one
// point per thread (operator API): moment += 2 gd Q, epsilonikdot = gd/mu Q
// with Q = s' - 2 Gk epsilonik.  eps and epsdot may be the same array (each
// point reads before it writes), as in the reference's corrector call.
struct TransArgs {
    Grid g;
    const TransLayer *L;
    const float *dg0;        // weak-zone perturbation or null
    const float *sig;        // 6 x nh
    const float *eps;        // 6 x nh
    float *m;                // 6 x nh, accumulated
    float *epsdot;           // 6 x nh
    float muinv;
    float *tm_part;          // [gridDim.x]
};

__global__ void __launch_bounds__(RELAX_NTHREADS) k_transient(TransArgs a)
{
    __shared__ float shf[32];
    const Grid &g = a.g;
    const size_t nh = g.nh;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    float tm = 3.0e38f;
    if (q < nh) {
        const TransLayer L = a.L[q / g.plane];
        const float g0 = a.dg0 ? L.g0 + a.dg0[q] : L.g0;
        if (1.0e-20f > g0) {
            for (int c = 0; c < 6; c++) a.epsdot[c * nh + q] = 0.f;
        } else {
            float s[6], e[6];
            for (int c = 0; c < 6; c++) { s[c] = a.sig[c * nh + q]; e[c] = a.eps[c * nh + q]; }
            const float tr3 = (s[0] + s[3] + s[5]) * (1.f / 3.f);
            const float Q[6] = {(s[0] - tr3) - L.gk2 * e[0], s[1] - L.gk2 * e[1], s[2] - L.gk2 * e[2],
                                (s[3] - tr3) - L.gk2 * e[3], s[4] - L.gk2 * e[4], (s[5] - tr3) - L.gk2 * e[5]};
            const float x = tnorm6(Q[0], Q[1], Q[2], Q[3], Q[4], Q[5]) * a.muinv;
            const float pe = L.power - 1.f;
            float gd;
            if (pe == 0.f) gd = g0;
            else if (pe == 1.f) gd = g0 * x;
            else if (pe == 2.f) gd = g0 * x * x;
            else gd = g0 * powf(x, pe);
            const float rq = gd * a.muinv, gd2 = 2.f * gd;
            for (int c = 0; c < 6; c++) {
                a.epsdot[c * nh + q] = rq * Q[c];
                a.m[c * nh + q] += gd2 * Q[c];
            }
            tm = 1.f / gd;
        }
    }
    tm = block_min(tm, shf);
    if (threadIdx.x == 0) a.tm_part[blockIdx.x] = tm;
}

// builddgammadot0 (src/viscoelastic3d.f90:320-435): the fluidity perturbation
// of tapered ductile zones (bricks, spheres, cylinders) at the physical
// points, one point per thread
__global__ void k_dgammadot0(Grid g, const relax_weakzone *zones, int nz, double beta, float *out)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int j1 = (int)(q % g.sx1), j2 = (int)((q / g.sx1) % g.sx2), j3 = (int)(q / g.plane);
    const double x1 = (j1 < g.sx1 / 2 ? j1 : j1 - g.sx1) * g.dx1;
    const double x2 = (j2 < g.sx2 / 2 ? j2 : j2 - g.sx2) * g.dx2;
    const double x3 = (double)j3 * g.dx3;
    double f = 0.0;
    for (int i = 0; i < nz; i++) {
        const relax_weakzone &z = zones[i];
        const double dg = z.dgammadot0, W = z.length, L = z.width, D = z.thickness;
        const double Wp = W * (1.0 + 2.0 * beta) / 2.0, Lp = L * (1.0 + 2.0 * beta) / 2.0,
                     Dp = D * (1.0 + 2.0 * beta) / 2.0;
        const double LM = fmax(Wp, fmax(Lp, Dp));
        if (fabs(x3 - z.z) > LM || fabs(x1 - z.x) > LM || fabs(x2 - z.y) > LM) continue;
        const double cs = cos(z.strike), ss = sin(z.strike), cd = cos(z.dip), sd = sin(z.dip);
        double x2r = cs * z.x - ss * z.y;
        const double xr = cd * x2r - sd * z.z, yr = ss * z.x + cs * z.y, zr = sd * x2r + cd * z.z;
        x2r = cs * x1 - ss * x2;
        const double x1s = cd * x2r - sd * x3, x2s = ss * x1 + cs * x2, x3s = sd * x2r + cd * x3;
        if (D >= 0 && W >= 0 && L >= 0) {
            f = f + d_omega((x1s - xr) / D, beta) * d_omega((x2s - yr) / W, beta) * d_omega((x3s - zr) / L, beta) * dg;
        } else if (D < 0 && W < 0 && L < 0) {
            const double r = sqrt(((x1s - xr) / D) * ((x1s - xr) / D) + ((x2s - yr) / W) * ((x2s - yr) / W) +
                                  ((x3s - zr) / L) * ((x3s - zr) / L));
            f = f + d_omega(r, beta) * dg;
        } else if (D < 0 && W < 0) {
            const double rho = sqrt(((x1s - xr) / D) * ((x1s - xr) / D) + ((x2s - yr) / W) * ((x2s - yr) / W));
            f = f + d_omega(rho, beta) * d_omega((x3s - zr) / L, beta) * dg;
        } else if (D < 0 && L < 0) {
            const double rho = sqrt(((x1s - xr) / D) * ((x1s - xr) / D) + ((x3s - zr) / L) * ((x3s - zr) / L));
            f = f + d_omega(rho, beta) * d_omega((x2s - yr) / W, beta) * dg;
        } else if (W < 0 && L < 0) {
            const double rho = sqrt(((x2s - yr) / W) * ((x2s - yr) / W) + ((x3s - zr) / L) * ((x3s - zr) / L));
            f = f + d_omega(rho, beta) * d_omega((x1s - xr) / D, beta) * dg;
        }
    }
    out[q] = (float)f;
}

// ------------------------------------------------------------------------
// 3-D transform, pass 1: R2C along x1.
//   MODE_DIV: the input is the equivalent body force -div(m) of the moment
//             tensor (equivalentbodyforce, src/elastic3d.f90:1214-1506)
//             computed on the fly, and the traction t_i = m_i3(x3=0).
//   MODE_REAL: the input is read from real arrays (any pitches).
// Output: spectrum planes [0, nin) and the traction plane sx3, scaled by
// dx1 dx2 dx3 (dx1 dx2 for the traction), src/fourier.f90:195-199.
// ------------------------------------------------------------------------
enum { XIN_DIV = 0, XIN_REAL = 1 };

struct XfArgs {
    Grid g;
    float2 *S;
    FftPlan pm;              // complex length M = sx1/2
    const float2 *tw1;       // exp(-2 pi i k / sx1)
    int nin, rows;
    int has_trac;            // blockIdx.y == nin is the traction plane
    const float *m;          // XIN_DIV: 6 x nh moment
    float k1, k2, k3, k3b;
    Fir7 fx, fy;             // XIN_DIV: the x1, x2 differentiators (n = 7: fir7, k_xfwd only)
    const float *in[3];      // XIN_REAL
    size_t rp, pp;           // row / plane pitch (elements)
    const float *tin[3];
    size_t trp;
    const float *tload;      // optional surface load added to t3 (sx1 x sx2)
    float scale3, scale2;
    const struct XfArgs *tab;   // batched launch: one entry per member (blockIdx.z)
};

template <int XIN>
__global__ void __launch_bounds__(RELAX_NTHREADS) k_xfwd(XfArgs a)
{
    extern __shared__ float2 sm[];
    const Grid &g = a.g;
    const int M = g.M, ls = M + 1, rows = a.rows, L = 3 * rows;
    float2 *A = sm, *B = sm + (size_t)L * ls;
    const int i2base = blockIdx.x * rows;
    const int pi = blockIdx.y;                 // [0, nin] ; nin = traction
    const bool trac = a.has_trac && pi == a.nin;
    const int i3 = pi;
    const int nthr = blockDim.x;

    for (int t = threadIdx.x; t < L * M; t += nthr) {
        const int line = t / M, n = t % M;
        const int c = line / rows, r = line % rows, i2 = i2base + r;
        float v[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int i1 = 2 * n + h;
            float x;
            if (XIN == XIN_DIV) {
                const size_t rowo = (size_t)i2 * g.sx1;
                if (trac) {
                    const int cz = c == 0 ? 2 : c == 1 ? 4 : 5;
                    x = a.m[cz * g.nh + rowo + i1];
                    if (c == 2 && a.tload) x += a.tload[rowo + i1];
                    x *= a.scale2;
                } else {
                    const int cx = c == 0 ? 0 : c == 1 ? 1 : 2;
                    const int cy = c == 0 ? 1 : c == 1 ? 3 : 4;
                    const int cz = c == 0 ? 2 : c == 1 ? 4 : 5;
                    const size_t pl = (size_t)i3 * g.plane;
                    const float *mx = a.m + cx * g.nh + pl + rowo;
                    const float fx = a.fx.n == 7
                                         ? fir_x1(mx, i1, g.sx1, a.fx)
                                         : (__ldg(mx + (i1 + 1) % g.sx1) - __ldg(mx + (i1 + g.sx1 - 1) % g.sx1)) * a.k1;
                    const float *my = a.m + cy * g.nh + pl + i1;
                    const float fy = a.fy.n == 7
                                         ? fir_y1(my, i2, g.sx2, g.sx1, a.fy)
                                         : (__ldg(my + (size_t)((i2 + 1) % g.sx2) * g.sx1) -
                                            __ldg(my + (size_t)((i2 + g.sx2 - 1) % g.sx2) * g.sx1)) * a.k2;
                    const float *mz = a.m + cz * g.nh + rowo + i1;
                    float fz;
                    if (i3 == 0) fz = (__ldg(mz + g.plane) - __ldg(mz)) * a.k3b;
                    else if (i3 == g.sx3h - 1) fz = (__ldg(mz + pl) - __ldg(mz + pl - g.plane)) * a.k3b;
                    else fz = (__ldg(mz + pl + g.plane) - __ldg(mz + pl - g.plane)) * a.k3;
                    x = -(fx + fy + fz) * a.scale3;
                }
            } else {
                if (trac) {
                    x = a.tin[c][(size_t)i2 * a.trp + i1];
                    if (c == 2 && a.tload) x += a.tload[(size_t)i2 * g.sx1 + i1];
                    x *= a.scale2;
                } else {
                    x = a.in[c][(size_t)i3 * a.pp + (size_t)i2 * a.rp + i1] * a.scale3;
                }
            }
            v[h] = x;
        }
        A[line * ls + n] = make_float2(v[0], v[1]);
    }
    __syncthreads();
    float2 *R = fft_smem<-1>(A, B, a.pm, L, 1, ls);
    // unpack: X[k] = (Z_k + conj Z_{M-k})/2 - i/2 W^k (Z_k - conj Z_{M-k})
    const int p = trac ? g.sx3 : i3;
    for (int t = threadIdx.x; t < L * (M + 1); t += nthr) {
        const int line = t / (M + 1), k = t % (M + 1);
        const int c = line / rows, r = line % rows;
        const float2 zk = R[line * ls + (k == M ? 0 : k)];
        const float2 zm = cconj(R[line * ls + (k == 0 ? 0 : M - k)]);
        const float2 e = cscale(cadd(zk, zm), 0.5f);
        const float2 d = csub(zk, zm);
        const float2 w = __ldg(&a.tw1[k]);
        const float2 wd = cmul(w, d);
        const float2 X = make_float2(e.x + 0.5f * wd.y, e.y - 0.5f * wd.x);
        a.S[sidx(g, c, p, i2base + r, k)] = X;
    }
}


// pass 1, register-resident: -div(m) (or the traction m_i3, or real input
// rows) -> packed real FFT along x1 for rows of M = N1*N2 complex values; RW
// rows of one plane per block, N2 threads per row, components in turn.
// The body force of the block's rows is first built in the row buffers with
// float4 loads (x neighbours by warp shuffle, one wrap-around load per warp
// edge), then each row thread picks its stride-N2 elements from there.
template <int XIN, int N1, int N2, int RW, bool BATCH = false>
__global__ void __launch_bounds__(RW *N2, (RW * N2 <= 128) ? 8 : 4) k_xfwd_reg(const __grid_constant__ XfArgs a0)
{
    pdl_enter();
    const XfArgs &a = BATCH ? a0.tab[blockIdx.z] : a0;
    constexpr int M = N1 * N2, Q = N1 / N2, N2P = N2 + 1, NT = RW * N2;
    constexpr int RS0 = (N1 * N2P > M + 1 ? N1 * N2P : M + 1);
    constexpr int RS = RS0 + ((8 - RS0 % 16) + 16) % 16;
    constexpr int SX1 = 2 * M, R4 = SX1 / 4, ITS = RW * R4 / NT;
    static_assert(N1 % N2 == 0, "N1 must be a multiple of N2");
    static_assert(NT % 32 == 0 && (RW * R4) % NT == 0, "rows split evenly over the block");
    // x neighbours by shuffle when every warp stages part of one row
    constexpr bool SHFL = R4 % 32 == 0;
    static_assert(RS % 2 == 0, "row buffers start on 16 bytes");
    extern __shared__ float2 smx[];
    const Grid &g = a.g;
    const int t = threadIdx.x % N2, r = threadIdx.x / N2, lane = threadIdx.x & 31;
    const int i2 = blockIdx.x * RW + r, pi = blockIdx.y;
    const bool trac = a.has_trac && pi == a.nin;
    const int i3 = pi;
    float2 *T = smx + r * RS;
    const size_t rowo = (size_t)i2 * g.sx1;
#pragma unroll 1
    for (int c = 0; c < 3; c++) {
        float2 z[N1];
        if (XIN == XIN_DIV && !trac) {
            const int cx = c == 0 ? 0 : c == 1 ? 1 : 2;
            const int cy = c == 0 ? 1 : c == 1 ? 3 : 4;
            const int cz = c == 0 ? 2 : c == 1 ? 4 : 5;
            const size_t pl = (size_t)i3 * g.plane;
            size_t zp, zm;
            float kz;
            if (i3 == 0) { zp = g.plane; zm = 0; kz = a.k3b; }
            else if (i3 == g.sx3h - 1) { zp = pl; zm = pl - g.plane; kz = a.k3b; }
            else { zp = pl + g.plane; zm = pl - g.plane; kz = a.k3; }
#pragma unroll 4
            for (int it = 0; it < ITS; it++) {
                const int q = threadIdx.x + NT * it, rr = q / R4, x = 4 * (q % R4);
                const int row = blockIdx.x * RW + rr;
                const float *mx = a.m + cx * g.nh + pl + (size_t)row * SX1;
                const float4 xc = __ldg(reinterpret_cast<const float4 *>(mx + x));
                float xl, xr;
                if (SHFL) {
                    xl = __shfl_up_sync(0xffffffffu, xc.w, 1);
                    xr = __shfl_down_sync(0xffffffffu, xc.x, 1);
                    if (lane == 0) xl = __ldg(mx + (x + SX1 - 1) % SX1);
                    if (lane == 31) xr = __ldg(mx + (x + 4) % SX1);
                } else {
                    xl = __ldg(mx + (x + SX1 - 1) % SX1);
                    xr = __ldg(mx + (x + 4) % SX1);
                }
                const float *my = a.m + cy * g.nh + pl + x;
                const float4 yp = __ldg(reinterpret_cast<const float4 *>(my + (size_t)((row + 1) % g.sx2) * SX1));
                const float4 ym =
                    __ldg(reinterpret_cast<const float4 *>(my + (size_t)((row + g.sx2 - 1) % g.sx2) * SX1));
                const float *mz = a.m + cz * g.nh + (size_t)row * SX1 + x;
                const float4 zpv = __ldg(reinterpret_cast<const float4 *>(mz + zp));
                const float4 zmv = __ldg(reinterpret_cast<const float4 *>(mz + zm));
                float4 f;
                f.x = -((xc.y - xl) * a.k1 + (yp.x - ym.x) * a.k2 + (zpv.x - zmv.x) * kz) * a.scale3;
                f.y = -((xc.z - xc.x) * a.k1 + (yp.y - ym.y) * a.k2 + (zpv.y - zmv.y) * kz) * a.scale3;
                f.z = -((xc.w - xc.y) * a.k1 + (yp.z - ym.z) * a.k2 + (zpv.z - zmv.z) * kz) * a.scale3;
                f.w = -((xr - xc.z) * a.k1 + (yp.w - ym.w) * a.k2 + (zpv.w - zmv.w) * kz) * a.scale3;
                *reinterpret_cast<float4 *>(reinterpret_cast<float *>(smx + rr * RS) + x) = f;
            }
            __syncthreads();
#pragma unroll
            for (int j1 = 0; j1 < N1; j1++) z[j1] = T[N2 * j1 + t];
            __syncthreads();
        } else if (XIN == XIN_DIV) {
            const int cz = c == 0 ? 2 : c == 1 ? 4 : 5;
            {
                const float *mt = a.m + cz * g.nh + rowo;
#pragma unroll
                for (int j1 = 0; j1 < N1; j1++) {
                    const int i1 = 2 * (N2 * j1 + t);
                    float2 v = *reinterpret_cast<const float2 *>(mt + i1);
                    if (c == 2 && a.tload) {
                        const float2 l = *reinterpret_cast<const float2 *>(a.tload + rowo + i1);
                        v.x += l.x; v.y += l.y;
                    }
                    z[j1] = make_float2(v.x * a.scale2, v.y * a.scale2);
                }
            }
        } else {
#pragma unroll
            for (int j1 = 0; j1 < N1; j1++) {
                const int i1 = 2 * (N2 * j1 + t);
                float2 v;
                if (trac) {
                    v = make_float2(a.tin[c][(size_t)i2 * a.trp + i1], a.tin[c][(size_t)i2 * a.trp + i1 + 1]);
                    if (c == 2 && a.tload) { v.x += a.tload[rowo + i1]; v.y += a.tload[rowo + i1 + 1]; }
                    v.x *= a.scale2; v.y *= a.scale2;
                } else {
                    const float *src = a.in[c] + (size_t)i3 * a.pp + (size_t)i2 * a.rp + i1;
                    v = make_float2(src[0] * a.scale3, src[1] * a.scale3);
                }
                z[j1] = v;
            }
        }
        // complex FFT of length M of the packed row
        RDft<N1, -1>::run(z);
#pragma unroll
        for (int k1 = 1; k1 < N1; k1++)
            if (t) z[k1] = cmul(z[k1], twn<-1>(a.pm.tw, t * k1));
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) T[k1 * N2P + t] = z[k1];
        __syncthreads();
        float2 y[Q][N2];
#pragma unroll
        for (int q = 0; q < Q; q++) {
#pragma unroll
            for (int jj = 0; jj < N2; jj++) y[q][jj] = T[(t + N2 * q) * N2P + jj];
            RDft<N2, -1>::run(y[q]);
        }
        __syncthreads();
        // natural order Z[k1 + N1 k2] into the row buffer for the unpacking
#pragma unroll
        for (int q = 0; q < Q; q++)
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) T[(t + N2 * q) + N1 * k2] = y[q][k2];
        __syncthreads();
        const int p = trac ? g.sx3 : i3;
        float2 *dst = a.S + sidx(g, c, p, i2, 0);
        for (int k = t; k <= M; k += N2) {
            const float2 zk = T[k == M ? 0 : k];
            const float2 zm = cconj(T[k == 0 ? 0 : M - k]);
            const float2 e = cscale(cadd(zk, zm), 0.5f);
            const float2 d = csub(zk, zm);
            const float2 w = __ldg(&a.tw1[k]);
            const float2 wd = cmul(w, d);
            dst[k] = make_float2(e.x + 0.5f * wd.y, e.y - 0.5f * wd.x);
        }
        __syncthreads();
    }
}


// pass 2 / 4: complex transform along x2 for a tile of x1 wavenumbers
struct YArgs {
    Grid g;
    float2 *S;
    FftPlan py;
    int tw;            // tile width (k1 columns)
    int nbody;         // body planes [0, nbody)
    int traction;      // also the traction plane (index nbody of blockIdx.y)
    const struct YArgs *tab;   // batched launch: one entry per member (blockIdx.y)
};

template <int SIGN>
__global__ void __launch_bounds__(RELAX_NTHREADS) k_ypass(YArgs a)
{
    extern __shared__ float2 sm[];
    const Grid &g = a.g;
    const int TW = a.tw, n = g.sx2;
    const int k1t = blockIdx.x * TW, ncol = min(TW, g.K1 - k1t);
    const int p = (a.traction && (int)blockIdx.y == a.nbody) ? g.sx3 : (int)blockIdx.y;
    const int c = blockIdx.z;
    float2 *A = sm, *B = sm + (size_t)n * TW;
    const size_t base = sidx(g, c, p, 0, k1t);
    for (int t = threadIdx.x; t < n * TW; t += blockDim.x) {
        const int i2 = t / TW, col = t % TW;
        A[t] = col < ncol ? a.S[base + (size_t)i2 * g.K1 + col] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2 *R = fft_smem<SIGN>(A, B, a.py, TW, TW, 1);
    for (int t = threadIdx.x; t < n * TW; t += blockDim.x) {
        const int i2 = t / TW, col = t % TW;
        if (col < ncol) a.S[base + (size_t)i2 * g.K1 + col] = R[t];
    }
}

// ------------------------------------------------------------------------
// pass 3: the Fourier-domain Green's function on whole x3 columns.
// For a tile of x1 wavenumbers at one k2, all three components:
//   forward transform along x3 (input planes [0, nin), zero below),
//   elasticresponse (src/green.f90:51-101),
//   surfacetractioncowling (src/green.f90:327-377; the k3 sum in FP64,
//   fixed order), p = t - p (src/green.f90:1082-1084),
//   cerrutimodified (src/green.f90:520-612; per-column coefficients FP64),
//   inverse transform along x3, planes [0, nout) written back.
// ------------------------------------------------------------------------
struct ZArgs {
    Grid g;
    float2 *S;
    FftPlan pz;
    int tw, nin, nout;
    float ratio1, ratio2;            // elastic response constants
    double lambda, mu, gam;
    const struct ZArgs *tab;         // batched launch: one entry per member (blockIdx.y)
};

__global__ void __launch_bounds__(RELAX_NTHREADS) k_zspec(ZArgs a)
{
    extern __shared__ float2 sm[];
    const Grid &g = a.g;
    const int TW = a.tw, n = g.sx3, L = 3 * TW;
    const int k1t = blockIdx.x * TW, ncol = min(TW, g.K1 - k1t);
    const int k2i = blockIdx.y;
    const int nthr = blockDim.x;
    float2 *A = sm, *B = sm + (size_t)n * L;
    double *red = reinterpret_cast<double *>(sm + 2 * (size_t)n * L);      // [P][TW][6]
    const int P = nthr / TW;
    float *colc = reinterpret_cast<float *>(red + (size_t)P * TW * 6);     // [TW][10]

    for (int t = threadIdx.x; t < n * L; t += nthr) {
        const int j = t / L, line = t % L, c = line / TW, col = line % TW;
        A[t] = (j < a.nin && col < ncol) ? a.S[sidx(g, c, j, k2i, k1t + col)] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2 *R = fft_smem<-1>(A, B, a.pz, L, L, 1);
    float2 *O = R == A ? B : A;

    const double PI2 = 6.28318530717958623199592693708837032318;
    const double k2v = (k2i < g.sx2 / 2) ? (double)k2i / (g.sx2 * g.dx2) : -(double)(g.sx2 - k2i) / (g.sx2 * g.dx2);
    // elastic response + surface-traction partial sums
    {
        const int col = threadIdx.x % TW, part = threadIdx.x / TW;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        if (part < P) {
            const double k1v = (double)(k1t + col) / (g.sx1 * g.dx1);
            const float k1f = (float)k1v, k2f = (float)k2v;
            const double modulus = a.lambda + 2.0 * a.mu;
            const double alpha = (a.lambda + a.mu) / (a.lambda + 2.0 * a.mu);
            const double grav = 2.0 * a.mu * alpha * a.gam;
            for (int j = part; j < n; j += P) {
                const double k3v = (j < n / 2) ? (double)j / (n * g.dx3) : -(double)(n - j) / (n * g.dx3);
                const float k3f = (float)k3v;
                float2 *p0 = R + (size_t)j * L + col;
                float2 c1 = p0[0], c2 = p0[TW], c3 = p0[2 * TW];
                const float r2 = k1f * k1f + k2f * k2f + k3f * k3f;
                float2 u1, u2, u3;
                if (r2 > 0.f && col < ncol) {
                    const float den = a.ratio1 / (r2 * r2);
                    const float a1 = k2f * k2f + k3f * k3f + a.ratio2 * r2;
                    const float a2 = k1f * k1f + k3f * k3f + a.ratio2 * r2;
                    const float a3 = k1f * k1f + k2f * k2f + a.ratio2 * r2;
                    u1.x = (a1 * c1.x - k1f * (k2f * c2.x + k3f * c3.x)) * den;
                    u1.y = (a1 * c1.y - k1f * (k2f * c2.y + k3f * c3.y)) * den;
                    u2.x = (a2 * c2.x - k2f * (k1f * c1.x + k3f * c3.x)) * den;
                    u2.y = (a2 * c2.y - k2f * (k1f * c1.y + k3f * c3.y)) * den;
                    u3.x = (a3 * c3.x - k3f * (k1f * c1.x + k2f * c2.x)) * den;
                    u3.y = (a3 * c3.y - k3f * (k1f * c1.y + k2f * c2.y)) * den;
                } else {
                    u1 = u2 = u3 = make_float2(0.f, 0.f);
                }
                p0[0] = u1; p0[TW] = u2; p0[2 * TW] = u3;
                // i 2 pi (...) terms, src/green.f90:363-366
                const double a1r = a.mu * (k3v * u1.x + k1v * u3.x), a1i = a.mu * (k3v * u1.y + k1v * u3.y);
                const double a2r = a.mu * (k3v * u2.x + k2v * u3.x), a2i = a.mu * (k3v * u2.y + k2v * u3.y);
                const double a3r = modulus * k3v * u3.x + a.lambda * (k1v * u1.x + k2v * u2.x);
                const double a3i = modulus * k3v * u3.y + a.lambda * (k1v * u1.y + k2v * u2.y);
                acc[0] += -PI2 * a1i; acc[1] += PI2 * a1r;
                acc[2] += -PI2 * a2i; acc[3] += PI2 * a2r;
                acc[4] += -PI2 * a3i - grav * u3.x; acc[5] += PI2 * a3r - grav * u3.y;
            }
            for (int q = 0; q < 6; q++) red[((size_t)part * TW + col) * 6 + q] = acc[q];
        }
    }
    __syncthreads();
    // fixed-order reduction over the parts, then p = t - sum/(sx3 dx3) and
    // the per-column Cerruti coefficients
    if (threadIdx.x < TW) {
        const int col = threadIdx.x;
        double s[6] = {0, 0, 0, 0, 0, 0};
        for (int pp = 0; pp < P; pp++)
            for (int q = 0; q < 6; q++) s[q] += red[((size_t)pp * TW + col) * 6 + q];
        float *cc = colc + col * 12;
        for (int q = 0; q < 12; q++) cc[q] = 0.f;
        const double k1v = (double)(k1t + col) / (g.sx1 * g.dx1);
        if (col < ncol && !(k1v == 0.0 && k2v == 0.0)) {
            const double d = (double)n * g.dx3;
            double p[6];
            for (int c = 0; c < 3; c++) {
                const float2 tc = a.S[sidx(g, c, g.sx3, k2i, k1t + col)];
                p[2 * c] = (double)tc.x - s[2 * c] / d;
                p[2 * c + 1] = (double)tc.y - s[2 * c + 1] / d;
            }
            const double alpha = (a.lambda + a.mu) / (a.lambda + 2.0 * a.mu);
            const double beta = PI2 * sqrt(k1v * k1v + k2v * k2v);
            const double h = a.gam / beta;
            const double c0 = 1.0 / (2.0 * a.mu * beta * beta * beta);
            // b1' = p1 c0, b2' = p2 c0 (b_i = fi b_i'), Q = b1' k1 + b2' k2
            const double b1r = p[0] * c0, b1i = p[1] * c0, b2r = p[2] * c0, b2i = p[3] * c0;
            const double qr = PI2 * k1v * p[0] + PI2 * k2v * p[2], qi = PI2 * k1v * p[1] + PI2 * k2v * p[3];
            const double den = 2.0 * alpha * a.mu * beta * beta * beta * beta * (1 + h);
            const double b3r = (beta * p[4] + (1.0 - alpha) * qi) / den;
            const double b3i = (beta * p[5] - (1.0 - alpha) * qr) / den;
            cc[0] = (float)b1r; cc[1] = (float)b1i; cc[2] = (float)b2r; cc[3] = (float)b2i;
            cc[4] = (float)b3r; cc[5] = (float)b3i;
            cc[6] = (float)(b1r * k1v + b2r * k2v); cc[7] = (float)(b1i * k1v + b2i * k2v);
            cc[8] = (float)beta; cc[9] = (float)k1v; cc[10] = (float)k2v; cc[11] = 1.f;
        }
    }
    __syncthreads();
    // cerrutimodified, applied to every k3
    {
        const float alpha = (float)((a.lambda + a.mu) / (a.lambda + 2.0 * a.mu));
        const float pi2 = 6.28318530717958623f;
        for (int t = threadIdx.x; t < n * TW; t += nthr) {
            const int j = t / TW, col = t % TW;
            const float *cc = colc + col * 12;
            if (cc[11] == 0.f) continue;
            const float beta = cc[8], k1f = cc[9], k2f = cc[10];
            const float k3f = (float)((j < n / 2) ? (double)j / (n * g.dx3) : -(double)(n - j) / (n * g.dx3));
            const float fi = (2.f * beta) / ((pi2 * pi2) * (k3f * k3f) + beta * beta);
            const float gg = pi2 * k3f * fi;
            const float b3r = cc[4], b3i = cc[5];
            // tmp = alpha i beta 2pi b3 (1 - 1/alpha - i g)
            const float er = 1.f - 1.f / alpha, ei = -gg;
            const float gr = b3r * er - b3i * ei, gi = b3r * ei + b3i * er;
            const float ab = alpha * beta * pi2;
            const float tmr = -ab * gi, tmi = ab * gr;
            // v3 = -alpha beta^2 b3 (1/alpha - i g)
            const float hr = 1.f / alpha, hi = -gg, ab2 = -alpha * beta * beta;
            const float v3r = ab2 * (b3r * hr - b3i * hi), v3i = ab2 * (b3r * hi + b3i * hr);
            // S = fi Q ; C = S (1 - i g)
            const float sr = fi * cc[6], si = fi * cc[7];
            const float cr = sr + si * gg, ci = si - sr * gg;
            const float ap = alpha * pi2 * pi2, bb2 = 2.f * beta * beta * fi;
            float2 *p0 = R + (size_t)j * L + col;
            float2 u1 = p0[0], u2 = p0[TW], u3 = p0[2 * TW];
            u1.x += tmr * k1f * fi - bb2 * cc[0] + ap * k1f * cr;
            u1.y += tmi * k1f * fi - bb2 * cc[1] + ap * k1f * ci;
            u2.x += tmr * k2f * fi - bb2 * cc[2] + ap * k2f * cr;
            u2.y += tmi * k2f * fi - bb2 * cc[3] + ap * k2f * ci;
            const float ak = alpha * beta * pi2 * pi2 * k3f * fi;
            u3.x += v3r * fi + ak * sr;
            u3.y += v3i * fi + ak * si;
            p0[0] = u1; p0[TW] = u2; p0[2 * TW] = u3;
        }
    }
    __syncthreads();
    float2 *R2 = fft_smem<+1>(R, O, a.pz, L, L, 1);
    for (int t = threadIdx.x; t < a.nout * L; t += nthr) {
        const int j = t / L, line = t % L, c = line / TW, col = line % TW;
        if (col < ncol) a.S[sidx(g, c, j, k2i, k1t + col)] = R2[t];
    }
}


// ------------------------------------------------------------------------
// Register-resident variants of passes 2-4 (see rfft.cuh): columns of
// length n = N1*N2, CW columns per block, N2 threads per column.
// ------------------------------------------------------------------------

// pass 2 / 4 along x2.  Register budgets as measured fastest: the 128-point
// transform (128 threads a block) takes the registers it asks for (78
// instead of 54-64 on 128 x 128 boxes), the 256-point one 3 blocks of 256
// threads per SM (80 registers instead of 64: forward pass 30.4 -> 27.4 us
// on the 256 x 256 x 128 box), the 512-point one 2 blocks per SM (128
// registers instead of 85: 192 -> 187 us forward, 193 -> 185 us inverse on
// the 512 x 512 x 256 box)
template <int N1, int N2, int CW, int SIGN, bool BATCH = false>
__global__ void __launch_bounds__(CW *N2, (N1 == 16 && N2 == 8) ? 1 : (N1 == 16 && N2 == 16) ? 3 : (N1 == 32) ? 2 : 0) k_ypass_reg(const __grid_constant__ YArgs a0)
{
    pdl_enter();
    const YArgs &a = BATCH ? a0.tab[blockIdx.y] : a0;
    constexpr int n = N1 * N2, Q = N1 / N2;
    static_assert(N1 % N2 == 0, "N1 must be a multiple of N2");
    extern __shared__ float2 smy[];
    const Grid &g = a.g;
    const int c = threadIdx.x % CW, t = threadIdx.x / CW;
    // columns (component, plane, k1) flattened: f = (cp np + pi) K1 + k1
    const int np = a.nbody + a.traction;
    const int f = blockIdx.x * CW + c;
    const bool ok = f < 3 * np * g.K1;
    const int cp = ok ? f / (np * g.K1) : 0, rem = ok ? f % (np * g.K1) : 0;
    const int pi = rem / g.K1, k1c = rem % g.K1;
    const int p = (a.traction && pi == a.nbody) ? g.sx3 : pi;
    const size_t base = sidx(g, cp, p, 0, k1c);
    float2 x[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++)
        x[j1] = ok ? a.S[base + (size_t)(N2 * j1 + t) * g.K1] : make_float2(0.f, 0.f);
    RDft<N1, SIGN>::run(x);
#pragma unroll
    for (int k1 = 1; k1 < N1; k1++)
        if (t) x[k1] = cmul(x[k1], twn<SIGN>(a.py.tw, t * k1));
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) smy[(k1 * N2 + t) * CW + c] = x[k1];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; q++) {
        float2 y[N2];
        const int k1 = t + N2 * q;
#pragma unroll
        for (int jj = 0; jj < N2; jj++) y[jj] = smy[(k1 * N2 + jj) * CW + c];
        RDft<N2, SIGN>::run(y);
        if (ok) {
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) a.S[base + (size_t)(k1 + N1 * k2) * g.K1] = y[k2];
        }
    }
    (void)n;
}

// pass 3, register/shared-memory version.  The three components of CW
// columns stay in shared memory (U[cp][k1][j2][c]) between the phases, so a
// thread holds one N1 or 3 x N2 group at a time.  PRUNED: input planes
// [n/2, n) are zero and only output planes [0, n/2) are wanted (the step's
// Green's functions); otherwise nin/nout are honoured.
constexpr int ZCOL = 26;   // floats of per-column constants in k_zspec_sm

template <int N1, int N2, int CW, bool PRUNED, bool BATCH = false>
__global__ void __launch_bounds__(CW *N2, (CW * N2 >= 256) ? 2 : 4) k_zspec_sm(const __grid_constant__ ZArgs a0)
{
    pdl_enter();
    const ZArgs &a = BATCH ? a0.tab[blockIdx.y] : a0;
    constexpr int n = N1 * N2, Q = N1 / N2;
    static_assert(N1 % N2 == 0, "N1 must be a multiple of N2");
    extern __shared__ float2 smz[];
    float2 *U = smz;                                                   // [3][N1][N2][CW]
    float *red = reinterpret_cast<float *>(smz + 3 * n * CW);          // [N2][12][CW]
    // per column, ZCOL floats: the Cerruti coefficients cc[14], the surface
    // traction (6 floats), then beta, c0, 1/den as doubles (float offset 20)
    float *colc = red + N2 * 12 * CW;                                  // [CW][ZCOL]
    const Grid &g = a.g;
    const int c = threadIdx.x % CW, t = threadIdx.x / CW;
    // columns (k1, k2) flattened over the plane: col = k2 K1 + k1
    const int col = blockIdx.x * CW + c;
    const bool ok = col < g.sx2 * g.K1;
    const int k2i = ok ? col / g.K1 : 0, k1c = ok ? col % g.K1 : 0;
    const double PI2 = 6.28318530717958623199592693708837032318;
    const double inv_l3 = 1.0 / (n * g.dx3);
    auto uidx = [&](int cp, int k1, int j) { return ((cp * N1 + k1) * N2 + j) * CW + c; };

    // forward stage A: all loads first, then the three transforms
    constexpr int NL = PRUNED ? N1 / 2 : N1;
    float2 x[3][NL];
#pragma unroll
    for (int cp = 0; cp < 3; cp++)
#pragma unroll
        for (int j1 = 0; j1 < NL; j1++) {
            const int i3 = N2 * j1 + t;
            const bool ld = ok && (PRUNED || i3 < a.nin);
            x[cp][j1] = ld ? a.S[sidx(g, cp, i3, k2i, k1c)] : make_float2(0.f, 0.f);
        }
    // while those loads are in flight, one thread per column reads the
    // surface traction and forms the column's data-independent FP64
    // constants of cerrutisolmodified (src/green.f90:578-609): beta =
    // 2 pi |k|, c0 = 1/(2 mu beta^3), 1/den = 1/(2 alpha mu beta^4 (1 + gam/beta))
    if (t == N2 - 1) {
        float *cc = colc + c * ZCOL;
        if (ok) {
#pragma unroll
            for (int cp = 0; cp < 3; cp++) {
                const float2 tc = a.S[sidx(g, cp, g.sx3, k2i, k1c)];
                cc[14 + 2 * cp] = tc.x;
                cc[15 + 2 * cp] = tc.y;
            }
        }
        double *cd = reinterpret_cast<double *>(cc + 20);
        const double k1d = (double)k1c / (g.sx1 * g.dx1);
        const double k2d = (k2i < g.sx2 / 2) ? (double)k2i / (g.sx2 * g.dx2) : -(double)(g.sx2 - k2i) / (g.sx2 * g.dx2);
        if (ok && !(k1d == 0.0 && k2d == 0.0)) {
            const double alpha = (a.lambda + a.mu) / (a.lambda + 2.0 * a.mu);
            const double beta = PI2 * sqrt(k1d * k1d + k2d * k2d);
            const double h = a.gam / beta;
            cd[0] = beta;
            cd[1] = 1.0 / (2.0 * a.mu * beta * beta * beta);
            cd[2] = 1.0 / (2.0 * alpha * a.mu * beta * beta * beta * beta * (1 + h));
        }
    }
    {
        float2 tw[N1];   // W_n^(t k1), shared by the three components
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) tw[k1] = twn<-1>(a.pz.tw, t * k1);
#pragma unroll
        for (int cp = 0; cp < 3; cp++) {
            float2 z[N1];
#pragma unroll
            for (int j1 = 0; j1 < N1; j1++) z[j1] = j1 < NL ? x[cp][j1] : make_float2(0.f, 0.f);
            RDft<N1, -1>::run(z);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) U[uidx(cp, k1, t)] = k1 ? cmul(z[k1], tw[k1]) : z[k1];
        }
    }
    __syncthreads();

    // stage B, elastic response, surface-traction moments
    const double k1v = (double)k1c / (g.sx1 * g.dx1);
    const double k2v = (k2i < g.sx2 / 2) ? (double)k2i / (g.sx2 * g.dx2) : -(double)(g.sx2 - k2i) / (g.sx2 * g.dx2);
    const float k1f = (float)k1v, k2f = (float)k2v;
    const double alpha = (a.lambda + a.mu) / (a.lambda + 2.0 * a.mu);
    // elasticresponse as u = A c - B k (k.c) with A = ratio1 (1 + ratio2) / r2,
    // B = ratio1 / r2^2 (src/green.f90:78-90 rearranged); surface traction
    // from the FP64 sums Sk_i = sum k3 u_i and S_i = sum u_i over k3
    const float ra = a.ratio1 * (1.f + a.ratio2);
    const float il3f = (float)inv_l3;   // k3 = jw / (n dx3)
    // FP32 partial sums of jw u_i (k3 = jw / (n dx3)) and of u_i over this
    // thread's k3; the reference accumulates these in REAL*4 over all k3
    // (src/green.f90:365-367)
    float acc[12] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < Q; q++) {
        const int k1 = t + N2 * q;
        // SEQ (N2 >= 16): one component's DFT at a time, back to the
        // thread's own slots of U, so that 3 N2 values never sit in
        // registers together; otherwise the three stay in registers
        constexpr bool SEQ = N2 >= 16;
        float2 y[SEQ ? 1 : 3][N2];
#pragma unroll
        for (int cp = 0; cp < 3; cp++) {
            float2 *v = y[SEQ ? 0 : cp];
#pragma unroll
            for (int jj = 0; jj < N2; jj++) v[jj] = U[uidx(cp, k1, jj)];
            RDft<N2, -1>::run(v);
            if (SEQ) {
#pragma unroll
                for (int jj = 0; jj < N2; jj++) U[uidx(cp, k1, jj)] = v[jj];
            }
        }
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) {
            const int j = k1 + N1 * k2;
            const int jw = j < n / 2 ? j : j - n;
            const float w = (float)jw;
            const float k3f = w * il3f;
            const float2 c1 = SEQ ? U[uidx(0, k1, k2)] : y[0][k2];
            const float2 c2 = SEQ ? U[uidx(1, k1, k2)] : y[SEQ ? 0 : 1][k2];
            const float2 c3 = SEQ ? U[uidx(2, k1, k2)] : y[SEQ ? 0 : 2][k2];
            const float r2 = k1f * k1f + k2f * k2f + k3f * k3f;
            float2 u1, u2, u3;
            if (r2 > 0.f) {
                const float ir2 = rcp_fast(r2);
                const float A = ra * ir2, B = a.ratio1 * ir2 * ir2;
                const float kcr = k1f * c1.x + k2f * c2.x + k3f * c3.x;
                const float kci = k1f * c1.y + k2f * c2.y + k3f * c3.y;
                u1 = make_float2(A * c1.x - B * k1f * kcr, A * c1.y - B * k1f * kci);
                u2 = make_float2(A * c2.x - B * k2f * kcr, A * c2.y - B * k2f * kci);
                u3 = make_float2(A * c3.x - B * k3f * kcr, A * c3.y - B * k3f * kci);
            } else {
                u1 = u2 = u3 = make_float2(0.f, 0.f);
            }
            U[uidx(0, k1, k2)] = u1;
            U[uidx(1, k1, k2)] = u2;
            U[uidx(2, k1, k2)] = u3;
            acc[0] += w * u1.x; acc[1] += w * u1.y; acc[2] += w * u2.x;
            acc[3] += w * u2.y; acc[4] += w * u3.x; acc[5] += w * u3.y;
            acc[6] += u1.x; acc[7] += u1.y; acc[8] += u2.x; acc[9] += u2.y; acc[10] += u3.x; acc[11] += u3.y;
        }
    }
#pragma unroll
    for (int qq = 0; qq < 12; qq++) red[(t * 12 + qq) * CW + c] = acc[qq];
    __syncthreads();
    if (t == 0) {
        double s[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int tt = 0; tt < N2; tt++)
            for (int qq = 0; qq < 12; qq++) s[qq] += (double)red[(tt * 12 + qq) * CW + c];
        for (int qq = 0; qq < 6; qq++) s[qq] *= inv_l3;
        float *cc = colc + c * ZCOL;
        const double *cd = reinterpret_cast<const double *>(cc + 20);
        float tr[6];
#pragma unroll
        for (int qq = 0; qq < 6; qq++) tr[qq] = cc[14 + qq];
#pragma unroll
        for (int qq = 0; qq < 14; qq++) cc[qq] = 0.f;
        if (ok && !(k1v == 0.0 && k2v == 0.0)) {
            // surfacetractioncowling (src/green.f90:356-366): i 2pi (...) - grav u3
            const double modulus = a.lambda + 2.0 * a.mu;
            const double grav = 2.0 * a.mu * alpha * a.gam;
            const double a1r = a.mu * (s[0] + k1v * s[10]), a1i = a.mu * (s[1] + k1v * s[11]);
            const double a2r = a.mu * (s[2] + k2v * s[10]), a2i = a.mu * (s[3] + k2v * s[11]);
            const double a3r = modulus * s[4] + a.lambda * (k1v * s[6] + k2v * s[8]);
            const double a3i = modulus * s[5] + a.lambda * (k1v * s[7] + k2v * s[9]);
            const double sum[6] = {-PI2 * a1i, PI2 * a1r, -PI2 * a2i, PI2 * a2r,
                                   -PI2 * a3i - grav * s[10], PI2 * a3r - grav * s[11]};
            const double id = inv_l3;   // 1 / (n dx3)
            double p[6];
#pragma unroll
            for (int qq = 0; qq < 6; qq++) p[qq] = (double)tr[qq] - sum[qq] * id;
            // cerrutisolmodified (src/green.f90:578-609) written as
            // u_i += fi (P_i + g R_i), g = 2 pi k3 fi, with per-column P_i, R_i
            const double beta = cd[0], c0 = cd[1], iden = cd[2];
            const double b1r = p[0] * c0, b1i = p[1] * c0, b2r = p[2] * c0, b2i = p[3] * c0;
            const double qr = PI2 * k1v * p[0] + PI2 * k2v * p[2], qi = PI2 * k1v * p[1] + PI2 * k2v * p[3];
            const double b3r = (beta * p[4] + (1.0 - alpha) * qi) * iden;
            const double b3i = (beta * p[5] - (1.0 - alpha) * qr) * iden;
            const double Qr = b1r * k1v + b2r * k2v, Qi = b1i * k1v + b2i * k2v;
            const double ialpha = (a.lambda + 2.0 * a.mu) / (a.lambda + a.mu);   // 1 / alpha
            const double ab = alpha * beta * PI2, er = 1.0 - ialpha, ab2 = -alpha * beta * beta;
            const double ap = alpha * PI2 * PI2, bb = 2.0 * beta * beta;
            // P_1 = i k1 ab er b3 - 2 beta^2 b1' + ap k1 Q ; R_1 = k1 ab b3 - i ap k1 Q
            cc[0] = (float)(-k1v * ab * er * b3i - bb * b1r + ap * k1v * Qr);
            cc[1] = (float)(k1v * ab * er * b3r - bb * b1i + ap * k1v * Qi);
            cc[2] = (float)(k1v * ab * b3r + ap * k1v * Qi);
            cc[3] = (float)(k1v * ab * b3i - ap * k1v * Qr);
            cc[4] = (float)(-k2v * ab * er * b3i - bb * b2r + ap * k2v * Qr);
            cc[5] = (float)(k2v * ab * er * b3r - bb * b2i + ap * k2v * Qi);
            cc[6] = (float)(k2v * ab * b3r + ap * k2v * Qi);
            cc[7] = (float)(k2v * ab * b3i - ap * k2v * Qr);
            // P_3 = ab2 b3 / alpha ; R_3 = -i ab2 b3 + alpha beta 2pi Q
            cc[8] = (float)(ab2 * b3r * ialpha);
            cc[9] = (float)(ab2 * b3i * ialpha);
            cc[10] = (float)(ab2 * b3i + alpha * beta * PI2 * Qr);
            cc[11] = (float)(-ab2 * b3r + alpha * beta * PI2 * Qi);
            cc[12] = (float)beta;
            cc[13] = 1.f;
        }
    }
    __syncthreads();

    // Cerruti correction, inverse stage B, twiddle (in place in U)
    {
        float cc[14];
#pragma unroll
        for (int qq = 0; qq < 14; qq++) cc[qq] = colc[c * ZCOL + qq];
        const bool cerr = cc[13] != 0.f;
        const float pi2 = 6.28318530717958623f;
        const float beta = cc[12], b2 = beta * beta;
        const float il3 = (float)inv_l3;
#pragma unroll
        for (int q = 0; q < Q; q++) {
            const int k1 = t + N2 * q;
            constexpr bool SEQ = N2 >= 16;   // as in stage B
            float2 y[SEQ ? 1 : 3][N2];
            if (!SEQ || cerr) {
#pragma unroll
                for (int k2 = 0; k2 < N2; k2++) {
                    float2 u1 = U[uidx(0, k1, k2)], u2 = U[uidx(1, k1, k2)], u3 = U[uidx(2, k1, k2)];
                    if (cerr) {
                        const int j = k1 + N1 * k2;
                        const float k3f = (float)(j < n / 2 ? j : j - n) * il3;
                        const float fi = (2.f * beta) * rcp_fast((pi2 * pi2) * (k3f * k3f) + b2);
                        const float gg = pi2 * k3f * fi;
                        u1.x += fi * (cc[0] + gg * cc[2]); u1.y += fi * (cc[1] + gg * cc[3]);
                        u2.x += fi * (cc[4] + gg * cc[6]); u2.y += fi * (cc[5] + gg * cc[7]);
                        u3.x += fi * (cc[8] + gg * cc[10]); u3.y += fi * (cc[9] + gg * cc[11]);
                    }
                    if (SEQ) {
                        U[uidx(0, k1, k2)] = u1; U[uidx(1, k1, k2)] = u2; U[uidx(2, k1, k2)] = u3;
                    } else {
                        y[0][k2] = u1; y[SEQ ? 0 : 1][k2] = u2; y[SEQ ? 0 : 2][k2] = u3;
                    }
                }
            }
            float2 tw[N2];   // W_n^(-jj k1), shared by the three components
#pragma unroll
            for (int jj = 0; jj < N2; jj++) tw[jj] = twn<+1>(a.pz.tw, jj * k1);
#pragma unroll
            for (int cp = 0; cp < 3; cp++) {
                float2 *v = y[SEQ ? 0 : cp];
                if (SEQ) {
#pragma unroll
                    for (int jj = 0; jj < N2; jj++) v[jj] = U[uidx(cp, k1, jj)];
                }
                RDft<N2, +1>::run(v);
#pragma unroll
                for (int jj = 0; jj < N2; jj++) U[uidx(cp, k1, jj)] = jj ? cmul(v[jj], tw[jj]) : v[jj];
            }
        }
    }
    __syncthreads();

    // inverse stage A and store
#pragma unroll
    for (int cp = 0; cp < 3; cp++) {
        float2 z[N1];
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) z[k1] = U[uidx(cp, k1, t)];
        RDft<N1, +1>::run(z);
        if (ok) {
#pragma unroll
            for (int j1 = 0; j1 < N1; j1++) {
                const int i3 = N2 * j1 + t;
                if (PRUNED ? j1 < N1 / 2 : i3 < a.nout) a.S[sidx(g, cp, i3, k2i, k1c)] = z[j1];
            }
        }
    }
    (void)x;
}

// pass 5: C2R along x1, scaled by 2/(sx1 dx1 sx2 dx2 sx3 dx3), with the
// field update out = base + coef * w  (fieldadd, src/elastic3d.f90:3774-3812)
struct XiArgs {
    Grid g;
    const float2 *S;
    FftPlan pm;
    const float2 *tw1;
    int rows;
    float *out[3];
    const float *base[3];
    size_t rp, pp;           // pitches of out/base
    const StepState *st;     // coef = cmul * Dt (or cmul when st is null)
    float cmul, scale;
    const struct XiArgs *tab;   // batched launch: one entry per member (blockIdx.z / 3)
    float *vout[3];          // optional copy of the transformed field (the
    int vplanes;             // velocity v) for planes i3 < vplanes, pitches rp/pp
};

__global__ void __launch_bounds__(RELAX_NTHREADS) k_xinv(XiArgs a)
{
    extern __shared__ float2 sm[];
    const Grid &g = a.g;
    const int M = g.M, ls = M + 1, rows = a.rows, L = 3 * rows;
    float2 *A = sm, *B = sm + (size_t)L * ls;
    const int i2base = blockIdx.x * rows, i3 = blockIdx.y;
    const int nthr = blockDim.x;
    for (int t = threadIdx.x; t < L * M; t += nthr) {
        const int line = t / M, k = t % M;
        const int c = line / rows, r = line % rows;
        const size_t base = sidx(g, c, i3, i2base + r, 0);
        float2 xk = a.S[base + k], xm = a.S[base + (M - k)];
        if (k == 0) { xk.y = 0.f; xm.y = 0.f; }
        const float2 e = cscale(cadd(xk, cconj(xm)), 0.5f);
        const float2 d = cscale(csub(xk, cconj(xm)), 0.5f);
        const float2 o = cmul(d, cconj(__ldg(&a.tw1[k])));
        A[line * ls + k] = make_float2(e.x - o.y, e.y + o.x);   // E + i O
    }
    __syncthreads();
    float2 *R = fft_smem<+1>(A, B, a.pm, L, 1, ls);
    const float coef = a.st ? (float)(a.cmul * a.st->Dt) : a.cmul;
    for (int t = threadIdx.x; t < L * M; t += nthr) {
        const int line = t / M, nn = t % M;
        const int c = line / rows, r = line % rows, i2 = i2base + r;
        const float2 z = R[line * ls + nn];
        const size_t o = (size_t)i3 * a.pp + (size_t)i2 * a.rp + 2 * nn;
        float w0 = z.x * a.scale, w1 = z.y * a.scale;
        if (a.vout[c] && i3 < a.vplanes) *reinterpret_cast<float2 *>(a.vout[c] + o) = make_float2(w0, w1);
        if (a.base[c]) {
            w0 = a.base[c][o] + coef * w0;
            w1 = a.base[c][o + 1] + coef * w1;
        }
        *reinterpret_cast<float2 *>(a.out[c] + o) = make_float2(w0, w1);
    }
}


// pass 5, register-resident: C2R along x1 for rows of M = N1*N2 complex
// values, RW rows of one plane and one component per block, N2 threads per
// row, with the field update out = base + coef * w.  Shared-memory rows are
// padded (N2+1 per k1 group, row stride = 8 mod 16 float2) so both transpose
// access patterns are free of bank conflicts.  Register budgets as measured:
// 3 blocks per SM for M = 128 (33.6 -> 32.5 us on the 256 x 256 x 128 box),
// the registers asked for at M = 64.
template <int N1, int N2, int RW, int V, bool BATCH = false>
__global__ void __launch_bounds__(RW *N2, (N1 * N2 == 128) ? 3 : (N1 * N2 == 64) ? 1 : 0) k_xinv_reg(const __grid_constant__ XiArgs a0)
{
    pdl_enter();
    const XiArgs &a = BATCH ? a0.tab[blockIdx.z / 3] : a0;
    // RW rows of one plane and component per block, N2 threads per row.
    // (A) the block's spectrum rows, one contiguous run of RW*K1 values
    //     in S, are staged in shared memory with 16-byte loads;
    // (B) each row thread unpacks its stride-N2 inputs, transforms in
    //     registers and leaves the real row in shared memory;
    // (C) out = base + coef * scale * row with V-wide accesses (V = 4 for
    //     16-byte aligned rows, else 2).
    constexpr int M = N1 * N2, Q = N1 / N2, N2P = N2 + 1, K1 = M + 1, NT = RW * N2, SX1 = 2 * M;
    constexpr int RS0 = (N1 * N2P > K1 ? N1 * N2P : K1), RS = RS0 + ((8 - RS0 % 16) + 16) % 16;
    static_assert(N1 % N2 == 0, "N1 must be a multiple of N2");
    static_assert(RS % 2 == 0 && (RW * K1) % 2 == 0, "float4 staging");
    static_assert(V == 2 || V == 4, "V");
    extern __shared__ float2 smx[];
    const Grid &g = a.g;
    const int t = threadIdx.x % N2, r = threadIdx.x / N2;
    const int i2b = blockIdx.x * RW, i3 = blockIdx.y, c = blockIdx.z % 3;

    // (A) rows i2b .. i2b+RW-1 are contiguous: sidx is linear in i2
    {
        const float4 *src = reinterpret_cast<const float4 *>(a.S + sidx(g, c, i3, i2b, 0));
        constexpr int NF = RW * K1 / 2, ITS = (NF + NT - 1) / NT;
#pragma unroll
        for (int it = 0; it < ITS; it++) {
            const int f = threadIdx.x + NT * it;
            if (f < NF) {
                const float4 v = __ldg(src + f);
                const int e0 = 2 * f, e1 = 2 * f + 1;
                smx[(e0 / K1) * RS + e0 % K1] = make_float2(v.x, v.y);
                smx[(e1 / K1) * RS + e1 % K1] = make_float2(v.z, v.w);
            }
        }
    }
    __syncthreads();
    float2 *T = smx + r * RS;
    float2 x[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) {
        const int k = N2 * j1 + t;
        float2 xk = T[k], xm = T[M - k];
        if (k == 0) { xk.y = 0.f; xm.y = 0.f; }
        const float2 e = cscale(cadd(xk, cconj(xm)), 0.5f);
        const float2 d = cscale(csub(xk, cconj(xm)), 0.5f);
        const float2 o = cmul(d, cconj(__ldg(&a.tw1[k])));
        x[j1] = make_float2(e.x - o.y, e.y + o.x);   // E + i O
    }
    __syncthreads();
    RDft<N1, +1>::run(x);
#pragma unroll
    for (int k1 = 1; k1 < N1; k1++)
        if (t) x[k1] = cmul(x[k1], twn<+1>(a.pm.tw, t * k1));
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) T[k1 * N2P + t] = x[k1];
    __syncthreads();
    float2 y[Q][N2];
#pragma unroll
    for (int q = 0; q < Q; q++) {
        const int k1 = t + N2 * q;
#pragma unroll
        for (int jj = 0; jj < N2; jj++) y[q][jj] = T[k1 * N2P + jj];
        RDft<N2, +1>::run(y[q]);
    }
    __syncthreads();
    // real row in natural order: float2 nn holds x1 = 2 nn, 2 nn + 1
#pragma unroll
    for (int q = 0; q < Q; q++)
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) T[(t + N2 * q) + N1 * k2] = y[q][k2];
    __syncthreads();

    // (C)
    const float coef = a.st ? (float)(a.cmul * a.st->Dt) : a.cmul;
    float *out = a.out[c];
    const float *bs = a.base[c];
    float *vo = i3 < a.vplanes ? a.vout[c] : nullptr;
    constexpr int RV = SX1 / V, ITC = RW * RV / NT;
    static_assert((RW * RV) % NT == 0, "rows split evenly");
#pragma unroll
    for (int it = 0; it < ITC; it++) {
        const int f = threadIdx.x + NT * it, rr = f / RV, x0 = V * (f % RV);
        const size_t o = (size_t)i3 * a.pp + (size_t)(i2b + rr) * a.rp + x0;
        const float *row = reinterpret_cast<const float *>(smx + rr * RS) + x0;
        if (V == 4) {
            const float4 w4 = *reinterpret_cast<const float4 *>(row);
            float w[4] = {w4.x * a.scale, w4.y * a.scale, w4.z * a.scale, w4.w * a.scale};
            if (vo) *reinterpret_cast<float4 *>(vo + o) = make_float4(w[0], w[1], w[2], w[3]);
            if (bs) {
                const float4 b = __ldg(reinterpret_cast<const float4 *>(bs + o));
                w[0] = b.x + coef * w[0]; w[1] = b.y + coef * w[1];
                w[2] = b.z + coef * w[2]; w[3] = b.w + coef * w[3];
            }
            *reinterpret_cast<float4 *>(out + o) = make_float4(w[0], w[1], w[2], w[3]);
        } else {
            const float2 w2 = *reinterpret_cast<const float2 *>(row);
            float w0 = w2.x * a.scale, w1 = w2.y * a.scale;
            if (vo) *reinterpret_cast<float2 *>(vo + o) = make_float2(w0, w1);
            if (bs) {
                const float2 b = *reinterpret_cast<const float2 *>(bs + o);
                w0 = b.x + coef * w0;
                w1 = b.y + coef * w1;
            }
            *reinterpret_cast<float2 *>(out + o) = make_float2(w0, w1);
        }
    }
}

// postseismic displacement, src/relax.f90:839-850: ur += Dt v over the
// planes i3 < nur and inter += Dt v in plane i3s (3 components each; v with
// component stride vstride)
__global__ void k_relax_accum(const float *v, size_t vstride, float *ur, int nur, float *inter, int i3s,
                              size_t plane, const StepState *st)
{
    const float dt = (float)st->Dt;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nu = (size_t)nur * plane;
    if (q < 3 * nu) {
        const size_t c = q / nu, r = q % nu;
        ur[q] += dt * v[c * vstride + r];
    } else if (inter && q - 3 * nu < 3 * plane) {
        const size_t p = q - 3 * nu, c = p / plane, r = p % plane;
        inter[p] += dt * v[c * vstride + (size_t)i3s * plane + r];
    }
}

// ------------------------------------------------------------------------
// time step: reduction of the Maxwell-time minima and integrationstep
// (src/relax.f90:650-677, :1420-1452), one block.
// ------------------------------------------------------------------------
// host-side inputs of one step's time-step choice
struct DtIn {
    double t, dt_override;
    int oi, use_override;
};

__device__ __forceinline__ void dt_body(StepState *st, const DtPolicy &pol, const DtIn &in, const float *tm_part,
                                        int ntm, const float *fr_part, int nfr)
{
    __shared__ float shf[32];
    float m0 = 3.0e38f, m1 = 3.0e38f, m2 = 3.0e38f;
    if (ntm == 0 && threadIdx.x == 0) {
        // minima already reduced by the stress kernel's last block
        m0 = st->tmin[0];
        m1 = st->tmin[1];
    }
    for (int i = threadIdx.x; i < ntm; i += blockDim.x) {
        m0 = fminf(m0, tm_part[i]);
        m1 = fminf(m1, tm_part[ntm + i]);
    }
    for (int i = threadIdx.x; i < nfr; i += blockDim.x) m2 = fminf(m2, fr_part[i]);
    m0 = block_min(m0, shf);
    __syncthreads();
    m1 = block_min(m1, shf);
    __syncthreads();
    m2 = block_min(m2, shf);
    if (threadIdx.x == 0) {
        const double STEP_MAX = 1e7;
        // mechanisms of src/relax.f90:660-664: linear, power law, fault
        // creep, linear and nonlinear transient
        double mw[5];
        const float mf[5] = {m0, m1, m2, ntm == 0 ? st->tmin[2] : 3.0e38f, ntm == 0 ? st->tmin[3] : 3.0e38f};
        for (int k = 0; k < 5; k++) {
            // tm = min(REAL(STEP_MAX), min over cells), src/viscoelastic3d.f90:242-245
            const float v = fminf((float)STEP_MAX, mf[k]);
            mw[k] = pol.mech[k] ? (double)v : STEP_MAX;
            st->maxwell[k] = mw[k];
        }
        double tm = 1.0 / ((double)pol.mech[0] / mw[0] + (double)pol.mech[1] / mw[1] +
                           (double)pol.mech[2] / mw[2] + (double)pol.mech[3] / mw[3] +
                           (double)pol.mech[4] / mw[4]);
        if (tm > STEP_MAX) tm = STEP_MAX;
        if (pol.has_inter && tm == STEP_MAX) tm = pol.interval / 20.0;
        st->tm = tm;
        double Dt = tm / 10.0;
        const double t = in.t;
        st->t = in.t;
        st->oi = in.oi;
        if (0 == pol.skip) {
            if ((t + Dt) >= ((double)in.oi * pol.odt) - Dt * 0.04) Dt = (double)in.oi * pol.odt - t;
        } else {
            Dt = Dt * pol.tscale;
            if (pol.has_next_event)
                if ((t + Dt - pol.next_event_time) >= 0.0) Dt = pol.next_event_time - t;
        }
        if (in.use_override) Dt = in.dt_override;
        // an invalid step is reported by the host; Dt = 0 leaves the state
        // unchanged meanwhile
        const bool ok = Dt > 0.0 && isfinite(Dt);
        st->dt_raw = Dt;
        st->Dt = ok ? Dt : 0.0;
        // t + Dt on the next event: the step ends with the event branch
        // (src/relax.f90:859) instead of the END stress pass
        st->fire = ok && pol.has_next_event && fabs((t + Dt) - pol.next_event_time) < 1e-6;
    }
}

__global__ void k_dt(StepState *st, DtPolicy pol, DtIn in, const float *tm_part, int ntm,
                     const float *fr_part, int nfr)
{
    dt_body(st, pol, in, tm_part, ntm, fr_part, nfr);
}

// the same with the policy and the step's inputs in device memory, written
// by the host before each step (the form a captured step graph launches)
struct DtParams {
    DtPolicy pol;
    DtIn in;
};

__global__ void k_dt_dev(StepState *st, const DtParams *p, const float *fr_part, int nfr)
{
    dt_body(st, p->pol, p->in, nullptr, 0, fr_part, nfr);
}

// one block per member of a batch
struct DtArgs {
    StepState *st;
    DtPolicy pol;
    DtIn in;
    const float *fr_part;
    int nfr;
};

__global__ void k_dt_batch(const DtArgs *tab)
{
    const DtArgs &a = tab[blockIdx.x];
    dt_body(a.st, a.pol, a.in, nullptr, 0, a.fr_part, a.nfr);
}

// fixed-order sums of the amplitude partials -> power, C:E^i of the log
__global__ void k_reduce_amp(StepState *st, const double *amp_part, int n, const double *amp_alt,
                             double dv)
{
    __shared__ double shd[32];
    double a0 = 0.0, a1 = 0.0;
    const double *pp = amp_alt ? amp_alt : amp_part;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a0 += pp[i];
        a1 += amp_part[n + i];
    }
    a0 = block_sum(a0, shd);
    __syncthreads();
    a1 = block_sum(a1, shd);
    if (threadIdx.x == 0) {
        st->power = a0 * dv;
        st->cei = a1 * dv;
    }
}

// ------------------------------------------------------------------------
// coseismic sources (setup): source (src/elastic3d.f90:2064-2252, CPU
// branch), momentdensityshear (:2661-2750).  L = width, W = length as the
// call sites pass them (src/relax.f90:1148-1152, :1191-1196).
// ------------------------------------------------------------------------
struct SrcArgs {
    Grid g;
    double mu, s, x, y, z, L, W, strike, dip, rake, beta;
    double lambda;           // tensile and point sources
    float *f[3];             // body force (3 x nh, physical layers; whole box: 3 x 2 nh)
    float *t[3];             // traction (3 x plane)
    float *tau;              // 6 x nh (momentdensityshear)
};

__global__ void k_source_force(SrcArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = i3 * g.dx3;
    const double cs = cos(a.strike), ss = sin(a.strike), cd = cos(a.dip), sd = sin(a.dip);
    const double cr = cos(a.rake), sr = sin(a.rake), scale = -a.mu * a.s;
    const double Wp = a.W * (1.0 + 2.0 * a.beta) / 2.0, Lp = a.L * (1.0 + 2.0 * a.beta) / 2.0;
    const double mlw = Wp > Lp ? Wp : Lp;
    const double x2r0 = cs * a.x - ss * a.y;
    const double xr = cd * x2r0 - sd * a.z, yr = ss * a.x + cs * a.y, zr = sd * x2r0 + cd * a.z;
    if (fabs(x3 - a.z) > Lp && fabs(x3 + a.z) > Lp) return;
    if (fabs(x1 - a.x) > mlw || fabs(x2 - a.y) > mlw) return;
    const double x2r = cs * x1 - ss * x2;
    const double x1s = cd * x2r - sd * x3, x1i = cd * x2r + sd * x3;
    if (fabs(x1s - xr) > 7.01 * g.dx1 && fabs(x1i - xr) > 7.01 * g.dx1) return;
    const double x2s = ss * x1 + cs * x2;
    const double x3s = sd * x2r + cd * x3, x3i = -sd * x2r + cd * x3;
    double temp1 = d_gauss(x1s - xr, g.dx1), temp2 = d_omega((x2s - yr) / a.W, a.beta);
    double temp3 = d_omega((x3s - zr) / a.L, a.beta);
    const double sourc = scale * d_gaussp(x1s - xr, g.dx1) * temp2 * temp3;
    const double dblcp = scale / a.W * temp1 * d_omegap((x2s - yr) / a.W, a.beta) * temp3;
    const double dipcs = scale / a.L * temp1 * temp2 * d_omegap((x3s - zr) / a.L, a.beta);
    temp1 = d_gauss(x1i - xr, g.dx1);
    temp3 = d_omega((x3i + zr) / a.L, a.beta);
    const double image = scale * d_gaussp(x1i - xr, g.dx1) * temp2 * temp3;
    const double cplei = scale / a.W * temp1 * d_omegap((x2s - yr) / a.W, a.beta) * temp3;
    float &f1 = a.f[0][q], &f2 = a.f[1][q], &f3 = a.f[2][q];
    if (2.01 * 0.01745329251994329547437168059786927 > a.dip) {
        f1 = (float)(f1 + cr * ss * (sourc + image) + cr * cd * cs * (dblcp + cplei));
        f2 = (float)(f2 + cr * cs * (sourc + image) - cr * cd * ss * (dblcp + cplei));
        f3 = (float)(f3 - cr * sd * (dblcp - cplei));
    } else {
        f1 = (float)(f1 + cr * ss * (sourc) + cr * cd * cs * (dblcp));
        f2 = (float)(f2 + cr * cs * (sourc) - cr * cd * ss * (dblcp));
        f3 = (float)(f3 - cr * sd * (dblcp));
    }
    f1 = (float)(f1 + cd * sr * cs * dipcs + sd * sr * cs * sourc);
    f2 = (float)(f2 - cd * sr * ss * dipcs - sd * sr * ss * sourc);
    f3 = (float)(f3 + cd * sr * sourc - sd * sr * dipcs);
}

__global__ void k_source_traction(SrcArgs a)
{
    const Grid &g = a.g;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (int)g.plane) return;
    const int i1 = q % g.sx1, i2 = q / g.sx1;
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = 0.0;
    const double cs = cos(a.strike), ss = sin(a.strike), cd = cos(a.dip), sd = sin(a.dip);
    const double cr = cos(a.rake), sr = sin(a.rake);
    const double Wp = a.W * (1.0 + 2.0 * a.beta) / 2.0, Lp = a.L * (1.0 + 2.0 * a.beta) / 2.0;
    const double mlw = Wp > Lp ? Wp : Lp;
    const double x2r0 = cs * a.x - ss * a.y;
    const double xr = cd * x2r0 - sd * a.z, yr = ss * a.x + cs * a.y, zr = sd * x2r0 + cd * a.z;
    if (fabs(x1 - a.x) > mlw || fabs(x2 - a.y) > mlw) return;
    const double x2r = cs * x1 - ss * x2;
    const double x1s = cd * x2r - sd * x3, x1i = cd * x2r + sd * x3;
    const double w701 = (double)7.01f;   // default-real literal of src/elastic3d.f90:2139
    if (fabs(x1s - xr) > w701 * g.dx1 && fabs(x1i - xr) > w701 * g.dx1) return;
    const double x2s = ss * x1 + cs * x2;
    const double x3s = sd * x2r + cd * x3, x3i = -sd * x2r + cd * x3;
    double temp1 = d_gauss(x1s - xr, g.dx1), temp2 = d_omega((x2s - yr) / a.W, a.beta);
    double temp3 = d_omega((x3s - zr) / a.L, a.beta);
    double sourc = temp1 * temp2 * temp3;
    temp1 = d_gauss(x1i - xr, g.dx1);
    temp3 = d_omega((x3i + zr) / a.L, a.beta);
    sourc = sourc + temp1 * temp2 * temp3;
    const double n[3] = {cd * cs * sourc, -cd * ss * sourc, -sd * sourc};
    const double b[3] = {a.mu * a.s * (ss * cr + cs * sd * sr), a.mu * a.s * (cs * cr - ss * sd * sr),
                         a.mu * a.s * (cd * sr)};
    a.t[0][q] += (float)((n[0] * b[2] + n[2] * b[0]) / 2.0);
    a.t[1][q] += (float)((n[1] * b[2] + n[2] * b[1]) / 2.0);
    a.t[2][q] += (float)(n[2] * b[2]);
}

__global__ void k_moment_shear(SrcArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = i3 * g.dx3;
    const double cs = cos(a.strike), ss = sin(a.strike), cd = cos(a.dip), sd = sin(a.dip);
    const double cr = cos(a.rake), sr = sin(a.rake);
    const double Wp = a.W * (1.0 + 2.0 * a.beta) / 2.0, Lp = a.L * (1.0 + 2.0 * a.beta) / 2.0;
    const double x2r0 = cs * a.x - ss * a.y;
    const double xr = cd * x2r0 - sd * a.z, yr = ss * a.x + cs * a.y, zr = sd * x2r0 + cd * a.z;
    if (fabs(x3 - a.z) > Lp) return;
    if (fabs(x1 - a.x) > Wp || fabs(x2 - a.y) > Wp) return;
    const double x2r = cs * x1 - ss * x2;
    const double x1s = cd * x2r - sd * x3, x1i = cd * x2r + sd * x3;
    const double w701 = (double)7.01f;   // default-real literal of src/elastic3d.f90:2712
    if (fabs(x1s - xr) > w701 * g.dx1 && fabs(x1i - xr) > w701 * g.dx1) return;
    const double x2s = ss * x1 + cs * x2;
    const double x3s = sd * x2r + cd * x3, x3i = -sd * x2r + cd * x3;
    double temp1 = d_gauss(x1s - xr, g.dx1), temp2 = d_omega((x2s - yr) / a.W, a.beta);
    double temp3 = d_omega((x3s - zr) / a.L, a.beta);
    double ap = temp1 * temp2 * temp3;
    temp1 = d_gauss(x1i - xr, g.dx1);
    temp3 = d_omega((x3i + zr) / a.L, a.beta);
    ap = ap + temp1 * temp2 * temp3;
    const double n[3] = {cd * cs * ap, -cd * ss * ap, -sd * ap};
    const double s[3] = {a.s * (ss * cr + cs * sd * sr), a.s * (cs * cr - ss * sd * sr), a.s * (cd * sr)};
    const float rmu = 2.0f * (float)a.mu;
    const float e[6] = {(float)(n[0] * s[0]), (float)((n[0] * s[1] + n[1] * s[0]) / 2.0),
                        (float)((n[0] * s[2] + n[2] * s[0]) / 2.0), (float)(n[1] * s[1]),
                        (float)((n[1] * s[2] + n[2] * s[1]) / 2.0), (float)(n[2] * s[2])};
    for (int c = 0; c < 6; c++) a.tau[c * g.nh + q] += rmu * e[c];
}

// tensilesource (src/elastic3d.f90:2315-2411): equivalent body force of an
// opening crack (a.s = opening) over the whole box, sx3 layers (x3 < 0
// holds the image), f[k] of sx1 sx2 sx3 floats each
__global__ void k_source_tensile(SrcArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 2 * g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = (i3 < g.sx3 / 2 ? i3 : i3 - g.sx3) * g.dx3;
    const double Wp = a.W * (1.0 + 2.0 * a.beta) / 2.0, Lp = a.L * (1.0 + 2.0 * a.beta) / 2.0;
    if (fabs(x3 - a.z) > Lp && fabs(x3 + a.z) > Lp) return;
    if (fabs(x1 - a.x) > Wp || fabs(x2 - a.y) > Wp) return;
    const double cs = cos(a.strike), ss = sin(a.strike), cd = cos(a.dip), sd = sin(a.dip);
    const double x2r0 = cs * a.x - ss * a.y;
    const double xr = cd * x2r0 - sd * a.z, yr = ss * a.x + cs * a.y, zr = sd * x2r0 + cd * a.z;
    const double scale1 = -a.s * (a.lambda + 2.0 * a.mu), scale2 = -a.s * a.lambda;
    const double x2r = cs * x1 - ss * x2;
    const double x1s = cd * x2r - sd * x3, x1i = cd * x2r + sd * x3;
    const double w701 = (double)7.01f;   // default-real literal
    if (fabs(x1s - xr) > w701 * g.dx1 && fabs(x1i - xr) > w701 * g.dx1) return;
    const double x2s = ss * x1 + cs * x2;
    const double x3s = sd * x2r + cd * x3, x3i = -sd * x2r + cd * x3;
    double temp1 = d_gauss(x1s - xr, g.dx1), temp2 = d_omega((x2s - yr) / a.W, a.beta);
    double temp3 = d_omega((x3s - zr) / a.L, a.beta);
    const double sourc = scale1 * d_gaussp(x1s - xr, g.dx1) * temp2 * temp3;
    const double dblcp = scale2 / a.W * temp1 * d_omegap((x2s - yr) / a.W, a.beta) * temp3;
    const double dipcs = scale2 / a.L * temp1 * temp2 * d_omegap((x3s - zr) / a.L, a.beta);
    temp1 = d_gauss(x1i - xr, g.dx1);
    temp3 = d_omega((x3i + zr) / a.L, a.beta);
    const double image = scale1 * d_gaussp(x1i - xr, g.dx1) * temp2 * temp3;
    const double cplei = scale2 / a.W * temp1 * d_omegap((x2s - yr) / a.W, a.beta) * temp3;
    const double dipci = scale2 / a.L * temp1 * temp2 * d_omegap((x3i + zr) / a.L, a.beta);
    a.f[0][q] = (float)(a.f[0][q] + cs * cd * (sourc + image) + ss * (dblcp + cplei) + cs * sd * (dipcs + dipci));
    a.f[1][q] = (float)(a.f[1][q] - ss * cd * (sourc + image) + cs * (dblcp + cplei) - ss * sd * (dipcs + dipci));
    a.f[2][q] = (float)(a.f[2][q] - sd * (sourc - image) + cd * (dipcs - dipci));
}

// mogisource (src/elastic3d.f90:2458-2509): a dilatation point source of
// amplitude a.s and its image over the whole box
__global__ void k_source_mogi(SrcArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 2 * g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = (i3 < g.sx3 / 2 ? i3 : i3 - g.sx3) * g.dx3;
    const double W6 = 6.0 * fmax(g.dx1, fmax(g.dx2, g.dx3));
    if (fabs(x3 - a.z) > W6 && fabs(x3 + a.z) > W6) return;
    if (fabs(x1 - a.x) > W6 || fabs(x2 - a.y) > W6) return;
    const double scale = -(a.lambda + 2.0 * a.mu / 3.0) * a.s;
    const double temp1 = d_gauss(x1 - a.x, g.dx1), temp2 = d_gauss(x2 - a.y, g.dx2);
    double temp3 = d_gauss(x3 - a.z, g.dx3);
    const double source1 = scale * d_gaussp(x1 - a.x, g.dx1) * temp2 * temp3;
    const double source2 = scale * temp1 * d_gaussp(x2 - a.y, g.dx2) * temp3;
    const double source3 = scale * temp1 * temp2 * d_gaussp(x3 - a.z, g.dx3);
    temp3 = d_gauss(x3 + a.z, g.dx3);
    const double image1 = scale * d_gaussp(x1 - a.x, g.dx1) * temp2 * temp3;
    const double image2 = scale * temp1 * d_gaussp(x2 - a.y, g.dx2) * temp3;
    const double image3 = scale * temp1 * temp2 * d_gaussp(x3 + a.z, g.dx3);
    a.f[0][q] = (float)(a.f[0][q] + (source1 + image1));
    a.f[1][q] = (float)(a.f[1][q] + (source2 + image2));
    a.f[2][q] = (float)(a.f[2][q] + (source3 - image3));
}

// momentdensitytensile (src/elastic3d.f90:3137-3215): isotropic Hooke's law
// of the crack's eigenstrain n (x) (opening n), added to a.tau (6 x nh)
__global__ void k_moment_tensile(SrcArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = i3 * g.dx3;
    const double Wp = a.W * (1.0 + 2.0 * a.beta) / 2.0, Lp = a.L * (1.0 + 2.0 * a.beta) / 2.0;
    if (fabs(x3 - a.z) > Lp) return;
    if (fabs(x1 - a.x) > Wp || fabs(x2 - a.y) > Wp) return;
    const double cs = cos(a.strike), ss = sin(a.strike), cd = cos(a.dip), sd = sin(a.dip);
    const double x2r0 = cs * a.x - ss * a.y;
    const double xr = cd * x2r0 - sd * a.z, yr = ss * a.x + cs * a.y, zr = sd * x2r0 + cd * a.z;
    const double x2r = cs * x1 - ss * x2;
    const double x1s = cd * x2r - sd * x3, x1i = cd * x2r + sd * x3;
    const double w701 = (double)7.01f;
    if (fabs(x1s - xr) > w701 * g.dx1 && fabs(x1i - xr) > w701 * g.dx1) return;
    const double x2s = ss * x1 + cs * x2;
    const double x3s = sd * x2r + cd * x3, x3i = -sd * x2r + cd * x3;
    double temp1 = d_gauss(x1s - xr, g.dx1), temp2 = d_omega((x2s - yr) / a.W, a.beta);
    double temp3 = d_omega((x3s - zr) / a.L, a.beta);
    double ap = temp1 * temp2 * temp3;
    temp1 = d_gauss(x1i - xr, g.dx1);
    temp3 = d_omega((x3i + zr) / a.L, a.beta);
    ap = ap + temp1 * temp2 * temp3;
    const double n[3] = {cd * cs * ap, -cd * ss * ap, -sd * ap};
    const double s[3] = {a.s * n[0], a.s * n[1], a.s * n[2]};
    float e[6] = {(float)(n[0] * s[0]), (float)((n[0] * s[1] + n[1] * s[0]) / 2.0),
                  (float)((n[0] * s[2] + n[2] * s[0]) / 2.0), (float)(n[1] * s[1]),
                  (float)((n[1] * s[2] + n[2] * s[1]) / 2.0), (float)(n[2] * s[2])};
    // isotropicstressstrain, src/elastic3d.f90:129-142
    const double epskk = (double)(e[0] + e[3] + e[5]);
    const float mu2 = (float)(2.0 * a.mu);
    for (int c = 0; c < 6; c++) e[c] = mu2 * e[c];
    e[0] = (float)(e[0] + a.lambda * epskk);
    e[3] = (float)(e[3] + a.lambda * epskk);
    e[5] = (float)(e[5] + a.lambda * epskk);
    for (int c = 0; c < 6; c++) a.tau[c * g.nh + q] += e[c];
}

// momentdensitymogi (src/elastic3d.f90:3240-3286): kappa o delta_ij at the
// point source, added to a.tau (6 x nh)
__global__ void k_moment_mogi(SrcArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = i3 * g.dx3;
    const double W6 = 6.0 * fmax(g.dx1, fmax(g.dx2, g.dx3));
    if (fabs(x3 - a.z) > W6) return;
    if (fabs(x1 - a.x) > W6 || fabs(x2 - a.y) > W6) return;
    const double kappa = a.lambda + 2.0 / 3.0 * a.mu;
    const float gm = (float)(kappa * (a.s * d_gauss(x1 - a.x, g.dx1) * d_gauss(x2 - a.y, g.dx2) *
                                      d_gauss(x3 - a.z, g.dx3)));
    a.tau[0 * g.nh + q] += gm;
    a.tau[3 * g.nh + q] += gm;
    a.tau[5 * g.nh + q] += gm;
}

// ------------------------------------------------------------------------
// eigenstrain sources (--with-eigenstrain, --with-curvilinear): body forces
// into a.f (physical layers of the whole-box arrays) and moment densities
// into a.tau (6 x nh)
// ------------------------------------------------------------------------
struct EigArgs {
    Grid g;
    double lambda, mu, beta;
    float e[6];                          // the eigenstrain e11 e12 e13 e22 e23 e33
    // cuboid: centre, L = width, W = length, T = thickness (as dislocations
    // passes them, src/relax.f90:1157-1166), strike, dip (radians)
    double x, y, z, L, W, T, strike, dip;
    float sdy[6][6];                     // s.s, n.s, s.d, n.n, n.d, d.d (momentDensityCuboid)
    // tetrahedron: outward unit normals and centroids of the faces BCD, CDA,
    // DAB, ABC, and the tractions (c : e) n of each face
    double n[4][3], cen[4][3], tr[4][3];
    float *f[3];
    float *tau;
};

__device__ __forceinline__ double d_gaussi(double x, double s) { return (1.0 + erf(x / sqrt(2.0) / s)) / 2.0; }

// cuboidSource, src/elastic3d.f90:1680-1884 (the surface-traction loop there
// stores nothing)
__global__ void k_source_cuboid(EigArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = i3 * g.dx3;
    const double Wp = a.W * (1.0 + 2.0 * a.beta) / 2.0, Lp = a.L * (1.0 + 2.0 * a.beta) / 2.0,
                 Tp = a.T * (1.0 + 2.0 * a.beta) / 2.0;
    const double r2 = (double)1.41421354f * fmax(Wp, fmax(Lp, Tp));   // SQRT(2.) of default kind
    if (fabs(x3 - a.z) > r2 || fabs(x1 - a.x) > r2 || fabs(x2 - a.y) > r2) return;
    const double cs = cos(a.strike), ss = sin(a.strike), cd = cos(a.dip), sd = sin(a.dip);
    const double x2r0 = cs * a.x - ss * a.y;
    const double xr = cd * x2r0 - sd * a.z, yr = ss * a.x + cs * a.y, zr = sd * x2r0 + cd * a.z;
    const double x2r = cs * x1 - ss * x2;
    const double x1s = cd * x2r - sd * x3, x1i = cd * x2r + sd * x3;
    const double x2s = ss * x1 + cs * x2;
    const double x3s = sd * x2r + cd * x3, x3i = -sd * x2r + cd * x3;
    const double T = a.T, W = a.W, L = a.L, b = a.beta;
    double t1 = d_omega((x1s - xr) / T, b);
    const double t2 = d_omega((x2s - yr) / W, b);
    double t3 = d_omega((x3s - zr) / L, b);
    const double sourc = 1.0 / T * d_omegap((x1s - xr) / T, b) * t2 * t3;
    const double dblcp = 1.0 / W * t1 * d_omegap((x2s - yr) / W, b) * t3;
    const double dipcs = 1.0 / L * t1 * t2 * d_omegap((x3s - zr) / L, b);
    t1 = d_omega((x1i - xr) / T, b);
    t3 = d_omega((x3i + zr) / L, b);
    const double image = 1.0 / T * d_omegap((x1i - xr) / T, b) * t2 * t3;
    const double cplei = 1.0 / W * t1 * d_omegap((x2s - yr) / W, b) * t3;
    const double mu = a.mu;
    const double ekk = (double)(a.e[0] + a.e[3] + a.e[5]);
    const double e12 = a.e[1], e13 = a.e[2], e23 = a.e[4];
    const double s11 = a.lambda * ekk + 2.0 * mu * a.e[0], s22 = a.lambda * ekk + 2.0 * mu * a.e[3],
                 s33 = a.lambda * ekk + 2.0 * mu * a.e[5];
    double f1, f2, f3;
    if (2.01 * 0.01745329251994329547437168059786927 > a.dip) {
        // method of images for subvertical sources
        f1 = 2.0 * mu * e12 * ss * (sourc + image) + 2.0 * mu * e12 * cd * cs * (dblcp + cplei) -
             s11 * ss * (dblcp + cplei) - s22 * cd * cs * (sourc + image);
        f2 = 2.0 * mu * e12 * cs * (sourc + image) - 2.0 * mu * e12 * cd * ss * (dblcp + cplei) -
             s11 * cs * (dblcp + cplei) + s22 * cd * ss * (sourc + image);
        f3 = -2.0 * mu * e12 * sd * (dblcp - cplei) + s22 * sd * (sourc - image);
    } else {
        f1 = 2.0 * mu * e12 * ss * sourc + 2.0 * mu * e12 * cd * cs * dblcp - s11 * ss * dblcp - s22 * cd * cs * sourc;
        f2 = 2.0 * mu * e12 * cs * sourc - 2.0 * mu * e12 * cd * ss * dblcp - s11 * cs * dblcp + s22 * cd * ss * sourc;
        f3 = -2.0 * mu * e12 * sd * dblcp + s22 * sd * sourc;
    }
    float *p1 = a.f[0] + q, *p2 = a.f[1] + q, *p3 = a.f[2] + q;
    *p1 = (float)(*p1 + f1);
    *p2 = (float)(*p2 + f2);
    *p3 = (float)(*p3 + f3);
    // vertical shear components
    *p1 = (float)(*p1 + 2.0 * mu * e13 * cd * ss * dipcs + 2.0 * mu * e13 * sd * cs * dblcp -
                  2.0 * mu * e23 * cd * cs * dipcs - 2.0 * mu * e23 * sd * cs * sourc - s33 * sd * dipcs * cs);
    *p2 = (float)(*p2 + 2.0 * mu * e13 * cd * cs * dipcs - 2.0 * mu * e13 * sd * ss * dblcp +
                  2.0 * mu * e23 * cd * ss * dipcs + 2.0 * mu * e23 * sd * ss * sourc + s33 * sd * dipcs * ss);
    *p3 = (float)(*p3 + 2.0 * mu * e13 * cd * dblcp - 2.0 * mu * e23 * cd * sourc - s33 * cd * dipcs);
}

// the signed distances of a point to the four faces (positive inside)
__device__ __forceinline__ void tet_dist(const EigArgs &a, double x1, double x2, double x3, double d[4])
{
#pragma unroll
    for (int f = 0; f < 4; f++)
        d[f] = (a.cen[f][0] - x1) * a.n[f][0] + (a.cen[f][1] - x2) * a.n[f][1] + (a.cen[f][2] - x3) * a.n[f][2];
}

// tetrahedronSource, src/elastic3d.f90:1916-2039: face tractions times a
// Gaussian across the face and error-function steps across the others
__global__ void k_source_tetra(EigArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = i3 * g.dx3;
    double d[4];
    tet_dist(a, x1, x2, x3, d);
    const double lim = 7.0 * g.dx1;
    if (fabs(d[0]) > lim && fabs(d[1]) > lim && fabs(d[2]) > lim && fabs(d[3]) > lim) return;
    double H[4], G[4];
#pragma unroll
    for (int f = 0; f < 4; f++) {
        H[f] = d_gaussi(d[f], g.dx1);
        G[f] = d_gauss(d[f], g.dx1);
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float *p = a.f[k] + q;
        *p = (float)(*p + a.tr[0][k] * G[0] * H[1] * H[2] * H[3] + a.tr[1][k] * H[0] * G[1] * H[2] * H[3] +
                     a.tr[2][k] * H[0] * H[1] * G[2] * H[3] + a.tr[3][k] * H[0] * H[1] * H[2] * G[3]);
    }
}

// tau += trace(E) lambda delta + 2 mu E for an eigenstrain E (FP32 as the
// reference's REAL*4 tensors)
__device__ __forceinline__ void tau_add_eigen(float *tau, size_t nh, size_t q, const float E[6], float lambda,
                                              float rmu)
{
    const float ekk = (float)(double)(E[0] + E[3] + E[5]);
    const float lam[6] = {lambda, 0.f, 0.f, lambda, 0.f, lambda};
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const float t = __fadd_rn(tau[c * nh + q], __fmul_rn(ekk, lam[c]));
        tau[c * nh + q] = __fadd_rn(t, __fmul_rn(rmu, E[c]));
    }
}

// momentDensityCuboid, src/elastic3d.f90:2927-3029 (the image term is not
// used there)
__global__ void k_moment_cuboid(EigArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = i3 * g.dx3;
    const double Wp = a.W * (1.0 + 2.0 * a.beta) / 2.0, Lp = a.L * (1.0 + 2.0 * a.beta) / 2.0,
                 Tp = a.T * (1.0 + 2.0 * a.beta) / 2.0;
    const double r2 = (double)1.41421354f * fmax(Wp, fmax(Lp, Tp));
    if (fabs(x3 - a.z) > r2 || fabs(x1 - a.x) > r2 || fabs(x2 - a.y) > r2) return;
    const double cs = cos(a.strike), ss = sin(a.strike), cd = cos(a.dip), sd = sin(a.dip);
    const double x2r0 = cs * a.x - ss * a.y;
    const double xr = cd * x2r0 - sd * a.z, yr = ss * a.x + cs * a.y, zr = sd * x2r0 + cd * a.z;
    const double x2r = cs * x1 - ss * x2;
    const double x1s = cd * x2r - sd * x3, x2s = ss * x1 + cs * x2, x3s = sd * x2r + cd * x3;
    const float ap = (float)(d_omega((x1s - xr) / a.T, a.beta) * d_omega((x2s - yr) / a.W, a.beta) *
                             d_omega((x3s - zr) / a.L, a.beta));
    float ea[6];
#pragma unroll
    for (int c = 0; c < 6; c++) ea[c] = __fmul_rn(ap, a.e[c]);
    // E = e11 s.s + 2 e12 n.s + 2 e13 s.d + e22 n.n + 2 e23 n.d + e33 d.d
    const float w[6] = {ea[0], __fmul_rn(2.f, ea[1]), __fmul_rn(2.f, ea[2]), ea[3], __fmul_rn(2.f, ea[4]), ea[5]};
    float E[6];
#pragma unroll
    for (int c = 0; c < 6; c++) {
        float v = __fmul_rn(w[0], a.sdy[0][c]);
#pragma unroll
        for (int k = 1; k < 6; k++) v = __fadd_rn(v, __fmul_rn(w[k], a.sdy[k][c]));
        E[c] = v;
    }
    tau_add_eigen(a.tau, g.nh, q, E, (float)a.lambda, __fmul_rn(2.f, (float)a.mu));
}

// momentDensityTetrahedron, src/elastic3d.f90:2788-2873; a point is left
// out when all four signed distances are below 7 dx1, as the source reads
__global__ void k_moment_tetra(EigArgs a)
{
    const Grid &g = a.g;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    const double x1 = (i1 < g.sx1 / 2 ? i1 : i1 - g.sx1) * g.dx1;
    const double x2 = (i2 < g.sx2 / 2 ? i2 : i2 - g.sx2) * g.dx2;
    const double x3 = i3 * g.dx3;
    double d[4];
    tet_dist(a, x1, x2, x3, d);
    const double lim = 7.0 * g.dx1;
    if (d[0] < lim && d[1] < lim && d[2] < lim && d[3] < lim) return;
    const double H = d_gaussi(d[0], g.dx1) * d_gaussi(d[1], g.dx1) * d_gaussi(d[2], g.dx1) * d_gaussi(d[3], g.dx1);
    const float h = (float)H;
    float E[6];
#pragma unroll
    for (int c = 0; c < 6; c++) E[c] = __fmul_rn(h, a.e[c]);
    tau_add_eigen(a.tau, g.nh, q, E, (float)a.lambda, __fmul_rn(2.f, (float)a.mu));
}

// ------------------------------------------------------------------------
// layout conversion between RELAX's arrays and the device layout
// ------------------------------------------------------------------------
// AoS TENSOR (sx1, sx2, sx3h) <-> SoA
__global__ void k_aos_to_soa(const relax_tensor *src, float *dst, size_t n)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const relax_tensor t = src[q];
    dst[q] = t.s11; dst[n + q] = t.s12; dst[2 * n + q] = t.s13;
    dst[3 * n + q] = t.s22; dst[4 * n + q] = t.s23; dst[5 * n + q] = t.s33;
}
__global__ void k_soa_to_aos(const float *src, relax_tensor *dst, size_t n)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    relax_tensor t;
    t.s11 = src[q]; t.s12 = src[n + q]; t.s13 = src[2 * n + q];
    t.s22 = src[3 * n + q]; t.s23 = src[4 * n + q]; t.s33 = src[5 * n + q];
    dst[q] = t;
}
// padded (sx1+2) rows <-> compact rows, nrows rows of sx1
__global__ void k_unpad(const float *src, float *dst, int sx1, size_t nrows)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nrows * sx1) return;
    const size_t r = q / sx1, i = q % sx1;
    dst[q] = src[r * (sx1 + 2) + i];
}
__global__ void k_pad(const float *src, float *dst, int sx1, size_t nrows)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nrows * (sx1 + 2)) return;
    const size_t r = q / (sx1 + 2), i = q % (sx1 + 2);
    dst[q] = i < (size_t)sx1 ? src[r * sx1 + i] : 0.f;
}

// compact rows back into the first sx1 entries of padded rows
__global__ void k_repad(const float *src, float *dst, int sx1, size_t nrows)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nrows * sx1) return;
    const size_t r = q / sx1, i = q % sx1;
    dst[r * (sx1 + 2) + i] = src[q];
}

// standalone equivalentbodyforce (for the operator API): c_i -= div(sig),
// t_i += sig_i3(x3=0) on padded arrays
__global__ void k_bodyforce(Grid g, const float *m, float *c1, float *c2, float *c3, float *t1,
                            float *t2, float *t3, float k1, float k2, float k3, float k3b, Fir7 firx,
                            Fir7 fir)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nh) return;
    const int i1 = (int)(q % g.sx1), i2 = (int)((q / g.sx1) % g.sx2), i3 = (int)(q / g.plane);
    float *cc[3] = {c1, c2, c3}, *tt[3] = {t1, t2, t3};
    const size_t rowo = (size_t)i2 * g.sx1, pl = (size_t)i3 * g.plane;
    const size_t po = ((size_t)i3 * g.sx2 + i2) * (g.sx1 + 2) + i1;
    for (int c = 0; c < 3; c++) {
        const int cx = c == 0 ? 0 : c == 1 ? 1 : 2;
        const int cy = c == 0 ? 1 : c == 1 ? 3 : 4;
        const int cz = c == 0 ? 2 : c == 1 ? 4 : 5;
        const float *mx = m + cx * g.nh + pl + rowo;
        const float fx = firx.n == 7 ? fir_x1(mx, i1, g.sx1, firx)
                                     : (mx[(i1 + 1) % g.sx1] - mx[(i1 + g.sx1 - 1) % g.sx1]) * k1;
        const float *my = m + cy * g.nh + pl + i1;
        const float fy = fir.n == 7 ? fir_y1(my, i2, g.sx2, g.sx1, fir)
                                    : (my[(size_t)((i2 + 1) % g.sx2) * g.sx1] -
                                       my[(size_t)((i2 + g.sx2 - 1) % g.sx2) * g.sx1]) * k2;
        const float *mz = m + cz * g.nh + rowo + i1;
        float fz;
        if (i3 == 0) fz = (mz[g.plane] - mz[0]) * k3b;
        else if (i3 == g.sx3h - 1) fz = (mz[pl] - mz[pl - g.plane]) * k3b;
        else fz = (mz[pl + g.plane] - mz[pl - g.plane]) * k3;
        cc[c][po] = cc[c][po] - (fx + fy + fz);
        if (i3 == 0) tt[c][(size_t)i2 * (g.sx1 + 2) + i1] += m[cz * g.nh + rowo + i1];
    }
}

}  // namespace
}  // namespace relax
