// zspec_tc.cuh -- pass 3 of the Green's function (greenfunctioncowling,
// src/green.f90:1008-1129: the transform along x3 of fft3, elasticresponse,
// surfacetractioncowling, cerrutimodified and the inverse transform) with
// its DFT sub-transforms on the 5th-generation tensor cores (tcgen05).
//
// Mixed-precision form of k_zspec_sm for a 128-deep FFT box and the step's
// pruned transform (input planes [0, 64) non-zero, output planes [0, 64)
// wanted).  A column of 128 points splits into two interleaved length-64
// DFTs:
//   X[2k + p] = sum_{n<64} (x[n] W128^(p n)) W64^(n k)                 p = 0, 1
//   y[n]      = sum_k Y[2k] W64^(-n k) + W128^(-n) sum_k Y[2k+1] W64^(-n k)
// and the length-64 DFTs of a tile of 64 columns are one matrix product
// D[128 x 128] = A[128 x 128] B^T each:
//   A rows: the (parity p, column) vectors, (Re, Im) interleaved along K;
//   B:      the real 128 x 128 form of the DFT-64 matrix;
// in split precision, A = Ah + Al and B = Bh + Bl with BF16 parts, D =
// Ah Bh + Ah Bl + Al Bh accumulated in FP32 in tensor memory (the dropped
// Al Bl term and the parts' rounding leave a relative error of about 2^-16
// per product).  The inverse uses the transpose of the same B (the forward
// matrix read as an MN-major operand).
//
// One CTA per SM walks the tiles.  Per tile the three components go
// through: forward product (tcgen05.mma, two operand buffers so that
// building one component's operand overlaps the previous product), the
// elastic response and surface-traction sums on the CUDA cores (FP32, the
// response written back into tensor memory), the per-column FP64
// coefficients of the traction solve, the Cerruti correction folded into
// the inverse operand, the inverse product, and the recombination of the
// two parities with the W128^(-n) twiddle on the way out.  Every wait on
// the tensor cores is bounded: on a time-out the kernel raises a flag,
// stops and frees its tensor memory.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace relax {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of an operand in the no-swizzle canonical
// layout: 8 rows x 16 bytes core matrices; lbo / sbo the byte strides of the
// leading / stride dimension blocks; version 1 (sm_100).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> FP32, M x N, A K-major,
// B K-major (b_mn = 0) or MN-major (b_mn = 1).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)b_mn << 16) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

// D (tensor memory) (+)= A (shared) . B (shared); one thread issues it
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

// arrive on an mbarrier once every tcgen05 operation issued so far by this
// thread has completed
__device__ __forceinline__ void commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for the phase `parity` of an mbarrier to complete
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (int it = 0; it < (1 << 22); it++)
        if (mbar_try(bar, parity)) return true;
    return false;
}

// 32 lanes x 32 columns of FP32 from tensor memory (lane = row of the warp's
// quarter, one column per register) and back
__device__ __forceinline__ void tld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tst32(uint32_t taddr, const float (&v)[32])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};"
        :
        : "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
          "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
          "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
          "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
          "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
          "r"(__float_as_uint(v[15])), "r"(__float_as_uint(v[16])), "r"(__float_as_uint(v[17])),
          "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])), "r"(__float_as_uint(v[20])),
          "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])), "r"(__float_as_uint(v[23])),
          "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])), "r"(__float_as_uint(v[26])),
          "r"(__float_as_uint(v[27])), "r"(__float_as_uint(v[28])), "r"(__float_as_uint(v[29])),
          "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31]))
        : "memory");
}

__device__ __forceinline__ void tld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tst_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// byte offset of the 16-byte chunk (K elements [8 kb, 8 kb + 8)) of row r in
// a 128-row operand of K = 128 BF16 elements: core matrices of 8 rows x 16 B,
// row blocks 128 B apart (SBO), K blocks 2048 B apart (LBO)
__device__ __forceinline__ uint32_t opoff(int r, int kb) { return ((uint32_t)(kb * 16 + (r >> 3)) << 7) + ((r & 7) << 4); }

// BF16 hi / lo parts of a complex pair, packed (Re low, Im high)
__device__ __forceinline__ void split2(float re, float im, uint32_t &hi, uint32_t &lo)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(re - hf.x, im - hf.y);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}

}  // namespace tc

struct ZtcArgs {
    ZArgs z;          // grid, spectrum and elastic constants (z.nin = z.nout = 64)
    int ncol;         // sx2 * K1 columns
    int ntiles;       // ceil(ncol / 64)
    int *err;         // raised (1 << RELAX_ERR_CUDA) when a wait on the tensor cores times out
    const uint4 *tab; // k_ztc_tables: the DFT-64 matrix (hi, lo) in operand layout, then W128^n
};

constexpr int ZT_COLS = 64;
constexpr int ZT_THREADS = 256;
constexpr int ZT_TMEM_COLS = 512;                    // three 128-column accumulators
// shared memory map (bytes)
constexpr uint32_t ZT_BH = 0, ZT_BL = 32768;         // DFT-64 matrix, BF16 hi and lo parts
constexpr uint32_t ZT_OP = 65536;                    // operand buffers [2][hi, lo] of 32 KB
constexpr uint32_t ZT_TW = ZT_OP + 4 * 32768;        // W128^n, n < 128 (float2)
constexpr uint32_t ZT_RED = ZT_TW + 128 * 8;         // FP32 partial sums [4 parts][12][64 columns]
constexpr uint32_t ZT_CC = ZT_RED + 4 * 12 * 64 * 4; // per-column coefficients [14][64]
constexpr uint32_t ZT_COLC = ZT_CC + 14 * 64 * 4;   // per-column FP64 constants [12][64]
constexpr uint32_t ZT_BAR = ZT_COLC + 12 * 64 * 8;   // 2 mbarriers, TMEM base
constexpr uint32_t ZT_SMEM = ZT_BAR + 64;
constexpr uint32_t ZT_TAB_BYTES = 65536 + 128 * 8;   // the table k_ztc_tables writes

// The constant operands of k_zspec_tc, computed once per device buffer: the
// BF16 hi / lo parts of the DFT-64 matrix B[nn][kq] (nn = 2k + ro: output k,
// Re / Im; kq = 2n + ri: input n, Re / Im; e^{-i 2 pi n k / 64}) in the
// kernel's shared-memory operand layout, followed by W128^n, n < 128.
__global__ void k_ztc_tables(uint4 *tab)
{
    unsigned char *dst = reinterpret_cast<unsigned char *>(tab);
    const int ch = blockIdx.x * blockDim.x + threadIdx.x;
    if (ch < 128 * 16) {
        const int nn = ch >> 4, kb = ch & 15;
        const int k = nn >> 1, ro = nn & 1;
        uint32_t hv[4], lv[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int n = kb * 4 + e;
            double sn, cs;
            sincospi((double)((n * k) & 63) / 32.0, &sn, &cs);
            const float w0 = ro == 0 ? (float)cs : (float)(-sn), w1 = ro == 0 ? (float)sn : (float)cs;
            tc::split2(w0, w1, hv[e], lv[e]);
        }
        const uint32_t o = tc::opoff(nn, kb);
        *reinterpret_cast<uint4 *>(dst + o) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
        *reinterpret_cast<uint4 *>(dst + 32768 + o) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
    }
    if (ch < 128) {
        double sn, cs;
        sincospi(-(double)ch / 64.0, &sn, &cs);           // W128^n = e^{-2 pi i n / 128}
        reinterpret_cast<float2 *>(dst + 65536)[ch] = make_float2((float)cs, (float)sn);
    }
}

__global__ void __launch_bounds__(ZT_THREADS, 1) k_zspec_tc(const __grid_constant__ ZtcArgs t)
{
    extern __shared__ __align__(1024) unsigned char zsm[];
    const ZArgs &a = t.z;
    const Grid &g = a.g;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = tc::smem_u32(zsm);
    const uint32_t bar[2] = {sbase + ZT_BAR, sbase + ZT_BAR + 8};
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(zsm + ZT_BAR + 16);
    float2 *tw = reinterpret_cast<float2 *>(zsm + ZT_TW);
    float *red = reinterpret_cast<float *>(zsm + ZT_RED);
    float *ccs = reinterpret_cast<float *>(zsm + ZT_CC);
    double *colc = reinterpret_cast<double *>(zsm + ZT_COLC);   // [12][64]

    // ---- set-up: DFT-64 matrix (hi/lo) and twiddles from the table,
    // barriers, tensor memory
    for (int q = tid; q < 4096; q += ZT_THREADS) reinterpret_cast<uint4 *>(zsm + ZT_BH)[q] = t.tab[q];
    if (tid < 64) reinterpret_cast<uint4 *>(zsm + ZT_TW)[tid] = t.tab[4096 + tid];
    if (tid == 0) {
        tc::mbar_init(bar[0], 1);
        tc::mbar_init(bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(sbase + ZT_BAR + 16, ZT_TMEM_COLS);
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tmem_slot;

    const uint32_t idf = tc::idesc_bf16(128, 128, 0), idi = tc::idesc_bf16(128, 128, 1);
    const uint32_t opA[2] = {sbase + ZT_OP, sbase + ZT_OP + 65536};   // hi at +0, lo at +32768
    // per buffer: the parity of its barrier's next phase, and whether a
    // committed product on it has not been waited for (at most one)
    uint32_t ph[2] = {0, 0};
    int pend[2] = {0, 0};
    bool aborted = false;

    // the three split products of one length-64 DFT set; fwd: B K-major,
    // inverse: the transpose of B read MN-major
    auto issue = [&](int buf, int comp, bool fwd) {
        pend[buf] = 1;
        if (tid != 0) return;
        tc::fence_after();
        const uint32_t d = tmem + comp * 128;
        const uint32_t ah = opA[buf], al = opA[buf] + 32768;
        const uint32_t bh = sbase + ZT_BH, bl = sbase + ZT_BL;
#pragma unroll 1
        for (int prod = 0; prod < 3; prod++) {
            const uint32_t aa = prod == 2 ? al : ah, bb = prod == 1 ? bl : bh;
#pragma unroll 1
            for (int s = 0; s < 8; s++) {
                const uint64_t da = tc::sdesc(aa + s * 4096, 2048, 128);
                const uint64_t db = fwd ? tc::sdesc(bb + s * 4096, 2048, 128) : tc::sdesc(bb + s * 256, 128, 2048);
                tc::mma_bf16(d, da, db, fwd ? idf : idi, (prod > 0 || s > 0) ? 1u : 0u);
            }
        }
        tc::commit(bar[buf]);
    };
    // bounded wait on a buffer's barrier; every thread takes the same branch
    auto wait_buf = [&](int buf) -> bool {
        const bool ok = tc::mbar_wait(bar[buf], ph[buf]);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(t.err, 1 << RELAX_ERR_CUDA);
            aborted = true;
            return false;
        }
        ph[buf] ^= 1u;
        pend[buf] = 0;
        tc::fence_after();
        return true;
    };

    const size_t PS = (size_t)g.sx2 * g.K1;                 // plane stride of the spectrum
    const double inv_l3 = 1.0 / (128.0 * g.dx3);
    const float il3 = (float)inv_l3;
    const int lq = warp & 3, hv = warp >> 2;                // TMEM lane quarter, column half
    const int row = 32 * lq + lane, par = row >> 6, rcol = row & 63;
    const uint32_t trow = tmem + ((uint32_t)(32 * lq) << 16);

    // the loader's share of a tile: one column, a quarter of the 64 planes
    const int lcol = tid & 63, zq = tid >> 6;
    float2 x[16];
    auto load_tile = [&](int tl, int comp) {
        const int q0 = tl * ZT_COLS, nq = min(ZT_COLS, t.ncol - q0);
        const float2 *src = a.S + sidx(g, comp, 0, 0, 0) + q0 + lcol;
#pragma unroll
        for (int i = 0; i < 16; i++)
            x[i] = lcol < nq ? src[(size_t)(16 * zq + i) * PS] : make_float2(0.f, 0.f);
    };
    if (blockIdx.x < t.ntiles) load_tile(blockIdx.x, 0);

#pragma unroll 1
    for (int tile = blockIdx.x; tile < t.ntiles && !aborted; tile += gridDim.x) {
        const int p0 = tile * ZT_COLS;
        const int np = min(ZT_COLS, t.ncol - p0);
        auto load = [&](int comp) { load_tile(tile, comp); };

        // the columns' constants of the traction solve, ahead of their sums
        // (src/green.f90:356-366, :578-609): wavenumbers, beta, 1/(2 mu
        // beta^3), 1/(2 alpha mu beta^4 (1 + gamma/beta)), the surface traction
        if (tid < 64) {
            const int c = tid, pc = p0 + c;
            double v[12];
#pragma unroll
            for (int q = 0; q < 12; q++) v[q] = 0.0;
            if (c < np) {
                const int ck2 = pc / g.K1, ck1 = pc % g.K1;
                const double ck1v = (double)ck1 / (g.sx1 * g.dx1);
                const double ck2v = (ck2 < g.sx2 / 2) ? (double)ck2 / (g.sx2 * g.dx2)
                                                      : -(double)(g.sx2 - ck2) / (g.sx2 * g.dx2);
                if (!(ck1v == 0.0 && ck2v == 0.0)) {
                    const double PI2 = 6.28318530717958623199592693708837032318;
                    const double alpha = (a.lambda + a.mu) / (a.lambda + 2.0 * a.mu);
                    const double beta = PI2 * sqrt(ck1v * ck1v + ck2v * ck2v);
                    const double h = a.gam / beta;
                    v[0] = ck1v; v[1] = ck2v; v[2] = beta;
                    v[3] = 1.0 / (2.0 * a.mu * beta * beta * beta);
                    v[4] = 1.0 / (2.0 * alpha * a.mu * beta * beta * beta * beta * (1 + h));
                    for (int cp = 0; cp < 3; cp++) {
                        const float2 tcv = a.S[sidx(g, cp, g.sx3, ck2, ck1)];
                        v[5 + 2 * cp] = tcv.x;
                        v[6 + 2 * cp] = tcv.y;
                    }
                    v[11] = 1.0;
                }
            }
#pragma unroll
            for (int q = 0; q < 12; q++) colc[q * 64 + c] = v[q];
        }

        // ---- forward products of the three components ----------------
        auto build_fwd = [&](int buf) {
            unsigned char *hi = zsm + ZT_OP + buf * 65536, *lo = hi + 32768;
#pragma unroll
            for (int b = 0; b < 4; b++) {
                uint32_t h0[4], l0[4], h1[4], l1[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int i = 4 * b + e, n = 16 * zq + i;
                    tc::split2(x[i].x, x[i].y, h0[e], l0[e]);
                    const float2 w = tw[n];
                    tc::split2(x[i].x * w.x - x[i].y * w.y, x[i].x * w.y + x[i].y * w.x, h1[e], l1[e]);
                }
                const int kb = 4 * zq + b;
                const uint32_t o0 = tc::opoff(lcol, kb), o1 = tc::opoff(64 + lcol, kb);
                *reinterpret_cast<uint4 *>(hi + o0) = make_uint4(h0[0], h0[1], h0[2], h0[3]);
                *reinterpret_cast<uint4 *>(lo + o0) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
                *reinterpret_cast<uint4 *>(hi + o1) = make_uint4(h1[0], h1[1], h1[2], h1[3]);
                *reinterpret_cast<uint4 *>(lo + o1) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
            }
            tc::fence_async_smem();
        };
        build_fwd(0);                                       // comp 0 was loaded ahead
        __syncthreads();
        issue(0, 0, true);
        load(1);
        build_fwd(1);
        __syncthreads();
        issue(1, 1, true);
        load(2);
        if (!wait_buf(0)) break;                            // product 0 has read buffer 0
        build_fwd(0);
        __syncthreads();
        issue(0, 2, true);
        if (!wait_buf(1) || !wait_buf(0)) break;

        // ---- elastic response, surface-traction partial sums ----------
        const int pcol = p0 + rcol;
        const bool colok = rcol < np;
        const int k2i = colok ? pcol / g.K1 : 0, k1c = colok ? pcol % g.K1 : 0;
        const double k1v = (double)k1c / (g.sx1 * g.dx1);
        const double k2v = (k2i < g.sx2 / 2) ? (double)k2i / (g.sx2 * g.dx2)
                                             : -(double)(g.sx2 - k2i) / (g.sx2 * g.dx2);
        {
            const float k1f = (float)k1v, k2f = (float)k2v;
            const float ra = a.ratio1 * (1.f + a.ratio2);
            float acc[12];
#pragma unroll
            for (int q = 0; q < 12; q++) acc[q] = 0.f;
#pragma unroll 1
            for (int q = 0; q < 2; q++) {
                const uint32_t col = 64 * hv + 32 * q;      // columns 2k + ri, k in [32 hv + 16 q, +16)
                float f0[32], f1[32], f2[32];
                tc::tld32(trow + col, f0);
                tc::tld32(trow + 128 + col, f1);
                tc::tld32(trow + 256 + col, f2);
                tc::tld_wait();
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int j = 2 * (32 * hv + 16 * q + i) + par;
                    const int jw = j < 64 ? j : j - 128;
                    const float k3f = (float)((double)jw * inv_l3);
                    const float r2 = k1f * k1f + k2f * k2f + k3f * k3f;
                    const float2 c1 = make_float2(f0[2 * i], f0[2 * i + 1]);
                    const float2 c2 = make_float2(f1[2 * i], f1[2 * i + 1]);
                    const float2 c3 = make_float2(f2[2 * i], f2[2 * i + 1]);
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
                    f0[2 * i] = u1.x; f0[2 * i + 1] = u1.y;
                    f1[2 * i] = u2.x; f1[2 * i + 1] = u2.y;
                    f2[2 * i] = u3.x; f2[2 * i + 1] = u3.y;
                    const float w = (float)jw;
                    acc[0] += w * u1.x; acc[1] += w * u1.y; acc[2] += w * u2.x;
                    acc[3] += w * u2.y; acc[4] += w * u3.x; acc[5] += w * u3.y;
                    acc[6] += u1.x; acc[7] += u1.y; acc[8] += u2.x; acc[9] += u2.y;
                    acc[10] += u3.x; acc[11] += u3.y;
                }
                tc::tst32(trow + col, f0);
                tc::tst32(trow + 128 + col, f1);
                tc::tst32(trow + 256 + col, f2);
            }
            tc::tst_wait();
            const int part = par * 2 + hv;
#pragma unroll
            for (int q = 0; q < 12; q++) red[(part * 12 + q) * 64 + rcol] = acc[q];
        }
        __syncthreads();
        // per-column FP64 combination (fixed order), surface traction, and the
        // Cerruti coefficients of k_zspec_sm (src/green.f90:356-366, :578-609)
        if (tid < 64) {
            const int c = tid;
            float cc[14];
#pragma unroll
            for (int q = 0; q < 14; q++) cc[q] = 0.f;
            {
                const double ck1v = colc[0 * 64 + c], ck2v = colc[1 * 64 + c];
                if (colc[11 * 64 + c] != 0.0) {
                    const double PI2 = 6.28318530717958623199592693708837032318;
                    double s[12];
                    for (int q = 0; q < 12; q++) {
                        s[q] = 0.0;
                        for (int pt = 0; pt < 4; pt++) s[q] += (double)red[(pt * 12 + q) * 64 + c];
                    }
                    for (int q = 0; q < 6; q++) s[q] *= inv_l3;
                    const double alpha = (a.lambda + a.mu) / (a.lambda + 2.0 * a.mu);
                    const double modulus = a.lambda + 2.0 * a.mu;
                    const double grav = 2.0 * a.mu * alpha * a.gam;
                    const double a1r = a.mu * (s[0] + ck1v * s[10]), a1i = a.mu * (s[1] + ck1v * s[11]);
                    const double a2r = a.mu * (s[2] + ck2v * s[10]), a2i = a.mu * (s[3] + ck2v * s[11]);
                    const double a3r = modulus * s[4] + a.lambda * (ck1v * s[6] + ck2v * s[8]);
                    const double a3i = modulus * s[5] + a.lambda * (ck1v * s[7] + ck2v * s[9]);
                    const double sum[6] = {-PI2 * a1i, PI2 * a1r, -PI2 * a2i, PI2 * a2r,
                                           -PI2 * a3i - grav * s[10], PI2 * a3r - grav * s[11]};
                    const double id = 1.0 / (128.0 * g.dx3);
                    double p[6];
                    for (int q = 0; q < 6; q++) p[q] = colc[(5 + q) * 64 + c] - sum[q] * id;
                    const double beta = colc[2 * 64 + c], c0 = colc[3 * 64 + c], iden = colc[4 * 64 + c];
                    const double b1r = p[0] * c0, b1i = p[1] * c0, b2r = p[2] * c0, b2i = p[3] * c0;
                    const double qr = PI2 * ck1v * p[0] + PI2 * ck2v * p[2];
                    const double qi = PI2 * ck1v * p[1] + PI2 * ck2v * p[3];
                    const double b3r = (beta * p[4] + (1.0 - alpha) * qi) * iden;
                    const double b3i = (beta * p[5] - (1.0 - alpha) * qr) * iden;
                    const double Qr = b1r * ck1v + b2r * ck2v, Qi = b1i * ck1v + b2i * ck2v;
                    const double ab = alpha * beta * PI2, er = 1.0 - 1.0 / alpha, ab2 = -alpha * beta * beta;
                    const double ap = alpha * PI2 * PI2, bb = 2.0 * beta * beta;
                    cc[0] = (float)(-ck1v * ab * er * b3i - bb * b1r + ap * ck1v * Qr);
                    cc[1] = (float)(ck1v * ab * er * b3r - bb * b1i + ap * ck1v * Qi);
                    cc[2] = (float)(ck1v * ab * b3r + ap * ck1v * Qi);
                    cc[3] = (float)(ck1v * ab * b3i - ap * ck1v * Qr);
                    cc[4] = (float)(-ck2v * ab * er * b3i - bb * b2r + ap * ck2v * Qr);
                    cc[5] = (float)(ck2v * ab * er * b3r - bb * b2i + ap * ck2v * Qi);
                    cc[6] = (float)(ck2v * ab * b3r + ap * ck2v * Qi);
                    cc[7] = (float)(ck2v * ab * b3i - ap * ck2v * Qr);
                    cc[8] = (float)(ab2 * b3r / alpha);
                    cc[9] = (float)(ab2 * b3i / alpha);
                    cc[10] = (float)(ab2 * b3i + alpha * beta * PI2 * Qr);
                    cc[11] = (float)(-ab2 * b3r + alpha * beta * PI2 * Qi);
                    cc[12] = (float)beta;
                    cc[13] = 1.f;
                }
            }
#pragma unroll
            for (int q = 0; q < 14; q++) ccs[q * 64 + c] = cc[q];
        }
        __syncthreads();

        // ---- inverse operands (response + Cerruti), products, epilogues --
        // the next tile's first component is read while this one finishes
        if (tile + (int)gridDim.x < t.ntiles) load_tile(tile + gridDim.x, 0);
        float cc[14];
#pragma unroll
        for (int q = 0; q < 14; q++) cc[q] = ccs[q * 64 + rcol];
        const bool cerr = cc[13] != 0.f;
        auto build_inv = [&](int buf, int comp) {
            unsigned char *hi = zsm + ZT_OP + buf * 65536, *lo = hi + 32768;
            const float pi2 = 6.28318530717958623f;
            const float beta = cc[12], b2 = beta * beta;
            const float Pr = cc[4 * comp], Pi = cc[4 * comp + 1], Rr = cc[4 * comp + 2], Ri = cc[4 * comp + 3];
#pragma unroll 1
            for (int q = 0; q < 2; q++) {
                float u[32];
                tc::tld32(trow + comp * 128 + 64 * hv + 32 * q, u);
                tc::tld_wait();
                if (cerr) {
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        const int j = 2 * (32 * hv + 16 * q + i) + par;
                        const float k3f = (float)(j < 64 ? j : j - 128) * il3;
                        const float fi = (2.f * beta) * rcp_fast((pi2 * pi2) * (k3f * k3f) + b2);
                        const float gg = pi2 * k3f * fi;
                        u[2 * i] += fi * (Pr + gg * Rr);
                        u[2 * i + 1] += fi * (Pi + gg * Ri);
                    }
                }
#pragma unroll
                for (int b = 0; b < 4; b++) {
                    uint32_t h[4], l[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) tc::split2(u[8 * b + 2 * e], u[8 * b + 2 * e + 1], h[e], l[e]);
                    const uint32_t o = tc::opoff(row, 8 * hv + 4 * q + b);
                    *reinterpret_cast<uint4 *>(hi + o) = make_uint4(h[0], h[1], h[2], h[3]);
                    *reinterpret_cast<uint4 *>(lo + o) = make_uint4(l[0], l[1], l[2], l[3]);
                }
            }
            tc::fence_async_smem();
            tc::fence_before();
        };
        // y[n] = z0[n] + W128^(-n) z1[n]: the parity-0 row keeps n in the lower
        // 16 of its 32, the parity-1 row the upper 16; each hands the other
        // half to its partner through `buf`
        auto epilogue = [&](int buf, int comp) {
            float2 *xch = reinterpret_cast<float2 *>(zsm + ZT_OP + buf * 65536);   // [par][hv][16][64]
            float z[2][32];
            tc::tld32(trow + comp * 128 + 64 * hv, z[0]);
            tc::tld32(trow + comp * 128 + 64 * hv + 32, z[1]);
            tc::tld_wait();
#pragma unroll
            for (int i = 0; i < 16; i++) {
                // parity 0 hands over its upper half, parity 1 its lower half
                float2 v = par == 0 ? make_float2(z[1][2 * i], z[1][2 * i + 1])
                                    : make_float2(z[0][2 * i], z[0][2 * i + 1]);
                if (par == 1) {
                    const float2 w = tw[32 * hv + i];                      // n = 32 hv + i
                    v = make_float2(v.x * w.x + v.y * w.y, v.y * w.x - v.x * w.y);
                }
                xch[((par * 2 + hv) * 16 + i) * 64 + rcol] = v;
            }
            tc::fence_before();
            __syncthreads();
            float2 *dst = a.S + sidx(g, comp, 0, 0, 0) + p0 + rcol;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const float2 o = xch[(((1 - par) * 2 + hv) * 16 + i) * 64 + rcol];
                const int n = 32 * hv + 16 * par + i;
                float2 y;
                if (par == 0) {
                    y = make_float2(z[0][2 * i] + o.x, z[0][2 * i + 1] + o.y);
                } else {
                    const float2 w = tw[n];
                    const float zr = z[1][2 * i], zi = z[1][2 * i + 1];
                    y = make_float2(o.x + zr * w.x + zi * w.y, o.y + zi * w.x - zr * w.y);
                }
                if (colok) dst[(size_t)n * PS] = y;
            }
            __syncthreads();
        };
        build_inv(0, 0);
        __syncthreads();
        issue(0, 0, false);
        build_inv(1, 1);
        __syncthreads();
        issue(1, 1, false);
        if (!wait_buf(0)) break;
        epilogue(0, 0);
        build_inv(0, 2);
        __syncthreads();
        issue(0, 2, false);
        if (!wait_buf(1)) break;
        epilogue(1, 1);
        if (!wait_buf(0)) break;
        epilogue(1, 2);
    }

    // ---- tear-down: no product in flight, tensor memory released ---------
    if (aborted) {
        // a wait timed out: give the products still outstanding one more
        // bounded wait before the tensor memory goes back
        for (int b = 0; b < 2; b++)
            if (pend[b]) tc::mbar_wait(bar[b], ph[b]);
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after();
        tc::tmem_free(tmem, ZT_TMEM_COLS);
    }
}

// The tensor-core DFT-64 of k_zspec_tc on its own, for the operator tests:
// 128 vectors of 64 complex values (in[r][n], FP32 pairs) to their
// forward (sign -1) or inverse (sign +1, unnormalised) DFT, with the same
// operand layout, split products and B matrix (read K-major forward,
// MN-major inverse) as the z pass.  One CTA of 128 threads.
constexpr uint32_t DP_SMEM = 4 * 32768 + 64;

__global__ void __launch_bounds__(128, 1) k_dft64_tc(const float2 *in, float2 *out, int inverse, int *err)
{
    extern __shared__ __align__(1024) unsigned char psm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = tc::smem_u32(psm);
    const uint32_t bar = sbase + 4 * 32768;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(psm + 4 * 32768 + 16);
    for (int ch = tid; ch < 128 * 16; ch += 128) {
        const int nn = ch >> 4, kb = ch & 15;
        const int k = nn >> 1, ro = nn & 1;
        uint32_t hv[4], lv[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int n = kb * 4 + e;
            double s, c;
            sincospi((double)((n * k) & 63) / 32.0, &s, &c);
            const float w0 = ro == 0 ? (float)c : (float)(-s), w1 = ro == 0 ? (float)s : (float)c;
            tc::split2(w0, w1, hv[e], lv[e]);
        }
        const uint32_t o = tc::opoff(nn, kb);
        *reinterpret_cast<uint4 *>(psm + o) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
        *reinterpret_cast<uint4 *>(psm + 32768 + o) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
    }
    // operand: row r = tid, K = 2n + ri
    for (int kb = 0; kb < 16; kb++) {
        uint32_t h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const float2 v = in[tid * 64 + kb * 4 + e];
            tc::split2(v.x, v.y, h[e], l[e]);
        }
        const uint32_t o = tc::opoff(tid, kb);
        *reinterpret_cast<uint4 *>(psm + 65536 + o) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(psm + 98304 + o) = make_uint4(l[0], l[1], l[2], l[3]);
    }
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(sbase + 4 * 32768 + 16, 128);
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tmem_slot;
    const bool fwd = inverse == 0;
    if (tid == 0) {
        const uint32_t id = tc::idesc_bf16(128, 128, fwd ? 0 : 1);
        for (int prod = 0; prod < 3; prod++) {
            const uint32_t aa = sbase + (prod == 2 ? 98304 : 65536), bb = sbase + (prod == 1 ? 32768 : 0);
            for (int s = 0; s < 8; s++) {
                const uint64_t da = tc::sdesc(aa + s * 4096, 2048, 128);
                const uint64_t db = fwd ? tc::sdesc(bb + s * 4096, 2048, 128) : tc::sdesc(bb + s * 256, 128, 2048);
                tc::mma_bf16(tmem, da, db, id, (prod > 0 || s > 0) ? 1u : 0u);
            }
        }
        tc::commit(bar);
    }
    const bool ok = tc::mbar_wait(bar, 0);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicOr(err, 1 << RELAX_ERR_CUDA);
        tc::mbar_wait(bar, 0);
    } else {
        tc::fence_after();
        const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
        for (int q = 0; q < 4; q++) {
            float v[32];
            tc::tld32(trow + 32 * q, v);
            tc::tld_wait();
            for (int i = 0; i < 16; i++) out[(32 * warp + lane) * 64 + 16 * q + i] = make_float2(v[2 * i], v[2 * i + 1]);
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after();
        tc::tmem_free(tmem, 128);
    }
}

}  // namespace relax
