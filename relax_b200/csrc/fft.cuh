// fft.cuh -- batched complex FFT in shared memory (Stockham autosort,
// radix 2/3/4/8), the building block of the 3-D real<->complex transform of
// the Fourier-domain Green's function (the role FFTW/cuFFT play in
// src/fourier.f90:177-201 and src/cugreen.cu:166-206).
//
// A pass of radix R over a line of length n with span p (product of the
// radices already applied) maps, for i in [0, n/R):
//     k = i mod p
//     v_r = in[i + r n/R] * w^(r k n/(p R))          r = 0..R-1
//     V   = DFT_R(v)
//     out[(i - k) R + k + s p] = V_s                   s = 0..R-1
// with w = exp(SIGN 2 pi i / n).  Lines live in shared memory at
// base + line*ls + j*es, all threads of the block cooperate, passes
// ping-pong between two buffers.  Twiddles come from a table of
// exp(-2 pi i j / n), j < n, computed on the host in double precision.
#pragma once

#include <cuda_runtime.h>

namespace relax {

struct FftPlan {
    int n;          // transform length
    int nr;         // number of passes
    int r[12];      // radices, first pass first
    const float2 *tw;  // exp(-2 pi i j / n), j = 0..n-1 (device)
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// SIGN * i * z
template <int SIGN>
__device__ __forceinline__ float2 mul_si(float2 z)
{
    return SIGN < 0 ? make_float2(z.y, -z.x) : make_float2(-z.y, z.x);
}

template <int R, int SIGN> struct Dft;

template <int SIGN> struct Dft<2, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int SIGN> struct Dft<4, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        float2 t2 = cadd(v[1], v[3]), t3 = mul_si<SIGN>(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    }
};

template <int SIGN> struct Dft<8, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        const float h = 0.70710678118654752440f;   // 1/sqrt(2)
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4, SIGN>::run(e);
        Dft<4, SIGN>::run(o);
        // w8^k = exp(SIGN 2 pi i k / 8)
        float2 o1 = make_float2(h * (o[1].x - SIGN * o[1].y), h * (o[1].y + SIGN * o[1].x));
        float2 o2 = mul_si<SIGN>(o[2]);
        float2 o3 = make_float2(h * (-o[3].x - SIGN * o[3].y), h * (-o[3].y + SIGN * o[3].x));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
};

template <int SIGN> struct Dft<3, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        const float s3 = 0.86602540378443864676f;   // sqrt(3)/2
        float2 t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        float2 a = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
        float2 b = cscale(mul_si<SIGN>(d), s3);
        v[0] = cadd(v[0], t);
        v[1] = cadd(a, b);
        v[2] = csub(a, b);
    }
};

template <int R, int SIGN>
__device__ __forceinline__ void fft_pass(const float2 *__restrict__ in, float2 *__restrict__ out,
                                         const FftPlan &P, int p, int nlines, int es, int ls)
{
    const int n = P.n, nr = n / R, ntask = nlines * nr, tstride = n / (p * R);
    const int nthr = blockDim.x * blockDim.y;
    for (int t = threadIdx.x + blockDim.x * threadIdx.y; t < ntask; t += nthr) {
        const int line = t % nlines, i = t / nlines;
        const int k = i % p;
        float2 v[R];
        const float2 *src = in + line * ls;
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = src[(i + r * nr) * es];
        if (k) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                float2 w = __ldg(&P.tw[r * k * tstride]);
                if (SIGN > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        Dft<R, SIGN>::run(v);
        const int j = (i - k) * R + k;
        float2 *dst = out + line * ls;
#pragma unroll
        for (int r = 0; r < R; r++) dst[(j + r * p) * es] = v[r];
    }
}

// Transforms nlines lines held in buffer a; b is scratch of the same size.
// Returns the buffer that holds the result.  The caller must __syncthreads()
// after filling a; this function ends with a __syncthreads().
template <int SIGN>
__device__ float2 *fft_smem(float2 *a, float2 *b, const FftPlan &P, int nlines, int es, int ls)
{
    int p = 1;
    for (int s = 0; s < P.nr; ++s) {
        const int R = P.r[s];
        if (R == 8) fft_pass<8, SIGN>(a, b, P, p, nlines, es, ls);
        else if (R == 4) fft_pass<4, SIGN>(a, b, P, p, nlines, es, ls);
        else if (R == 2) fft_pass<2, SIGN>(a, b, P, p, nlines, es, ls);
        else fft_pass<3, SIGN>(a, b, P, p, nlines, es, ls);
        __syncthreads();
        float2 *t = a;
        a = b;
        b = t;
        p *= R;
    }
    return a;
}

}  // namespace relax
