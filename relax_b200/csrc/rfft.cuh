// rfft.cuh -- register-resident column transforms for the Green's function
// passes.  A length n = N1*N2 transform of a column is split as
//     X[k1 + N1 k2] = sum_j2 W_N2^(j2 k2) [ W_n^(j2 k1) sum_j1 x[N2 j1 + j2] W_N1^(j1 k1) ]
// Stage A: N2 threads per column each hold the N1 values x[N2 j1 + j2] in
// registers and transform them; stage B: after one shared-memory transpose
// each thread holds N1/N2 groups of N2 values and transforms those.  One
// shared-memory round trip per transform instead of one per radix pass.
#pragma once

#include "fft.cuh"

namespace relax {
namespace {

// exp(-2 pi i m / 16), m = 0..15
__constant__ float2 c_w16[16] = {
    {1.000000000e+00f, 0.000000000e+00f}, {9.238795325e-01f, -3.826834324e-01f}, {7.071067812e-01f, -7.071067812e-01f}, {3.826834324e-01f, -9.238795325e-01f},
    {0.000000000e+00f, -1.000000000e+00f}, {-3.826834324e-01f, -9.238795325e-01f}, {-7.071067812e-01f, -7.071067812e-01f}, {-9.238795325e-01f, -3.826834324e-01f},
    {-1.000000000e+00f, 0.000000000e+00f}, {-9.238795325e-01f, 3.826834324e-01f}, {-7.071067812e-01f, 7.071067812e-01f}, {-3.826834324e-01f, 9.238795325e-01f},
    {0.000000000e+00f, 1.000000000e+00f}, {3.826834324e-01f, 9.238795325e-01f}, {7.071067812e-01f, 7.071067812e-01f}, {9.238795325e-01f, 3.826834324e-01f},
};
// exp(-2 pi i m / 32), m = 0..31
__constant__ float2 c_w32[32] = {
    {1.000000000e+00f, 0.000000000e+00f}, {9.807852804e-01f, -1.950903220e-01f}, {9.238795325e-01f, -3.826834324e-01f}, {8.314696123e-01f, -5.555702330e-01f},
    {7.071067812e-01f, -7.071067812e-01f}, {5.555702330e-01f, -8.314696123e-01f}, {3.826834324e-01f, -9.238795325e-01f}, {1.950903220e-01f, -9.807852804e-01f},
    {0.000000000e+00f, -1.000000000e+00f}, {-1.950903220e-01f, -9.807852804e-01f}, {-3.826834324e-01f, -9.238795325e-01f}, {-5.555702330e-01f, -8.314696123e-01f},
    {-7.071067812e-01f, -7.071067812e-01f}, {-8.314696123e-01f, -5.555702330e-01f}, {-9.238795325e-01f, -3.826834324e-01f}, {-9.807852804e-01f, -1.950903220e-01f},
    {-1.000000000e+00f, 0.000000000e+00f}, {-9.807852804e-01f, 1.950903220e-01f}, {-9.238795325e-01f, 3.826834324e-01f}, {-8.314696123e-01f, 5.555702330e-01f},
    {-7.071067812e-01f, 7.071067812e-01f}, {-5.555702330e-01f, 8.314696123e-01f}, {-3.826834324e-01f, 9.238795325e-01f}, {-1.950903220e-01f, 9.807852804e-01f},
    {0.000000000e+00f, 1.000000000e+00f}, {1.950903220e-01f, 9.807852804e-01f}, {3.826834324e-01f, 9.238795325e-01f}, {5.555702330e-01f, 8.314696123e-01f},
    {7.071067812e-01f, 7.071067812e-01f}, {8.314696123e-01f, 5.555702330e-01f}, {9.238795325e-01f, 3.826834324e-01f}, {9.807852804e-01f, 1.950903220e-01f},
};

// exp(-2 pi i m / 24), m = 0..23
__constant__ float2 c_w24[24] = {
    {1.000000000e+00f, 0.000000000e+00f}, {9.659258263e-01f, -2.588190451e-01f}, {8.660254038e-01f, -5.000000000e-01f}, {7.071067812e-01f, -7.071067812e-01f},
    {5.000000000e-01f, -8.660254038e-01f}, {2.588190451e-01f, -9.659258263e-01f}, {0.000000000e+00f, -1.000000000e+00f}, {-2.588190451e-01f, -9.659258263e-01f},
    {-5.000000000e-01f, -8.660254038e-01f}, {-7.071067812e-01f, -7.071067812e-01f}, {-8.660254038e-01f, -5.000000000e-01f}, {-9.659258263e-01f, -2.588190451e-01f},
    {-1.000000000e+00f, 0.000000000e+00f}, {-9.659258263e-01f, 2.588190451e-01f}, {-8.660254038e-01f, 5.000000000e-01f}, {-7.071067812e-01f, 7.071067812e-01f},
    {-5.000000000e-01f, 8.660254038e-01f}, {-2.588190451e-01f, 9.659258263e-01f}, {0.000000000e+00f, 1.000000000e+00f}, {2.588190451e-01f, 9.659258263e-01f},
    {5.000000000e-01f, 8.660254038e-01f}, {7.071067812e-01f, 7.071067812e-01f}, {8.660254038e-01f, 5.000000000e-01f}, {9.659258263e-01f, 2.588190451e-01f},
};

template <int N, int SIGN>
__device__ __forceinline__ float2 wc(int m)
{
    float2 w = N == 16 ? c_w16[m & 15] : N == 24 ? c_w24[m % 24] : c_w32[m & 31];
    if (SIGN > 0) w.y = -w.y;
    return w;
}

// in-register DFT of size R, natural order in and out
template <int R, int SIGN> struct RDft;

template <int SIGN> struct RDft<4, SIGN> {
    __device__ __forceinline__ static void run(float2 *v) { Dft<4, SIGN>::run(v); }
};
template <int SIGN> struct RDft<8, SIGN> {
    __device__ __forceinline__ static void run(float2 *v) { Dft<8, SIGN>::run(v); }
};
// 16 = 4 x 4: n = n1 + 4 n2, k = k2 + 4 k1
template <int SIGN> struct RDft<16, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a[4][4];
#pragma unroll
        for (int n1 = 0; n1 < 4; n1++) {
            float2 t[4] = {v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]};
            Dft<4, SIGN>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++) a[n1][k2] = (n1 && k2) ? cmul(t[k2], wc<16, SIGN>(n1 * k2)) : t[k2];
        }
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) {
            float2 t[4] = {a[0][k2], a[1][k2], a[2][k2], a[3][k2]};
            Dft<4, SIGN>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < 4; k1++) v[k2 + 4 * k1] = t[k1];
        }
    }
};
// 32 = 4 x 8: n = n1 + 4 n2, k = k2 + 8 k1
template <int SIGN> struct RDft<32, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a[4][8];
#pragma unroll
        for (int n1 = 0; n1 < 4; n1++) {
            float2 t[8];
#pragma unroll
            for (int n2 = 0; n2 < 8; n2++) t[n2] = v[n1 + 4 * n2];
            Dft<8, SIGN>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < 8; k2++) a[n1][k2] = (n1 && k2) ? cmul(t[k2], wc<32, SIGN>(n1 * k2)) : t[k2];
        }
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) {
            float2 t[4] = {a[0][k2], a[1][k2], a[2][k2], a[3][k2]};
            Dft<4, SIGN>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < 4; k1++) v[k2 + 8 * k1] = t[k1];
        }
    }
};

// 24 = 3 x 8: n = n1 + 3 n2, k = k2 + 8 k1
template <int SIGN> struct RDft<24, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a[3][8];
#pragma unroll
        for (int n1 = 0; n1 < 3; n1++) {
            float2 t[8];
#pragma unroll
            for (int n2 = 0; n2 < 8; n2++) t[n2] = v[n1 + 3 * n2];
            Dft<8, SIGN>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < 8; k2++) a[n1][k2] = (n1 && k2) ? cmul(t[k2], wc<24, SIGN>(n1 * k2)) : t[k2];
        }
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) {
            float2 t[3] = {a[0][k2], a[1][k2], a[2][k2]};
            Dft<3, SIGN>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < 3; k1++) v[k2 + 8 * k1] = t[k1];
        }
    }
};

// twiddle exp(SIGN 2 pi i m / n) from the table exp(-2 pi i j / n)
template <int SIGN>
__device__ __forceinline__ float2 twn(const float2 *tw, int m)
{
    float2 w = __ldg(&tw[m]);
    if (SIGN > 0) w.y = -w.y;
    return w;
}

}  // namespace
}  // namespace relax
