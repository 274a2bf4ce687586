/*
 * relax_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of RELAX's per-time-step relaxation loop (the reference's
 * CPU path: src/relax.f90, src/elastic3d.f90, src/viscoelastic3d.f90,
 * src/friction3d.f90, src/green.f90, src/fourier.f90).  It is the checker
 * for the CUDA library and the timed CPU baseline; nothing in the product
 * links or calls it.
 *
 * Built twice from this file (see oracle/Makefile):
 *   liboracle32.so  ORC_REAL=float  -- the reference's own precision: FP32
 *                   storage, FP64 intermediates wherever the Fortran source
 *                   converts to REAL*8 (the "FP32 parity build");
 *   liboracle64.so  ORC_REAL=double -- every field in FP64 (the "FP64
 *                   oracle" the mixed/plain GPU forms are scored against).
 *
 * Parity pin: the reference cannot be compiled in this environment (no
 * Fortran compiler, no FFTW/netCDF), so this restatement is pinned against
 * the reference's captured run logs examples/tutorials/output2.param
 * (power-law n=3) and output3.param (afterslip), whose per-step Dt, Maxwell
 * times, "power" and "C:E^i" it reproduces to the logs' 3 significant
 * figures (tests/test_oracle_pins.py), and against analytic known answers
 * (FFT vs numpy.fft, Green's function of one Fourier mode, divergence of a
 * constant tensor, linear Maxwell tm = 1/gammadot0).
 *
 * The FFT (third-party FFTW/MKL in the reference) is restated as a
 * mixed-radix Stockham transform in double precision, rounded to ORC_REAL
 * between passes, with FFTW's unnormalised sign convention (forward
 * exp(-2 pi i jk/n)) and RELAX's normalisation (src/fourier.f90:177-201).
 *
 * Array layouts are the reference's: Fortran column-major with i1 fastest;
 * vector fields padded to sx1+2 (src/relax.f90:250-252); tensors are
 * structs of 6 values.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/relax_b200.h"

#ifndef ORC_REAL
#define ORC_REAL float
#endif
typedef ORC_REAL real;

/* F32(x): a REAL*4 rounding the Fortran source performs (CMPLX/REAL of
 * kind 4); identity in the FP64 build. */
#define F32(x) ((real)(x))

typedef struct otensor {
    real s11, s12, s13, s22, s23, s33;
} otensor;

typedef struct otensor_layer {
    real z, dum;
    otensor t;
} otensor_layer;

static const double PI = 3.141592653589793115997963468544185161;
static const double PI2 = 6.28318530717958623199592693708837032318;
static const double DEG2RAD = 0.01745329251994329547437168059786927;

#define ORC_OK 0
#define ORC_ERR_ARG 1
#define ORC_ERR_NOMEM 3
#define ORC_ERR_UNSUPPORTED 4
#define ORC_ERR_FRICTION 6
#define ORC_ERR_POWER 7

#define IDX3(i1, i2, i3, n1, n2) ((size_t)(i1) + (size_t)(n1) * ((size_t)(i2) + (size_t)(n2) * (size_t)(i3)))

/* ------------------------------------------------------------------ */
/* scalar helpers                                                     */
/* ------------------------------------------------------------------ */

/* fix, src/elastic3d.f90:69-80 */
static int orc_fix(double number)
{
    int f = (int)floor(number), c = (int)ceil(number);
    return (number - f) > 0.5 ? c : f;
}

/* my_sinh, src/elastic3d.f90:86-95 */
static double my_sinh(double x)
{
    if (fabs(x) > 11.0) return copysign(1.0, x) * sinh(11.0);
    return sinh(x);
}

/* gauss, src/elastic3d.f90:525-530 */
static double gauss(double x, double sigma)
{
    return exp(-0.5 * (x / sigma) * (x / sigma)) / sqrt(PI2) / sigma;
}

/* gaussp, src/elastic3d.f90:537-542 */
static double gaussp(double x, double sigma)
{
    return -x * exp(-0.5 * (x / sigma) * (x / sigma)) / sqrt(PI2) / (sigma * sigma * sigma);
}

/* omega, src/elastic3d.f90:549-562 */
static double omega(double x, double beta)
{
    double ax = fabs(x);
    if (ax <= (1.0 - 2.0 * beta) / (1.0 - beta) / 2.0) return 1.0;
    if (ax < 1.0 / (1.0 - beta) / 2.0) {
        double c = cos(PI * ((1.0 - beta) * ax - 0.5 + beta) / 2.0 / beta);
        return c * c;
    }
    return 0.0;
}

/* omegap, src/elastic3d.f90:570-581 */
static double omegap(double x, double beta)
{
    double ax = fabs(x);
    if (ax > (1.0 - 2.0 * beta) / (1.0 - beta) / 2.0 && ax < 1.0 / (1.0 - beta) / 2.0)
        return -copysign(1.0, x) * PI * (1.0 - beta) / 2.0 / beta *
               sin(PI * ((1.0 - beta) * ax - 0.5 + beta) / beta);
    return 0.0;
}

/* shiftedcoordinates, src/elastic3d.f90:4027-4048 (1-based indices) */
static void shiftedcoordinates(int i1, int i2, int i3, int sx1, int sx2, int sx3,
                               double dx1, double dx2, double dx3,
                               double *x1, double *x2, double *x3)
{
    *x1 = (i1 <= sx1 / 2) ? (double)(i1 - 1) * dx1 : (double)(i1 - sx1 - 1) * dx1;
    *x2 = (i2 <= sx2 / 2) ? (double)(i2 - 1) * dx2 : (double)(i2 - sx2 - 1) * dx2;
    *x3 = (i3 <= sx3 / 2) ? (double)(i3 - 1) * dx3 : (double)(i3 - sx3 - 1) * dx3;
}

/* ------------------------------------------------------------------ */
/* tensor algebra, src/elastic3d.f90:129-319                          */
/* ------------------------------------------------------------------ */

/* tensortrace (:296-302): REAL*4 sum returned as REAL*8 */
static double ttrace(const otensor *t) { return (double)(t->s11 + t->s22 + t->s33); }

#define SQ(x) ((double)((x) * (x)))
/* tensornorm (:311-319): squares of REAL*4 components, sum in REAL*8 */
static double tnorm(const otensor *t)
{
    return sqrt((SQ(t->s11) + 2.0 * SQ(t->s12) + 2.0 * SQ(t->s13) + SQ(t->s22) +
                 2.0 * SQ(t->s23) + SQ(t->s33)) / 2.0);
}

/* tensordeviatoric (:275-290) */
static otensor tdev(const otensor *t)
{
    real diag = (real)(ttrace(t) / 3.0);
    otensor d = {t->s11 - diag, t->s12, t->s13, t->s22 - diag, t->s23, t->s33 - diag};
    return d;
}

static otensor tplus(otensor a, otensor b)
{
    otensor r = {a.s11 + b.s11, a.s12 + b.s12, a.s13 + b.s13, a.s22 + b.s22, a.s23 + b.s23, a.s33 + b.s33};
    return r;
}

static otensor tminus(otensor a, otensor b)
{
    otensor r = {a.s11 - b.s11, a.s12 - b.s12, a.s13 - b.s13, a.s22 - b.s22, a.s23 - b.s23, a.s33 - b.s33};
    return r;
}

static otensor ttimes(real c, otensor a)
{
    otensor r = {c * a.s11, c * a.s12, c * a.s13, c * a.s22, c * a.s23, c * a.s33};
    return r;
}

/* tensorsymmetricdyadprod (:203-214) */
static otensor sdyad(const double a[3], const double b[3])
{
    otensor r = {(real)(a[0] * b[0]), (real)((a[0] * b[1] + a[1] * b[0]) / 2.0),
                 (real)((a[0] * b[2] + a[2] * b[0]) / 2.0), (real)(a[1] * b[1]),
                 (real)((a[1] * b[2] + a[2] * b[1]) / 2.0), (real)(a[2] * b[2])};
    return r;
}

/* tensorvectordotprod (:222-231) */
static void tdot(const otensor *t, const double v[3], double out[3])
{
    out[0] = t->s11 * v[0] + t->s12 * v[1] + t->s13 * v[2];
    out[1] = t->s12 * v[0] + t->s22 * v[1] + t->s23 * v[2];
    out[2] = t->s13 * v[0] + t->s23 * v[1] + t->s33 * v[2];
}

/* isotropicstressstrain (:129-142) */
static void isotropic(otensor *t, double lambda, double mu)
{
    double epskk = ttrace(t);
    *t = ttimes((real)(2.0 * mu), *t);
    t->s11 = (real)(t->s11 + lambda * epskk);
    t->s22 = (real)(t->s22 + lambda * epskk);
    t->s33 = (real)(t->s33 + lambda * epskk);
}

/* ------------------------------------------------------------------ */
/* depth structures, src/elastic3d.f90:630-829                         */
/* ------------------------------------------------------------------ */

int orc_viscoelastic_structure(const relax_layer *layers, int nv, double dx3, int sx3,
                               relax_layer *vs)
{
    if (nv <= 0) return ORC_ERR_ARG;
    for (int k = 0; k < sx3; k++) {
        vs[k].z = 0; vs[k].gammadot0 = 0; vs[k].friction = 0.6; vs[k].cohesion = 0;
        vs[k].stressexponent = layers[0].stressexponent; vs[k].Gk = 0;
    }
    double z0 = orc_fix(layers[0].z / dx3) * dx3, z1 = z0;
    double g0 = 0, p0 = 0, f0 = 0, c0 = 0, k0 = 0, g1 = 0, p1 = 0, f1 = 0, c1 = 0, k1 = 0;
    int i3e = 1;
    for (int k = 0; k < nv; k++) {
        z1 = orc_fix(layers[k].z / dx3) * dx3;
        if (z1 < z0) return ORC_ERR_ARG;
        g1 = layers[k].gammadot0; p1 = layers[k].stressexponent; f1 = layers[k].friction;
        c1 = layers[k].cohesion; k1 = layers[k].Gk;
        if (z1 == z0) {
            i3e = orc_fix(z1 / dx3 + 1);
        } else {
            int i3s = orc_fix(z0 / dx3) + 1;
            i3e = orc_fix(z1 / dx3 + 1);
            if (i3e > sx3) i3e = sx3;
            for (int i3 = i3s; i3 <= i3e; i3++) {
                double z = (i3 - 1.0) * dx3;
                if (i3 < 1) continue;
                vs[i3 - 1].gammadot0 = ((z - z0) * g1 + (z1 - z) * g0) / (z1 - z0);
                vs[i3 - 1].stressexponent = ((z - z0) * p1 + (z1 - z) * p0) / (z1 - z0);
                vs[i3 - 1].friction = ((z - z0) * f1 + (z1 - z) * f0) / (z1 - z0);
                vs[i3 - 1].cohesion = ((z - z0) * c1 + (z1 - z) * c0) / (z1 - z0);
                vs[i3 - 1].Gk = ((z - z0) * k1 + (z1 - z) * k0) / (z1 - z0);
            }
        }
        z0 = z1; g0 = g1; p0 = p1; f0 = f1; c0 = c1; k0 = k1;
    }
    if (orc_fix(z1 / dx3) < sx3 - 1) {
        for (int i3 = (i3e < 1 ? 1 : i3e); i3 <= sx3; i3++) {
            /* REAL(...) conversions of src/elastic3d.f90:821-825 */
            vs[i3 - 1].gammadot0 = (float)g1;
            vs[i3 - 1].stressexponent = (float)p1;
            vs[i3 - 1].friction = (float)f1;
            vs[i3 - 1].cohesion = (float)c1;
            vs[i3 - 1].Gk = (float)k1;
        }
    }
    return ORC_OK;
}

int orc_tensor_structure(const relax_tensor_layer *layers, int nv, double dx3, int sx3,
                         relax_tensor_layer *vs)
{
    if (nv <= 0) return ORC_ERR_ARG;
    memset(vs, 0, sizeof(relax_tensor_layer) * (size_t)sx3);
    double z0 = orc_fix(layers[0].z / dx3) * dx3, z1 = z0;
    relax_tensor t0 = {0, 0, 0, 0, 0, 0}, t1 = {0, 0, 0, 0, 0, 0};
    int i3e = 1;
    for (int k = 0; k < nv; k++) {
        z1 = orc_fix(layers[k].z / dx3) * dx3;
        if (z1 < z0) return ORC_ERR_ARG;
        t1 = layers[k].t;
        if (z1 == z0) {
            i3e = orc_fix(z1 / dx3 + 1);
        } else {
            int i3s = orc_fix(z0 / dx3) + 1;
            i3e = orc_fix(z1 / dx3 + 1);
            if (i3e > sx3) i3e = sx3;
            for (int i3 = i3s; i3 <= i3e; i3++) {
                double z = (i3 - 1.0) * dx3;
                float a = (float)(z - z0), b = (float)(z1 - z), s = (float)(1.0 / (z1 - z0));
                relax_tensor t;
                t.s11 = s * (a * t1.s11 + b * t0.s11);
                t.s12 = s * (a * t1.s12 + b * t0.s12);
                t.s13 = s * (a * t1.s13 + b * t0.s13);
                t.s22 = s * (a * t1.s22 + b * t0.s22);
                t.s23 = s * (a * t1.s23 + b * t0.s23);
                t.s33 = s * (a * t1.s33 + b * t0.s33);
                if (i3 >= 1) vs[i3 - 1].t = t;
            }
        }
        z0 = z1; t0 = t1;
    }
    if (orc_fix(z1 / dx3) < sx3 - 1)
        for (int i3 = (i3e < 1 ? 1 : i3e); i3 <= sx3; i3++) vs[i3 - 1].t = t1;
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* FIR differentiators, src/elastic3d.f90:846-907, src/kernel*.inc     */
/* (the Fortran literals are default-real, i.e. single precision)      */
/* ------------------------------------------------------------------ */
static const float FIR7[7] = {8.77856e-01f, -2.81913e-01f, +6.22696e-02f, +2.82441e-02f,
                              -5.09029e-02f, +4.20471e-02f, -1.59409e-02f};

/* The periodic neighbour index.  The reference's mod(sx+i-1-l,sx)+1 keeps
 * the dividend's sign (Fortran MOD), so for a 7-point filter on an axis of
 * 5 or 6 samples it indexes outside the axis (i - 1 - l < -sx); here the
 * index wraps, which is the periodic neighbour the filter means. */
static inline int pmod(int a, int n)
{
    const int r = a % n;
    return r < 0 ? r + n : r;
}

static int optimalfilter(int sx1, int sx2, int sx3, double *k1, double *k2, double *k3,
                         int *l1, int *l2, int *l3)
{
    int sx[3] = {sx1, sx2, sx3}, *len[3] = {l1, l2, l3};
    double *ker[3] = {k1, k2, k3};
    for (int d = 0; d < 3; d++) {
        int n = sx[d];
        if (d < 2 && n >= 2 && n <= 4) { *len[d] = 1; ker[d][0] = 0.5; }
        else if (n >= 5 && n <= 14) {
            *len[d] = 7;
            for (int l = 0; l < 7; l++) ker[d][l] = (double)FIR7[l];
        } else if (n >= 15) { *len[d] = 1; ker[d][0] = 0.5; }
        else return ORC_ERR_ARG;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* stressupdate, src/elastic3d.f90:956-1180                             */
/* u: (sx1+2, sx2, sx3) padded; sig: (sx1, sx2, sx3); sx3 = physical.  */
/* ------------------------------------------------------------------ */
int orc_stressupdate(const real *v1, const real *v2, const real *v3, double lambda, double mu,
                     double dx1, double dx2, double dx3, int sx1, int sx2, int sx3, otensor *sig)
{
    double ker1[16] = {0}, ker2[16] = {0}, ker3[16] = {0};
    int len1, len2, len3;
    if (optimalfilter(sx1, sx2, sx3, ker1, ker2, ker3, &len1, &len2, &len3)) return ORC_ERR_ARG;
    for (int l = 0; l < len1; l++) ker1[l] /= dx1;
    for (int l = 0; l < len2; l++) ker2[l] /= dx2;
    for (int l = 0; l < len3; l++) ker3[l] /= dx3;
    const int n1 = sx1 + 2;

#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        int boundary = !((i3 > len3) && (i3 < (sx3 - len3 + 1)));
        double px3 = 0;
        int i3m = 0, i3p = 0;
        if (boundary) {
            if (i3 == 1) { px3 = dx3; i3p = 2; i3m = 1; }
            else if (i3 == sx3) { px3 = dx3; i3p = sx3; i3m = sx3 - 1; }
            else { px3 = dx3 * 2.0; i3m = i3 - 1; i3p = i3 + 1; }
        }
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                otensor e = {0, 0, 0, 0, 0, 0};
#define V(a, j1, j2, j3) (a)[IDX3((j1) - 1, (j2) - 1, (j3) - 1, n1, sx2)]
                for (int l = 1; l <= len1; l++) {
                    int i1m = pmod(sx1 + i1 - 1 - l, sx1) + 1, i1p = (i1 - 1 + l) % sx1 + 1;
                    e.s11 = (real)(e.s11 + (real)(V(v1, i1p, i2, i3) - V(v1, i1m, i2, i3)) * ker1[l - 1]);
                    e.s12 = (real)(e.s12 + (real)(V(v2, i1p, i2, i3) - V(v2, i1m, i2, i3)) * ker1[l - 1]);
                    e.s13 = (real)(e.s13 + (real)(V(v3, i1p, i2, i3) - V(v3, i1m, i2, i3)) * ker1[l - 1]);
                }
                for (int l = 1; l <= len2; l++) {
                    int i2m = pmod(sx2 + i2 - 1 - l, sx2) + 1, i2p = (i2 - 1 + l) % sx2 + 1;
                    e.s12 = (real)(e.s12 + (real)(V(v1, i1, i2p, i3) - V(v1, i1, i2m, i3)) * ker2[l - 1]);
                    e.s22 = (real)(e.s22 + (real)(V(v2, i1, i2p, i3) - V(v2, i1, i2m, i3)) * ker2[l - 1]);
                    e.s23 = (real)(e.s23 + (real)(V(v3, i1, i2p, i3) - V(v3, i1, i2m, i3)) * ker2[l - 1]);
                }
                if (boundary) {
                    /* localstrain_ani, :1140-1175 */
                    e.s13 = (real)(e.s13 + (real)(V(v1, i1, i2, i3p) - V(v1, i1, i2, i3m)) / px3);
                    e.s23 = (real)(e.s23 + (real)(V(v2, i1, i2, i3p) - V(v2, i1, i2, i3m)) / px3);
                    e.s33 = (real)((real)(V(v3, i1, i2, i3p) - V(v3, i1, i2, i3m)) / px3);
                } else {
                    /* localstrain_fir2, :1060-1100 */
                    for (int l = 1; l <= len3; l++) {
                        int m = i3 - l, p = i3 + l;
                        e.s13 = (real)(e.s13 + (real)(V(v1, i1, i2, p) - V(v1, i1, i2, m)) * ker3[l - 1]);
                        e.s23 = (real)(e.s23 + (real)(V(v2, i1, i2, p) - V(v2, i1, i2, m)) * ker3[l - 1]);
                        e.s33 = (real)(e.s33 + (real)(V(v3, i1, i2, p) - V(v3, i1, i2, m)) * ker3[l - 1]);
                    }
                }
#undef V
                e.s12 = (real)(e.s12 / 2.0);
                e.s13 = (real)(e.s13 / 2.0);
                e.s23 = (real)(e.s23 / 2.0);
                isotropic(&e, lambda, mu);
                otensor *s = &sig[IDX3(i1 - 1, i2 - 1, i3 - 1, sx1, sx2)];
                *s = tplus(*s, e);
            }
        }
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* equivalentbodyforce, src/elastic3d.f90:1214-1506                    */
/* c: (sx1+2, sx2, >=sx3) padded; t: (sx1+2, sx2); sx3 = physical.    */
/* ------------------------------------------------------------------ */
int orc_equivalentbodyforce(const otensor *sig, double dx1, double dx2, double dx3, int sx1,
                            int sx2, int sx3, real *c1, real *c2, real *c3, real *t1, real *t2,
                            real *t3)
{
    double ker1[16] = {0}, ker2[16] = {0}, ker3[16] = {0};
    int len1, len2, len3;
    if (optimalfilter(sx1, sx2, sx3, ker1, ker2, ker3, &len1, &len2, &len3)) return ORC_ERR_ARG;
    for (int l = 0; l < len1; l++) ker1[l] /= dx1;
    for (int l = 0; l < len2; l++) ker2[l] /= dx2;
    for (int l = 0; l < len3; l++) ker3[l] /= dx3;
    const int n1 = sx1 + 2;

    for (int i2 = 0; i2 < sx2; i2++)
        for (int i1 = 0; i1 < sx1; i1++) {
            const otensor *s = &sig[IDX3(i1, i2, 0, sx1, sx2)];
            t1[i1 + (size_t)n1 * i2] += s->s13;
            t2[i1 + (size_t)n1 * i2] += s->s23;
            t3[i1 + (size_t)n1 * i2] += s->s33;
        }

#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        int boundary = !((i3 > len3) && (i3 < (sx3 - len3 + 1)));
        double px3 = 0;
        int i3m = 0, i3p = 0;
        if (boundary) {
            if (i3 == 1) { px3 = dx3; i3p = 2; i3m = 1; }
            else if (i3 == sx3) { px3 = dx3; i3p = sx3; i3m = sx3 - 1; }
            else { px3 = dx3 * 2.0; i3m = i3 - 1; i3p = i3 + 1; }
        }
#define S(j1, j2, j3) sig[IDX3((j1) - 1, (j2) - 1, (j3) - 1, sx1, sx2)]
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double f1 = 0, f2 = 0, f3 = 0;
                for (int l = 1; l <= len1; l++) {
                    int i1m = pmod(sx1 + i1 - 1 - l, sx1) + 1, i1p = (i1 - 1 + l) % sx1 + 1;
                    f1 += (real)(S(i1p, i2, i3).s11 - S(i1m, i2, i3).s11) * ker1[l - 1];
                    f2 += (real)(S(i1p, i2, i3).s12 - S(i1m, i2, i3).s12) * ker1[l - 1];
                    f3 += (real)(S(i1p, i2, i3).s13 - S(i1m, i2, i3).s13) * ker1[l - 1];
                }
                for (int l = 1; l <= len2; l++) {
                    int i2m = pmod(sx2 + i2 - 1 - l, sx2) + 1, i2p = (i2 - 1 + l) % sx2 + 1;
                    f1 += (real)(S(i1, i2p, i3).s12 - S(i1, i2m, i3).s12) * ker2[l - 1];
                    f2 += (real)(S(i1, i2p, i3).s22 - S(i1, i2m, i3).s22) * ker2[l - 1];
                    f3 += (real)(S(i1, i2p, i3).s23 - S(i1, i2m, i3).s23) * ker2[l - 1];
                }
                if (boundary) {
                    f1 += (real)(S(i1, i2, i3p).s13 - S(i1, i2, i3m).s13) / px3;
                    f2 += (real)(S(i1, i2, i3p).s23 - S(i1, i2, i3m).s23) / px3;
                    f3 += (real)(S(i1, i2, i3p).s33 - S(i1, i2, i3m).s33) / px3;
                } else {
                    for (int l = 1; l <= len3; l++) {
                        f1 += (real)(S(i1, i2, i3 + l).s13 - S(i1, i2, i3 - l).s13) * ker3[l - 1];
                        f2 += (real)(S(i1, i2, i3 + l).s23 - S(i1, i2, i3 - l).s23) * ker3[l - 1];
                        f3 += (real)(S(i1, i2, i3 + l).s33 - S(i1, i2, i3 - l).s33) * ker3[l - 1];
                    }
                }
                size_t o = IDX3(i1 - 1, i2 - 1, i3 - 1, n1, sx2);
                c1[o] = c1[o] - (real)f1;
                c2[o] = c2[o] - (real)f2;
                c3[o] = c3[o] - (real)f3;
            }
        }
#undef S
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* viscouseigenstress, src/viscoelastic3d.f90:217-314                  */
/* ------------------------------------------------------------------ */
int orc_viscouseigenstress(double mu, const relax_layer *structure,
                           const relax_tensor_layer *prestress, const otensor *sig, int sx1,
                           int sx2, int sx3, otensor *moment, double *maxwelltime, real *gamma,
                           const real *dgammadot0)
{
    real tm = maxwelltime ? (real)*maxwelltime : (real)1e30;
    int err = ORC_OK;
    for (int i3 = 0; i3 < sx3; i3++)
        if (structure[i3].stressexponent < 0.999999) err = ORC_ERR_POWER;
    if (err) return err;
#pragma omp parallel for schedule(static) reduction(min : tm)
    for (int i3 = 0; i3 < sx3; i3++) {
        double power = structure[i3].stressexponent, cohesion = structure[i3].cohesion;
        otensor p;
        if (prestress) {
            const relax_tensor *q = &prestress[i3].t;
            p.s11 = (real)q->s11; p.s12 = (real)q->s12; p.s13 = (real)q->s13;
            p.s22 = (real)q->s22; p.s23 = (real)q->s23; p.s33 = (real)q->s33;
        } else {
            memset(&p, 0, sizeof p);
        }
        otensor sp = tdev(&p);
        double taup = tnorm(&sp);
        for (int i2 = 0; i2 < sx2; i2++) {
            for (int i1 = 0; i1 < sx1; i1++) {
                size_t o = IDX3(i1, i2, i3, sx1, sx2);
                double gammadot0 = structure[i3].gammadot0;
                if (dgammadot0) gammadot0 = gammadot0 + dgammadot0[o];
                if (1.0e-20 > gammadot0) continue;
                otensor s = tdev(&sig[o]);
                otensor ssp = tplus(s, sp);
                double tau = tnorm(&ssp);
                double tauc = tau - cohesion > 0.0 ? tau - cohesion : 0.0;
                if (tauc <= 1.0e-20) continue;
                double gammadot = gammadot0 * pow(tauc / mu, power - 1);
                double gammadotp = gammadot0 * pow(taup / mu, power - 1);
                moment[o] = tplus(moment[o], tminus(ttimes((real)(2.0 * gammadot), s),
                                                    ttimes((real)(2.0 * gammadotp), sp)));
                real r = (real)(1.0 / gammadot);
                tm = tm < r ? tm : r;
                if (gamma) gamma[IDX3(i1, i2, i3, sx1 + 2, sx2)] = (real)(gammadot * tauc / mu);
            }
        }
    }
    if (maxwelltime) *maxwelltime = (double)tm < *maxwelltime ? (double)tm : *maxwelltime;
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* transienteigenstress, src/viscoelastic3d.f90:123-202: Burgers creep    */
/* with the transient strain epsilonik.  epsilonik and epsilonikdot may   */
/* be the same array (the corrector's call, src/relax.f90:768-786): each  */
/* point reads epsilonik before it writes epsilonikdot.                   */
/* ------------------------------------------------------------------ */
int orc_transienteigenstress(double mu, const relax_layer *structure, const otensor *sig,
                             const otensor *epsilonik, int sx1, int sx2, int sx3, otensor *moment,
                             otensor *epsilonikdot, double *maxwelltime, const real *dgammadot0)
{
    real tm = maxwelltime ? (real)*maxwelltime : (real)1e30;
    for (int i3 = 0; i3 < sx3; i3++)
        if (structure[i3].stressexponent < 0.999999) return ORC_ERR_POWER;
#pragma omp parallel for schedule(static) reduction(min : tm)
    for (int i3 = 0; i3 < sx3; i3++) {
        double power = structure[i3].stressexponent, muk = structure[i3].Gk;
        for (int i2 = 0; i2 < sx2; i2++) {
            for (int i1 = 0; i1 < sx1; i1++) {
                size_t o = IDX3(i1, i2, i3, sx1, sx2);
                double gammadot0 = structure[i3].gammadot0;
                if (dgammadot0) gammadot0 = gammadot0 + dgammadot0[o];
                if (1.0e-20 > gammadot0) {
                    memset(&epsilonikdot[o], 0, sizeof(otensor));
                    continue;
                }
                otensor s = tdev(&sig[o]);
                otensor Q = tminus(s, ttimes((real)(2.0 * muk), epsilonik[o]));
                double nq = tnorm(&Q);
                double gammadot = gammadot0 * pow(nq / mu, power - 1);
                epsilonikdot[o] = ttimes((real)(gammadot / mu), Q);
                moment[o] = tplus(moment[o], ttimes((real)(2.0 * gammadot), Q));
                real r = (real)(1.0 / gammadot);
                tm = tm < r ? tm : r;
            }
        }
    }
    if (maxwelltime) *maxwelltime = (double)tm < *maxwelltime ? (double)tm : *maxwelltime;
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* tensile cracks and dilatation point sources                          */
/* ------------------------------------------------------------------ */

/* tensilesource, src/elastic3d.f90:2315-2411: equivalent body force of an
 * opening crack over the whole box (sx3 layers: the image lies in the
 * lower half), padded (sx1+2, sx2, sx3) arrays */
void orc_tensilesource(double lambda, double mu, double s, double x, double y, double z, double L,
                       double W, double strike, double dip, double beta, int sx1, int sx2, int sx3,
                       double dx1, double dx2, double dx3, real *f1, real *f2, real *f3)
{
    const int n1 = sx1 + 2;
    double cstrike = cos(strike), sstrike = sin(strike), cdip = cos(dip), sdip = sin(dip);
    double Wp = W * (1.0 + 2.0 * beta) / 2.0, Lp = L * (1.0 + 2.0 * beta) / 2.0;
    double x2r0 = cstrike * x - sstrike * y;
    double xr = cdip * x2r0 - sdip * z, yr = sstrike * x + cstrike * y, zr = sdip * x2r0 + cdip * z;
    double scale1 = -s * (lambda + 2.0 * mu), scale2 = -s * lambda;
    const double w701 = (double)7.01f;   /* default-real literal */
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        double x1, x2, x3;
        shiftedcoordinates(1, 1, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &x3);
        if (fabs(x3 - z) > Lp && fabs(x3 + z) > Lp) continue;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &x3);
                if (fabs(x1 - x) > Wp || fabs(x2 - y) > Wp) continue;
                double x2r = cstrike * x1 - sstrike * x2;
                double x1s = cdip * x2r - sdip * x3, x1i = cdip * x2r + sdip * x3;
                if (fabs(x1s - xr) > w701 * dx1 && fabs(x1i - xr) > w701 * dx1) continue;
                double x2s = sstrike * x1 + cstrike * x2;
                double x3s = sdip * x2r + cdip * x3, x3i = -sdip * x2r + cdip * x3;
                double temp1 = gauss(x1s - xr, dx1), temp2 = omega((x2s - yr) / W, beta);
                double temp3 = omega((x3s - zr) / L, beta);
                double sourc = scale1 * gaussp(x1s - xr, dx1) * temp2 * temp3;
                double dblcp = scale2 / W * temp1 * omegap((x2s - yr) / W, beta) * temp3;
                double dipcs = scale2 / L * temp1 * temp2 * omegap((x3s - zr) / L, beta);
                temp1 = gauss(x1i - xr, dx1);
                temp3 = omega((x3i + zr) / L, beta);
                double image = scale1 * gaussp(x1i - xr, dx1) * temp2 * temp3;
                double cplei = scale2 / W * temp1 * omegap((x2s - yr) / W, beta) * temp3;
                double dipci = scale2 / L * temp1 * temp2 * omegap((x3i + zr) / L, beta);
                size_t o = IDX3(i1 - 1, i2 - 1, i3 - 1, n1, sx2);
                f1[o] = (real)(f1[o] + cstrike * cdip * (sourc + image) + sstrike * (dblcp + cplei) +
                               cstrike * sdip * (dipcs + dipci));
                f2[o] = (real)(f2[o] - sstrike * cdip * (sourc + image) + cstrike * (dblcp + cplei) -
                               sstrike * sdip * (dipcs + dipci));
                f3[o] = (real)(f3[o] - sdip * (sourc - image) + cdip * (dipcs - dipci));
            }
        }
    }
}

/* mogisource, src/elastic3d.f90:2458-2509: equivalent body force of a
 * dilatation point source and its image over the whole box */
void orc_mogisource(double lambda, double mu, double o, double xs, double ys, double zs, int sx1, int sx2,
                    int sx3, double dx1, double dx2, double dx3, real *f1, real *f2, real *f3)
{
    const int n1 = sx1 + 2;
    double scale = -(lambda + 2.0 * mu / 3.0) * o;
    double mx = dx1 > dx2 ? dx1 : dx2;
    if (dx3 > mx) mx = dx3;
    double Wp = 6.0 * mx, Lp = 6.0 * mx;
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        double x1, x2, x3;
        shiftedcoordinates(1, 1, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &x3);
        if (fabs(x3 - zs) > Lp && fabs(x3 + zs) > Lp) continue;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &x3);
                if (fabs(x1 - xs) > Wp || fabs(x2 - ys) > Wp) continue;
                double temp1 = gauss(x1 - xs, dx1), temp2 = gauss(x2 - ys, dx2), temp3 = gauss(x3 - zs, dx3);
                double source1 = scale * gaussp(x1 - xs, dx1) * temp2 * temp3;
                double source2 = scale * temp1 * gaussp(x2 - ys, dx2) * temp3;
                double source3 = scale * temp1 * temp2 * gaussp(x3 - zs, dx3);
                temp3 = gauss(x3 + zs, dx3);
                double image1 = scale * gaussp(x1 - xs, dx1) * temp2 * temp3;
                double image2 = scale * temp1 * gaussp(x2 - ys, dx2) * temp3;
                double image3 = scale * temp1 * temp2 * gaussp(x3 + zs, dx3);
                size_t q = IDX3(i1 - 1, i2 - 1, i3 - 1, n1, sx2);
                f1[q] = (real)(f1[q] + (source1 + image1));
                f2[q] = (real)(f2[q] + (source2 + image2));
                f3[q] = (real)(f3[q] + (source3 - image3));
            }
        }
    }
}

/* momentdensitytensile, src/elastic3d.f90:3137-3215 (physical layers) */
void orc_momentdensitytensile(double lambda, double mu, double slip, double x, double y, double z, double L,
                              double W, double strike, double dip, double beta, int sx1, int sx2, int sx3,
                              double dx1, double dx2, double dx3, otensor *sig)
{
    double cstrike = cos(strike), sstrike = sin(strike), cdip = cos(dip), sdip = sin(dip);
    double Wp = W * (1.0 + 2.0 * beta) / 2.0, Lp = L * (1.0 + 2.0 * beta) / 2.0;
    double x2r0 = cstrike * x - sstrike * y;
    double xr = cdip * x2r0 - sdip * z, yr = sstrike * x + cstrike * y, zr = sdip * x2r0 + cdip * z;
    const double w701 = (double)7.01f;
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        double x3 = (double)(i3 - 1) * dx3;
        if (fabs(x3 - z) > Lp) continue;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double x1, x2, dum;
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &dum);
                if (fabs(x1 - x) > Wp || fabs(x2 - y) > Wp) continue;
                double x2r = cstrike * x1 - sstrike * x2;
                double x1s = cdip * x2r - sdip * x3, x1i = cdip * x2r + sdip * x3;
                if (fabs(x1s - xr) > w701 * dx1 && fabs(x1i - xr) > w701 * dx1) continue;
                double x2s = sstrike * x1 + cstrike * x2;
                double x3s = sdip * x2r + cdip * x3, x3i = -sdip * x2r + cdip * x3;
                double temp1 = gauss(x1s - xr, dx1), temp2 = omega((x2s - yr) / W, beta);
                double temp3 = omega((x3s - zr) / L, beta);
                double aperture = temp1 * temp2 * temp3;
                temp1 = gauss(x1i - xr, dx1);
                temp3 = omega((x3i + zr) / L, beta);
                aperture = aperture + temp1 * temp2 * temp3;
                double n[3] = {+cdip * cstrike * aperture, -cdip * sstrike * aperture, -sdip * aperture};
                double sn[3] = {slip * n[0], slip * n[1], slip * n[2]};
                otensor Ei = sdyad(n, sn);
                isotropic(&Ei, lambda, mu);
                size_t o = IDX3(i1 - 1, i2 - 1, i3 - 1, sx1, sx2);
                sig[o] = tplus(sig[o], Ei);
            }
        }
    }
}

/* momentdensitymogi, src/elastic3d.f90:3240-3286 (physical layers) */
void orc_momentdensitymogi(double lambda, double mu, double o, double xs, double ys, double zs, int sx1,
                           int sx2, int sx3, double dx1, double dx2, double dx3, otensor *sig)
{
    double kappa = lambda + 2.0 / 3.0 * mu;
    double mx = dx1 > dx2 ? dx1 : dx2;
    if (dx3 > mx) mx = dx3;
    double Wp = 6.0 * mx, Lp = 6.0 * mx;
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        double x3 = (double)(i3 - 1) * dx3;
        if (fabs(x3 - zs) > Lp) continue;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double x1, x2, dum;
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &dum);
                if (fabs(x1 - xs) > Wp || fabs(x2 - ys) > Wp) continue;
                double gamma = o * gauss(x1 - xs, dx1) * gauss(x2 - ys, dx2) * gauss(x3 - zs, dx3);
                gamma = kappa * gamma;
                otensor m = {(real)gamma, 0, 0, (real)gamma, 0, (real)gamma};
                size_t q = IDX3(i1 - 1, i2 - 1, i3 - 1, sx1, sx2);
                sig[q] = tplus(sig[q], m);
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* builddgammadot0 / fdgammadot0, src/viscoelastic3d.f90:320-435        */
/* ------------------------------------------------------------------ */
void orc_builddgammadot0(int sx1, int sx2, int sx3, double dx1, double dx2, double dx3, double beta,
                         int nz, const relax_weakzone *zones, real *dgammadot0)
{
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        double x3 = (double)(i3 - 1) * dx3;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double x1, x2, dum;
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &dum);
                double f = 0.0;
                for (int i = 0; i < nz; i++) {
                    const relax_weakzone *z = &zones[i];
                    double dg = z->dgammadot0, x = z->x, y = z->y, zz = z->z;
                    double W = z->length, L = z->width, D = z->thickness;
                    double Wp = W * (1.0 + 2.0 * beta) / 2.0, Lp = L * (1.0 + 2.0 * beta) / 2.0;
                    double Dp = D * (1.0 + 2.0 * beta) / 2.0;
                    double LM = Wp > Lp ? Wp : Lp;
                    if (Dp > LM) LM = Dp;
                    if (fabs(x3 - zz) > LM || fabs(x1 - x) > LM || fabs(x2 - y) > LM) continue;
                    double cs = cos(z->strike), ss = sin(z->strike), cd = cos(z->dip), sd = sin(z->dip);
                    double x2r = cs * x - ss * y;
                    double xr = cd * x2r - sd * zz, yr = ss * x + cs * y, zr = sd * x2r + cd * zz;
                    x2r = cs * x1 - ss * x2;
                    double x1s = cd * x2r - sd * x3, x2s = ss * x1 + cs * x2, x3s = sd * x2r + cd * x3;
                    if (D >= 0 && W >= 0 && L >= 0) {
                        f = f + omega((x1s - xr) / D, beta) * omega((x2s - yr) / W, beta) *
                                    omega((x3s - zr) / L, beta) * dg;
                    } else if (D < 0 && W < 0 && L < 0) {
                        double r = sqrt(SQ((x1s - xr) / D) + SQ((x2s - yr) / W) + SQ((x3s - zr) / L));
                        f = f + omega(r, beta) * dg;
                    } else if (D < 0 && W < 0) {
                        double rho = sqrt(SQ((x1s - xr) / D) + SQ((x2s - yr) / W));
                        f = f + omega(rho, beta) * omega((x3s - zr) / L, beta) * dg;
                    } else if (D < 0 && L < 0) {
                        double rho = sqrt(SQ((x1s - xr) / D) + SQ((x3s - zr) / L));
                        f = f + omega(rho, beta) * omega((x2s - yr) / W, beta) * dg;
                    } else if (W < 0 && L < 0) {
                        double rho = sqrt(SQ((x2s - yr) / W) + SQ((x3s - zr) / L));
                        f = f + omega(rho, beta) * omega((x1s - xr) / D, beta) * dg;
                    }
                }
                dgammadot0[IDX3(i1 - 1, i2 - 1, i3 - 1, sx1, sx2)] = (real)f;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* frictioneigenstress, src/friction3d.f90:82-241 (CPU branch)          */
/* ------------------------------------------------------------------ */
int orc_frictioneigenstress(double x, double y, double z, double L, double W, double strike,
                            double dip, double rake, double beta, const otensor *sig, double mu,
                            const relax_layer *structure, int sx1, int sx2, int sx3, double dx1,
                            double dx2, double dx3, otensor *moment, double *maxwelltime)
{
    real tm = maxwelltime ? (real)*maxwelltime : (real)1e30;
    double cstrike = cos(strike), sstrike = sin(strike), cdip = cos(dip), sdip = sin(dip);
    double cr = cos(rake), sr = sin(rake);
    double Wp = W * (1.0 + 2.0 * beta) / 2.0, Lp = L * (1.0 + 2.0 * beta) / 2.0;
    double x2r = cstrike * x - sstrike * y;
    double xr = cdip * x2r - sdip * z, yr = sstrike * x + cstrike * y, zr = sdip * x2r + cdip * z;
    double n[3] = {+cdip * cstrike, -cdip * sstrike, -sdip};
    double r[3] = {sstrike * cr + cstrike * sdip * sr, cstrike * cr - sstrike * sdip * sr, cdip * sr};
    double mwp = Wp > Lp ? Wp : Lp;
    int err = ORC_OK;

    for (int i3 = 1; i3 <= sx3; i3++) {
        double x3 = (double)(i3 - 1) * dx3;
        if (fabs(x3 - z) > Lp && fabs(x3 + z) > Lp) continue;
        double vo = structure[i3 - 1].gammadot0, tauc = structure[i3 - 1].stressexponent;
        double friction = structure[i3 - 1].friction, cohesion = structure[i3 - 1].cohesion;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double x1, x2, dum;
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &dum);
                if (fabs(x1 - x) > mwp || fabs(x2 - y) > mwp) continue;
                double x2rr = cstrike * x1 - sstrike * x2;
                double x1s = cdip * x2rr - sdip * x3, x1i = cdip * x2rr + sdip * x3;
                if (fabs(x1s - xr) > 7.01 * dx1 && fabs(x1i - xr) > 7.01 * dx1) continue;
                double x2s = sstrike * x1 + cstrike * x2;
                double x3s = sdip * x2rr + cdip * x3, x3i = -sdip * x2rr + cdip * x3;
                double temp1 = gauss(x1s - xr, dx1), temp2 = omega((x2s - yr) / W, beta);
                double temp3 = omega((x3s - zr) / L, beta);
                double sourc = temp1 * temp2 * temp3;
                temp1 = gauss(x1i - xr, dx1);
                temp3 = omega((x3i + zr) / L, beta);
                double image = temp1 * temp2 * temp3;
                double impulse = sourc + image;
                size_t o = IDX3(i1 - 1, i2 - 1, i3 - 1, sx1, sx2);
                otensor s = sig[o];
                double t[3], ts[3];
                tdot(&s, n, t);
                double taun = t[0] * n[0] + t[1] * n[1] + t[2] * n[2];
                for (int k = 0; k < 3; k++) ts[k] = t[k] - taun * n[k];
                double taus = sqrt(ts[0] * ts[0] + ts[1] * ts[1] + ts[2] * ts[2]);
                double tau = taus + friction * taun - cohesion;
                if (tau < 0.0) tau = 0.0;
                if ((ts[0] * r[0] + ts[1] * r[1] + ts[2] * r[2]) < 0.0 && fabs(rake) < PI2 * 1.5)
                    continue;
                if ((tau / tauc) > 20) err = ORC_ERR_FRICTION;
                for (int k = 0; k < 3; k++) ts[k] = ts[k] / taus;
                double gammadot = vo * 2.0 * my_sinh(tau / tauc);
                real cand = (real)(tau / mu / gammadot * ((L < W ? L : W) / sqrt(dx1 * dx3)));
                if (cand < tm) tm = cand; /* a NaN candidate (0/0) leaves tm */
                double b[3];
                for (int k = 0; k < 3; k++) b[k] = (2.0 * mu * impulse * gammadot) * n[k];
                moment[o] = tplus(moment[o], sdyad(ts, b));
            }
        }
    }
    if (maxwelltime) *maxwelltime = (double)tm < *maxwelltime ? (double)tm : *maxwelltime;
    return err;
}

/* ------------------------------------------------------------------ */
/* monitorfriction / frictionadd, src/friction3d.f90:263-453           */
/* ------------------------------------------------------------------ */
int orc_monitorfriction(double x, double y, double z, double L, double W, double strike,
                        double dip, double rake, double beta, int sx1, int sx2, int sx3,
                        double dx1, double dx2, double dx3, const otensor *sig,
                        const relax_layer *structure, int px2, int px3, relax_slippatch *patch)
{
    (void)L; (void)W; (void)beta;
    double cstrike = cos(strike), sstrike = sin(strike), cdip = cos(dip), sdip = sin(dip);
    double cr = cos(rake), sr = sin(rake);
    double sv[3] = {sstrike, cstrike, 0.0}, dv[3] = {-cstrike * sdip, +sstrike * sdip, -cdip};
    double n[3] = {+cdip * cstrike, -cdip * sstrike, -sdip};
    double r[3] = {sstrike * cr + cstrike * sdip * sr, cstrike * cr - sstrike * sdip * sr, cdip * sr};
    for (int j3 = 1; j3 <= px3; j3++) {
        for (int j2 = 1; j2 <= px2; j2++) {
            relax_slippatch *p = &patch[(j2 - 1) + (size_t)px2 * (j3 - 1)];
            /* ref2local */
            double x2 = cstrike * x - sstrike * y;
            double xr = cdip * x2 - sdip * z, yr = sstrike * x + cstrike * y, zr = sdip * x2 + cdip * z;
            yr = (double)(F32(yr) + F32(((double)j2 - (double)px2 / 2.0 - 1.0) * dx2));
            zr = (double)(F32(zr) + F32(((double)j3 - (double)px3 / 2.0 - 1.0) * dx3));
            /* local2ref */
            double x2p = cdip * xr + sdip * zr;
            double x1 = cstrike * x2p + sstrike * yr;
            double xx2 = -sstrike * x2p + cstrike * yr;
            double x3 = -sdip * xr + cdip * zr;
            p->x1 = x1; p->x2 = xx2; p->x3 = x3; p->lx = yr; p->lz = zr;
            /* bounds: the physical half-space holds sx3 (= sx3/2 of the box) layers */
            if (x1 > (double)(sx1 / 2 - 1) * dx1 || x1 < -(double)(sx1 / 2) * dx1 ||
                xx2 > (double)(sx2 / 2 - 1) * dx2 || xx2 < -(double)(sx2 / 2) * dx2 ||
                x3 > (double)(sx3 - 1) * dx3 || x3 < 0.0)
                continue;
            /* shiftedindex, src/elastic3d.f90:4064-4101 */
            int i1 = (sx1 + orc_fix(x1 / dx1)) % sx1 + 1;
            int i2 = (sx2 + orc_fix(xx2 / dx2)) % sx2 + 1;
            int i3 = orc_fix(x3 / dx3) + 1;
            if (i3 > sx3) continue;
            double vo = structure[i3 - 1].gammadot0, tauc = structure[i3 - 1].stressexponent;
            double friction = structure[i3 - 1].friction, cohesion = structure[i3 - 1].cohesion;
            otensor s = sig[IDX3(i1 - 1, i2 - 1, i3 - 1, sx1, sx2)];
            p->sig.s11 = (float)s.s11; p->sig.s12 = (float)s.s12; p->sig.s13 = (float)s.s13;
            p->sig.s22 = (float)s.s22; p->sig.s23 = (float)s.s23; p->sig.s33 = (float)s.s33;
            double t[3], ts[3];
            tdot(&s, n, t);
            double taun = t[0] * n[0] + t[1] * n[1] + t[2] * n[2];
            for (int k = 0; k < 3; k++) ts[k] = t[k] - taun * n[k];
            double taus = sqrt(ts[0] * ts[0] + ts[1] * ts[1] + ts[2] * ts[2]);
            double tau = taus + friction * taun - cohesion;
            if (tau < 0.0) tau = 0.0;
            if ((ts[0] * r[0] + ts[1] * r[1] + ts[2] * r[2]) < 0.0 && fabs(rake) < PI2 * 1.5) continue;
            p->taus = taus;
            p->v = vo * 2.0 * my_sinh(tau / tauc);
            for (int k = 0; k < 3; k++) ts[k] = ts[k] / taus;
            p->vss = p->v * (ts[0] * sv[0] + ts[1] * sv[1] + ts[2] * sv[2]);
            p->vds = p->v * (ts[0] * dv[0] + ts[1] * dv[1] + ts[2] * dv[2]);
        }
    }
    return ORC_OK;
}

void orc_frictionadd(int npatch, relax_slippatch *patch, double dt)
{
    for (int k = 0; k < npatch; k++) {
        patch[k].ss = patch[k].ss + dt * patch[k].vss;
        patch[k].ds = patch[k].ds + dt * patch[k].vds;
        patch[k].slip = pow(patch[k].ds * patch[k].ds + patch[k].ss * patch[k].ss, 0.5);
    }
}

/* ------------------------------------------------------------------ */
/* field algebra, src/elastic3d.f90:3774-3959                          */
/* ------------------------------------------------------------------ */
void orc_fieldadd(real *u, const real *v, size_t n, int has_c1, real c1, int has_c2, real c2)
{
    if (has_c1 && has_c2) for (size_t i = 0; i < n; i++) u[i] = c1 * u[i] + c2 * v[i];
    else if (has_c1) for (size_t i = 0; i < n; i++) u[i] = c1 * u[i] + v[i];
    else if (has_c2) for (size_t i = 0; i < n; i++) u[i] = u[i] + c2 * v[i];
    else for (size_t i = 0; i < n; i++) u[i] = u[i] + v[i];
}

void orc_tensorfieldadd(otensor *t1, const otensor *t2, size_t n, int has_c1, real c1,
                        int has_c2, real c2)
{
    if (has_c1 && has_c2) {
        if (c1 == 0) {
            if (c2 == 0) memset(t1, 0, n * sizeof(otensor));
            else for (size_t i = 0; i < n; i++) t1[i] = ttimes(c2, t2[i]);
        } else {
            for (size_t i = 0; i < n; i++) t1[i] = tplus(ttimes(c1, t1[i]), ttimes(c2, t2[i]));
        }
    } else if (has_c1) {
        for (size_t i = 0; i < n; i++) t1[i] = tplus(ttimes(c1, t1[i]), t2[i]);
    } else if (has_c2) {
        for (size_t i = 0; i < n; i++) t1[i] = tplus(t1[i], ttimes(c2, t2[i]));
    } else {
        for (size_t i = 0; i < n; i++) t1[i] = tplus(t2[i], t2[i]);
    }
}

/* tensoramplitude, src/elastic3d.f90:446-466 */
double orc_tensoramplitude(const otensor *t, size_t n, double dx1, double dx2, double dx3)
{
    double a = 0;
    for (size_t i = 0; i < n; i++) a += tnorm(&t[i]);
    return a * (dx1 * dx2 * dx3);
}

/* ------------------------------------------------------------------ */
/* FFT: mixed-radix Stockham, double precision internally               */
/* ------------------------------------------------------------------ */
typedef struct { double re, im; } cpx;

static int factorize(int n, int *f)
{
    int m = 0;
    while (n % 4 == 0) { f[m++] = 4; n /= 4; }
    while (n % 2 == 0) { f[m++] = 2; n /= 2; }
    for (int p = 3; n > 1; p += 2)
        while (n % p == 0) { f[m++] = p; n /= p; }
    return m;
}

/* forward (sign=-1): X[k] = sum x[j] exp(-2 pi i jk/n), no scaling */
static void fft_c(cpx *x, int n, int sign, cpx *y)
{
    int f[40], m = factorize(n, f), p = 1;
    cpx *in = x, *out = y;
    for (int s = 0; s < m; s++) {
        int R = f[s], nr = n / R;
        for (int i = 0; i < nr; i++) {
            int k = i % p;
            cpx v[64], w[64];
            for (int r = 0; r < R; r++) {
                cpx a = in[i + r * nr];
                long q = ((long)r * k) % ((long)p * R);
                double ang = sign * PI2 * (double)q / (double)(p * R);
                double c = cos(ang), sn = sin(ang);
                v[r].re = a.re * c - a.im * sn;
                v[r].im = a.re * sn + a.im * c;
            }
            for (int t = 0; t < R; t++) {
                double re = 0, im = 0;
                for (int r = 0; r < R; r++) {
                    long q = ((long)r * t) % R;
                    double ang = sign * PI2 * (double)q / (double)R;
                    double c = cos(ang), sn = sin(ang);
                    re += v[r].re * c - v[r].im * sn;
                    im += v[r].re * sn + v[r].im * c;
                }
                w[t].re = re; w[t].im = im;
            }
            int j = (i - k) * R + k;
            for (int t = 0; t < R; t++) out[j + t * p] = w[t];
        }
        cpx *tmp = in; in = out; out = tmp;
        p *= R;
    }
    if (in != x) memcpy(x, in, sizeof(cpx) * (size_t)n);
}

void orc_fft_c(double *xy, int n, int sign)
{
    cpx *y = malloc(sizeof(cpx) * (size_t)n);
    fft_c((cpx *)xy, n, sign, y);
    free(y);
}

/* in-place real<->complex 2-D/3-D transform on a (sx1+2, sx2, sx3) array,
 * src/fourier.f90:177-201 (FFTW) / :372-401 (fft2) semantics:
 * forward result x (dx1 dx2 dx3) in REAL*4, inverse / (sx1 dx1 ...).
 * The c2r along x1 uses Re of the k1=0 and k1=sx1/2 bins. */
static void fft_rc(real *data, int sx1, int sx2, int sx3, int direction, real scale)
{
    const int n1 = sx1 + 2, K1 = sx1 / 2 + 1;
    int nmax = sx1 > sx2 ? sx1 : sx2;
    if (sx3 > nmax) nmax = sx3;
    if (direction < 0) {
#pragma omp parallel
        {
            cpx *a = malloc(sizeof(cpx) * (size_t)nmax), *w = malloc(sizeof(cpx) * (size_t)nmax);
#pragma omp for schedule(static)
            for (int row = 0; row < sx2 * sx3; row++) {
                real *r = data + (size_t)row * n1;
                for (int i = 0; i < sx1; i++) { a[i].re = r[i]; a[i].im = 0; }
                fft_c(a, sx1, -1, w);
                for (int k = 0; k < K1; k++) { r[2 * k] = (real)a[k].re; r[2 * k + 1] = (real)a[k].im; }
            }
#pragma omp for schedule(static)
            for (int line = 0; line < K1 * sx3; line++) {
                int k1 = line % K1, i3 = line / K1;
                for (int i2 = 0; i2 < sx2; i2++) {
                    real *c = data + IDX3(2 * k1, i2, i3, n1, sx2);
                    a[i2].re = c[0]; a[i2].im = c[1];
                }
                fft_c(a, sx2, -1, w);
                for (int i2 = 0; i2 < sx2; i2++) {
                    real *c = data + IDX3(2 * k1, i2, i3, n1, sx2);
                    c[0] = (real)a[i2].re; c[1] = (real)a[i2].im;
                }
            }
            if (sx3 > 1) {
#pragma omp for schedule(static)
                for (int line = 0; line < K1 * sx2; line++) {
                    int k1 = line % K1, i2 = line / K1;
                    for (int i3 = 0; i3 < sx3; i3++) {
                        real *c = data + IDX3(2 * k1, i2, i3, n1, sx2);
                        a[i3].re = c[0]; a[i3].im = c[1];
                    }
                    fft_c(a, sx3, -1, w);
                    for (int i3 = 0; i3 < sx3; i3++) {
                        real *c = data + IDX3(2 * k1, i2, i3, n1, sx2);
                        c[0] = (real)a[i3].re; c[1] = (real)a[i3].im;
                    }
                }
            }
            free(a); free(w);
        }
        size_t tot = (size_t)n1 * sx2 * sx3;
        for (size_t i = 0; i < tot; i++) data[i] = data[i] * scale;
    } else {
#pragma omp parallel
        {
            cpx *a = malloc(sizeof(cpx) * (size_t)nmax), *w = malloc(sizeof(cpx) * (size_t)nmax);
            if (sx3 > 1) {
#pragma omp for schedule(static)
                for (int line = 0; line < K1 * sx2; line++) {
                    int k1 = line % K1, i2 = line / K1;
                    for (int i3 = 0; i3 < sx3; i3++) {
                        real *c = data + IDX3(2 * k1, i2, i3, n1, sx2);
                        a[i3].re = c[0]; a[i3].im = c[1];
                    }
                    fft_c(a, sx3, +1, w);
                    for (int i3 = 0; i3 < sx3; i3++) {
                        real *c = data + IDX3(2 * k1, i2, i3, n1, sx2);
                        c[0] = (real)a[i3].re; c[1] = (real)a[i3].im;
                    }
                }
            }
#pragma omp for schedule(static)
            for (int line = 0; line < K1 * sx3; line++) {
                int k1 = line % K1, i3 = line / K1;
                for (int i2 = 0; i2 < sx2; i2++) {
                    real *c = data + IDX3(2 * k1, i2, i3, n1, sx2);
                    a[i2].re = c[0]; a[i2].im = c[1];
                }
                fft_c(a, sx2, +1, w);
                for (int i2 = 0; i2 < sx2; i2++) {
                    real *c = data + IDX3(2 * k1, i2, i3, n1, sx2);
                    c[0] = (real)a[i2].re; c[1] = (real)a[i2].im;
                }
            }
#pragma omp for schedule(static)
            for (int row = 0; row < sx2 * sx3; row++) {
                real *r = data + (size_t)row * n1;
                a[0].re = r[0]; a[0].im = 0;
                for (int k = 1; k < K1 - 1; k++) {
                    a[k].re = r[2 * k]; a[k].im = r[2 * k + 1];
                    a[sx1 - k].re = r[2 * k]; a[sx1 - k].im = -r[2 * k + 1];
                }
                a[sx1 / 2].re = r[2 * (K1 - 1)]; a[sx1 / 2].im = 0;
                fft_c(a, sx1, +1, w);
                for (int i = 0; i < sx1; i++) r[i] = (real)a[i].re;
                r[sx1] = 0; r[sx1 + 1] = 0;
            }
            free(a); free(w);
        }
        size_t tot = (size_t)n1 * sx2 * sx3;
        for (size_t i = 0; i < tot; i++) data[i] = data[i] / scale;
    }
}

/* fft3, src/fourier.f90:177-201 */
void orc_fft3(real *data, int sx1, int sx2, int sx3, double dx1, double dx2, double dx3,
              int direction)
{
    if (direction < 0) fft_rc(data, sx1, sx2, sx3, -1, (real)(dx1 * dx2 * dx3));
    else fft_rc(data, sx1, sx2, sx3, +1, (real)(sx1 * dx1 * sx2 * dx2 * sx3 * dx3));
}

/* fft2, src/fourier.f90:372-401 */
void orc_fft2(real *data, int sx1, int sx2, double dx1, double dx2, int direction)
{
    if (direction < 0) fft_rc(data, sx1, sx2, 1, -1, (real)(dx1 * dx2));
    else fft_rc(data, sx1, sx2, 1, +1, (real)(sx1 * dx1 * sx2 * dx2));
}

/* wavenumbers, src/fourier.f90:64-81 (0-based j) */
static double wn(int j, int sx, double dx)
{
    return (j < sx / 2) ? (double)j / (sx * dx) : -((double)(sx - j)) / (sx * dx);
}

/* ------------------------------------------------------------------ */
/* Green's function, src/green.f90                                    */
/* ------------------------------------------------------------------ */

/* elasticresponse, src/green.f90:51-101 */
void orc_elasticresponse(double lambda, double mu, real *f1, real *f2, real *f3, int sx1,
                         int sx2, int sx3, double dx1, double dx2, double dx3)
{
    const int n1 = sx1 + 2;
    double ratio1 = (lambda + mu) / (lambda + 2.0 * mu) / mu / (PI2 * PI2);
    double ratio2 = mu / (lambda + mu);
#pragma omp parallel for schedule(static)
    for (int i3 = 0; i3 < sx3; i3++) {
        double k3 = wn(i3, sx3, dx3);
        for (int i2 = 0; i2 < sx2; i2++) {
            double k2 = wn(i2, sx2, dx2);
            for (int i1 = 0; i1 < sx1 / 2 + 1; i1++) {
                double k1 = (double)i1 / (sx1 * dx1);
                double r2 = k1 * k1 + k2 * k2 + k3 * k3;
                double denom = ratio1 / (r2 * r2);
                size_t o = IDX3(2 * i1, i2, i3, n1, sx2);
                double c1r = f1[o], c1i = f1[o + 1], c2r = f2[o], c2i = f2[o + 1];
                double c3r = f3[o], c3i = f3[o + 1];
                double a1 = k2 * k2 + k3 * k3 + ratio2 * r2;
                double a2 = k1 * k1 + k3 * k3 + ratio2 * r2;
                double a3 = k1 * k1 + k2 * k2 + ratio2 * r2;
                double b1r = (a1 * c1r - k1 * (k2 * c2r + k3 * c3r)) * denom;
                double b1i = (a1 * c1i - k1 * (k2 * c2i + k3 * c3i)) * denom;
                double b2r = (a2 * c2r - k2 * (k1 * c1r + k3 * c3r)) * denom;
                double b2i = (a2 * c2i - k2 * (k1 * c1i + k3 * c3i)) * denom;
                double b3r = (a3 * c3r - k3 * (k1 * c1r + k2 * c2r)) * denom;
                double b3i = (a3 * c3i - k3 * (k1 * c1i + k2 * c2i)) * denom;
                f1[o] = (real)b1r; f1[o + 1] = (real)b1i;
                f2[o] = (real)b2r; f2[o + 1] = (real)b2i;
                f3[o] = (real)b3r; f3[o + 1] = (real)b3i;
            }
        }
    }
    f1[0] = 0; f1[1] = 0; f2[0] = 0; f2[1] = 0; f3[0] = 0; f3[1] = 0;
}

/* surfacetractioncowling, src/green.f90:327-377 */
void orc_surfacetractioncowling(double lambda, double mu, double gamma, const real *u1,
                                const real *u2, const real *u3, int sx1, int sx2, int sx3,
                                double dx1, double dx2, double dx3, real *p1, real *p2, real *p3)
{
    const int n1 = sx1 + 2;
    double modulus = lambda + 2.0 * mu, alpha = (lambda + mu) / (lambda + 2.0 * mu);
    double grav = 2.0 * mu * alpha * gamma;
    memset(p1, 0, sizeof(real) * (size_t)n1 * sx2);
    memset(p2, 0, sizeof(real) * (size_t)n1 * sx2);
    memset(p3, 0, sizeof(real) * (size_t)n1 * sx2);
#pragma omp parallel for schedule(static)
    for (int i2 = 0; i2 < sx2; i2++) {
        double k2 = wn(i2, sx2, dx2);
        for (int i3 = 0; i3 < sx3; i3++) {
            double k3 = wn(i3, sx3, dx3);
            for (int i1 = 0; i1 < sx1 / 2 + 1; i1++) {
                double k1 = (double)i1 / (sx1 * dx1);
                size_t o = IDX3(2 * i1, i2, i3, n1, sx2);
                double c1r = u1[o], c1i = u1[o + 1], c2r = u2[o], c2i = u2[o + 1];
                double c3r = u3[o], c3i = u3[o + 1];
                /* i = (0, 2 pi) */
                double a1r = mu * (k3 * c1r + k1 * c3r), a1i = mu * (k3 * c1i + k1 * c3i);
                double a2r = mu * (k3 * c2r + k2 * c3r), a2i = mu * (k3 * c2i + k2 * c3i);
                double a3r = modulus * k3 * c3r + lambda * (k1 * c1r + k2 * c2r);
                double a3i = modulus * k3 * c3i + lambda * (k1 * c1i + k2 * c2i);
                double s1r = -PI2 * a1i, s1i = PI2 * a1r;
                double s2r = -PI2 * a2i, s2i = PI2 * a2r;
                double s3r = -PI2 * a3i - grav * c3r, s3i = PI2 * a3r - grav * c3i;
                size_t q = 2 * (size_t)i1 + (size_t)n1 * i2;
                p1[q] = p1[q] + (real)s1r; p1[q + 1] = p1[q + 1] + (real)s1i;
                p2[q] = p2[q] + (real)s2r; p2[q + 1] = p2[q + 1] + (real)s2i;
                p3[q] = p3[q] + (real)s3r; p3[q + 1] = p3[q + 1] + (real)s3i;
            }
        }
    }
    real d = (real)(sx3 * dx3);
    for (size_t q = 0; q < (size_t)n1 * sx2; q++) {
        p1[q] = p1[q] / d; p2[q] = p2[q] / d; p3[q] = p3[q] / d;
    }
}

/* cerrutimodified + cerrutisolmodified, src/green.f90:520-612 */
void orc_cerrutimodified(const real *p1, const real *p2, const real *p3, double lambda,
                         double mu, double gamma, real *u1, real *u2, real *u3, int sx1, int sx2,
                         int sx3, double dx1, double dx2, double dx3)
{
    const int n1 = sx1 + 2;
    double alpha = (lambda + mu) / (lambda + 2 * mu);
#pragma omp parallel for schedule(static)
    for (int i2 = 0; i2 < sx2; i2++) {
        double k2 = wn(i2, sx2, dx2);
        for (int i1 = 0; i1 < sx1 / 2 + 1; i1++) {
            double k1 = (double)i1 / (sx1 * dx1);
            size_t q = 2 * (size_t)i1 + (size_t)n1 * i2;
            /* COMPLEX(KIND=4) traction */
            real t1r = F32(p1[q]), t1i = F32(p1[q + 1]);
            real t2r = F32(p2[q]), t2i = F32(p2[q + 1]);
            real t3r = F32(p3[q]), t3i = F32(p3[q + 1]);
            if (k1 == 0 && k2 == 0) continue; /* u_i = 0 */
            double beta = PI2 * sqrt(k1 * k1 + k2 * k2);
            double h = gamma / beta;
            for (int i3 = 0; i3 < sx3; i3++) {
                double k3 = wn(i3, sx3, dx3);
                double fi = (2 * beta) / ((PI2 * PI2) * (k3 * k3) + beta * beta);
                double temp = (1.0 / (2.0 * mu * beta * beta * beta)) * fi;
                double b1r = temp * t1r, b1i = temp * t1i, b2r = temp * t2r, b2i = temp * t2i;
                /* b3 = (beta p3 - i (1-alpha)(2pi k1 p1 + 2pi k2 p2)) / (2 alpha mu beta^4 (1+h)) */
                double qr = PI2 * k1 * t1r + PI2 * k2 * t2r, qi = PI2 * k1 * t1i + PI2 * k2 * t2i;
                double den = 2.0 * alpha * mu * beta * beta * beta * beta * (1 + h);
                double b3r = (beta * t3r + (1.0 - alpha) * qi) / den;
                double b3i = (beta * t3i - (1.0 - alpha) * qr) / den;
                /* tmp = alpha i beta 2pi b3 (1 - 1/alpha - i 2pi k3 fi) */
                double er = 1.0 - 1.0 / alpha, ei = -PI2 * k3 * fi;
                double gr = b3r * er - b3i * ei, gi = b3r * ei + b3i * er;
                double ab = alpha * beta * PI2;
                double tmpr = -ab * gi, tmpi = ab * gr;
                double v1r = tmpr * k1 * fi, v1i = tmpi * k1 * fi;
                double v2r = tmpr * k2 * fi, v2i = tmpi * k2 * fi;
                /* v3 = -alpha beta^2 b3 (1/alpha - i fi 2pi k3) */
                double hr = 1.0 / alpha, hi = -fi * PI2 * k3;
                double ab2 = -alpha * beta * beta;
                double v3r = ab2 * (b3r * hr - b3i * hi), v3i = ab2 * (b3r * hi + b3i * hr);
                /* common: alpha 2pi^2 (b1 k1 + b2 k2)(1 - i 2pi k3 fi) */
                double sr = b1r * k1 + b2r * k2, si = b1i * k1 + b2i * k2;
                double mr = 1.0, mi = -PI2 * k3 * fi;
                double cr = sr * mr - si * mi, ci = sr * mi + si * mr;
                double ap = alpha * (PI2 * PI2);
                double w1r = v1r + (-(2.0 * beta * beta * b1r) + ap * k1 * cr);
                double w1i = v1i + (-(2.0 * beta * beta * b1i) + ap * k1 * ci);
                double w2r = v2r + (-(2.0 * beta * beta * b2r) + ap * k2 * cr);
                double w2i = v2i + (-(2.0 * beta * beta * b2i) + ap * k2 * ci);
                /* u3 = v3 fi + alpha beta 2pi (k1 b1 + k2 b2) 2pi k3 fi */
                double ak = alpha * beta * PI2 * PI2 * k3 * fi;
                double w3r = v3r * fi + ak * sr, w3i = v3i * fi + ak * si;
                size_t o = IDX3(2 * i1, i2, i3, n1, sx2);
                u1[o] = u1[o] + F32(w1r); u1[o + 1] = u1[o + 1] + F32(w1i);
                u2[o] = u2[o] + F32(w2r); u2[o + 1] = u2[o + 1] + F32(w2i);
                u3[o] = u3[o] + F32(w3r); u3[o + 1] = u3[o + 1] + F32(w3i);
            }
        }
    }
}

/* greenfunctioncowling, src/green.f90:1008-1129 (CPU branch) */
int orc_greenfunctioncowling(real *c1, real *c2, real *c3, real *t1, real *t2, real *t3,
                             int sx1, int sx2, int sx3, double dx1, double dx2, double dx3,
                             double lambda, double mu, double gamma)
{
    size_t np = (size_t)(sx1 + 2) * sx2;
    real *p1 = calloc(np, sizeof(real)), *p2 = calloc(np, sizeof(real)), *p3 = calloc(np, sizeof(real));
    if (!p1 || !p2 || !p3) { free(p1); free(p2); free(p3); return ORC_ERR_NOMEM; }
    orc_fft3(c1, sx1, sx2, sx3, dx1, dx2, dx3, -1);
    orc_fft3(c2, sx1, sx2, sx3, dx1, dx2, dx3, -1);
    orc_fft3(c3, sx1, sx2, sx3, dx1, dx2, dx3, -1);
    orc_fft2(t1, sx1, sx2, dx1, dx2, -1);
    orc_fft2(t2, sx1, sx2, dx1, dx2, -1);
    orc_fft2(t3, sx1, sx2, dx1, dx2, -1);
    orc_elasticresponse(lambda, mu, c1, c2, c3, sx1, sx2, sx3, dx1, dx2, dx3);
    orc_surfacetractioncowling(lambda, mu, gamma, c1, c2, c3, sx1, sx2, sx3, dx1, dx2, dx3, p1, p2, p3);
    for (size_t q = 0; q < np; q++) {
        p1[q] = t1[q] - p1[q]; p2[q] = t2[q] - p2[q]; p3[q] = t3[q] - p3[q];
    }
    orc_cerrutimodified(p1, p2, p3, lambda, mu, gamma, c1, c2, c3, sx1, sx2, sx3, dx1, dx2, dx3);
    orc_fft3(c1, sx1, sx2, sx3, dx1, dx2, dx3, +1);
    orc_fft3(c2, sx1, sx2, sx3, dx1, dx2, dx3, +1);
    orc_fft3(c3, sx1, sx2, sx3, dx1, dx2, dx3, +1);
    orc_fft2(t1, sx1, sx2, dx1, dx2, +1);
    orc_fft2(t2, sx1, sx2, dx1, dx2, +1);
    orc_fft2(t3, sx1, sx2, dx1, dx2, +1);
    free(p1); free(p2); free(p3);
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* coseismic sources                                                   */
/* ------------------------------------------------------------------ */

/* source, src/elastic3d.f90:2064-2252 (CPU branch).  L = width and
 * W = length as passed by dislocations (src/relax.f90:1148-1152). */
void orc_source(double mu, double s, double x, double y, double z, double L, double W,
                double strike, double dip, double rake, double beta, int sx1, int sx2, int sx3,
                double dx1, double dx2, double dx3, real *f1, real *f2, real *f3, real *t1,
                real *t2, real *t3)
{
    const int n1 = sx1 + 2;
    double cstrike = cos(strike), sstrike = sin(strike), cdip = cos(dip), sdip = sin(dip);
    double cr = cos(rake), sr = sin(rake), scale = -mu * s;
    double Wp = W * (1.0 + 2.0 * beta) / 2.0, Lp = L * (1.0 + 2.0 * beta) / 2.0;
    double x2r0 = cstrike * x - sstrike * y;
    double xr = cdip * x2r0 - sdip * z, yr = sstrike * x + cstrike * y, zr = sdip * x2r0 + cdip * z;
    double mlw = Lp > Wp ? Lp : Wp;
    const double w701s = (double)7.01f; /* default-real literal, :2139 */

    /* equivalent surface traction (i3 = 1) */
    for (int i2 = 1; i2 <= sx2; i2++) {
        for (int i1 = 1; i1 <= sx1; i1++) {
            double x1, x2, x3;
            shiftedcoordinates(i1, i2, 1, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &x3);
            if (fabs(x1 - x) > mlw || fabs(x2 - y) > mlw) continue;
            double x2r = cstrike * x1 - sstrike * x2;
            double x1s = cdip * x2r - sdip * x3, x1i = cdip * x2r + sdip * x3;
            if (fabs(x1s - xr) > w701s * dx1 && fabs(x1i - xr) > w701s * dx1) continue;
            double x2s = sstrike * x1 + cstrike * x2;
            double x3s = sdip * x2r + cdip * x3, x3i = -sdip * x2r + cdip * x3;
            double temp1 = gauss(x1s - xr, dx1), temp2 = omega((x2s - yr) / W, beta);
            double temp3 = omega((x3s - zr) / L, beta);
            double sourc = temp1 * temp2 * temp3;
            temp1 = gauss(x1i - xr, dx1);
            temp3 = omega((x3i + zr) / L, beta);
            sourc = sourc + temp1 * temp2 * temp3;
            double n[3] = {+cdip * cstrike * sourc, -cdip * sstrike * sourc, -sdip * sourc};
            double b[3];
            b[0] = sstrike * cr + cstrike * sdip * sr;
            b[1] = cstrike * cr - sstrike * sdip * sr;
            b[2] = +cdip * sr;
            double mb[3] = {mu * s * b[0], mu * s * b[1], mu * s * b[2]};
            otensor m = sdyad(n, mb);
            size_t q = (size_t)(i1 - 1) + (size_t)n1 * (i2 - 1);
            t1[q] = t1[q] + m.s13;
            t2[q] = t2[q] + m.s23;
            t3[q] = t3[q] + m.s33;
        }
    }

    /* equivalent body-force density */
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3 / 2; i3++) {
        double x1, x2, x3;
        shiftedcoordinates(1, 1, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &x3);
        if (fabs(x3 - z) > Lp && fabs(x3 + z) > Lp) continue;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &x3);
                if (fabs(x1 - x) > mlw || fabs(x2 - y) > mlw) continue;
                double x2r = cstrike * x1 - sstrike * x2;
                double x1s = cdip * x2r - sdip * x3, x1i = cdip * x2r + sdip * x3;
                if (fabs(x1s - xr) > 7.01 * dx1 && fabs(x1i - xr) > 7.01 * dx1) continue;
                double x2s = sstrike * x1 + cstrike * x2;
                double x3s = sdip * x2r + cdip * x3, x3i = -sdip * x2r + cdip * x3;
                double temp1 = gauss(x1s - xr, dx1), temp2 = omega((x2s - yr) / W, beta);
                double temp3 = omega((x3s - zr) / L, beta);
                double sourc = scale * gaussp(x1s - xr, dx1) * temp2 * temp3;
                double dblcp = scale / W * temp1 * omegap((x2s - yr) / W, beta) * temp3;
                double dipcs = scale / L * temp1 * temp2 * omegap((x3s - zr) / L, beta);
                temp1 = gauss(x1i - xr, dx1);
                temp3 = omega((x3i + zr) / L, beta);
                double image = scale * gaussp(x1i - xr, dx1) * temp2 * temp3;
                double cplei = scale / W * temp1 * omegap((x2s - yr) / W, beta) * temp3;
                /* dipci (:2189-2191) is computed by the reference but never used */
                size_t o = IDX3(i1 - 1, i2 - 1, i3 - 1, n1, sx2);
                if (2.01 * DEG2RAD > dip) {
                    f1[o] = (real)(f1[o] + cr * sstrike * (sourc + image) + cr * cdip * cstrike * (dblcp + cplei));
                    f2[o] = (real)(f2[o] + cr * cstrike * (sourc + image) - cr * cdip * sstrike * (dblcp + cplei));
                    f3[o] = (real)(f3[o] - cr * sdip * (dblcp - cplei));
                } else {
                    f1[o] = (real)(f1[o] + cr * sstrike * (sourc) + cr * cdip * cstrike * (dblcp));
                    f2[o] = (real)(f2[o] + cr * cstrike * (sourc) - cr * cdip * sstrike * (dblcp));
                    f3[o] = (real)(f3[o] - cr * sdip * (dblcp));
                }
                f1[o] = (real)(f1[o] + cdip * sr * cstrike * dipcs + sdip * sr * cstrike * sourc);
                f2[o] = (real)(f2[o] - cdip * sr * sstrike * dipcs - sdip * sr * sstrike * sourc);
                f3[o] = (real)(f3[o] + cdip * sr * sourc - sdip * sr * dipcs);
            }
        }
    }
}

/* momentdensityshear, src/elastic3d.f90:2661-2750; sx3 = physical layers */
void orc_momentdensityshear(double mu, double slip, double x, double y, double z, double L,
                            double W, double strike, double dip, double rake, double beta,
                            int sx1, int sx2, int sx3, double dx1, double dx2, double dx3,
                            otensor *sig)
{
    real rmu = (real)2 * F32(mu);
    double cstrike = cos(strike), sstrike = sin(strike), cdip = cos(dip), sdip = sin(dip);
    double cr = cos(rake), sr = sin(rake);
    double Wp = W * (1.0 + 2.0 * beta) / 2.0, Lp = L * (1.0 + 2.0 * beta) / 2.0;
    double x2r0 = cstrike * x - sstrike * y;
    double xr = cdip * x2r0 - sdip * z, yr = sstrike * x + cstrike * y, zr = sdip * x2r0 + cdip * z;
    const double w701s = (double)7.01f; /* default-real literal, :2712 */
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        double x3 = (double)(i3 - 1) * dx3;
        if (fabs(x3 - z) > Lp) continue;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double x1, x2, dum;
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &dum);
                if (fabs(x1 - x) > Wp || fabs(x2 - y) > Wp) continue;
                double x2r = cstrike * x1 - sstrike * x2;
                double x1s = cdip * x2r - sdip * x3, x1i = cdip * x2r + sdip * x3;
                if (fabs(x1s - xr) > w701s * dx1 && fabs(x1i - xr) > w701s * dx1) continue;
                double x2s = sstrike * x1 + cstrike * x2;
                double x3s = sdip * x2r + cdip * x3, x3i = -sdip * x2r + cdip * x3;
                double temp1 = gauss(x1s - xr, dx1), temp2 = omega((x2s - yr) / W, beta);
                double temp3 = omega((x3s - zr) / L, beta);
                double aperture = temp1 * temp2 * temp3;
                temp1 = gauss(x1i - xr, dx1);
                temp3 = omega((x3i + zr) / L, beta);
                aperture = aperture + temp1 * temp2 * temp3;
                double n[3] = {+cdip * cstrike * aperture, -cdip * sstrike * aperture, -sdip * aperture};
                double s[3] = {sstrike * cr + cstrike * sdip * sr, cstrike * cr - sstrike * sdip * sr, +cdip * sr};
                double ss[3] = {slip * s[0], slip * s[1], slip * s[2]};
                otensor Ei = sdyad(n, ss);
                size_t o = IDX3(i1 - 1, i2 - 1, i3 - 1, sx1, sx2);
                sig[o] = tplus(sig[o], ttimes(rmu, Ei));
            }
        }
    }
}

/* traction, src/elastic3d.f90:2517-2590 */
void orc_traction(double mu, const relax_event *e, int sx1, int sx2, double dx1, double dx2,
                  double t, double Dt, real *t3, int rate)
{
    (void)mu;
    const int n1 = sx1 + 2;
    for (int i = 0; i < e->nl; i++) {
        const relax_source *l = &e->l[i];
        double x = l->x, y = l->y, period = l->period, phi = l->phase, L = l->length, W = l->width;
        double beta = l->beta;
        double Lp = L * (1.0 + 2.0 * beta) / 2.0, Wp = W * (1.0 + 2.0 * beta) / 2.0;
        if (Lp == 0 || Wp == 0) continue;
        double m = Lp > Wp ? Lp : Wp;
        for (int i2 = 1; i2 <= sx2; i2++)
            for (int i1 = 1; i1 <= sx1; i1++) {
                double x1, x2, x3;
                shiftedcoordinates(i1, i2, 1, sx1, sx2, 1, dx1, dx2, 1.0e8, &x1, &x2, &x3);
                if (fabs(x1 - x) > m || fabs(x2 - y) > m) continue;
                double amp = omega((x1 - x) / L, beta) * omega((x2 - y) / W, beta) * l->slip;
                size_t q = (size_t)(i1 - 1) + (size_t)n1 * (i2 - 1);
                if (rate) {
                    if (period != 0)
                        t3[q] = (real)(t3[q] - amp * (sin(2 * PI * (t + Dt) / period + phi) -
                                                      sin(2 * PI * t / period + phi)) / Dt);
                } else {
                    if (period == 0) t3[q] = (real)(t3[q] - amp);
                    else t3[q] = (real)(t3[q] - amp * sin(2 * PI * t / period + phi));
                }
            }
    }
}

/* ------------------------------------------------------------------ */
/* the time loop, src/relax.f90:555-890 + integrationstep :1420-1452    */
/* ------------------------------------------------------------------ */
/* ------------------------------------------------------------------ */
/* Okada (1992), Bull. Seism. Soc. Am. 82(2), 1018-1040: displacement of a
 * rectangular dislocation in a half-space, the space-domain solution RELAX
 * adds for small coseismic sources (dislocations_disp, src/relax.f90:
 * 1298-1349; okada / grnfct_okada, src/okada/green_space.f90:29-144, over
 * the reference's DC3D, src/okada/dc3d.f).  Restated from the paper's
 * Table 6: f^A, f^B, f^C per corner, Chinnery's alternating sum over the
 * corners, the real source (d = c + z) and its image (d = c - z).  FP64.
 * ------------------------------------------------------------------ */
typedef struct {
    double xi, et, q, r, yt, dt, th, lx, le, x11, y11, x32, y32;
} okc;

static void okada_c(double xi, double et, double q, double sd, double cd, int kx, int ke, okc *c)
{
    if (fabs(xi) < 1e-6) xi = 0;
    if (fabs(et) < 1e-6) et = 0;
    if (fabs(q) < 1e-6) q = 0;
    c->xi = xi; c->et = et; c->q = q;
    c->r = sqrt(xi * xi + et * et + q * q);
    c->yt = et * cd + q * sd;
    c->dt = et * sd - q * cd;
    c->th = q == 0 ? 0 : atan(xi * et / (q * c->r));
    if (kx) { c->lx = -log(c->r - xi); c->x11 = 0; c->x32 = 0; }
    else {
        c->lx = log(c->r + xi);
        c->x11 = 1 / (c->r * (c->r + xi));
        c->x32 = (2 * c->r + xi) / (c->r * c->r * c->r * (c->r + xi) * (c->r + xi));
    }
    if (ke) { c->le = -log(c->r - et); c->y11 = 0; c->y32 = 0; }
    else {
        c->le = log(c->r + et);
        c->y11 = 1 / (c->r * (c->r + et));
        c->y32 = (2 * c->r + et) / (c->r * c->r * c->r * (c->r + et) * (c->r + et));
    }
}

/* f^A, f^B, f^C of Table 6 for the dislocation (u1, u2, u3) */
static void okada_f(const okc *c, double z, double al, double sd, double cd, const double U[3], int part,
                    double f[3])
{
    const double a1 = (1 - al) / 2, a2 = al / 2, a3 = (1 - al) / al, a4 = 1 - al;
    const double xi = c->xi, et = c->et, q = c->q, R = c->r, yt = c->yt, dt = c->dt, th = c->th;
    f[0] = f[1] = f[2] = 0;
    if (part == 0) {
        f[0] = U[0] * (th / 2 + a2 * xi * q * c->y11) + U[1] * (a2 * q / R) +
               U[2] * (-a1 * c->le - a2 * q * q * c->y11);
        f[1] = U[0] * (a2 * q / R) + U[1] * (th / 2 + a2 * et * q * c->x11) +
               U[2] * (-a1 * c->lx - a2 * q * q * c->x11);
        f[2] = U[0] * (a1 * c->le - a2 * q * q * c->y11) + U[1] * (a1 * c->lx - a2 * q * q * c->x11) +
               U[2] * (th / 2 - a2 * q * (et * c->x11 + xi * c->y11));
    } else if (part == 1) {
        const double Rd = R + dt;
        double I3, I4;
        if (cd != 0) {
            const double X = sqrt(xi * xi + q * q);
            I4 = xi == 0 ? 0
                         : sd / cd * xi / Rd +
                               2 / (cd * cd) * atan((et * (X + q * cd) + X * (R + X) * sd) / (xi * (R + X) * cd));
            I3 = yt / (cd * Rd) - (c->le - sd * log(Rd)) / (cd * cd);
        } else {
            I3 = 0.5 * (et / Rd + yt * q / (Rd * Rd) - c->le);
            I4 = 0.5 * xi * yt / (Rd * Rd);
        }
        const double I1 = -xi / Rd * cd - I4 * sd, I2 = log(Rd) + I3 * sd;
        f[0] = U[0] * (-xi * q * c->y11 - th - a3 * I1 * sd) + U[1] * (-q / R + a3 * I3 * sd * cd) +
               U[2] * (q * q * c->y11 - a3 * I3 * sd * sd);
        f[1] = U[0] * (-q / R + a3 * yt / Rd * sd) + U[1] * (-et * q * c->x11 - th - a3 * xi / Rd * sd * cd) +
               U[2] * (q * q * c->x11 + a3 * xi / Rd * sd * sd);
        f[2] = U[0] * (q * q * c->y11 - a3 * I2 * sd) + U[1] * (q * q * c->x11 + a3 * I4 * sd * cd) +
               U[2] * (q * (et * c->x11 + xi * c->y11) - th - a3 * I4 * sd * sd);
    } else {
        const double cb = dt + z, R3 = R * R * R, h = q * cd - z;
        const double Z32 = sd / R3 - h * c->y32;
        f[0] = U[0] * (a4 * xi * c->y11 * cd - al * xi * q * Z32) +
               U[1] * (a4 * cd / R - q * c->y11 * sd - al * cb * q / R3) +
               U[2] * (-a4 * (sd / R + q * c->y11 * cd) - al * (z * c->y11 - q * q * Z32));
        f[1] = U[0] * (a4 * (cd / R + 2 * q * c->y11 * sd) - al * cb * q / R3) +
               U[1] * (a4 * yt * c->x11 - al * cb * et * q * c->x32) +
               U[2] * (a4 * 2 * xi * c->y11 * sd + dt * c->x11 - al * cb * (c->x11 - q * q * c->x32));
        f[2] = U[0] * (a4 * q * c->y11 * cd - al * (cb * et / R3 - z * c->y11 + xi * xi * Z32)) +
               U[1] * (-dt * c->x11 - xi * c->y11 * sd - al * cb * (c->x11 - q * q * c->x32)) +
               U[2] * (a4 * (yt * c->x11 + xi * c->y11 * cd) + al * q * (cb * et * c->x32 + xi * Z32));
    }
}

/* displacement at (x, y, z <= 0) in the fault frame; 0, or 1 on a fault edge */
static int okada_dc(double al, double x, double y, double z, double c0, double dipd, double L, double W,
                    const double U[3], double u[3])
{
    double sd = sin(dipd * 0.01745329251994329547437168059786927);
    double cd = cos(dipd * 0.01745329251994329547437168059786927);
    if (fabs(cd) < 1e-6) { cd = 0; sd = sd > 0 ? 1 : -1; }
    double xi[2] = {x, x - L};
    for (int i = 0; i < 2; i++) if (fabs(xi[i]) < 1e-6) xi[i] = 0;
    u[0] = u[1] = u[2] = 0;
    for (int img = 0; img < 2; img++) {
        const double d = img ? c0 - z : c0 + z;
        const double p = y * cd + d * sd;
        double q = y * sd - d * cd;
        double et[2] = {p + W, p};
        if (fabs(q) < 1e-6) q = 0;
        for (int i = 0; i < 2; i++) if (fabs(et[i]) < 1e-6) et[i] = 0;
        if (q == 0 && ((xi[0] * xi[1] <= 0 && et[0] * et[1] == 0) || (et[0] * et[1] <= 0 && xi[0] * xi[1] == 0))) {
            u[0] = u[1] = u[2] = 0;
            return 1;
        }
        int kx[2] = {0, 0}, ke[2] = {0, 0};
        if (xi[0] < 0 && sqrt(xi[1] * xi[1] + et[0] * et[0] + q * q) + xi[1] < 1e-6) kx[0] = 1;
        if (xi[0] < 0 && sqrt(xi[1] * xi[1] + et[1] * et[1] + q * q) + xi[1] < 1e-6) kx[1] = 1;
        if (et[0] < 0 && sqrt(xi[0] * xi[0] + et[1] * et[1] + q * q) + et[1] < 1e-6) ke[0] = 1;
        if (et[0] < 0 && sqrt(xi[1] * xi[1] + et[1] * et[1] + q * q) + et[1] < 1e-6) ke[1] = 1;
        for (int j = 0; j < 2; j++)
            for (int i = 0; i < 2; i++) {
                okc c;
                okada_c(xi[i], et[j], q, sd, cd, kx[j], ke[i], &c);
                if (c.r == 0) continue;
                double w[3], fa[3];
                okada_f(&c, z, al, sd, cd, U, 0, fa);
                if (!img) {
                    w[0] = -fa[0];
                    w[1] = -fa[1] * cd + fa[2] * sd;
                    w[2] = -fa[1] * sd - fa[2] * cd;
                } else {
                    double fb[3], fc[3];
                    okada_f(&c, z, al, sd, cd, U, 1, fb);
                    okada_f(&c, z, al, sd, cd, U, 2, fc);
                    w[0] = fa[0] + fb[0] + z * fc[0];
                    w[1] = (fa[1] + fb[1] + z * fc[1]) * cd - (fa[2] + fb[2] + z * fc[2]) * sd;
                    w[2] = (fa[1] + fb[1] - z * fc[1]) * sd + (fa[2] + fb[2] - z * fc[2]) * cd;
                }
                const double sg = (i + j) % 2 ? -1.0 : 1.0;
                for (int k = 0; k < 3; k++) u[k] += sg * w[k] / (2 * M_PI);
            }
    }
    return 0;
}

/* monitorstressfield / monitorfield, src/elastic3d.f90:3404-3762: the field f
 * (nc = 6 tensor components or nc = 1 scalar, each sx1 x sx2 x sx3 floats,
 * x1 fastest; sx3 the stored half) sampled on the (px2+1) x (px3+1) points of
 * a plane (L along dip, W along strike, as the reference names them); out:
 * 5 + nc doubles per point (x1, x2, x3, yr, zr, values) or NULL to size. */
static double orc_sinc(double x)
{
    const double pi = 3.141592653589793115997963468544185161;
    return x != 0 ? sin(pi * x) / (pi * x) : 1.0;
}

void orc_monitor_plane(const float *f, int nc, int sx1, int sx2, int sx3, double dx1, double dx2, double dx3,
                       double x, double y, double z, double L, double W, double strike, double dip, double beta,
                       int *px2_out, int *px3_out, double *out)
{
    const double cstrike = cos(strike), sstrike = sin(strike), cdip = cos(dip), sdip = sin(dip);
    const double Wp = W * (1.0 + 2.0 * beta), Lp = L * (1.0 + 2.0 * beta);
    const int px3 = orc_fix(Lp / dx3), px2 = orc_fix(Wp / dx2);
    const size_t nh = (size_t)sx1 * sx2 * sx3;
    *px2_out = px2;
    *px3_out = px3;
    if (!out) return;
    for (int j3 = 1; j3 <= px3 + 1; j3++)
        for (int j2 = 1; j2 <= px2 + 1; j2++) {
            /* ref2local */
            const double xa = cstrike * x - sstrike * y;
            const double xr = cdip * xa - sdip * z;
            double yr = sstrike * x + cstrike * y;
            double zr = sdip * xa + cdip * z;
            yr = (double)((float)yr + (float)(((double)j2 - (double)px2 / 2.0 - 1.0) * dx2));
            zr = (double)((float)zr + (float)(((double)j3 - (double)px3 / 2.0 - 1.0) * dx3));
            /* local2ref */
            const double x2p = cdip * xr + sdip * zr;
            const double x1 = cstrike * x2p + sstrike * yr;
            const double x2 = -sstrike * x2p + cstrike * yr;
            const double x3 = -sdip * xr + cdip * zr;
            double *o = out + (size_t)(5 + nc) * ((size_t)(j2 - 1) + (size_t)(px2 + 1) * (j3 - 1));
            o[0] = x1; o[1] = x2; o[2] = x3; o[3] = yr; o[4] = zr;
            float lsig[6] = {0, 0, 0, 0, 0, 0};
            double value = 0;
            if (!(x1 > (double)(sx1 / 2 - 1) * dx1 || x1 < -(double)(sx1 / 2) * dx1 ||
                  x2 > (double)(sx2 / 2 - 1) * dx2 || x2 < -(double)(sx2 / 2) * dx2 ||
                  x3 > (double)(sx3 - 1) * dx3 || x3 < 0)) {
                /* sampletensor / sample */
                const int i = (sx1 + orc_fix(x1 / dx1)) % sx1 + 1;
                const int j = (sx2 + orc_fix(x2 / dx2)) % sx2 + 1;
                const int k = orc_fix(x3 / dx3) + 1;
                const double xs = (double)(i <= sx1 / 2 ? i - 1 : i - sx1 - 1) * dx1;
                const double ys = (double)(j <= sx2 / 2 ? j - 1 : j - sx2 - 1) * dx2;
                const double zs = (double)(k <= sx3 ? k - 1 : k - 2 * sx3 - 1) * dx3;
                const double EPS = (double)1e-2f;
                if (fabs(xs - x1) < EPS * dx1 && fabs(ys - x2) < EPS * dx2 && fabs(zs - x3) < EPS * dx3) {
                    const size_t c = (size_t)(i - 1) + (size_t)sx1 * ((size_t)(j - 1) + (size_t)sx2 * (k - 1));
                    if (nc == 1) value = f[c];
                    else for (int m = 0; m < 6; m++) lsig[m] = f[m * nh + c];
                } else {
                    double sum = 0;
                    for (int l3 = -2; l3 <= 2; l3++) {
                        if (k + l3 <= 0 || k + l3 > sx3) continue;
                        const int i3p = l3 >= 0 ? (k - 1 + l3) % sx3 + 1 : (sx3 + k - 1 + l3) % sx3 + 1;
                        for (int l2 = -2; l2 <= 2; l2++) {
                            const int i2p = l2 >= 0 ? (j - 1 + l2) % sx2 + 1 : (sx2 + j - 1 + l2) % sx2 + 1;
                            for (int l1 = -2; l1 <= 2; l1++) {
                                const int i1p = l1 >= 0 ? (i - 1 + l1) % sx1 + 1 : (sx1 + i - 1 + l1) % sx1 + 1;
                                const double weight = orc_sinc(((xs + l1 * dx1) - x1) / dx1) * dx1 *
                                                      orc_sinc(((ys + l2 * dx2) - x2) / dx2) * dx2 *
                                                      orc_sinc(((zs + l3 * dx3) - x3) / dx3) * dx3;
                                const size_t c = (size_t)(i1p - 1) +
                                                 (size_t)sx1 * ((size_t)(i2p - 1) + (size_t)sx2 * (i3p - 1));
                                if (nc == 1) {
                                    value = value + weight * f[c];
                                } else {
                                    const float w = (float)weight;
                                    for (int m = 0; m < 6; m++) lsig[m] = lsig[m] + w * f[m * nh + c];
                                }
                                sum = sum + weight;
                            }
                        }
                    }
                    if (sum > (double)1e-6f) {
                        if (nc == 1) {
                            value = value / sum;
                        } else {
                            const float r = (float)(1.0 / sum);
                            for (int m = 0; m < 6; m++) lsig[m] = r * lsig[m];
                        }
                    }
                }
            }
            if (nc == 1) o[5] = value;
            else for (int m = 0; m < 6; m++) o[5 + m] = lsig[m];
        }
}

/* okada, src/okada/green_space.f90:29-105: source in the input convention
 * (north, east, depth of the top edge; degrees), receiver (north, east,
 * depth); displacement with x3 down */
void orc_okada(double lambda, double mu, double slip, double opening, double x1, double x2, double x3, double width,
               double length, double strike, double dip, double rake, double xr, double yr, double zr, double *d)
{
    const double rad = 0.01745329251994329547437168059786927;
    const double cs = cos(strike * rad), ss = sin(strike * rad);
    const double U[3] = {slip * cos(rake * rad), slip * sin(rake * rad), opening};
    double u[3];
    if (okada_dc((lambda + mu) / (lambda + 2 * mu), (xr - x1) * cs + (yr - x2) * ss, (xr - x1) * ss - (yr - x2) * cs,
                 -zr, x3, dip, length, width, U, u)) {
        d[0] = d[1] = d[2] = 0;
        return;
    }
    d[0] = u[0] * cs + u[1] * ss;
    d[1] = u[0] * ss - u[1] * cs;
    d[2] = -u[2];
}

/* grnfct_okada, src/okada/green_space.f90:114-144, into the padded v */
static void grnfct_okada(double lambda, double mu, double slip, double opening, double x, double y, double z,
                         double width, double length, double strike, double dip, double rake, int sx1, int sx2,
                         int sx3h, double dx1, double dx2, double dx3, real *u1, real *u2, real *u3)
{
#pragma omp parallel for schedule(static)
    for (int i3 = 0; i3 < sx3h; i3++)
        for (int i2 = 0; i2 < sx2; i2++)
            for (int i1 = 0; i1 < sx1; i1++) {
                const double x1 = (i1 < sx1 / 2 ? i1 : i1 - sx1) * dx1, x2 = (i2 < sx2 / 2 ? i2 : i2 - sx2) * dx2;
                double d[3];
                orc_okada(lambda, mu, slip, opening, x, y, z, width, length, strike, dip, rake, x1, x2, i3 * dx3, d);
                const size_t o = (size_t)i1 + (size_t)(sx1 + 2) * (i2 + (size_t)sx2 * i3);
                u1[o] += (real)d[0];
                u2[o] += (real)d[1];
                u3[o] += (real)d[2];
            }
}

/* the input-file form of a configured source: wangconvention and the
 * rotation (src/input.f90:1780-1822) undone */
static void input_form(const relax_config *c, const relax_source *s, double *x, double *y, double *z,
                       double *strike, double *dip, double *rake)
{
    const double rad = 0.01745329251994329547437168059786927;
    const double st = s->strike - c->rot * rad, a = -c->rot * rad;
    const double xx = s->x * cos(a) + s->y * sin(a), yy = -s->x * sin(a) + s->y * cos(a);
    *x = xx + c->x0 + s->length / 2 * sin(st) - s->width / 2 * sin(s->dip) * cos(st);
    *y = yy + c->y0 + s->length / 2 * cos(st) + s->width / 2 * sin(s->dip) * sin(st);
    *z = s->z - s->width / 2 * cos(s->dip);
    *strike = -90 - st / rad;
    *dip = 90 - s->dip / rad;
    *rake = s->rake / rad;
}

typedef struct orc_state {
    relax_config cfg;
    int sx1, sx2, sx3, sx3h;
    size_t nv, nu, nt, n2;
    real *v[3], *u[3], *t[3], *gamma;
    otensor *tau, *sig, *moment;
    otensor *eps, *epsdot;          /* transient strain and its rate (with a transient structure) */
    relax_slippatch **patch;
    double time;
    int i, e, oi;
} orc_state;

static void integrationstep(double tm, double *Dt, double t, int oi, double odt, int skip,
                            double tscale, const relax_event *events, int e, int ne)
{
    *Dt = tm / 10.0;
    if (0 == skip) {
        if ((t + *Dt) >= ((double)oi * odt) - *Dt * 0.04) *Dt = (double)oi * odt - t;
    } else {
        *Dt = *Dt * tscale;
        if (e < ne - 1)
            if ((t + *Dt - events[e + 1].time) >= 0.0) *Dt = events[e + 1].time - t;
    }
}

/* ------------------------------------------------------------------ */
/* DC3D of Okada (1992), src/okada/dc3d.f (displacement rows only), as */
/* src/okada/green_space.f90:14-89 (okada) calls it: REAL*4 arguments, */
/* REAL*8 arithmetic inside, REAL*4 results.  A second restatement of  */
/* the half-space solution, from the reference's own routine, that     */
/* checks the oracle's orc_okada and the library's okada.cuh.          */
/* ------------------------------------------------------------------ */
typedef struct dc3d_c0 { double alp1, alp2, alp3, alp4, alp5, sd, cd, sdsd, cdcd, sdcd; } dc3d_c0;
typedef struct dc3d_c2 { double xi2, et2, q2, r, r2, r3, r5, y, d, tt, alx, ale, x11, y11, x32, y32; } dc3d_c2;

/* DCCON0, dc3d.f:509-545 */
static void dc3d_con0(double alpha, double dip, dc3d_c0 *c)
{
    const double pi2 = 6.283185307179586;
    c->alp1 = (1.0 - alpha) / 2.0;
    c->alp2 = alpha / 2.0;
    c->alp3 = (1.0 - alpha) / alpha;
    c->alp4 = 1.0 - alpha;
    c->alp5 = alpha;
    const double p18 = pi2 / 360.0;
    c->sd = sin(dip * p18);
    c->cd = cos(dip * p18);
    if (fabs(c->cd) < 1e-6) {
        c->cd = 0.0;
        if (c->sd > 0.0) c->sd = 1.0;
        if (c->sd < 0.0) c->sd = -1.0;
    }
    c->sdsd = c->sd * c->sd;
    c->cdcd = c->cd * c->cd;
    c->sdcd = c->sd * c->cd;
}

/* DCCON2, dc3d.f:596-665 (the quantities the displacement rows read) */
static void dc3d_con2(double xi, double et, double q, double sd, double cd, int kxi, int ket, dc3d_c2 *c)
{
    if (fabs(xi) < 1e-6) xi = 0.0;
    if (fabs(et) < 1e-6) et = 0.0;
    if (fabs(q) < 1e-6) q = 0.0;
    c->xi2 = xi * xi;
    c->et2 = et * et;
    c->q2 = q * q;
    c->r2 = c->xi2 + c->et2 + c->q2;
    c->r = sqrt(c->r2);
    if (c->r == 0.0) return;
    c->r3 = c->r * c->r2;
    c->r5 = c->r3 * c->r2;
    c->y = et * cd + q * sd;
    c->d = et * sd - q * cd;
    c->tt = (q == 0.0) ? 0.0 : atan(xi * et / (q * c->r));
    if (kxi == 1) {
        c->alx = -log(c->r - xi);
        c->x11 = 0.0;
        c->x32 = 0.0;
    } else {
        const double rxi = c->r + xi;
        c->alx = log(rxi);
        c->x11 = 1.0 / (c->r * rxi);
        c->x32 = (c->r + rxi) * c->x11 * c->x11 / c->r;
    }
    if (ket == 1) {
        c->ale = -log(c->r - et);
        c->y11 = 0.0;
        c->y32 = 0.0;
    } else {
        const double ret = c->r + et;
        c->ale = log(ret);
        c->y11 = 1.0 / (c->r * ret);
        c->y32 = (c->r + ret) * c->y11 * c->y11 / c->r;
    }
}

/* UA, UB, UC, dc3d.f:200-508: the displacement rows u(1..3) */
static void dc3d_ua(double xi, double et, double q, const double disl[3], const dc3d_c0 *k, const dc3d_c2 *c,
                    double u[3])
{
    const double pi2 = 6.283185307179586;
    const double qx = q * c->x11, qy = q * c->y11;
    double du[3];
    u[0] = u[1] = u[2] = 0.0;
    if (disl[0] != 0.0) {
        du[0] = c->tt / 2.0 + k->alp2 * xi * qy;
        du[1] = k->alp2 * q / c->r;
        du[2] = k->alp1 * c->ale - k->alp2 * q * qy;
        for (int i = 0; i < 3; i++) u[i] = u[i] + disl[0] / pi2 * du[i];
    }
    if (disl[1] != 0.0) {
        du[0] = k->alp2 * q / c->r;
        du[1] = c->tt / 2.0 + k->alp2 * et * qx;
        du[2] = k->alp1 * c->alx - k->alp2 * q * qx;
        for (int i = 0; i < 3; i++) u[i] = u[i] + disl[1] / pi2 * du[i];
    }
    if (disl[2] != 0.0) {
        du[0] = -k->alp1 * c->ale - k->alp2 * q * qy;
        du[1] = -k->alp1 * c->alx - k->alp2 * q * qx;
        du[2] = c->tt / 2.0 - k->alp2 * (et * qx + xi * qy);
        for (int i = 0; i < 3; i++) u[i] = u[i] + disl[2] / pi2 * du[i];
    }
}

static void dc3d_ub(double xi, double et, double q, const double disl[3], const dc3d_c0 *k, const dc3d_c2 *c,
                    double u[3])
{
    const double pi2 = 6.283185307179586;
    const double rd = c->r + c->d, sd = k->sd, cd = k->cd;
    double ai3, ai4;
    if (cd != 0.0) {
        if (xi == 0.0) {
            ai4 = 0.0;
        } else {
            const double x = sqrt(c->xi2 + c->q2);
            ai4 = 1.0 / k->cdcd *
                  (xi / rd * k->sdcd + 2.0 * atan((et * (x + q * cd) + x * (c->r + x) * sd) / (xi * (c->r + x) * cd)));
        }
        ai3 = (c->y * cd / rd - c->ale + sd * log(rd)) / k->cdcd;
    } else {
        const double rd2 = rd * rd;
        ai3 = (et / rd + c->y * q / rd2 - c->ale) / 2.0;
        ai4 = xi * c->y / rd2 / 2.0;
    }
    const double ai1 = -xi / rd * cd - ai4 * sd;
    const double ai2 = log(rd) + ai3 * sd;
    const double qx = q * c->x11, qy = q * c->y11;
    double du[3];
    u[0] = u[1] = u[2] = 0.0;
    if (disl[0] != 0.0) {
        du[0] = -xi * qy - c->tt - k->alp3 * ai1 * sd;
        du[1] = -q / c->r + k->alp3 * c->y / rd * sd;
        du[2] = q * qy - k->alp3 * ai2 * sd;
        for (int i = 0; i < 3; i++) u[i] = u[i] + disl[0] / pi2 * du[i];
    }
    if (disl[1] != 0.0) {
        du[0] = -q / c->r + k->alp3 * ai3 * k->sdcd;
        du[1] = -et * qx - c->tt - k->alp3 * xi / rd * k->sdcd;
        du[2] = q * qx + k->alp3 * ai4 * k->sdcd;
        for (int i = 0; i < 3; i++) u[i] = u[i] + disl[1] / pi2 * du[i];
    }
    if (disl[2] != 0.0) {
        du[0] = q * qy - k->alp3 * ai3 * k->sdsd;
        du[1] = q * qx + k->alp3 * xi / rd * k->sdsd;
        du[2] = et * qx + xi * qy - c->tt - k->alp3 * ai4 * k->sdsd;
        for (int i = 0; i < 3; i++) u[i] = u[i] + disl[2] / pi2 * du[i];
    }
}

static void dc3d_uc(double xi, double et, double q, double z, const double disl[3], const dc3d_c0 *k,
                    const dc3d_c2 *c, double u[3])
{
    const double pi2 = 6.283185307179586;
    const double sd = k->sd, cd = k->cd;
    const double cc = c->d + z;
    const double h = q * cd - z;
    const double z32 = sd / c->r3 - h * c->y32;
    const double xy = xi * c->y11, qy = q * c->y11;
    double du[3];
    u[0] = u[1] = u[2] = 0.0;
    if (disl[0] != 0.0) {
        du[0] = k->alp4 * xy * cd - k->alp5 * xi * q * z32;
        du[1] = k->alp4 * (cd / c->r + 2.0 * qy * sd) - k->alp5 * cc * q / c->r3;
        du[2] = k->alp4 * qy * cd - k->alp5 * (cc * et / c->r3 - z * c->y11 + c->xi2 * z32);
        for (int i = 0; i < 3; i++) u[i] = u[i] + disl[0] / pi2 * du[i];
    }
    if (disl[1] != 0.0) {
        du[0] = k->alp4 * cd / c->r - qy * sd - k->alp5 * cc * q / c->r3;
        du[1] = k->alp4 * c->y * c->x11 - k->alp5 * cc * et * q * c->x32;
        du[2] = -c->d * c->x11 - xy * sd - k->alp5 * cc * (c->x11 - c->q2 * c->x32);
        for (int i = 0; i < 3; i++) u[i] = u[i] + disl[1] / pi2 * du[i];
    }
    if (disl[2] != 0.0) {
        du[0] = -k->alp4 * (sd / c->r + qy * cd) - k->alp5 * (z * c->y11 - c->q2 * z32);
        du[1] = k->alp4 * 2.0 * xy * sd + c->d * c->x11 - k->alp5 * cc * (c->x11 - c->q2 * c->x32);
        du[2] = k->alp4 * (c->y * c->x11 + xy * cd) + k->alp5 * q * (cc * et * c->x32 + xi * z32);
        for (int i = 0; i < 3; i++) u[i] = u[i] + disl[2] / pi2 * du[i];
    }
}

/* DC3D, dc3d.f:1-199 (displacement only); float arguments as the routine
 * declares them.  Returns 0, or 1 for a point on a fault edge (zero). */
static int dc3d_disp(float alpha, float x, float y, float z, float depth, float dip, float al1, float al2, float aw1,
                     float aw2, float disl1, float disl2, float disl3, float out[3])
{
    const double eps = 1e-6;
    dc3d_c0 k;
    dc3d_c2 c;
    memset(&c, 0, sizeof c);
    double u[3] = {0, 0, 0};
    dc3d_con0(alpha, dip, &k);
    const double zz = z, dd[3] = {disl1, disl2, disl3};
    double xi[2] = {(double)x - al1, (double)x - al2};
    for (int j = 0; j < 2; j++)
        if (fabs(xi[j]) < eps) xi[j] = 0.0;
    for (int part = 0; part < 2; part++) {
        /* part 0: the real source at d = depth + z; part 1: the image at depth - z */
        const double d = part == 0 ? (double)depth + z : (double)depth - z;
        const double p = y * k.cd + d * k.sd;
        double q = y * k.sd - d * k.cd;
        double et[2] = {p - aw1, p - aw2};
        if (fabs(q) < eps) q = 0.0;
        for (int j = 0; j < 2; j++)
            if (fabs(et[j]) < eps) et[j] = 0.0;
        if (q == 0.0 && ((xi[0] * xi[1] <= 0.0 && et[0] * et[1] == 0.0) ||
                         (et[0] * et[1] <= 0.0 && xi[0] * xi[1] == 0.0))) {
            out[0] = out[1] = out[2] = 0.0f;
            return 1;
        }
        int kxi[2] = {0, 0}, ket[2] = {0, 0};
        const double r12 = sqrt(xi[0] * xi[0] + et[1] * et[1] + q * q);
        const double r21 = sqrt(xi[1] * xi[1] + et[0] * et[0] + q * q);
        const double r22 = sqrt(xi[1] * xi[1] + et[1] * et[1] + q * q);
        if (xi[0] < 0.0 && r21 + xi[1] < eps) kxi[0] = 1;
        if (xi[0] < 0.0 && r22 + xi[1] < eps) kxi[1] = 1;
        if (et[0] < 0.0 && r12 + et[1] < eps) ket[0] = 1;
        if (et[0] < 0.0 && r22 + et[1] < eps) ket[1] = 1;
        for (int kk = 0; kk < 2; kk++) {
            for (int j = 0; j < 2; j++) {
                /* the loop indices as DC3D passes them: KXI(K), KET(J) */
                dc3d_con2(xi[j], et[kk], q, k.sd, k.cd, kxi[kk], ket[j], &c);
                double xj = fabs(xi[j]) < eps ? 0.0 : xi[j], ek = fabs(et[kk]) < eps ? 0.0 : et[kk];
                double du[3], ua[3];
                dc3d_ua(xj, ek, q, dd, &k, &c, ua);
                if (part == 0) {
                    du[0] = -ua[0];
                    du[1] = -ua[1] * k.cd + ua[2] * k.sd;
                    du[2] = -ua[1] * k.sd - ua[2] * k.cd;
                } else {
                    double ub[3], uc[3];
                    dc3d_ub(xj, ek, q, dd, &k, &c, ub);
                    dc3d_uc(xj, ek, q, zz, dd, &k, &c, uc);
                    du[0] = ua[0] + ub[0] + z * uc[0];
                    du[1] = (ua[1] + ub[1] + z * uc[1]) * k.cd - (ua[2] + ub[2] + z * uc[2]) * k.sd;
                    du[2] = (ua[1] + ub[1] - z * uc[1]) * k.sd + (ua[2] + ub[2] - z * uc[2]) * k.cd;
                }
                for (int i = 0; i < 3; i++) u[i] = (j + kk != 1) ? u[i] + du[i] : u[i] - du[i];
            }
        }
    }
    for (int i = 0; i < 3; i++) out[i] = (float)u[i];
    return 0;
}

/* okada, src/okada/green_space.f90:14-89: a source in RELAX's input
 * convention (degrees; x3 the depth of the top edge's reference point)
 * at a receiver (xrec, yrec, zrec >= 0 depth) */
void orc_okada_dc3d(double lambda, double mu, double slip, double opening, double x1, double x2, double x3,
                    double width, double length, double strike, double dipd, double rake, double xrec, double yrec,
                    double zrec, double *disp)
{
    const double degtorad = (double)1.745329252E-02f;        /* a default-real literal */
    const float alpha = (float)((lambda + mu) / (lambda + 2.0 * mu));
    const float z = (float)(-zrec);
    disp[0] = disp[1] = disp[2] = 0.0;
    const double st = strike * degtorad, csst = cos(st), ssst = sin(st);
    const double ra = rake * degtorad, csra = cos(ra), ssra = sin(ra);
    const float x = (float)((xrec - x1) * csst + (yrec - x2) * ssst);
    const float y = (float)((xrec - x1) * ssst - (yrec - x2) * csst);
    float u[3];
    const int iret = dc3d_disp(alpha, x, y, z, (float)x3, (float)dipd, 0.0f, (float)length, -(float)width, 0.0f,
                               (float)(slip * csra), (float)(slip * ssra), (float)opening, u);
    if (iret == 0) {
        disp[0] = disp[0] + (double)u[0] * csst + (double)u[1] * ssst;
        disp[1] = disp[1] + (double)u[0] * ssst - (double)u[1] * csst;
        disp[2] = disp[2] - (double)u[2];
    }
    (void)mu;
}

/* ------------------------------------------------------------------ */
/* eigenstrain sources (--with-eigenstrain, --with-curvilinear)        */
/* ------------------------------------------------------------------ */

/* gaussi, src/elastic3d.f90:513-518 */
static double gaussi(double x, double sigma) { return (1.0 + erf(x / sqrt(2.0) / sigma)) / 2.0; }

/* cuboidSource, src/elastic3d.f90:1680-1884: body force of an eigenstrain
 * e in a cuboid (L, W, T as passed by dislocations: L = width, W = length,
 * src/relax.f90:1157-1166), physical layers of the (sx1+2, sx2, sx3) box.
 * The surface-traction loop of the source computes a moment it does not
 * store (its additions are commented out there) and is left out. */
void orc_cuboidsource(double lambda, double mu, const relax_tensor *e, double x, double y, double z, double L,
                      double W, double T, double strike, double dip, double beta, int sx1, int sx2, int sx3,
                      double dx1, double dx2, double dx3, real *f1, real *f2, real *f3)
{
    const double ekk = (double)((real)e->s11 + (real)e->s22 + (real)e->s33);
    const double e11 = e->s11, e12 = e->s12, e13 = e->s13, e22 = e->s22, e23 = e->s23, e33 = e->s33;
    const double cstrike = cos(strike), sstrike = sin(strike), cdip = cos(dip), sdip = sin(dip);
    const double Wp = W * (1.0 + 2.0 * beta) / 2.0, Lp = L * (1.0 + 2.0 * beta) / 2.0,
                 Tp = T * (1.0 + 2.0 * beta) / 2.0;
    double mx = Wp > Lp ? Wp : Lp;
    if (Tp > mx) mx = Tp;
    const double r2 = (double)sqrtf(2.0f) * mx;              /* SQRT(2.) is default-real */
    const double x2r0 = cstrike * x - sstrike * y;
    const double xr = cdip * x2r0 - sdip * z, yr = sstrike * x + cstrike * y, zr = sdip * x2r0 + cdip * z;
    const int sx1p = sx1 + 2;
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3 / 2; i3++) {
        const double x3 = (double)(i3 - 1) * dx3;
        if (fabs(x3 - z) > r2) continue;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double x1, x2, dum;
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &dum);
                if (fabs(x1 - x) > r2 || fabs(x2 - y) > r2 || fabs(x3 - z) > r2) continue;
                const double x2r = cstrike * x1 - sstrike * x2;
                const double x1s = cdip * x2r - sdip * x3, x1i = cdip * x2r + sdip * x3;
                const double x2s = sstrike * x1 + cstrike * x2;
                const double x3s = sdip * x2r + cdip * x3, x3i = -sdip * x2r + cdip * x3;
                double temp1 = omega((x1s - xr) / T, beta), temp2 = omega((x2s - yr) / W, beta);
                double temp3 = omega((x3s - zr) / L, beta);
                const double sourc = 1.0 / T * omegap((x1s - xr) / T, beta) * temp2 * temp3;
                const double dblcp = 1.0 / W * temp1 * omegap((x2s - yr) / W, beta) * temp3;
                const double dipcs = 1.0 / L * temp1 * temp2 * omegap((x3s - zr) / L, beta);
                temp1 = omega((x1i - xr) / T, beta);
                temp3 = omega((x3i + zr) / L, beta);
                const double image = 1.0 / T * omegap((x1i - xr) / T, beta) * temp2 * temp3;
                const double cplei = 1.0 / W * temp1 * omegap((x2s - yr) / W, beta) * temp3;
                const double dipci = 1.0 / L * temp1 * temp2 * omegap((x3i + zr) / L, beta);
                (void)dipci;
                const size_t o = (size_t)(i1 - 1) + (size_t)sx1p * ((size_t)(i2 - 1) + (size_t)sx2 * (i3 - 1));
                const double s11 = lambda * ekk + 2.0 * mu * e11, s22 = lambda * ekk + 2.0 * mu * e22;
                const double s33 = lambda * ekk + 2.0 * mu * e33;
                if (2.01 * DEG2RAD > dip) {
                    /* method of images for subvertical sources */
                    f1[o] = (real)(f1[o] + 2.0 * mu * e12 * sstrike * (sourc + image) +
                                   2.0 * mu * e12 * cdip * cstrike * (dblcp + cplei) -
                                   s11 * sstrike * (dblcp + cplei) - s22 * cdip * cstrike * (sourc + image));
                    f2[o] = (real)(f2[o] + 2.0 * mu * e12 * cstrike * (sourc + image) -
                                   2.0 * mu * e12 * cdip * sstrike * (dblcp + cplei) -
                                   s11 * cstrike * (dblcp + cplei) + s22 * cdip * sstrike * (sourc + image));
                    f3[o] = (real)(f3[o] - 2.0 * mu * e12 * sdip * (dblcp - cplei) + s22 * sdip * (sourc - image));
                } else {
                    f1[o] = (real)(f1[o] + 2.0 * mu * e12 * sstrike * sourc + 2.0 * mu * e12 * cdip * cstrike * dblcp -
                                   s11 * sstrike * dblcp - s22 * cdip * cstrike * sourc);
                    f2[o] = (real)(f2[o] + 2.0 * mu * e12 * cstrike * sourc - 2.0 * mu * e12 * cdip * sstrike * dblcp -
                                   s11 * cstrike * dblcp + s22 * cdip * sstrike * sourc);
                    f3[o] = (real)(f3[o] - 2.0 * mu * e12 * sdip * dblcp + s22 * sdip * sourc);
                }
                /* vertical shear components */
                f1[o] = (real)(f1[o] + 2.0 * mu * e13 * cdip * sstrike * dipcs + 2.0 * mu * e13 * sdip * cstrike * dblcp -
                               2.0 * mu * e23 * cdip * cstrike * dipcs - 2.0 * mu * e23 * sdip * cstrike * sourc -
                               s33 * sdip * dipcs * cstrike);
                f2[o] = (real)(f2[o] + 2.0 * mu * e13 * cdip * cstrike * dipcs - 2.0 * mu * e13 * sdip * sstrike * dblcp +
                               2.0 * mu * e23 * cdip * sstrike * dipcs + 2.0 * mu * e23 * sdip * sstrike * sourc +
                               s33 * sdip * dipcs * sstrike);
                f3[o] = (real)(f3[o] + 2.0 * mu * e13 * cdip * dblcp - 2.0 * mu * e23 * cdip * sourc -
                               s33 * cdip * dipcs);
            }
        }
    }
}

/* the outward unit normals of a tetrahedron's faces BCD, CDA, DAB, ABC and
 * the faces' centroids (tetrahedronSource / momentDensityTetrahedron,
 * src/elastic3d.f90:1946-1980, :2816-2848); 0 for a tetrahedron without
 * volume */
static int tet_faces(const double A[3], const double B[3], const double C[3], const double D[3], double n[4][3],
                     double cen[4][3])
{
    const double *P[4] = {A, B, C, D};
    /* nA = (C-B) x (D-B), nB = (D-C) x (A-C), nC = (A-D) x (B-D), nD = (B-A) x (C-A) */
    const int tri[4][3] = {{1, 2, 3}, {2, 3, 0}, {3, 0, 1}, {0, 1, 2}};
    for (int f = 0; f < 4; f++) {
        const double *p = P[tri[f][0]], *q = P[tri[f][1]], *r = P[tri[f][2]];
        const double u[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
        const double v[3] = {r[0] - p[0], r[1] - p[1], r[2] - p[2]};
        n[f][0] = u[1] * v[2] - u[2] * v[1];
        n[f][1] = u[2] * v[0] - u[0] * v[2];
        n[f][2] = u[0] * v[1] - u[1] * v[0];
    }
    for (int f = 0; f < 4; f++)
        if (0.0 == sqrt(n[f][0] * n[f][0] + n[f][1] * n[f][1] + n[f][2] * n[f][2])) return 0;
    for (int f = 0; f < 4; f++) {
        const double nn = sqrt(n[f][0] * n[f][0] + n[f][1] * n[f][1] + n[f][2] * n[f][2]);
        for (int k = 0; k < 3; k++) n[f][k] = n[f][k] / nn;
    }
    for (int f = 0; f < 4; f++) {
        const double *p = P[tri[f][0]], *q = P[tri[f][1]], *r = P[tri[f][2]];
        for (int k = 0; k < 3; k++) cen[f][k] = (p[k] + q[k] + r[k]) / 3;
        /* outward: the opposite vertex lies behind the face */
        const double *o = P[f];
        const double d = n[f][0] * (o[0] - cen[f][0]) + n[f][1] * (o[1] - cen[f][1]) + n[f][2] * (o[2] - cen[f][2]);
        if (d > 0) for (int k = 0; k < 3; k++) n[f][k] = -n[f][k];
    }
    return 1;
}

/* tetrahedronSource, src/elastic3d.f90:1916-2039: body force of an
 * eigenstrain e in a tetrahedron ABCD, the faces smoothed with Gaussians of
 * width dx1, physical layers of the (sx1+2, sx2, sx3) box. */
void orc_tetrahedronsource(double lambda, double mu, const relax_tensor *e, const double A[3], const double B[3],
                           const double C[3], const double D[3], int sx1, int sx2, int sx3, double dx1, double dx2,
                           double dx3, real *f1, real *f2, real *f3)
{
    otensor m = {e->s11, e->s12, e->s13, e->s22, e->s23, e->s33};
    isotropic(&m, lambda, mu);
    double n[4][3], cen[4][3];
    if (!tet_faces(A, B, C, D, n, cen)) return;
    double tr[4][3];
    for (int f = 0; f < 4; f++) tdot(&m, n[f], tr[f]);
    const int sx1p = sx1 + 2;
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3 / 2; i3++) {
        double x[3];
        x[2] = (double)(i3 - 1) * dx3;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double dum;
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x[0], &x[1], &dum);
                double d[4];
                for (int f = 0; f < 4; f++)
                    d[f] = (cen[f][0] - x[0]) * n[f][0] + (cen[f][1] - x[1]) * n[f][1] + (cen[f][2] - x[2]) * n[f][2];
                if (fabs(d[0]) > 7.0 * dx1 && fabs(d[1]) > 7.0 * dx1 && fabs(d[2]) > 7.0 * dx1 &&
                    fabs(d[3]) > 7.0 * dx1)
                    continue;
                double H[4], G[4];
                for (int f = 0; f < 4; f++) H[f] = gaussi(d[f], dx1);
                for (int f = 0; f < 4; f++) G[f] = gauss(d[f], dx1);
                const size_t o = (size_t)(i1 - 1) + (size_t)sx1p * ((size_t)(i2 - 1) + (size_t)sx2 * (i3 - 1));
                real *fk[3] = {f1, f2, f3};
                for (int k = 0; k < 3; k++)
                    fk[k][o] = (real)(fk[k][o] + tr[0][k] * G[0] * H[1] * H[2] * H[3] +
                                      tr[1][k] * H[0] * G[1] * H[2] * H[3] + tr[2][k] * H[0] * H[1] * G[2] * H[3] +
                                      tr[3][k] * H[0] * H[1] * H[2] * G[3]);
            }
        }
    }
}

/* momentDensityCuboid, src/elastic3d.f90:2927-3029: moment density of the
 * eigenstrain e (strike, normal, dip frame) in a cuboid, physical layers
 * (sx3 of them); the image term is computed but not used there */
void orc_momentdensitycuboid(double mu, double lambda, const relax_tensor *e, double x, double y, double z,
                             double L, double W, double T, double strike, double dip, double beta, int sx1, int sx2,
                             int sx3, double dx1, double dx2, double dx3, otensor *sig)
{
    const otensor lamdij = {(real)lambda, 0, 0, (real)lambda, 0, (real)lambda};
    const real rmu = (real)2 * (real)mu;
    const double cstrike = cos(strike), sstrike = sin(strike), cdip = cos(dip), sdip = sin(dip);
    const double Wp = W * (1.0 + 2.0 * beta) / 2.0, Lp = L * (1.0 + 2.0 * beta) / 2.0,
                 Tp = T * (1.0 + 2.0 * beta) / 2.0;
    double mx = Wp > Lp ? Wp : Lp;
    if (Tp > mx) mx = Tp;
    const double r2 = (double)sqrtf(2.0f) * mx;
    const double x2r0 = cstrike * x - sstrike * y;
    const double xr = cdip * x2r0 - sdip * z, yr = sstrike * x + cstrike * y, zr = sdip * x2r0 + cdip * z;
    const double n[3] = {+cdip * cstrike, -cdip * sstrike, -sdip};
    const double s[3] = {-sstrike, -cstrike, 0};
    const double d[3] = {+cstrike * sdip, -sstrike * sdip, +cdip};
    const otensor ss = sdyad(s, s), ns = sdyad(n, s), sd = sdyad(s, d), nn = sdyad(n, n), nd = sdyad(n, d),
                  dd = sdyad(d, d);
    const otensor et = {e->s11, e->s12, e->s13, e->s22, e->s23, e->s33};
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        const double x3 = (double)(i3 - 1) * dx3;
        if (fabs(x3 - z) > r2) continue;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double x1, x2, dum;
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x1, &x2, &dum);
                if (fabs(x1 - x) > r2 || fabs(x2 - y) > r2 || fabs(x3 - z) > r2) continue;
                const double x2r = cstrike * x1 - sstrike * x2;
                const double x1s = cdip * x2r - sdip * x3;
                const double x2s = sstrike * x1 + cstrike * x2;
                const double x3s = sdip * x2r + cdip * x3;
                const real aperture = (real)(omega((x1s - xr) / T, beta) * omega((x2s - yr) / W, beta) *
                                             omega((x3s - zr) / L, beta));
                const otensor ea = ttimes(aperture, et);
                otensor Ei = ttimes(ea.s11, ss);
                Ei = tplus(Ei, ttimes((real)2 * ea.s12, ns));
                Ei = tplus(Ei, ttimes((real)2 * ea.s13, sd));
                Ei = tplus(Ei, ttimes(ea.s22, nn));
                Ei = tplus(Ei, ttimes((real)2 * ea.s23, nd));
                Ei = tplus(Ei, ttimes(ea.s33, dd));
                const real ekk = (real)ttrace(&Ei);
                const size_t o = IDX3(i1 - 1, i2 - 1, i3 - 1, sx1, sx2);
                sig[o] = tplus(tplus(sig[o], ttimes(ekk, lamdij)), ttimes(rmu, Ei));
            }
        }
    }
}

/* momentDensityTetrahedron, src/elastic3d.f90:2788-2873: moment density of
 * the eigenstrain e in a tetrahedron ABCD (physical layers, sx3 of them).
 * A point is left out when its signed distances to all four faces are
 * below 7 dx1, as the reference's test reads. */
void orc_momentdensitytetrahedron(double mu, double lambda, const relax_tensor *e, const double A[3],
                                  const double B[3], const double C[3], const double D[3], int sx1, int sx2,
                                  int sx3, double dx1, double dx2, double dx3, otensor *sig)
{
    const otensor lamdij = {(real)lambda, 0, 0, (real)lambda, 0, (real)lambda};
    const real rmu = (real)2 * (real)mu;
    double n[4][3], cen[4][3];
    if (!tet_faces(A, B, C, D, n, cen)) return;
    const otensor et = {e->s11, e->s12, e->s13, e->s22, e->s23, e->s33};
#pragma omp parallel for schedule(static)
    for (int i3 = 1; i3 <= sx3; i3++) {
        double x[3];
        x[2] = (double)(i3 - 1) * dx3;
        for (int i2 = 1; i2 <= sx2; i2++) {
            for (int i1 = 1; i1 <= sx1; i1++) {
                double dum;
                shiftedcoordinates(i1, i2, i3, sx1, sx2, sx3, dx1, dx2, dx3, &x[0], &x[1], &dum);
                double d[4];
                for (int f = 0; f < 4; f++)
                    d[f] = (cen[f][0] - x[0]) * n[f][0] + (cen[f][1] - x[1]) * n[f][1] + (cen[f][2] - x[2]) * n[f][2];
                if (d[0] < 7.0 * dx1 && d[1] < 7.0 * dx1 && d[2] < 7.0 * dx1 && d[3] < 7.0 * dx1) continue;
                const double H = gaussi(d[0], dx1) * gaussi(d[1], dx1) * gaussi(d[2], dx1) * gaussi(d[3], dx1);
                const otensor ea = ttimes((real)H, et);
                const real ekk = (real)ttrace(&ea);
                const size_t o = IDX3(i1 - 1, i2 - 1, i3 - 1, sx1, sx2);
                sig[o] = tplus(tplus(sig[o], ttimes(ekk, lamdij)), ttimes(rmu, ea));
            }
        }
    }
}


/* dislocations without eigenstress, src/relax.f90:1116-1289: shear,
 * cuboid and tetrahedral eigenstrain, tensile and point sources */
static int orc_dislocations(orc_state *S, const relax_event *ev)
{
    const relax_config *c = &S->cfg;
    double mind = c->dx1 < c->dx2 ? c->dx1 : c->dx2;
    if (c->dx3 < mind) mind = c->dx3;
    for (int i = 0; i < ev->ns; i++) {
        const relax_source *s = &ev->s[i];
        if (c->nyquist * mind < s->length || c->nyquist * mind < s->width)
            orc_source(c->mu, s->slip, s->x, s->y, s->z, s->width, s->length, s->strike, s->dip,
                       s->rake, s->beta, S->sx1, S->sx2, S->sx3, c->dx1, c->dx2, c->dx3,
                       S->v[0], S->v[1], S->v[2], S->t[0], S->t[1], S->t[2]);
    }
    /* cuboid and tetrahedral eigenstrain (src/relax.f90:1154-1181): the
     * cuboid's L = width, W = length, T = thickness, the global beta */
    for (int i = 0; i < ev->nc; i++) {
        const relax_weakzone *q = &ev->c[i];
        orc_cuboidsource(c->lambda, c->mu, &q->e, q->x, q->y, q->z, q->width, q->length, q->thickness, q->strike,
                         q->dip, c->beta, S->sx1, S->sx2, S->sx3, c->dx1, c->dx2, c->dx3, S->v[0], S->v[1],
                         S->v[2]);
    }
    for (int i = 0; i < ev->ntet; i++) {
        const relax_tetrahedron *q = &ev->tet[i];
        orc_tetrahedronsource(c->lambda, c->mu, &q->e, ev->vert + 3 * (q->i1 - 1), ev->vert + 3 * (q->i2 - 1),
                              ev->vert + 3 * (q->i3 - 1), ev->vert + 3 * (q->i4 - 1), S->sx1, S->sx2, S->sx3,
                              c->dx1, c->dx2, c->dx3, S->v[0], S->v[1], S->v[2]);
    }
    for (int i = 0; i < ev->ns; i++) {
        const relax_source *s = &ev->s[i];
        orc_momentdensityshear(c->mu, s->slip, s->x, s->y, s->z, s->width, s->length, s->strike,
                               s->dip, s->rake, s->beta, S->sx1, S->sx2, S->sx3h, c->dx1, c->dx2,
                               c->dx3, S->tau);
    }
    /* their moment densities into tau (src/relax.f90:1208-1224) */
    for (int i = 0; i < ev->nc; i++) {
        const relax_weakzone *q = &ev->c[i];
        orc_momentdensitycuboid(c->mu, c->lambda, &q->e, q->x, q->y, q->z, q->width, q->length, q->thickness,
                                q->strike, q->dip, c->beta, S->sx1, S->sx2, S->sx3h, c->dx1, c->dx2, c->dx3,
                                S->tau);
    }
    for (int i = 0; i < ev->ntet; i++) {
        const relax_tetrahedron *q = &ev->tet[i];
        orc_momentdensitytetrahedron(c->mu, c->lambda, &q->e, ev->vert + 3 * (q->i1 - 1), ev->vert + 3 * (q->i2 - 1),
                                     ev->vert + 3 * (q->i3 - 1), ev->vert + 3 * (q->i4 - 1), S->sx1, S->sx2,
                                     S->sx3h, c->dx1, c->dx2, c->dx3, S->tau);
    }
    /* tensile cracks (src/relax.f90:1226-1260): L = width, W = length, the
     * global beta, the crack's opening */
    for (int i = 0; i < ev->nt; i++) {
        const relax_source *s = &ev->ts[i];
        if (c->nyquist * mind < s->length || c->nyquist * mind < s->width)
            orc_tensilesource(c->lambda, c->mu, s->opening, s->x, s->y, s->z, s->width, s->length,
                              s->strike, s->dip, c->beta, S->sx1, S->sx2, S->sx3, c->dx1, c->dx2, c->dx3,
                              S->v[0], S->v[1], S->v[2]);
    }
    for (int i = 0; i < ev->nt; i++) {
        const relax_source *s = &ev->ts[i];
        orc_momentdensitytensile(c->lambda, c->mu, s->opening, s->x, s->y, s->z, s->width, s->length,
                                 s->strike, s->dip, c->beta, S->sx1, S->sx2, S->sx3h, c->dx1, c->dx2,
                                 c->dx3, S->tau);
    }
    /* dilatation point sources (src/relax.f90:1262-1287): amplitude in slip */
    for (int i = 0; i < ev->nm; i++) {
        const relax_source *s = &ev->m[i];
        orc_mogisource(c->lambda, c->mu, s->slip, s->x, s->y, s->z, S->sx1, S->sx2, S->sx3, c->dx1, c->dx2,
                       c->dx3, S->v[0], S->v[1], S->v[2]);
    }
    for (int i = 0; i < ev->nm; i++) {
        const relax_source *s = &ev->m[i];
        orc_momentdensitymogi(c->lambda, c->mu, s->slip, s->x, s->y, s->z, S->sx1, S->sx2, S->sx3h, c->dx1,
                              c->dx2, c->dx3, S->tau);
    }
    return ORC_OK;
}

static void zero_vt(orc_state *S)
{
    for (int k = 0; k < 3; k++) {
        memset(S->v[k], 0, sizeof(real) * S->nv);
        memset(S->t[k], 0, sizeof(real) * S->n2);
    }
}

static int green(orc_state *S)
{
    const relax_config *c = &S->cfg;
    return orc_greenfunctioncowling(S->v[0], S->v[1], S->v[2], S->t[0], S->t[1], S->t[2], S->sx1,
                                    S->sx2, S->sx3, c->dx1, c->dx2, c->dx3, c->lambda, c->mu, c->gam);
}

static int stressupdate_s(orc_state *S, real **w)
{
    const relax_config *c = &S->cfg;
    return orc_stressupdate(w[0], w[1], w[2], c->lambda, c->mu, c->dx1, c->dx2, c->dx3, S->sx1,
                            S->sx2, S->sx3h, S->sig);
}

static int eigen_all(orc_state *S, double *maxwell, int with_gamma, double Dt)
{
    const relax_config *c = &S->cfg;
    int err;
    const relax_layer *st[2] = {c->linearstruc, c->nonlinearstruc};
    const float *dg[2] = {c->lineardgammadot0, c->nonlineardgammadot0};
    real *dgr[2] = {NULL, NULL};
    for (int m = 0; m < 2; m++) {
        if (!st[m]) continue;
        if (dg[m]) {
            size_t n = S->nt;
            dgr[m] = malloc(sizeof(real) * n);
            for (size_t q = 0; q < n; q++) dgr[m][q] = (real)dg[m][q];
        }
        if (with_gamma) {
            memset(S->v[0], 0, sizeof(real) * S->nv);
            err = orc_viscouseigenstress(c->mu, st[m], c->stressstruc, S->sig, S->sx1, S->sx2,
                                         S->sx3h, S->moment, NULL, S->v[0], dgr[m]);
            if (!err) orc_fieldadd(S->gamma, S->v[0], S->nu, 0, 0, 1, (real)Dt);
        } else {
            err = orc_viscouseigenstress(c->mu, st[m], c->stressstruc, S->sig, S->sx1, S->sx2,
                                         S->sx3h, S->moment, &maxwell[m], NULL, dgr[m]);
        }
        free(dgr[m]);
        if (err) return err;
    }
    return ORC_OK;
}

void orc_state_free(orc_state *S)
{
    if (!S) return;
    for (int k = 0; k < 3; k++) { free(S->v[k]); free(S->u[k]); free(S->t[k]); }
    free(S->gamma); free(S->tau); free(S->sig); free(S->moment);
    free(S->eps); free(S->epsdot);
    if (S->patch) for (int k = 0; k < S->cfg.np; k++) free(S->patch[k]);
    free(S->patch);
    free(S);
}

orc_state *orc_state_create(const relax_config *cfg)
{
    orc_state *S = calloc(1, sizeof(orc_state));
    if (!S) return NULL;
    S->cfg = *cfg;
    S->sx1 = cfg->sx1; S->sx2 = cfg->sx2; S->sx3 = cfg->sx3; S->sx3h = cfg->sx3 / 2;
    S->nv = (size_t)(S->sx1 + 2) * S->sx2 * S->sx3;
    S->nu = (size_t)(S->sx1 + 2) * S->sx2 * S->sx3h;
    S->nt = (size_t)S->sx1 * S->sx2 * S->sx3h;
    S->n2 = (size_t)(S->sx1 + 2) * S->sx2;
    int ok = 1;
    for (int k = 0; k < 3; k++) {
        ok &= (S->v[k] = calloc(S->nv, sizeof(real))) != NULL;
        ok &= (S->u[k] = calloc(S->nu, sizeof(real))) != NULL;
        ok &= (S->t[k] = calloc(S->n2, sizeof(real))) != NULL;
    }
    ok &= (S->gamma = calloc(S->nu, sizeof(real))) != NULL;
    ok &= (S->tau = calloc(S->nt, sizeof(otensor))) != NULL;
    ok &= (S->sig = calloc(S->nt, sizeof(otensor))) != NULL;
    ok &= (S->moment = calloc(S->nt, sizeof(otensor))) != NULL;
    /* epsilonik starts at zero (allocated, src/relax.f90:299-302) */
    if (cfg->ltransientstruc || cfg->nltransientstruc) {
        ok &= (S->eps = calloc(S->nt, sizeof(otensor))) != NULL;
        ok &= (S->epsdot = calloc(S->nt, sizeof(otensor))) != NULL;
    }
    if (cfg->np > 0) {
        S->patch = calloc((size_t)cfg->np, sizeof(relax_slippatch *));
        for (int k = 0; k < cfg->np && S->patch; k++) {
            size_t n = (size_t)(cfg->planes[k].px2 > 0 ? cfg->planes[k].px2 : 0) *
                       (size_t)(cfg->planes[k].px3 > 0 ? cfg->planes[k].px3 : 0);
            S->patch[k] = calloc(n > 0 ? n : 1, sizeof(relax_slippatch));
            ok &= S->patch[k] != NULL;
        }
        ok &= S->patch != NULL;
    }
    if (!ok) { orc_state_free(S); return NULL; }
    /* tau = -prestress, src/relax.f90:287-297 */
    if (cfg->stressstruc)
        for (int i3 = 0; i3 < S->sx3h; i3++) {
            const relax_tensor *q = &cfg->stressstruc[i3].t;
            otensor p = {(real)q->s11, (real)q->s12, (real)q->s13, (real)q->s22, (real)q->s23, (real)q->s33};
            otensor m = ttimes((real)-1.0, p);
            for (size_t j = 0; j < (size_t)S->sx1 * S->sx2; j++) S->tau[j + (size_t)S->sx1 * S->sx2 * i3] = m;
        }
    return S;
}

/* coseismic solve of the first event, src/relax.f90:312-371 */
int orc_coseismic(orc_state *S, relax_step_log *log)
{
    const relax_config *c = &S->cfg;
    S->e = 0; S->oi = 1; S->time = 0; S->i = 0;
    zero_vt(S);
    if (c->ne <= 0) return ORC_ERR_ARG;
    int err = orc_dislocations(S, &c->events[0]);
    if (err) return err;
    orc_traction(c->mu, &c->events[0], S->sx1, S->sx2, c->dx1, c->dx2, 0.0, 0.0, S->t[2], 0);
    const relax_event *ev = &c->events[0];
    if (ev->nt || ev->ns || ev->nm || ev->nl || ev->nc || ev->ntet) {   /* src/relax.f90:344-350 */
        if ((err = green(S))) return err;
        /* dislocations_disp: the sources smaller than the Nyquist length
         * (src/relax.f90:355-360, :1320-1347) */
        double mind = c->dx1 < c->dx2 ? c->dx1 : c->dx2;
        if (c->dx3 < mind) mind = c->dx3;
        const double small = c->nyquist * mind;
        for (int i = 0; i < ev->ns + ev->nt; i++) {
            const int tens = i >= ev->ns;
            const relax_source *s = tens ? &ev->ts[i - ev->ns] : &ev->s[i];
            if (!(small >= s->length || small >= s->width)) continue;
            double x, y, z, strike, dip, rake;
            input_form(c, s, &x, &y, &z, &strike, &dip, &rake);
            grnfct_okada(c->lambda, c->mu, tens ? 0.0 : -s->slip, tens ? s->opening : 0.0, x, y, z, s->width,
                         s->length, strike, dip, tens ? 0.0 : rake, S->sx1, S->sx2, S->sx3h, c->dx1, c->dx2, c->dx3,
                         S->v[0], S->v[1], S->v[2]);
        }
    }
    for (int k = 0; k < 3; k++) memcpy(S->u[k], S->v[k], sizeof(real) * S->nu);
    orc_tensorfieldadd(S->sig, S->tau, S->nt, 1, 0, 1, -1);
    if ((err = stressupdate_s(S, S->u))) return err;
    if (log) {
        memset(log, 0, sizeof *log);
        log->cei = orc_tensoramplitude(S->tau, S->nt, c->dx1, c->dx2, c->dx3);
    }
    return ORC_OK;
}

/* the linear and nonlinear transient mechanisms in turn (src/relax.f90:614-645
 * in the predictor, :764-790 in the corrector): the input strain is `in`,
 * the rate goes to S->epsdot (each call overwrites it) */
static int transient_all(orc_state *S, const otensor *in, double *maxwell)
{
    const relax_config *c = &S->cfg;
    const relax_layer *st[2] = {c->ltransientstruc, c->nltransientstruc};
    const float *dg[2] = {c->ltransientdgammadot0, c->nltransientdgammadot0};
    for (int m = 0; m < 2; m++) {
        if (!st[m]) continue;
        real *dgr = NULL;
        if (dg[m]) {
            dgr = malloc(sizeof(real) * S->nt);
            if (!dgr) return ORC_ERR_ARG;
            for (size_t q = 0; q < S->nt; q++) dgr[q] = (real)dg[m][q];
        }
        int err = orc_transienteigenstress(c->mu, st[m], S->sig, in, S->sx1, S->sx2, S->sx3h, S->moment,
                                           S->epsdot, maxwell ? &maxwell[3 + m] : NULL, dgr);
        free(dgr);
        if (err) return err;
    }
    return ORC_OK;
}

/* one RK2 step, src/relax.f90:555-890 */
int orc_step(orc_state *S, const double *dt_override, relax_step_log *log)
{
    const relax_config *c = &S->cfg;
    const double STEP_MAX = 1e7;
    int err;
    if (S->time >= c->interval) { if (log) memset(log, 0, sizeof *log); return ORC_OK; }
    S->i++;
    double maxwell[5] = {STEP_MAX, STEP_MAX, STEP_MAX, STEP_MAX, STEP_MAX};
    double mech[5] = {0, 0, 0, 0, 0};
    /* predictor */
    orc_tensorfieldadd(S->moment, S->moment, S->nt, 1, 0, 1, 0);
    if ((err = eigen_all(S, maxwell, 0, 0.0))) return err;
    if (c->linearstruc) mech[0] = 1;
    if (c->nonlinearstruc) mech[1] = 1;
    if (c->faultcreepstruc) {
        for (int k = 0; k < c->np; k++) {
            const relax_plane *p = &c->planes[k];
            err = orc_frictioneigenstress(p->x, p->y, p->z, p->width, p->length, p->strike, p->dip,
                                          p->rake, c->beta, S->sig, c->mu, c->faultcreepstruc,
                                          S->sx1, S->sx2, S->sx3h, c->dx1, c->dx2, c->dx3,
                                          S->moment, &maxwell[2]);
            if (err) return err;
        }
        mech[2] = 1;
    }
    if (S->eps) {
        if ((err = transient_all(S, S->eps, maxwell))) return err;
        if (c->ltransientstruc) mech[3] = 1;
        if (c->nltransientstruc) mech[4] = 1;
    }
    double tm = 1.0 / (mech[0] / maxwell[0] + mech[1] / maxwell[1] + mech[2] / maxwell[2] +
                       mech[3] / maxwell[3] + mech[4] / maxwell[4]);
    if (tm > STEP_MAX) tm = STEP_MAX;
    if (c->inter.ns > 0 || c->inter.nt > 0)
        if (tm == STEP_MAX) tm = c->interval / 20.0;
    double Dt;
    integrationstep(tm, &Dt, S->time, S->oi, c->odt, c->skip, c->tscale, c->events, S->e, c->ne);
    if (dt_override) Dt = *dt_override;

    orc_tensorfieldadd(S->sig, S->moment, S->nt, 1, 0, 1, 1);
    zero_vt(S);
    orc_equivalentbodyforce(S->sig, c->dx1, c->dx2, c->dx3, S->sx1, S->sx2, S->sx3h, S->v[0],
                            S->v[1], S->v[2], S->t[0], S->t[1], S->t[2]);
    orc_traction(c->mu, &c->events[S->e], S->sx1, S->sx2, c->dx1, c->dx2, S->time, Dt / 2.0e8, S->t[2], 1);
    if ((err = green(S))) return err;
    for (int k = 0; k < 3; k++) orc_fieldadd(S->v[k], S->u[k], S->nu, 1, (real)(Dt / 2), 0, 0);
    /* epsilonikdot = Dt/2 epsilonikdot + epsilonik, src/relax.f90:693-695 */
    if (S->eps) orc_tensorfieldadd(S->epsdot, S->eps, S->nt, 1, (real)(Dt / 2), 1, 1);
    orc_tensorfieldadd(S->sig, S->tau, S->nt, 1, -(real)(Dt / 2), 1, -1);

    /* corrector */
    if ((err = stressupdate_s(S, S->v))) return err;
    orc_tensorfieldadd(S->moment, S->moment, S->nt, 1, 0, 1, 0);
    if ((err = eigen_all(S, maxwell, 1, Dt))) return err;
    if (c->faultcreepstruc) {
        for (int k = 0; k < c->np; k++) {
            const relax_plane *p = &c->planes[k];
            err = orc_frictioneigenstress(p->x, p->y, p->z, p->width, p->length, p->strike, p->dip,
                                          p->rake, c->beta, S->sig, c->mu, c->faultcreepstruc,
                                          S->sx1, S->sx2, S->sx3h, c->dx1, c->dx2, c->dx3,
                                          S->moment, NULL);
            if (err) return err;
            orc_monitorfriction(p->x, p->y, p->z, p->width, p->length, p->strike, p->dip, p->rake,
                                c->beta, S->sx1, S->sx2, S->sx3h, c->dx1, c->dx2, c->dx3, S->sig,
                                c->faultcreepstruc, p->px2, p->px3, S->patch[k]);
        }
    }
    if (S->eps) {
        /* both calls read epsilonikdot (src/relax.f90:768-786), then
         * epsilonik += Dt epsilonikdot and epsilonikdot = 0 (:789-790) */
        if ((err = transient_all(S, S->epsdot, NULL))) return err;
        orc_tensorfieldadd(S->eps, S->epsdot, S->nt, 0, 0, 1, (real)Dt);
        orc_tensorfieldadd(S->epsdot, S->epsdot, S->nt, 1, 0, 1, 0);
    }
    /* interseismic loading, src/relax.f90:796-800: dislocations(..., eigenstress=moment)
     * adds the moment densities to the moment and to tau */
    if (c->inter.ns > 0) {
        for (int i = 0; i < c->inter.ns; i++) {
            const relax_source *s = &c->inter.s[i];
            orc_momentdensityshear(c->mu, s->slip, s->x, s->y, s->z, s->width, s->length,
                                   s->strike, s->dip, s->rake, s->beta, S->sx1, S->sx2, S->sx3h,
                                   c->dx1, c->dx2, c->dx3, S->moment);
            orc_momentdensityshear(c->mu, s->slip, s->x, s->y, s->z, s->width, s->length,
                                   s->strike, s->dip, s->rake, s->beta, S->sx1, S->sx2, S->sx3h,
                                   c->dx1, c->dx2, c->dx3, S->tau);
        }
    }
    for (int i = 0; i < c->inter.nt; i++) {
        const relax_source *s = &c->inter.ts[i];
        orc_momentdensitytensile(c->lambda, c->mu, s->opening, s->x, s->y, s->z, s->width, s->length,
                                 s->strike, s->dip, c->beta, S->sx1, S->sx2, S->sx3h, c->dx1, c->dx2,
                                 c->dx3, S->moment);
    }
    for (int i = 0; i < c->inter.nt; i++) {
        const relax_source *s = &c->inter.ts[i];
        orc_momentdensitytensile(c->lambda, c->mu, s->opening, s->x, s->y, s->z, s->width, s->length,
                                 s->strike, s->dip, c->beta, S->sx1, S->sx2, S->sx3h, c->dx1, c->dx2,
                                 c->dx3, S->tau);
    }
    zero_vt(S);
    orc_equivalentbodyforce(S->moment, c->dx1, c->dx2, c->dx3, S->sx1, S->sx2, S->sx3h, S->v[0],
                            S->v[1], S->v[2], S->t[0], S->t[1], S->t[2]);
    orc_traction(c->mu, &c->events[S->e], S->sx1, S->sx2, c->dx1, c->dx2, S->time, Dt, S->t[2], 1);
    if ((err = green(S))) return err;
    for (int k = 0; k < 3; k++) orc_fieldadd(S->u[k], S->v[k], S->nu, 0, 0, 1, (real)Dt);
    orc_tensorfieldadd(S->tau, S->moment, S->nt, 0, 0, 1, (real)Dt);
    for (int k = 0; k < c->np; k++)
        orc_frictionadd(c->planes[k].px2 * c->planes[k].px3, S->patch[k], Dt);
    S->time = S->time + Dt;
    int fired = 0;
    if (S->e < c->ne - 1) {
        if (fabs(S->time - c->events[S->e + 1].time) < 1e-6) {
            S->e++;
            fired = 1;
            zero_vt(S);
            if ((err = orc_dislocations(S, &c->events[S->e]))) return err;
            orc_traction(c->mu, &c->events[S->e], S->sx1, S->sx2, c->dx1, c->dx2, S->time, 0.0, S->t[2], 0);
            if ((err = green(S))) return err;
            for (int k = 0; k < 3; k++) orc_fieldadd(S->u[k], S->v[k], S->nu, 0, 0, 0, 0);
        }
    }
    orc_tensorfieldadd(S->sig, S->tau, S->nt, 1, 0, 1, -1);
    if ((err = stressupdate_s(S, S->u))) return err;
    /* isoutput, src/relax.f90:1364-1376 */
    {
        double odt = c->odt, etime = c->events[S->e].time;
        if ((0 == c->skip && fabs(S->time - S->oi * odt) < 1e-6 * odt) ||
            (0 < c->skip && ((S->i - 1) % c->skip) == 0) || fabs(S->time - etime) < 1e-6)
            S->oi++;
    }
    if (log) {
        log->i = S->i; log->event = fired; log->dt = Dt;
        log->tm_ve = maxwell[0]; log->tm_pl = maxwell[1]; log->tm_as = maxwell[2];
        log->tm_tl = maxwell[3]; log->tm_tnl = maxwell[4];
        log->t = S->time;
        log->power = orc_tensoramplitude(S->moment, S->nt, c->dx1, c->dx2, c->dx3);
        log->cei = orc_tensoramplitude(S->tau, S->nt, c->dx1, c->dx2, c->dx3);
    }
    return ORC_OK;
}

/* field access in the reference layout */
int orc_get_field(orc_state *S, int which, void *dst)
{
    switch (which) {
    case RELAX_FIELD_U:
        for (int k = 0; k < 3; k++) memcpy((real *)dst + k * S->nu, S->u[k], sizeof(real) * S->nu);
        return ORC_OK;
    case RELAX_FIELD_SIG: memcpy(dst, S->sig, sizeof(otensor) * S->nt); return ORC_OK;
    case RELAX_FIELD_TAU: memcpy(dst, S->tau, sizeof(otensor) * S->nt); return ORC_OK;
    case RELAX_FIELD_MOMENT: memcpy(dst, S->moment, sizeof(otensor) * S->nt); return ORC_OK;
    case RELAX_FIELD_GAMMA: memcpy(dst, S->gamma, sizeof(real) * S->nu); return ORC_OK;
    case RELAX_FIELD_V:
        for (int k = 0; k < 3; k++) memcpy((real *)dst + k * S->nv, S->v[k], sizeof(real) * S->nv);
        return ORC_OK;
    default: return ORC_ERR_ARG;
    }
}

int orc_set_field(orc_state *S, int which, const void *src)
{
    switch (which) {
    case RELAX_FIELD_U:
        for (int k = 0; k < 3; k++) memcpy(S->u[k], (const real *)src + k * S->nu, sizeof(real) * S->nu);
        return ORC_OK;
    case RELAX_FIELD_SIG: memcpy(S->sig, src, sizeof(otensor) * S->nt); return ORC_OK;
    case RELAX_FIELD_TAU: memcpy(S->tau, src, sizeof(otensor) * S->nt); return ORC_OK;
    case RELAX_FIELD_MOMENT: memcpy(S->moment, src, sizeof(otensor) * S->nt); return ORC_OK;
    case RELAX_FIELD_GAMMA: memcpy(S->gamma, src, sizeof(real) * S->nu); return ORC_OK;
    default: return ORC_ERR_ARG;
    }
}

int orc_get_patches(orc_state *S, int k, relax_slippatch *dst)
{
    if (k < 0 || k >= S->cfg.np) return ORC_ERR_ARG;
    memcpy(dst, S->patch[k], sizeof(relax_slippatch) * (size_t)S->cfg.planes[k].px2 * S->cfg.planes[k].px3);
    return ORC_OK;
}

double orc_time(orc_state *S) { return S->time; }

int orc_real_size(void) { return (int)sizeof(real); }

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
