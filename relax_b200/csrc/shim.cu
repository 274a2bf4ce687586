// shim.cu -- the reference CUDA layer's entry points (src/cuelastic.cu,
// src/cugreen.cu), symbol for symbol, over this library's operators, so the
// reference Fortran GPU driver (src/curelax.f90) links against it unchanged.
//
// As in the reference, the fields live in one implicit device context in
// RELAX's own layout (padded vectors, TENSOR arrays), every call is
// synchronous, and the host arrays the Fortran side passes for fields are
// placeholders.  Errors are reported through the reference's iRet
// arguments where it has them and through relax_last_error().
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

using namespace relax;

namespace relax_shim {

struct ShimState {
    bool init = false;
    int sx1 = 0, sx2 = 0, sx3 = 0;
    double dx1 = 1, dx2 = 1, dx3 = 1;
    float *v[3] = {nullptr, nullptr, nullptr};   // (sx1+2, sx2, sx3)
    float *u[3] = {nullptr, nullptr, nullptr};   // (sx1+2, sx2, sx3/2)
    float *t[3] = {nullptr, nullptr, nullptr};   // (sx1+2, sx2)
    relax_tensor *sig = nullptr, *mom = nullptr, *tau = nullptr;
    float *work = nullptr;                        // 3 x sx1 sx2 sx3/2 + 3 x sx1 sx2
    // transient rheology (cuinflags_) and weak-zone fluidity fields
    // (E_GAMMADOT0_TYPE 1..4: linear, nonlinear, linear / nonlinear transient)
    bool transient = false;
    relax_tensor *eps = nullptr, *epsdot = nullptr;
    float *dg[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t nvec() const { return (size_t)(sx1 + 2) * sx2 * sx3; }
    size_t nhalf() const { return (size_t)(sx1 + 2) * sx2 * (sx3 / 2); }
    size_t ntens() const { return (size_t)sx1 * sx2 * (sx3 / 2); }
    size_t n2() const { return (size_t)(sx1 + 2) * sx2; }
};

ShimState S;

void release()
{
    for (int k = 0; k < 3; k++) {
        if (S.v[k]) cudaFree(S.v[k]);
        if (S.u[k]) cudaFree(S.u[k]);
        if (S.t[k]) cudaFree(S.t[k]);
        S.v[k] = S.u[k] = S.t[k] = nullptr;
    }
    if (S.sig) cudaFree(S.sig);
    if (S.mom) cudaFree(S.mom);
    if (S.tau) cudaFree(S.tau);
    if (S.work) cudaFree(S.work);
    if (S.eps) cudaFree(S.eps);
    if (S.epsdot) cudaFree(S.epsdot);
    for (int k = 0; k < 4; k++) {
        if (S.dg[k]) cudaFree(S.dg[k]);
        S.dg[k] = nullptr;
    }
    S.eps = S.epsdot = nullptr;
    S.sig = S.mom = S.tau = nullptr;
    S.work = nullptr;
    S.init = false;
}

relax_tensor *tensor_of(int type)
{
    // E_TENSOR_TYPE, src/cuinclude.h:121-129
    return type == 1 ? S.sig : type == 2 ? S.mom : type == 3 ? S.tau : type == 4 ? S.eps
                                                                   : type == 5 ? S.epsdot : nullptr;
}

__global__ void k_axpby_vec(float *a, const float *b, size_t n, float c1, float c2)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) a[q] = c1 * a[q] + c2 * b[q];
}

// tensorfieldadd, src/elastic3d.f90:3880-3959 (c1 = 0 branches included)
__global__ void k_axpby_tensor(relax_tensor *t1, const relax_tensor *t2, size_t n, float c1, float c2)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    float *a = reinterpret_cast<float *>(t1 + q);
    const float *b = reinterpret_cast<const float *>(t2 + q);
    for (int c = 0; c < 6; c++) {
        if (c1 == 0.f) a[c] = c2 == 0.f ? 0.f : c2 * b[c];
        else a[c] = c1 * a[c] + c2 * b[c];
    }
}

// add a compact (sx1, sx2, n3) field into a padded (sx1+2, sx2, n3) one
__global__ void k_add_padded(float *dst, const float *src, int sx1, size_t nrows)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nrows * sx1) return;
    const size_t r = q / sx1, i = q % sx1;
    dst[r * (sx1 + 2) + i] += src[q];
}

unsigned nb(size_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace relax_shim

using namespace relax_shim;

extern "C" {

void cuinflags_(int *istransient, int *nlwz, int *nnlwz, int *nltwz, int *nnltwz, int islinear,
                int isnonlinear, int isltransient, int isnltransient, int *iRet)
{
    (void)nlwz; (void)nnlwz; (void)nltwz; (void)nnltwz; (void)islinear; (void)isnonlinear;
    (void)isltransient; (void)isnltransient;
    // the weak-zone fields are allocated by cubuildgammadot_; epsilonik and
    // epsilonikdot by cuinit_ when the transient rheology is on
    S.transient = istransient && *istransient;
    if (iRet) *iRet = 0;
}

void cuinit_(int sx1, int sx2, int sx3, double dx1, double dx2, double dx3, int *iRet)
{
    release();
    S.sx1 = sx1; S.sx2 = sx2; S.sx3 = sx3; S.dx1 = dx1; S.dx2 = dx2; S.dx3 = dx3;
    bool ok = sx1 > 0 && sx2 > 0 && sx3 > 1;
    for (int k = 0; k < 3 && ok; k++) {
        ok &= cudaMalloc(&S.v[k], S.nvec() * sizeof(float)) == cudaSuccess;
        ok &= cudaMalloc(&S.u[k], S.nhalf() * sizeof(float)) == cudaSuccess;
        ok &= cudaMalloc(&S.t[k], S.n2() * sizeof(float)) == cudaSuccess;
        if (ok) {
            cudaMemset(S.v[k], 0, S.nvec() * sizeof(float));
            cudaMemset(S.u[k], 0, S.nhalf() * sizeof(float));
            cudaMemset(S.t[k], 0, S.n2() * sizeof(float));
        }
    }
    if (ok) {
        ok &= cudaMalloc(&S.sig, S.ntens() * sizeof(relax_tensor)) == cudaSuccess;
        ok &= cudaMalloc(&S.mom, S.ntens() * sizeof(relax_tensor)) == cudaSuccess;
        ok &= cudaMalloc(&S.tau, S.ntens() * sizeof(relax_tensor)) == cudaSuccess;
        ok &= cudaMalloc(&S.work, (3 * (size_t)sx1 * sx2 * (sx3 / 2) + 3 * (size_t)sx1 * sx2) * sizeof(float)) == cudaSuccess;
    }
    if (ok && S.transient) {
        ok &= cudaMalloc(&S.eps, S.ntens() * sizeof(relax_tensor)) == cudaSuccess;
        ok &= cudaMalloc(&S.epsdot, S.ntens() * sizeof(relax_tensor)) == cudaSuccess;
        if (ok) {
            cudaMemset(S.eps, 0, S.ntens() * sizeof(relax_tensor));
            cudaMemset(S.epsdot, 0, S.ntens() * sizeof(relax_tensor));
        }
    }
    if (ok) {
        cudaMemset(S.sig, 0, S.ntens() * sizeof(relax_tensor));
        cudaMemset(S.mom, 0, S.ntens() * sizeof(relax_tensor));
        cudaMemset(S.tau, 0, S.ntens() * sizeof(relax_tensor));
        ok &= cudaDeviceSynchronize() == cudaSuccess;
    }
    if (!ok) release();
    S.init = ok;
    if (iRet) *iRet = ok ? 0 : 1;
}

void cudeinit_(void)
{
    release();
}

void curesetvectors_(void)
{
    if (!S.init) return;
    for (int k = 0; k < 3; k++) {
        cudaMemset(S.v[k], 0, S.nvec() * sizeof(float));
        cudaMemset(S.t[k], 0, S.n2() * sizeof(float));
    }
    cudaDeviceSynchronize();
}

void cutensormemset_(int eType)
{
    relax_tensor *p = tensor_of(eType);
    if (!S.init || !p) return;
    cudaMemset(p, 0, S.ntens() * sizeof(relax_tensor));
    cudaDeviceSynchronize();
}

void copytau_(ST_TENSOR_C *host, int sx1, int sx2, int sx3h, int dir)
{
    if (!S.init || !host) return;
    const size_t n = (size_t)sx1 * sx2 * sx3h * sizeof(relax_tensor);
    if (dir == 1) cudaMemcpy(S.tau, host, n, cudaMemcpyHostToDevice);
    else cudaMemcpy(host, S.tau, n, cudaMemcpyDeviceToHost);
}

void cucopytraction_(float *t3, int sx1, int sx2, int *iRet)
{
    int r = 1;
    if (S.init && t3)
        r = cudaMemcpy(t3, S.t[2], (size_t)(sx1 + 2) * sx2 * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : 1;
    if (iRet) *iRet = r;
}

void cufieldadd_(int eType, float *a, float *b, float *c, float *d, float *e, float *f, int sx1p2, int sx2,
                 int sx3h, float c1, float c2)
{
    (void)a; (void)b; (void)c; (void)d; (void)e; (void)f;
    if (!S.init) return;
    const size_t n = (size_t)sx1p2 * sx2 * sx3h;
    for (int k = 0; k < 3; k++) {
        if (eType == 1) k_axpby_vec<<<nb(n), 256>>>(S.u[k], S.v[k], n, c1, c2);
        else if (eType == 2) k_axpby_vec<<<nb(n), 256>>>(S.v[k], S.u[k], n, c1, c2);
    }
    cudaDeviceSynchronize();
}

void cufieldrep_(int sx1p2, int sx2, int sx3h)
{
    float *dummy = nullptr;
    cufieldadd_(1, dummy, dummy, dummy, dummy, dummy, dummy, sx1p2, sx2, sx3h, 0.f, 1.f);
}

void cutensorfieldadd_(int eField, int sx1, int sx2, int sx3h, float c1, float c2)
{
    if (!S.init) return;
    // E_TENSOR_FIELD, src/cuinclude.h:100-111
    relax_tensor *pairs[9][2] = {{nullptr, nullptr}, {S.tau, S.tau}, {S.sig, S.tau},
                                 {S.mom, S.mom}, {S.sig, S.mom}, {S.tau, S.mom},
                                 {S.eps, S.epsdot}, {S.epsdot, S.eps}, {S.epsdot, S.epsdot}};
    if (eField < 1 || eField > 8 || !pairs[eField][0] || !pairs[eField][1]) return;
    const size_t n = (size_t)sx1 * sx2 * sx3h;
    k_axpby_tensor<<<nb(n), 256>>>(pairs[eField][0], pairs[eField][1], n, c1, c2);
    cudaDeviceSynchronize();
}

void custressupdatewrapper_(int eType, double lambda, double mu, double dx1, double dx2, double dx3, int sx1,
                            int sx2, int sx3h, float *u1, float *u2, float *u3, ST_TENSOR_C *sig)
{
    (void)u1; (void)u2; (void)u3; (void)sig;
    if (!S.init) return;
    float **w = eType == 2 ? S.v : S.u;
    relax_op_stressupdate(w[0], w[1], w[2], lambda, mu, dx1, dx2, dx3, sx1, sx2, sx3h, S.sig, nullptr);
    cudaDeviceSynchronize();
}

void cubodyforceswrapper_(int eType, double dx1, double dx2, double dx3, int sx1, int sx2, int sx3h, float *v1,
                          float *v2, float *v3, float *t1, float *t2, float *t3)
{
    (void)v1; (void)v2; (void)v3; (void)t1; (void)t2; (void)t3;
    if (!S.init) return;
    const relax_tensor *src = eType == 2 ? S.mom : S.sig;
    relax_op_bodyforce(src, dx1, dx2, dx3, sx1, sx2, sx3h, S.v[0], S.v[1], S.v[2], S.t[0], S.t[1], S.t[2],
                       nullptr);
    cudaDeviceSynchronize();
}

void calfftnelasic_(float *c1, float *c2, float *c3, float *t1, float *t2, float *t3, int sx1, int sx2, int sx3,
                    double dx1, double dx2, double dx3, double lambda, double mu, double gam, float *p1,
                    float *p2, float *p3, int *iRet)
{
    (void)c1; (void)c2; (void)c3; (void)t1; (void)t2; (void)t3; (void)p1; (void)p2; (void)p3;
    int r = 1;
    if (S.init)
        r = relax_op_green(S.v[0], S.v[1], S.v[2], S.t[0], S.t[1], S.t[2], sx1, sx2, sx3, dx1, dx2, dx3, lambda,
                           mu, gam, nullptr) == RELAX_OK ? 0 : 1;
    cudaDeviceSynchronize();
    if (iRet) *iRet = r;
}

void cuviscouseigen_(relax_layer *structure, relax_tensor_layer *prestress, double mu, int sx1, int sx2, int sx3h,
                     double dx1, double dx2, double dx3, int bMaxwell, double *tm, int gammadot0type)
{
    (void)dx1; (void)dx2; (void)dx3;
    if (!S.init) return;
    // E_GAMMADOT0_TYPE_LINEAR / _NONLINEAR: the field of cubuildgammadot_
    const float *dg = (gammadot0type == 1 || gammadot0type == 2) ? S.dg[gammadot0type - 1] : nullptr;
    relax_op_viscouseigenstress(mu, structure, prestress, S.sig, sx1, sx2, sx3h, S.mom, bMaxwell ? tm : nullptr,
                                nullptr, dg, nullptr);
    cudaDeviceSynchronize();
}

void cufrictioneigenstress_(double x, double y, double z, double L, double W, double strike, double dip,
                            double rake, double beta, double mu, relax_layer *structure, int sx1, int sx2,
                            int sx3h, double dx1, double dx2, double dx3, int bPresent, float *tm,
                            ST_TENSOR_C *moment, ST_TENSOR_C *sig)
{
    (void)moment; (void)sig;
    if (!S.init) return;
    double t = tm ? (double)*tm : 1e30;
    relax_op_frictioneigenstress(x, y, z, L, W, strike, dip, rake, beta, S.sig, mu, structure, sx1, sx2, sx3h,
                                 dx1, dx2, dx3, S.mom, bPresent ? &t : nullptr, nullptr);
    if (bPresent && tm) *tm = (float)t;
}

void cutensoramp_(int eType, int sx1, int sx2, int sx3h, double *amp)
{
    if (!S.init || !amp) return;
    const relax_tensor *p = eType == 1 ? S.mom : S.tau;   // E_TENSOR_AMP_TYPE
    relax_op_tensoramplitude(p, sx1, sx2, sx3h, 1.0, 1.0, 1.0, amp, nullptr);
}

void cusource_(double mu, double s, double x, double y, double z, double L, double W, double strike, double dip,
               double rake, double beta, int sx1, int sx2, int sx3, double dx1, double dx2, double dx3, float *f1,
               float *f2, float *f3, float *t1, float *t2, float *t3)
{
    (void)f1; (void)f2; (void)f3; (void)t1; (void)t2; (void)t3;
    if (!S.init) return;
    Grid g{};
    g.sx1 = sx1; g.sx2 = sx2; g.sx3 = sx3; g.sx3h = sx3 / 2; g.M = sx1 / 2; g.K1 = sx1 / 2 + 1;
    g.dx1 = dx1; g.dx2 = dx2; g.dx3 = dx3; g.plane = (size_t)sx1 * sx2; g.nh = g.plane * g.sx3h;
    const size_t nw = 3 * g.nh + 3 * g.plane;
    cudaMemset(S.work, 0, nw * sizeof(float));
    SrcArgs a{};
    a.g = g; a.mu = mu; a.s = s; a.x = x; a.y = y; a.z = z; a.L = L; a.W = W;
    a.strike = strike; a.dip = dip; a.rake = rake; a.beta = beta;
    for (int k = 0; k < 3; k++) {
        a.f[k] = S.work + k * g.nh;
        a.t[k] = S.work + 3 * g.nh + k * g.plane;
    }
    k_source_traction<<<nb(g.plane), 256>>>(a);
    k_source_force<<<nb(g.nh), 256>>>(a);
    for (int k = 0; k < 3; k++) {
        k_add_padded<<<nb(g.nh), 256>>>(S.v[k], a.f[k], sx1, (size_t)sx2 * g.sx3h);
        k_add_padded<<<nb(g.plane), 256>>>(S.t[k], a.t[k], sx1, (size_t)sx2);
    }
    cudaDeviceSynchronize();
}


// cutransienteigenwrapper_, src/cuelastic.cu:1085-1118: transienteigenstress
// on epsilonik (E_TENSOR_IK) or epsilonikdot (E_TENSOR_IKDOT, the
// corrector's in-place call) into epsilonikdot and the moment;
// E_GAMMADOT0_TYPE 3 / 4 select the transient weak-zone fields
void cutransienteigenwrapper_(int eType, relax_layer *structure, double mu, int sx1, int sx2, int sx3h,
                              double dx1, double dx2, double dx3, int bMaxwell, double *dMaxwell, int bgammadot)
{
    (void)dx1; (void)dx2; (void)dx3;
    if (!S.init || !S.eps) return;
    const relax_tensor *in = eType == 4 ? S.eps : eType == 5 ? S.epsdot : nullptr;
    if (!in) return;
    const float *dg = (bgammadot == 3 || bgammadot == 4) ? S.dg[bgammadot - 1] : nullptr;
    relax_op_transienteigenstress(mu, structure, S.sig, in, sx1, sx2, sx3h, S.mom, S.epsdot,
                                  bMaxwell ? dMaxwell : nullptr, dg, nullptr);
    cudaDeviceSynchronize();
}

// cubuildgammadot_, src/cuelastic.cu:1689-1750: the weak-zone field of one
// mechanism (beta = 0, as src/relax.f90:487-541 and the reference kernel)
void cubuildgammadot_(int sx1, int sx2, int sx3h, double dx1, double dx2, double dx3, int nz,
                      relax_weakzone *zones, int gammadotType)
{
    if (!S.init || gammadotType < 1 || gammadotType > 4) return;
    float *&d = S.dg[gammadotType - 1];
    const size_t n = (size_t)sx1 * sx2 * sx3h;
    if (!d && cudaMalloc(&d, n * sizeof(float)) != cudaSuccess) {
        d = nullptr;
        return;
    }
    relax_op_dgammadot0(zones, nz, sx1, sx2, sx3h, dx1, dx2, dx3, 0.0, d, nullptr);
    cudaDeviceSynchronize();
}

// cuexportspatial_, src/cuelastic.cu:1629-1650: one x3-plane of the padded
// displacement components to the host
void cuexportspatial_(float *u1, float *u2, float *u3, int i3)
{
    if (!S.init || i3 < 0 || i3 >= S.sx3 / 2) return;
    const size_t off = (size_t)i3 * S.n2();
    float *h[3] = {u1, u2, u3};
    for (int k = 0; k < 3; k++)
        if (h[k]) cudaMemcpy(h[k], S.u[k] + off, S.n2() * sizeof(float), cudaMemcpyDeviceToHost);
}

// cuexportpoints_, src/cuelastic.cu:1652-1687: displacement and stress at
// one grid point (0-based indices)
void cuexportpoints_(double *u1, double *u2, double *u3, ST_TENSOR_C *sig, int i1, int i2, int i3)
{
    if (!S.init || i1 < 0 || i1 >= S.sx1 || i2 < 0 || i2 >= S.sx2 || i3 < 0 || i3 >= S.sx3 / 2) return;
    const size_t iu = ((size_t)i3 * S.sx2 + i2) * (S.sx1 + 2) + i1;
    const size_t is = ((size_t)i3 * S.sx2 + i2) * S.sx1 + i1;
    double *h[3] = {u1, u2, u3};
    for (int k = 0; k < 3; k++) {
        float v = 0.f;
        cudaMemcpy(&v, S.u[k] + iu, sizeof(float), cudaMemcpyDeviceToHost);
        if (h[k]) *h[k] = (double)v;
    }
    if (sig) cudaMemcpy(sig, S.sig + is, sizeof(relax_tensor), cudaMemcpyDeviceToHost);
}

}  // extern "C"
