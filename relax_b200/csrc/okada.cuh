// okada.cuh -- displacement of a rectangular dislocation in an elastic
// half-space, Okada (1992), "Internal deformation due to shear and tensile
// faults in a half-space", Bull. Seism. Soc. Am. 82(2), 1018-1040.
//
// RELAX adds this space-domain solution for the coseismic sources smaller
// than the Nyquist length (dislocations_disp, src/relax.f90:1298-1349,
// through grnfct_okada / okada of src/okada/green_space.f90:29-144, which
// call the DC3D routine of src/okada/dc3d.f).  The paper's solution is
// restated here from its equations (displacement only): the sum over the
// four corners of the fault (Chinnery's notation) of
//
//   u = -A(real source, d = c + z) + [A + B + z C](image source, d = c - z)
//
// in the fault-aligned frame (x along strike, z up, observation z <= 0),
// with the paper's functions f^A, f^B, f^C of Table 6 and the integrals
// I1..I4 (cos(dip) = 0 handled by their limits).  Corners on the negative
// extension of a fault edge use the regularised logarithms; points on a
// fault edge give zero (the DC3D convention).  Arithmetic is FP64.
#pragma once

#include <math.h>

namespace relax {

struct OkadaConst {
    double alp1, alp2, alp3, alp4, alp5;   // (1-a)/2, a/2, (1-a)/a, 1-a, a
    double sd, cd;
};

struct OkadaCorner {
    double xi, et, q, r, y, d, tt, alx, ale, x11, y11, x32, y32;
};

__host__ __device__ inline void okada_corner(double xi, double et, double q, const OkadaConst &k, int kxi, int ket,
                                             OkadaCorner &c)
{
    const double eps = 1e-6;
    if (fabs(xi) < eps) xi = 0.0;
    if (fabs(et) < eps) et = 0.0;
    if (fabs(q) < eps) q = 0.0;
    c.xi = xi; c.et = et; c.q = q;
    const double r2 = xi * xi + et * et + q * q;
    c.r = sqrt(r2);
    c.y = et * k.cd + q * k.sd;      // y~ of the paper
    c.d = et * k.sd - q * k.cd;      // d~
    c.tt = (q == 0.0) ? 0.0 : atan(xi * et / (q * c.r));
    if (kxi) {
        c.alx = -log(c.r - xi); c.x11 = 0.0; c.x32 = 0.0;
    } else {
        const double rxi = c.r + xi;
        c.alx = log(rxi);
        c.x11 = 1.0 / (c.r * rxi);
        c.x32 = (c.r + rxi) * c.x11 * c.x11 / c.r;
    }
    if (ket) {
        c.ale = -log(c.r - et); c.y11 = 0.0; c.y32 = 0.0;
    } else {
        const double ret = c.r + et;
        c.ale = log(ret);
        c.y11 = 1.0 / (c.r * ret);
        c.y32 = (c.r + ret) * c.y11 * c.y11 / c.r;
    }
}

// f^A of Table 6 (per unit dislocation, without 1/2pi)
__host__ __device__ inline void okada_fa(const OkadaCorner &c, const OkadaConst &k, const double disl[3], double u[3])
{
    const double qx = c.q * c.x11, qy = c.q * c.y11;
    u[0] = u[1] = u[2] = 0.0;
    if (disl[0] != 0.0) {   // strike slip
        u[0] += disl[0] * (c.tt / 2.0 + k.alp2 * c.xi * qy);
        u[1] += disl[0] * (k.alp2 * c.q / c.r);
        u[2] += disl[0] * (k.alp1 * c.ale - k.alp2 * c.q * qy);
    }
    if (disl[1] != 0.0) {   // dip slip
        u[0] += disl[1] * (k.alp2 * c.q / c.r);
        u[1] += disl[1] * (c.tt / 2.0 + k.alp2 * c.et * qx);
        u[2] += disl[1] * (k.alp1 * c.alx - k.alp2 * c.q * qx);
    }
    if (disl[2] != 0.0) {   // tensile
        u[0] += disl[2] * (-k.alp1 * c.ale - k.alp2 * c.q * qy);
        u[1] += disl[2] * (-k.alp1 * c.alx - k.alp2 * c.q * qx);
        u[2] += disl[2] * (c.tt / 2.0 - k.alp2 * (c.et * qx + c.xi * qy));
    }
}

// f^B of Table 6 with the integrals I1..I4
__host__ __device__ inline void okada_fb(const OkadaCorner &c, const OkadaConst &k, const double disl[3], double u[3])
{
    const double rd = c.r + c.d;
    double ai3, ai4;
    if (k.cd != 0.0) {
        const double cdcd = k.cd * k.cd;
        if (c.xi == 0.0) {
            ai4 = 0.0;
        } else {
            const double x = sqrt(c.xi * c.xi + c.q * c.q);
            ai4 = (c.xi / rd * k.sd * k.cd +
                   2.0 * atan((c.et * (x + c.q * k.cd) + x * (c.r + x) * k.sd) / (c.xi * (c.r + x) * k.cd))) / cdcd;
        }
        ai3 = (c.y * k.cd / rd - c.ale + k.sd * log(rd)) / cdcd;
    } else {
        const double rd2 = rd * rd;
        ai3 = (c.et / rd + c.y * c.q / rd2 - c.ale) / 2.0;
        ai4 = c.xi * c.y / rd2 / 2.0;
    }
    const double ai1 = -c.xi / rd * k.cd - ai4 * k.sd;
    const double ai2 = log(rd) + ai3 * k.sd;
    const double qx = c.q * c.x11, qy = c.q * c.y11;
    const double sdcd = k.sd * k.cd, sdsd = k.sd * k.sd;
    u[0] = u[1] = u[2] = 0.0;
    if (disl[0] != 0.0) {
        u[0] += disl[0] * (-c.xi * qy - c.tt - k.alp3 * ai1 * k.sd);
        u[1] += disl[0] * (-c.q / c.r + k.alp3 * c.y / rd * k.sd);
        u[2] += disl[0] * (c.q * qy - k.alp3 * ai2 * k.sd);
    }
    if (disl[1] != 0.0) {
        u[0] += disl[1] * (-c.q / c.r + k.alp3 * ai3 * sdcd);
        u[1] += disl[1] * (-c.et * qx - c.tt - k.alp3 * c.xi / rd * sdcd);
        u[2] += disl[1] * (c.q * qx + k.alp3 * ai4 * sdcd);
    }
    if (disl[2] != 0.0) {
        u[0] += disl[2] * (c.q * qy - k.alp3 * ai3 * sdsd);
        u[1] += disl[2] * (c.q * qx + k.alp3 * c.xi / rd * sdsd);
        u[2] += disl[2] * (c.et * qx + c.xi * qy - c.tt - k.alp3 * ai4 * sdsd);
    }
}

// f^C of Table 6 (observation depth z <= 0)
__host__ __device__ inline void okada_fc(const OkadaCorner &c, double z, const OkadaConst &k, const double disl[3],
                                         double u[3])
{
    const double cc = c.d + z;                 // c-bar
    const double r3 = c.r * c.r * c.r;
    const double h = c.q * k.cd - z;
    const double z32 = k.sd / r3 - h * c.y32;
    const double xy = c.xi * c.y11, qy = c.q * c.y11, q2 = c.q * c.q;
    u[0] = u[1] = u[2] = 0.0;
    if (disl[0] != 0.0) {
        u[0] += disl[0] * (k.alp4 * xy * k.cd - k.alp5 * c.xi * c.q * z32);
        u[1] += disl[0] * (k.alp4 * (k.cd / c.r + 2.0 * qy * k.sd) - k.alp5 * cc * c.q / r3);
        u[2] += disl[0] * (k.alp4 * qy * k.cd - k.alp5 * (cc * c.et / r3 - z * c.y11 + c.xi * c.xi * z32));
    }
    if (disl[1] != 0.0) {
        u[0] += disl[1] * (k.alp4 * k.cd / c.r - qy * k.sd - k.alp5 * cc * c.q / r3);
        u[1] += disl[1] * (k.alp4 * c.y * c.x11 - k.alp5 * cc * c.et * c.q * c.x32);
        u[2] += disl[1] * (-c.d * c.x11 - xy * k.sd - k.alp5 * cc * (c.x11 - q2 * c.x32));
    }
    if (disl[2] != 0.0) {
        u[0] += disl[2] * (-k.alp4 * (k.sd / c.r + qy * k.cd) - k.alp5 * (z * c.y11 - q2 * z32));
        u[1] += disl[2] * (k.alp4 * 2.0 * xy * k.sd + c.d * c.x11 - k.alp5 * cc * (c.x11 - q2 * c.x32));
        u[2] += disl[2] * (k.alp4 * (c.y * c.x11 + xy * k.cd) + k.alp5 * c.q * (cc * c.et * c.x32 + c.xi * z32));
    }
}

// Displacement (ux, uy, uz) at (x, y, z <= 0) of the fault [al1, al2] x
// [aw1, aw2] (along strike, up dip) whose reference point is at depth
// `depth`, dip in degrees, dislocation (strike, dip, opening).  Returns 0,
// 1 on a fault edge (u = 0) or 2 for z > 0 (u = 0).
__host__ __device__ inline int okada_disp(double alpha, double x, double y, double z, double depth, double dipdeg,
                                          double al1, double al2, double aw1, double aw2, const double disl[3],
                                          double u[3])
{
    const double eps = 1e-6, pi2 = 6.283185307179586476925286766559;
    u[0] = u[1] = u[2] = 0.0;
    if (z > 0.0) return 2;
    OkadaConst k;
    k.alp1 = (1.0 - alpha) / 2.0; k.alp2 = alpha / 2.0; k.alp3 = (1.0 - alpha) / alpha;
    k.alp4 = 1.0 - alpha; k.alp5 = alpha;
    const double dip = dipdeg * 0.01745329251994329547437168059786927;
    k.sd = sin(dip); k.cd = cos(dip);
    if (fabs(k.cd) < eps) {
        k.cd = 0.0;
        k.sd = k.sd > 0.0 ? 1.0 : -1.0;
    }
    double xi[2] = {x - al1, x - al2};
    for (int i = 0; i < 2; i++)
        if (fabs(xi[i]) < eps) xi[i] = 0.0;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int pass = 0; pass < 2; pass++) {   // 0: real source, 1: image source
        const double d = pass == 0 ? depth + z : depth - z;
        const double p = y * k.cd + d * k.sd;
        double q = y * k.sd - d * k.cd;
        double et[2] = {p - aw1, p - aw2};
        if (fabs(q) < eps) q = 0.0;
        for (int i = 0; i < 2; i++)
            if (fabs(et[i]) < eps) et[i] = 0.0;
        // on a fault edge: singular
        if (q == 0.0 && ((xi[0] * xi[1] <= 0.0 && et[0] * et[1] == 0.0) || (et[0] * et[1] <= 0.0 && xi[0] * xi[1] == 0.0)))
            return 1;
        // on the negative extension of a fault edge: regularised logarithms
        int kxi[2] = {0, 0}, ket[2] = {0, 0};
        const double r12 = sqrt(xi[0] * xi[0] + et[1] * et[1] + q * q);
        const double r21 = sqrt(xi[1] * xi[1] + et[0] * et[0] + q * q);
        const double r22 = sqrt(xi[1] * xi[1] + et[1] * et[1] + q * q);
        if (xi[0] < 0.0 && r21 + xi[1] < eps) kxi[0] = 1;
        if (xi[0] < 0.0 && r22 + xi[1] < eps) kxi[1] = 1;
        if (et[0] < 0.0 && r12 + et[1] < eps) ket[0] = 1;
        if (et[0] < 0.0 && r22 + et[1] < eps) ket[1] = 1;
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++) {
                OkadaCorner c;
                okada_corner(xi[a], et[b], q, k, kxi[b], ket[a], c);
                if (c.r == 0.0) continue;
                double du[3];
                if (pass == 0) {
                    double fa[3];
                    okada_fa(c, k, disl, fa);
                    du[0] = -fa[0];
                    du[1] = -fa[1] * k.cd + fa[2] * k.sd;
                    du[2] = -fa[1] * k.sd - fa[2] * k.cd;
                } else {
                    double fa[3], fb[3], fc[3];
                    okada_fa(c, k, disl, fa);
                    okada_fb(c, k, disl, fb);
                    okada_fc(c, z, k, disl, fc);
                    du[0] = fa[0] + fb[0] + z * fc[0];
                    du[1] = (fa[1] + fb[1] + z * fc[1]) * k.cd - (fa[2] + fb[2] + z * fc[2]) * k.sd;
                    du[2] = (fa[1] + fb[1] - z * fc[1]) * k.sd + (fa[2] + fb[2] - z * fc[2]) * k.cd;
                }
                const double s = (a + b == 1) ? -1.0 : 1.0;   // Chinnery's alternating corners
                for (int i = 0; i < 3; i++) acc[i] += s * du[i];
            }
    }
    for (int i = 0; i < 3; i++) u[i] = acc[i] / pi2;
    return 0;
}

// okada of src/okada/green_space.f90:29-105: a source in RELAX's input
// convention (north x1, east x2, depth x3 of the top edge, strike/dip/rake
// in degrees) at a receiver (north, east, depth); displacement in RELAX's
// frame (x3 positive down).
__host__ __device__ inline void okada_relax(double lambda, double mu, double slip, double opening, double x1,
                                            double x2, double x3, double width, double length, double strike,
                                            double dipd, double rake, double xr, double yr, double zr, double d[3])
{
    const double deg = 0.01745329251994329547437168059786927;
    const double alpha = (lambda + mu) / (lambda + 2.0 * mu);
    const double st = strike * deg, ra = rake * deg;
    const double cs = cos(st), ss = sin(st);
    const double x = (xr - x1) * cs + (yr - x2) * ss;
    const double y = (xr - x1) * ss - (yr - x2) * cs;
    const double disl[3] = {slip * cos(ra), slip * sin(ra), opening};
    double u[3];
    const int iret = okada_disp(alpha, x, y, -zr, x3, dipd, 0.0, length, -width, 0.0, disl, u);
    if (iret != 0) {
        d[0] = d[1] = d[2] = 0.0;
        return;
    }
    d[0] = u[0] * cs + u[1] * ss;
    d[1] = u[0] * ss - u[1] * cs;
    d[2] = -u[2];
}

}  // namespace relax
