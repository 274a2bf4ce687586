// export.cu -- RELAX's output files written from the device fields:
//
//   * GMT grids: netCDF classic (CDF-1) files with the layout of
//     writeNetcdf, src/exportnetcdf.f90:54-127 (x, y double coordinates,
//     z float, long_name / actual_range attributes, node_offset = 1,
//     COARDS conventions), for the slices of exportgrd, src/export.f90:917-1057;
//   * VTK legacy binary files of a vector or a tensor field,
//     src/writevtk.c:72-141 and the tensor variant that follows it;
//   * the .ned time series at observation points, src/util.f90:83-124;
//   * the afterslip planes, the observation planes and the stress
//     observation segments, src/export.f90:308-849, :1364-2005;
//   * the step log line, formats 1100-1103 of src/relax.f90:1102-1105.
//
// The netCDF classic format is written directly (big-endian header and
// data, 4-byte alignment) from its published specification; no netCDF
// library is involved.
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <initializer_list>
#include <string>
#include <utility>
#include <vector>

#include "../../include/relax_b200.h"

extern "C" __attribute__((visibility("hidden"))) int relax_noalloc_fail(int code, const char *msg);

namespace {

int fail(int code, const char *fmt, ...)
{
    char msg[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, sizeof msg, fmt, ap);
    va_end(ap);
    return relax_noalloc_fail(code, msg);
}

// ---------------------------------------------------------------------------
// netCDF classic (CDF-1) writer for one 2-D grid
// ---------------------------------------------------------------------------
enum { NC_CHAR = 2, NC_INT = 4, NC_FLOAT = 5, NC_DOUBLE = 6 };
enum { NC_DIMENSION = 0x0A, NC_VARIABLE = 0x0B, NC_ATTRIBUTE = 0x0C };

struct Buf {
    std::vector<unsigned char> b;
    void u32(uint32_t v)
    {
        for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void f32(float v)
    {
        uint32_t u;
        memcpy(&u, &v, 4);
        u32(u);
    }
    void f64(double v)
    {
        uint64_t u;
        memcpy(&u, &v, 8);
        u32((uint32_t)(u >> 32));
        u32((uint32_t)u);
    }
    void pad()
    {
        while (b.size() % 4) b.push_back(0);
    }
    void name(const char *s)
    {
        const size_t n = strlen(s);
        u32((uint32_t)n);
        b.insert(b.end(), s, s + n);
        pad();
    }
};

struct Att {
    std::string name;
    int type;
    std::string text;
    std::vector<double> vals;
};

void put_atts(Buf &h, const std::vector<Att> &atts)
{
    if (atts.empty()) {
        h.u32(0);
        h.u32(0);
        return;
    }
    h.u32(NC_ATTRIBUTE);
    h.u32((uint32_t)atts.size());
    for (const Att &a : atts) {
        h.name(a.name.c_str());
        h.u32((uint32_t)a.type);
        if (a.type == NC_CHAR) {
            h.u32((uint32_t)a.text.size());
            h.b.insert(h.b.end(), a.text.begin(), a.text.end());
            h.pad();
        } else {
            h.u32((uint32_t)a.vals.size());
            for (double v : a.vals) {
                if (a.type == NC_INT) h.u32((uint32_t)(int32_t)v);
                else if (a.type == NC_FLOAT) h.f32((float)v);
                else h.f64(v);
            }
            h.pad();
        }
    }
}

// writeNetcdf with registration 1: z(nx, ny), x fastest
int write_grd(const float *z, int nx, int ny, double x0, double y0, double dx, double dy, const char *title,
              const char *filename)
{
    if (!z || !filename || nx < 2 || ny < 2) return fail(RELAX_ERR_ARG, "grid: null argument or size < 2");
    std::vector<double> x(nx), y(ny);
    for (int i = 0; i < nx; i++) x[i] = x0 + (double)i * dx;
    for (int i = 0; i < ny; i++) y[i] = y0 + (double)i * dy;
    float zmin = z[0], zmax = z[0];
    for (size_t i = 0; i < (size_t)nx * ny; i++) {
        zmin = std::fmin(zmin, z[i]);
        zmax = std::fmax(zmax, z[i]);
    }
    const std::vector<Att> gatts = {
        {"node_offset", NC_INT, "", {1.0}},
        {"title", NC_CHAR, title ? title : "", {}},
        {"history", NC_CHAR, "Relax output", {}},
        {"Conventions", NC_CHAR, "COARDS/CF-1.0", {}}};
    const std::vector<Att> xatts = {
        {"long_name", NC_CHAR, "x", {}},
        {"actual_range", NC_DOUBLE, "", {x[0] - 0.5 * (x[1] - x[0]), x[nx - 1] + 0.5 * (x[nx - 1] - x[nx - 2])}}};
    const std::vector<Att> yatts = {
        {"long_name", NC_CHAR, "y", {}},
        {"actual_range", NC_DOUBLE, "", {y[0] - 0.5 * (y[1] - y[0]), y[ny - 1] + 0.5 * (y[ny - 1] - y[ny - 2])}}};
    const std::vector<Att> zatts = {{"long_name", NC_CHAR, "z", {}},
                                    {"actual_range", NC_FLOAT, "", {(double)zmin, (double)zmax}}};
    const uint32_t xsize = 8u * nx, ysize = 8u * ny, zsize = 4u * (uint32_t)nx * ny;
    // the header twice: once to size it, once with the data offsets
    auto header = [&](uint32_t begin0) {
        Buf h;
        h.b = {'C', 'D', 'F', 1};
        h.u32(0);                       // numrecs
        h.u32(NC_DIMENSION);
        h.u32(2);
        h.name("x");
        h.u32((uint32_t)nx);
        h.name("y");
        h.u32((uint32_t)ny);
        put_atts(h, gatts);
        h.u32(NC_VARIABLE);
        h.u32(3);
        uint32_t begin = begin0;
        // x(x)
        h.name("x"); h.u32(1); h.u32(0); put_atts(h, xatts); h.u32(NC_DOUBLE); h.u32(xsize); h.u32(begin);
        begin += xsize;
        // y(y)
        h.name("y"); h.u32(1); h.u32(1); put_atts(h, yatts); h.u32(NC_DOUBLE); h.u32(ysize); h.u32(begin);
        begin += ysize;
        // z(y, x)
        h.name("z"); h.u32(2); h.u32(1); h.u32(0); put_atts(h, zatts); h.u32(NC_FLOAT); h.u32(zsize);
        h.u32(begin);
        return h;
    };
    const uint32_t hsize = (uint32_t)header(0).b.size();
    Buf f = header(hsize);
    for (double v : x) f.f64(v);
    for (double v : y) f.f64(v);
    for (size_t i = 0; i < (size_t)nx * ny; i++) f.f32(z[i]);
    FILE *fp = fopen(filename, "wb");
    if (!fp) return fail(RELAX_ERR_ARG, "cannot open %s: %s", filename, strerror(errno));
    const size_t w = fwrite(f.b.data(), 1, f.b.size(), fp);
    const int rc = fclose(fp);
    if (w != f.b.size() || rc != 0) return fail(RELAX_ERR_ARG, "writing %s failed", filename);
    return RELAX_OK;
}

// exportspatial with doflip, src/elastic3d.f90:4166-4207: fftshift and
// transpose of one (sx1, sx2) plane into p(sx2, sx1), x2 fastest
void exportspatial(const float *data, int sx1, int sx2, float *p)
{
    for (int j2 = 0; j2 < sx2; j2++) {
        const int j2s = j2 < sx2 / 2 ? sx2 / 2 + j2 : j2 - sx2 / 2;
        for (int j1 = 0; j1 < sx1; j1++) {
            const int j1s = j1 < sx1 / 2 ? sx1 / 2 + j1 : j1 - sx1 / 2;
            p[(size_t)j1s * sx2 + j2s] = data[(size_t)j2 * sx1 + j1];
        }
    }
}

// ---------------------------------------------------------------------------
// VTK legacy binary
// ---------------------------------------------------------------------------
void put_be(std::vector<unsigned char> &o, float v)
{
    uint32_t u;
    memcpy(&u, &v, 4);
    o.push_back((unsigned char)(u >> 24));
    o.push_back((unsigned char)(u >> 16));
    o.push_back((unsigned char)(u >> 8));
    o.push_back((unsigned char)u);
}

// Writes a structured-points file; plane(k3, pc) fills pc[0..ncomp) with
// the components of plane k3 (sx1 x sx2, x1 fastest) and returns a status.
template <class Plane>
int write_vtk(const char *filename, const char *title, const char *name, int ncomp, int sx1, int sx2, int sx3,
              double dx1, double dx2, double dx3, int j1, int j2, int j3, Plane plane)
{
    if (!filename || (ncomp != 3 && ncomp != 6)) return fail(RELAX_ERR_ARG, "vtk: 3 or 6 components");
    if (j1 < 1 || j2 < 1 || j3 < 1 || sx1 < 2 || sx2 < 2 || sx3 < 1) return fail(RELAX_ERR_ARG, "vtk: sizes");
    FILE *fp = fopen(filename, "wb");
    if (!fp) return fail(RELAX_ERR_ARG, "cannot open %s: %s", filename, strerror(errno));
    fprintf(fp, "# vtk DataFile Version 3.0\n");
    fprintf(fp, "%s\n", title ? title : "");
    fprintf(fp, "BINARY\n");
    fprintf(fp, "DATASET STRUCTURED_POINTS\n");
    fprintf(fp, "DIMENSIONS %i %i %i\n", sx1 / j1, sx2 / j2, sx3 / j3);
    fprintf(fp, "ORIGIN %f %f %f\n", -dx1 * (sx1 / 2), -dx2 * (sx2 / 2), 0.0);
    fprintf(fp, "SPACING %f %f %f\n", dx1 * j1, dx2 * j2, dx3 * j3);
    fprintf(fp, "POINT_DATA %i\n", (sx1 / j1) * (sx2 / j2) * (sx3 / j3));
    fprintf(fp, "%s %s float\n", ncomp == 3 ? "VECTORS" : "TENSORS", name ? name : "field");
    std::vector<unsigned char> o;
    const float *pc[6] = {};
    int rc = RELAX_OK;
    for (int k3 = 0; k3 < sx3 && rc == RELAX_OK; k3 += j3) {
        rc = plane(k3, pc);
        if (rc != RELAX_OK) break;
        o.clear();
        // x2 and x1 from -sx/2: the origin in the middle of the box
        for (int k2 = -sx2 / 2; k2 < sx2 / 2; k2 += j2) {
            const int i2 = (sx2 + k2) % sx2;
            for (int k1 = -sx1 / 2; k1 < sx1 / 2; k1 += j1) {
                const size_t q = (size_t)((sx1 + k1) % sx1) + (size_t)i2 * sx1;
                if (ncomp == 3) {
                    for (int k = 0; k < 3; k++) put_be(o, pc[k][q]);
                } else {
                    // the symmetric tensor as 3 x 3, row by row
                    static const int full[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
                    for (int k = 0; k < 9; k++) put_be(o, pc[full[k]][q]);
                }
            }
        }
        if (fwrite(o.data(), 1, o.size(), fp) != o.size()) rc = fail(RELAX_ERR_ARG, "writing %s failed", filename);
    }
    if (fclose(fp) != 0 && rc == RELAX_OK) rc = fail(RELAX_ERR_ARG, "writing %s failed", filename);
    return rc;
}

// ---------------------------------------------------------------------------
// Fortran edit descriptors of RELAX's text output
// ---------------------------------------------------------------------------
// ESw.dEe: one digit before the point, d after, an exponent of e digits;
// a field that does not fit is w asterisks.  e = 0 is ESw.d: E and two
// digits up to 99, a sign and three digits (no E) up to 999.
std::string es(double v, int w, int d, int e)
{
    char buf[64];
    snprintf(buf, sizeof buf, "%.*E", d, v);
    std::string s(buf);
    const size_t p = s.find('E');
    if (p == std::string::npos) return std::string(w, '*');
    std::string mant = s.substr(0, p);
    const int ex = atoi(s.c_str() + p + 1);
    const int ax = ex < 0 ? -ex : ex;
    if (e < 0 || e > 4) return std::string(w, '*');
    int lim = 1;
    for (int k = 0; k < (e > 0 ? e : 3); k++) lim *= 10;
    if (ax >= lim) return std::string(w, '*');
    char eb[16];
    if (e > 0) snprintf(eb, sizeof eb, "E%c%0*d", ex < 0 ? '-' : '+', e, ax);
    else if (ax <= 99) snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', ax);
    else snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', ax);
    std::string out = mant + eb;
    if ((int)out.size() > w) return std::string(w, '*');
    return std::string(w - out.size(), ' ') + out;
}

// Iw.m for a non-negative integer
std::string iw(int v, int w, int m)
{
    char buf[32];
    snprintf(buf, sizeof buf, "%0*d", m, v);
    if (v < 0 || (int)strlen(buf) > w) return std::string(w, '*');
    return std::string(w - strlen(buf), ' ') + buf;
}

int copy_out(const std::string &s, char *buf, size_t size)
{
    if (!buf || s.size() + 1 > size) return fail(RELAX_ERR_ARG, "buffer of %zu bytes too small", size);
    memcpy(buf, s.c_str(), s.size() + 1);
    return RELAX_OK;
}

// fix, src/elastic3d.f90:70-83: the nearest integer, halves rounded down
int fix(double x)
{
    const double f = std::floor(x), c = std::ceil(x);
    return (x - f) > 0.5 ? (int)c : (int)f;
}

// rotation, src/util.f90:153-166 (angle in degrees)
void rotation(double &x, double &y, double rot)
{
    const double a = rot * 0.01745329251994329547437168059786927;
    const double xx = x, yy = y;
    x = +xx * std::cos(a) + yy * std::sin(a);
    y = -xx * std::sin(a) + yy * std::cos(a);
}

std::string ned_row(double time, const double u[3], const relax_tensor &s)
{
    std::string r = es(time, 16, 8, 2);
    for (int k = 0; k < 3; k++) r += es(u[k], 16, 8, 2);
    const float c[6] = {s.s11, s.s12, s.s13, s.s22, s.s23, s.s33};
    for (int k = 0; k < 6; k++) r += es((double)c[k], 16, 8, 2);
    return r;
}

const char NED_HEADER[] = "#          t          u1          u2          u3         s11         s12         s13"
                          "         s22         s23         s33";

}  // namespace

extern "C" int relax_write_grd(const float *z, int nx, int ny, double x0, double y0, double dx, double dy,
                               const char *title, const char *filename)
{
    return write_grd(z, nx, ny, x0, y0, dx, dy, title, filename);
}

// exportgrd, src/export.f90:917-1057, for three unpadded (sx1, sx2) planes
extern "C" int relax_write_grd3(const float *c1, const float *c2, const float *c3, int sx1, int sx2, double dx1,
                                double dx2, double origx, double origy, const char *wdir, int index,
                                int convention)
{
    static const char *const suffix[7][3] = {
        {"north", "east", "up"}, {"relax-north", "relax-east", "relax-up"}, {"eqbf-north", "eqbf-east", "eqbf-up"},
        {"s11", "s12", "s13"},   {"s22", "s23", "s33"},                     {"e11", "e12", "e13"},
        {"e22", "e23", "e33"}};
    if (!c1 || !c2 || !c3 || !wdir) return fail(RELAX_ERR_ARG, "null argument");
    if (convention < 1 || convention > 7) return fail(RELAX_ERR_ARG, "convention %d outside 1..7", convention);
    if (sx1 < 2 || sx2 < 2) return fail(RELAX_ERR_ARG, "grid %d x %d", sx1, sx2);
    const size_t np = (size_t)sx1 * sx2;
    std::vector<float> p(np);
    const float *cs[3] = {c1, c2, c3};
    const std::string digit = iw(index, 3, 3);
    // x (east) from origy, y (north) from origx; pixel registration
    const double xmin = origy - (sx2 / 2) * dx2, ymin = origx - (sx1 / 2) * dx1;
    for (int k = 0; k < 3; k++) {
        exportspatial(cs[k], sx1, sx2, p.data());
        if (k == 2 && convention <= 3)
            for (float &v : p) v = -v;   // positive up
        const std::string title = digit + "-" + suffix[convention - 1][k];
        const std::string file = std::string(wdir) + "/" + title + ".grd";
        const int rc = write_grd(p.data(), sx2, sx1, xmin, ymin, dx2, dx1, title.c_str(), file.c_str());
        if (rc != RELAX_OK) return rc;
    }
    return RELAX_OK;
}

// The map-view grids of a context's field: U at plane int(oz/dx3) as
// NNN-north/east/up.grd (exportgrd, convention 1); SIG at plane fix(oz/dx3)
// as NNN-s11..s33.grd and EPS (the transient strain) as NNN-e11..e33.grd
// (exportstressgrd, src/export.f90:860-908, conventions 4/5 and 6/7).
extern "C" int relax_export_grd(relax_ctx *ctx, int which, double oz, double origx, double origy, const char *wdir,
                                int index)
{
    int sx[3];
    double dx[3];
    if (!ctx || !wdir) return fail(RELAX_ERR_ARG, "null argument");
    int rc = relax_get_grid(ctx, sx, dx);
    if (rc != RELAX_OK) return rc;
    const size_t np = (size_t)sx[0] * sx[1];
    if (which == RELAX_FIELD_U || which == RELAX_FIELD_UR) {
        std::vector<float> pl(3 * np);
        rc = relax_get_plane(ctx, which, (int)(oz / dx[2]), pl.data(), pl.size() * sizeof(float));
        if (rc != RELAX_OK) return rc;
        return relax_write_grd3(pl.data(), pl.data() + np, pl.data() + 2 * np, sx[0], sx[1], dx[0], dx[1], origx,
                                origy, wdir, index, which == RELAX_FIELD_U ? 1 : 2);
    }
    if (which != RELAX_FIELD_SIG && which != RELAX_FIELD_EPS)
        return fail(RELAX_ERR_ARG, "grids of field %d: U, UR, SIG or EPS", which);
    std::vector<float> pl(6 * np);
    rc = relax_get_plane(ctx, which, fix(oz / dx[2]), pl.data(), pl.size() * sizeof(float));
    if (rc != RELAX_OK) return rc;
    const int conv = which == RELAX_FIELD_SIG ? 4 : 6;
    const float *c = pl.data();
    rc = relax_write_grd3(c, c + np, c + 2 * np, sx[0], sx[1], dx[0], dx[1], origx, origy, wdir, index, conv);
    if (rc != RELAX_OK) return rc;
    return relax_write_grd3(c + 3 * np, c + 4 * np, c + 5 * np, sx[0], sx[1], dx[0], dx[1], origx, origy, wdir, index,
                            conv + 1);
}

// exportvtk_vectors_legacy / exportvtk_tensors_legacy, src/writevtk.c:72-225,
// for host fields: ncomp = 3 (vector) or 6 (s11 s12 s13 s22 s23 s33)
// component arrays of sx1 x sx2 x sx3 floats, x1 fastest.
extern "C" int relax_write_vtk(const float *const *comp, int ncomp, int sx1, int sx2, int sx3, double dx1,
                               double dx2, double dx3, int j1, int j2, int j3, const char *filename,
                               const char *title, const char *name)
{
    if (!comp || (ncomp != 3 && ncomp != 6)) return fail(RELAX_ERR_ARG, "vtk: 3 or 6 components");
    for (int k = 0; k < ncomp; k++)
        if (!comp[k]) return fail(RELAX_ERR_ARG, "null component");
    const size_t np = (size_t)sx1 * sx2;
    return write_vtk(filename, title, name, ncomp, sx1, sx2, sx3, dx1, dx2, dx3, j1, j2, j3,
                     [&](int k3, const float **pc) {
                         for (int k = 0; k < ncomp; k++) pc[k] = comp[k] + (size_t)k3 * np;
                         return RELAX_OK;
                     });
}

// The same for a context's field (U, V, UR or a tensor field), read plane
// by plane; sx3 (<= sx3/2 of the grid) is the depth exported, as the
// reference's sx3/4 for displacement and sx3/2 for stress and velocity.
extern "C" int relax_export_vtk(relax_ctx *ctx, int which, int sx3, int j1, int j2, int j3, const char *filename,
                                const char *title, const char *name)
{
    int sx[3];
    double dx[3];
    if (!ctx) return fail(RELAX_ERR_ARG, "null context");
    int rc = relax_get_grid(ctx, sx, dx);
    if (rc != RELAX_OK) return rc;
    if (sx3 < 1 || sx3 > sx[2] / 2) return fail(RELAX_ERR_ARG, "vtk depth %d outside [1, %d]", sx3, sx[2] / 2);
    int ncomp;
    switch (which) {
    case RELAX_FIELD_U:
    case RELAX_FIELD_V:
    case RELAX_FIELD_UR: ncomp = 3; break;
    case RELAX_FIELD_SIG:
    case RELAX_FIELD_TAU:
    case RELAX_FIELD_MOMENT:
    case RELAX_FIELD_EPS: ncomp = 6; break;
    default: return fail(RELAX_ERR_ARG, "vtk of field %d: U, V, UR or a tensor field", which);
    }
    const size_t np = (size_t)sx[0] * sx[1];
    std::vector<float> pl(ncomp * np);
    return write_vtk(filename, title, name, ncomp, sx[0], sx[1], sx3, dx[0], dx[1], dx[2], j1, j2, j3,
                     [&](int k3, const float **pc) {
                         const int r = relax_get_plane(ctx, which, k3, pl.data(), pl.size() * sizeof(float));
                         for (int k = 0; k < ncomp; k++) pc[k] = pl.data() + k * np;
                         return r;
                     });
}

// The afterslip planes' patches (src/export.f90:563-767): with
// RELAX_CREEP_TXT wdir/NNN.sKKKKK.creep.dat (every third patch along both
// directions, one patch per line, 18ES11.3E2; exportcreep_asc), with
// RELAX_CREEP_GRD the grids NNN.sKKKKK.slip-dip/slip-strike/slip.grd and
// NNN.sKKKKK.vel-strike/vel-dip/vel.grd (exportcreep_grd, which writes the
// dip-slip rate into vel-strike and the strike-slip rate into vel-dip; kept),
// with RELAX_CREEP_VTK wdir/creep-KKKKKs-NNN.vtk (exportcreep_vtk).
extern "C" int relax_export_creep(relax_ctx *ctx, const char *wdir, int index, int formats)
{
    int np = 0, sx[3];
    double dx[3];
    if (!ctx || !wdir) return fail(RELAX_ERR_ARG, "null argument");
    int rc = relax_num_planes(ctx, &np);
    if (rc == RELAX_OK) rc = relax_get_grid(ctx, sx, dx);
    if (rc != RELAX_OK) return rc;
    const std::string digit = iw(index, 3, 3);
    for (int k = 0; k < np; k++) {
        int n1 = 0, n2 = 0;
        if ((rc = relax_get_plane_shape(ctx, k, &n1, &n2)) != RELAX_OK) return rc;
        if (n1 <= 0 || n2 <= 0) continue;
        std::vector<relax_slippatch> p((size_t)n1 * n2);
        if ((rc = relax_get_patches(ctx, k, p.data(), p.size())) != RELAX_OK) return rc;
        const std::string stem = std::string(wdir) + "/" + digit + ".s" + iw(k + 1, 5, 5);
        if (formats & RELAX_CREEP_TXT) {
            FILE *fp = fopen((stem + ".creep.dat").c_str(), "w");
            if (!fp) return fail(RELAX_ERR_ARG, "could not open %s.creep.dat", stem.c_str());
            fprintf(fp, "#        x1         x2         x3          yr        yz       slip strike-slip  dip-slip"
                        "   velocity     ss vel     ds vel       taus      sig11      sig12      sig13      sig22"
                        "      sig23      sig33\n");
            for (int i2 = 0; i2 < n2; i2 += 3)
                for (int i1 = 0; i1 < n1; i1 += 3) {
                    const relax_slippatch &q = p[(size_t)i1 + (size_t)n1 * i2];
                    const double v[18] = {q.x1, q.x2, q.x3, q.lx, q.lz, q.slip, q.ss, q.ds, q.v, q.vss, q.vds,
                                          q.taus, q.sig.s11, q.sig.s12, q.sig.s13, q.sig.s22, q.sig.s23, q.sig.s33};
                    std::string line;
                    for (double x : v) line += es(x, 11, 3, 2);
                    fprintf(fp, "%s\n", line.c_str());
                }
            if (fclose(fp) != 0) return fail(RELAX_ERR_ARG, "writing %s.creep.dat failed", stem.c_str());
        }
        if (formats & RELAX_CREEP_VTK) {
            // exportcreep_vtk, src/export.f90:776-849: the patch centres as
            // points, two triangles per cell, the slip and rate fields
            char name[64];
            snprintf(name, sizeof name, "/creep-%05ds-%s.vtk", k + 1, digit.c_str());
            const std::string file = std::string(wdir) + name;
            FILE *fp = fopen(file.c_str(), "w");
            if (!fp) return fail(RELAX_ERR_ARG, "could not open %s", file.c_str());
            fprintf(fp, "# vtk DataFile Version 3.0\nafterslip\nASCII\nDATASET POLYDATA\nPOINTS %d float\n", n1 * n2);
            for (const auto &q : p) fprintf(fp, "%s\n", (es(q.x1, 11, 3, 2) + es(q.x2, 11, 3, 2) + es(q.x3, 11, 3, 2)).c_str());
            const int ncell = (n1 - 1) * (n2 - 1);
            fprintf(fp, "\nPOLYGONS %d %d\n", std::max(0, ncell) * 2, std::max(0, ncell) * 2 * 4);
            for (int i2 = 1; i2 <= n2 - 1; i2++)
                for (int i1 = 1; i1 <= n1 - 1; i1++) {
                    const int a0 = (i2 - 1) * n1 + i1 - 1;
                    fprintf(fp, "3 %d %d %d\n", a0, a0 + 1, i2 * n1 + i1);
                    fprintf(fp, "3 %d %d %d\n", a0, i2 * n1 + i1 - 1, i2 * n1 + i1);
                }
            fprintf(fp, "\nPOINT_DATA %d\n", n1 * n2);
            // list-directed output in the reference (the layout is the
            // compiler's); here one value per line, 17 significant digits
            const std::pair<const char *, double relax_slippatch::*> fields[7] = {
                {"afterslip", &relax_slippatch::slip},   {"strike_slip", &relax_slippatch::ss},
                {"dip-slip", &relax_slippatch::ds},      {"velocity", &relax_slippatch::v},
                {"velocity_strike_slip", &relax_slippatch::vss}, {"velocity_dip_slip", &relax_slippatch::vds},
                {"shear_stress", &relax_slippatch::taus}};
            for (const auto &f : fields) {
                fprintf(fp, "SCALARS %s float\nLOOKUP_TABLE default\n", f.first);
                for (const auto &q : p) fprintf(fp, " %.17G\n", q.*(f.second));
            }
            if (fclose(fp) != 0) return fail(RELAX_ERR_ARG, "writing %s failed", file.c_str());
        }
        if (formats & RELAX_CREEP_GRD) {
            if (n1 < 2 || n2 < 2) continue;   // a grid needs two nodes each way
            double xmin = p[0].lx, zmax = p[0].lz;
            for (const auto &q : p) {
                xmin = std::fmin(xmin, q.lx);
                zmax = std::fmax(zmax, q.lz);
            }
            std::vector<float> z((size_t)n1 * n2);
            auto grid = [&](double relax_slippatch::*f, const char *name) {
                for (int i2 = 0; i2 < n2; i2++)
                    for (int i1 = 0; i1 < n1; i1++)
                        z[(size_t)(n1 - 1 - i1) + (size_t)n1 * i2] = (float)(p[(size_t)i1 + (size_t)n1 * i2].*f);
                return write_grd(z.data(), n1, n2, xmin, -zmax, dx[1], dx[2], "monitor field",
                                 (stem + name).c_str());
            };
            if ((rc = grid(&relax_slippatch::ds, ".slip-dip.grd")) != RELAX_OK) return rc;
            if ((rc = grid(&relax_slippatch::ss, ".slip-strike.grd")) != RELAX_OK) return rc;
            if ((rc = grid(&relax_slippatch::slip, ".slip.grd")) != RELAX_OK) return rc;
            if ((rc = grid(&relax_slippatch::vds, ".vel-strike.grd")) != RELAX_OK) return rc;
            if ((rc = grid(&relax_slippatch::vss, ".vel-dip.grd")) != RELAX_OK) return rc;
            if ((rc = grid(&relax_slippatch::v, ".vel.grd")) != RELAX_OK) return rc;
        }
    }
    return RELAX_OK;
}

// exportplanestress / exporteigenstrain, src/export.f90:308-512
extern "C" int relax_export_plane_stress(relax_ctx *ctx, int which, int nop, const relax_obsplane *op, double x0,
                                         double y0, const char *wdir, int index)
{
    int sx[3];
    double dx[3];
    if (!ctx || !wdir || nop < 0 || (nop > 0 && !op)) return fail(RELAX_ERR_ARG, "null argument");
    if (which != RELAX_FIELD_SIG && which != RELAX_FIELD_GAMMA)
        return fail(RELAX_ERR_ARG, "plane exports sample the stress or gamma, not field %d", which);
    int rc = relax_get_grid(ctx, sx, dx);
    if (rc != RELAX_OK) return rc;
    const std::string digit = iw(index, 3, 3);
    for (int k = 0; k < nop; k++) {
        int px2 = 0, px3 = 0;
        if ((rc = relax_monitor_plane(ctx, which, &op[k], 0.0, nullptr, 0, &px2, &px3)) != RELAX_OK) return rc;
        const int n1 = px2 + 1, n2 = px3 + 1;
        std::vector<relax_slippatch> p((size_t)n1 * n2);
        if ((rc = relax_monitor_plane(ctx, which, &op[k], 0.0, p.data(), p.size(), &px2, &px3)) != RELAX_OK)
            return rc;
        double xmin = p[0].lx, zmax = p[0].lz;
        for (auto &q : p) {
            q.x1 += x0;
            q.x2 += y0;
            xmin = std::fmin(xmin, q.lx);
            zmax = std::fmax(zmax, q.lz);
        }
        std::vector<float> z((size_t)n1 * n2);
        auto grid = [&](auto value, const std::string &file, const char *title) {
            for (int i2 = 0; i2 < n2; i2++)
                for (int i1 = 0; i1 < n1; i1++)
                    z[(size_t)(n1 - 1 - i1) + (size_t)n1 * i2] = value(p[(size_t)i1 + (size_t)n1 * i2]);
            return write_grd(z.data(), n1, n2, xmin, -zmax, dx[1], dx[2], title, file.c_str());
        };
        if (which == RELAX_FIELD_GAMMA) {
            rc = grid([](const relax_slippatch &q) { return (float)q.slip; },
                      std::string(wdir) + "/" + digit + ".s" + iw(k + 1, 5, 5) + ".estrain.grd", "monitor field");
            if (rc != RELAX_OK) return rc;
            continue;
        }
        const std::string stem = std::string(wdir) + "/" + digit + ".op" + iw(k + 1, 3, 3) + "-s";
        float relax_tensor::*c[6] = {&relax_tensor::s11, &relax_tensor::s12, &relax_tensor::s13,
                                     &relax_tensor::s22, &relax_tensor::s23, &relax_tensor::s33};
        const char *suffix[6] = {"11", "12", "13", "22", "23", "33"};
        for (int m = 0; m < 6; m++) {
            rc = grid([&](const relax_slippatch &q) { return q.sig.*c[m]; }, stem + suffix[m] + ".grd",
                      "monitor tensor field");
            if (rc != RELAX_OK) return rc;
        }
    }
    return RELAX_OK;
}

namespace {

// The orientation and stress resolution of a segment, src/export.f90:1580-1622
struct SegStress {
    double n[3], s[3], d[3], t[3], ts[3];
    double taun, taus, taustrike, taudip, taucoulomb;
    relax_tensor sig;
};

SegStress resolve(const relax_segment &g, const relax_tensor *sig, const relax_tensor *sig0)
{
    SegStress r{};
    r.sig = sig ? *sig : relax_tensor{0, 0, 0, 0, 0, 0};
    if (sig && sig0) {
        r.sig.s11 = r.sig.s11 - sig0->s11;
        r.sig.s12 = r.sig.s12 - sig0->s12;
        r.sig.s13 = r.sig.s13 - sig0->s13;
        r.sig.s22 = r.sig.s22 - sig0->s22;
        r.sig.s23 = r.sig.s23 - sig0->s23;
        r.sig.s33 = r.sig.s33 - sig0->s33;
    }
    const double cs = std::cos(g.strike), ss = std::sin(g.strike), cd = std::cos(g.dip), sd = std::sin(g.dip);
    r.n[0] = cd * cs;   r.n[1] = -cd * ss; r.n[2] = -sd;
    r.s[0] = ss;        r.s[1] = cs;       r.s[2] = 0.0;
    r.d[0] = -cs * sd;  r.d[1] = ss * sd;  r.d[2] = -cd;
    const relax_tensor &t = r.sig;
    const double *n = r.n;
    r.t[0] = (double)t.s11 * n[0] + (double)t.s12 * n[1] + (double)t.s13 * n[2];
    r.t[1] = (double)t.s12 * n[0] + (double)t.s22 * n[1] + (double)t.s23 * n[2];
    r.t[2] = (double)t.s13 * n[0] + (double)t.s23 * n[1] + (double)t.s33 * n[2];
    r.taun = r.t[0] * n[0] + r.t[1] * n[1] + r.t[2] * n[2];
    for (int k = 0; k < 3; k++) r.ts[k] = r.t[k] - r.taun * n[k];
    r.taus = std::sqrt(r.ts[0] * r.ts[0] + r.ts[1] * r.ts[1] + r.ts[2] * r.ts[2]);
    r.taustrike = r.ts[0] * r.s[0] + r.ts[1] * r.s[1] + r.ts[2] * r.s[2];
    r.taudip = r.ts[0] * r.d[0] + r.ts[1] * r.d[1] + r.ts[2] * r.d[2];
    r.taucoulomb = r.taus + g.friction * r.taun;
    return r;
}

std::string row(std::initializer_list<double> v, int w, int d, int e)
{
    std::string out;
    for (double x : v) out += es(x, w, d, e);
    return out;
}

// the XML lines of exportvtk_rfaults_stress, src/export.f90:1777-1863
void vtp_array(FILE *fp, const char *type, const char *name, int ncomp, const char *extra)
{
    fprintf(fp, "        <DataArray type=\"%s\" Name=\"%s\"", type, name);
    if (ncomp > 0) fprintf(fp, " NumberOfComponents=\"%d\"", ncomp);
    fprintf(fp, " format=\"ascii\"%s>\n", extra);
}

}  // namespace

extern "C" int relax_write_segments(int kind, int n, const relax_segment *sop, const relax_tensor *sig,
                                    const relax_tensor *sig0, const char *filename)
{
    if (!filename || n < 0 || (n > 0 && !sop)) return fail(RELAX_ERR_ARG, "null argument");
    if (kind < RELAX_SEG_GMT || kind > RELAX_SEG_VTP) return fail(RELAX_ERR_ARG, "unknown segment export %d", kind);
    if (n == 0) return RELAX_OK;   // no file, as the reference
    FILE *fp = fopen(filename, "w");
    if (!fp) return fail(RELAX_ERR_ARG, "could not open %s for export", filename);
    if (kind == RELAX_SEG_TRACTION)
        fprintf(fp, "# position east, north, up, traction e, n, u, normal vector e, n, u\n");
    if (kind == RELAX_SEG_VTP) {
        fprintf(fp, "<?xml version=\"1.0\"?>\n<VTKFile type=\"PolyData\" version=\"0.1\">\n  <PolyData>\n");
    }
    for (int k = 0; k < n; k++) {
        const relax_segment &g = sop[k];
        const SegStress r = resolve(g, sig ? &sig[k] : nullptr, sig0 ? &sig0[k] : nullptr);
        const double x1 = g.x, x2 = g.y, x3 = g.z, W = g.width, L = g.length;
        const double *s = r.s, *d = r.d;
        if (kind == RELAX_SEG_GMT) {
            fprintf(fp, "> -Z%s\n", row({r.taus, r.taun, r.taucoulomb, r.taustrike, r.taudip}, 11, 2, 0).c_str());
            fprintf(fp, "%s\n", row({x2 - d[1] * W / 2 - s[1] * L / 2, x1 - d[0] * W / 2 - s[0] * L / 2}, 11, 2, 0).c_str());
            fprintf(fp, "%s\n", row({x2 - d[1] * W / 2 + s[1] * L / 2, x1 - d[0] * W / 2 + s[0] * L / 2}, 11, 2, 0).c_str());
            fprintf(fp, "%s\n", row({x2 + d[1] * W / 2 + s[1] * L / 2, x1 + d[0] * W / 2 + s[0] * L / 2}, 11, 2, 0).c_str());
            fprintf(fp, "%s\n", row({x2 + d[1] * W / 2 - s[1] * L / 2, x1 + d[0] * W / 2 - s[0] * L / 2}, 11, 2, 0).c_str());
        } else if (kind == RELAX_SEG_TRACTION) {
            fprintf(fp, "%s\n", row({x2, x1, -x3, r.ts[1], r.ts[0], -r.ts[2], r.n[1], r.n[0], -r.n[2]}, 11, 2, 0).c_str());
        } else {
            fprintf(fp, "    <Piece NumberOfPoints=\"4\" NumberOfPolys=\"1\">\n      <Points>\n");
            vtp_array(fp, "Float32", "Fault Patch", 3, "");
            fprintf(fp, "%s\n", row({x1 - d[0] * W / 2 - s[0] * L / 2, x2 - d[1] * W / 2 - s[1] * L / 2,
                                      x3 - d[2] * W / 2 - s[2] * L / 2, x1 - d[0] * W / 2 + s[0] * L / 2,
                                      x2 - d[1] * W / 2 + s[1] * L / 2, x3 - d[2] * W / 2 + s[2] * L / 2,
                                      x1 + d[0] * W / 2 + s[0] * L / 2, x2 + d[1] * W / 2 + s[1] * L / 2,
                                      x3 + d[2] * W / 2 + s[2] * L / 2, x1 + d[0] * W / 2 - s[0] * L / 2,
                                      x2 + d[1] * W / 2 - s[1] * L / 2, x3 + d[2] * W / 2 - s[2] * L / 2},
                                     11, 2, 0).c_str());
            fprintf(fp, "        </DataArray>\n      </Points>\n      <Polys>\n");
            vtp_array(fp, "Int32", "connectivity", 0, " RangeMin=\"0\" RangeMax=\"3\"");
            fprintf(fp, "0 1 2 3\n        </DataArray>\n");
            vtp_array(fp, "Int32", "offsets", 0, " RangeMin=\"4\" RangeMax=\"4\"");
            fprintf(fp, "          4\n        </DataArray>\n      </Polys>\n");
            fprintf(fp, "      <CellData Normals=\"stress\">\n");
            vtp_array(fp, "Float32", "stress tensor", 6, "");
            fprintf(fp, "%s\n        </DataArray>\n",
                    row({r.sig.s11, r.sig.s12, r.sig.s13, r.sig.s22, r.sig.s23, r.sig.s33}, 11, 2, 0).c_str());
            vtp_array(fp, "Float32", "traction vector", 3, "");
            fprintf(fp, "%s\n        </DataArray>\n", row({r.t[0], r.t[1], r.t[2]}, 11, 2, 0).c_str());
            vtp_array(fp, "Float32", "shear traction vector", 3, "");
            for (int m = 0; m < 3; m++) fprintf(fp, "%s\n", es(r.ts[m], 11, 2, 0).c_str());
            fprintf(fp, "        </DataArray>\n");
            const std::pair<const char *, double> scalars[5] = {{"shear stress", r.taus},
                                                                {"normal stress", r.taun},
                                                                {"Coulomb stress", r.taucoulomb},
                                                                {"stress in strike direction", r.taustrike},
                                                                {"stress in dip direction", r.taudip}};
            for (const auto &sc : scalars) {
                vtp_array(fp, "Float32", sc.first, 1, "");
                fprintf(fp, "%s\n        </DataArray>\n", es(sc.second, 11, 2, 0).c_str());
            }
            fprintf(fp, "      </CellData>\n    </Piece>\n");
        }
    }
    if (kind == RELAX_SEG_VTP) fprintf(fp, "  </PolyData>\n</VTKFile>\n");
    if (fclose(fp) != 0) return fail(RELAX_ERR_ARG, "writing %s failed", filename);
    return RELAX_OK;
}

// ---------------------------------------------------------------------------
// geometry files of the input reader (src/export.f90:1068-1206, 1216-1354,
// 2014-2153, 2295-2599)
// ---------------------------------------------------------------------------
namespace {

const char *const XML_HEAD = "<?xml version=\"1.0\"?>\n<VTKFile type=\"PolyData\" version=\"0.1\">\n  <PolyData>\n";
const char *const XML_TAIL = "  </PolyData>\n</VTKFile>\n";

// strike, dip and normal unit vectors of the rectangle writers (dip vector
// pointing down dip: d = (cs sd, -ss sd, cd))
struct Frame {
    double s[3], d[3], n[3];
    Frame(double strike, double dip)
    {
        const double cs = std::cos(strike), ss = std::sin(strike), cd = std::cos(dip), sd = std::sin(dip);
        s[0] = ss; s[1] = cs; s[2] = 0.0;
        d[0] = cs * sd; d[1] = -ss * sd; d[2] = cd;
        n[0] = cd * cs; n[1] = -cd * ss; n[2] = -sd;
    }
};

// corner (sd, ss, sn = +-1) of a brick of centre x, half-extents W/2 down
// dip, L/2 along strike, T/2 along the normal
void corner(const Frame &f, const double *x, double L, double W, double T, int sd, int ss, int sn, double *out)
{
    for (int k = 0; k < 3; k++) {
        out[k] = x[k] + sd * f.d[k] * W / 2 + ss * f.s[k] * L / 2;
        if (sn) out[k] = out[k] + sn * f.n[k] * T / 2.0;   // rectangles (sn = 0) have no normal term
    }
}

std::string row_es(const std::vector<double> &v, int w, int d, int e)
{
    std::string out;
    for (double x : v) out += es(x, w, d, e);
    return out;
}

void vtp_polys(FILE *fp, const char *conn, int rmax, const char *offsets, int omin, int omax)
{
    fprintf(fp, "      <Polys>\n        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\" "
                "RangeMin=\"0\" RangeMax=\"%d\">\n%s\n        </DataArray>\n", rmax, conn);
    fprintf(fp, "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\" RangeMin=\"%d\" "
                "RangeMax=\"%d\">\n%s\n        </DataArray>\n      </Polys>\n", omin, omax, offsets);
}

void vtp_points(FILE *fp, int npts, int npolys, const char *name, const std::string &coords)
{
    fprintf(fp, "    <Piece NumberOfPoints=\"%d\" NumberOfPolys=\"%d\">\n      <Points>\n", npts, npolys);
    fprintf(fp, "        <DataArray type=\"Float32\" Name=\"%s\" NumberOfComponents=\"3\" format=\"ascii\">\n"
                "%s\n        </DataArray>\n      </Points>\n", name, coords.c_str());
}

int closed(FILE *fp, const char *filename)
{
    if (fclose(fp) != 0) return fail(RELAX_ERR_ARG, "writing %s failed", filename);
    return RELAX_OK;
}

}  // namespace

// exportvtk_grid, src/export.f90:1068-1127
extern "C" int relax_write_vtk_grid(int sx1, int sx2, int sx3, double dx1, double dx2, double dx3,
                                    const char *filename)
{
    if (!filename) return fail(RELAX_ERR_ARG, "null argument");
    FILE *fp = fopen(filename, "w");
    if (!fp) return fail(RELAX_ERR_ARG, "could not open %s for export", filename);
    const double a = sx1 * dx1 / 2, b = sx2 * dx2 / 2, c = sx3 * dx3 / 2;
    fputs(XML_HEAD, fp);
    vtp_points(fp, 8, 6, "Computational Grid",
               row_es({-a, -b, c, a, -b, c, a, b, c, -a, b, c, -a, -b, 0.0, a, -b, 0.0, a, b, 0.0, -a, b, 0.0}, 9, 2,
                      1));
    vtp_polys(fp, "0 1 2 3 4 5 6 7 2 3 7 6 0 3 7 4 0 1 5 4 1 2 6 5", 7, "          4 8 12 16 20 24", 4, 24);
    fprintf(fp, "    </Piece>\n");
    fputs(XML_TAIL, fp);
    return closed(fp, filename);
}

// exportvtk_rectangle, src/export.f90:2014-2093
extern "C" int relax_write_vtk_rectangle(double x1, double x2, double x3, double L, double W, double strike,
                                         double dip, const char *filename)
{
    if (!filename) return fail(RELAX_ERR_ARG, "null argument");
    FILE *fp = fopen(filename, "w");
    if (!fp) return fail(RELAX_ERR_ARG, "could not open %s for export in ExportVTK_Rectangle", filename);
    const Frame f(strike, dip);
    const double x[3] = {x1, x2, x3};
    std::vector<double> v;
    const int sgn[4][2] = {{-1, -1}, {-1, 1}, {1, 1}, {1, -1}};
    for (const auto &q : sgn) {
        double c[3];
        corner(f, x, L, W, 0.0, q[0], q[1], 0, c);
        v.insert(v.end(), c, c + 3);
    }
    fputs(XML_HEAD, fp);
    vtp_points(fp, 4, 1, "Fault Patch", row_es(v, 11, 2, 0));
    vtp_polys(fp, "0 1 2 3", 3, "          4", 4, 4);
    fprintf(fp, "    </Piece>\n");
    fputs(XML_TAIL, fp);
    return closed(fp, filename);
}

// exportxy_brick, src/export.f90:2101-2153: the faces below and above the
// zone's mid-plane as two closed GMT polygons (east, north, depth)
extern "C" int relax_write_xy_brick(const relax_weakzone *z, const char *filename)
{
    if (!z || !filename) return fail(RELAX_ERR_ARG, "null argument");
    FILE *fp = fopen(filename, "w");
    if (!fp) return fail(RELAX_ERR_ARG, "could not open %s for export in ExportXY_Brick", filename);
    const Frame f(z->strike, z->dip);
    const double x[3] = {z->x, z->y, z->z};
    const int loop[5][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}, {-1, -1}};   // (strike, normal) signs
    for (int sd = -1; sd <= 1; sd += 2) {
        fprintf(fp, ">\n");
        for (const auto &q : loop) {
            double c[3];
            corner(f, x, z->length, z->width, z->thickness, sd, q[0], q[1], c);
            fprintf(fp, "%s\n", row_es({c[1], c[0], c[2]}, 11, 2, 0).c_str());
        }
    }
    return closed(fp, filename);
}

// exportvtk_allbricks, src/export.f90:2295-2599: two pieces per zone (three
// faces each) with the zone's strain
extern "C" int relax_write_vtk_bricks(int n, const relax_weakzone *z, const char *filename)
{
    if (!filename || n < 0 || (n > 0 && !z)) return fail(RELAX_ERR_ARG, "null argument");
    FILE *fp = fopen(filename, "w");
    if (!fp) return fail(RELAX_ERR_ARG, "could not open %s for export in ExportVTK_Brick", filename);
    fputs(XML_HEAD, fp);
    // the eight corners in the reference's order: (dip, strike, normal) signs
    const int order[8][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {1, -1, -1},
                             {1, -1, 1},   {-1, -1, 1}, {-1, 1, 1}, {1, 1, 1}};
    for (int i = 0; i < n; i++) {
        const relax_weakzone &w = z[i];
        const Frame f(w.strike, w.dip);
        const double x[3] = {w.x, w.y, w.z};
        std::vector<double> v;
        for (const auto &o : order) {
            double c[3];
            corner(f, x, w.length, w.width, w.thickness, o[0], o[1], o[2], c);
            v.insert(v.end(), c, c + 3);
        }
        const relax_tensor &e = w.e;
        const double ekk = (double)(e.s11 + e.s22 + e.s33);
        const double dev = std::sqrt((e.s11 - ekk / 3) * (e.s11 - ekk / 3) + (e.s22 - ekk / 3) * (e.s22 - ekk / 3) +
                                     (e.s33 - ekk / 3) * (e.s33 - ekk / 3) + (double)(2 * e.s12 * e.s12) +
                                     (double)(2 * e.s13 * e.s13) + (double)(2 * e.s23 * e.s23));
        const std::pair<const char *, double> cells[8] = {{"isotropic strain", ekk}, {"deviatoric strain", dev},
                                                          {"e11", e.s11}, {"e12", e.s12}, {"e13", e.s13},
                                                          {"e22", e.s22}, {"e23", e.s23}, {"e33", e.s33}};
        const char *conn[2] = {"7 4 5 6 7 4 3 2 7 2 1 6", "0 1 2 3 0 5 4 3 0 1 6 5"};
        const int rmax[2] = {6, 7};
        for (int piece = 0; piece < 2; piece++) {
            vtp_points(fp, 8, 1, "Weak Zone", row_es(v, 11, 2, 0));
            vtp_polys(fp, conn[piece], rmax[piece], "          12", 12, 12);
            fprintf(fp, "      <CellData Normals=\"slip\">\n");
            for (const auto &cell : cells) {
                vtp_array(fp, "Float32", cell.first, 1, "");
                fprintf(fp, "%s\n        </DataArray>\n", es(cell.second, 11, 2, 0).c_str());
            }
            fprintf(fp, "      </CellData>\n    </Piece>\n");
        }
    }
    fputs(XML_TAIL, fp);
    return closed(fp, filename);
}

// exportvtk_rfaults (kind RELAX_FAULTS_VTP, src/export.f90:1216-1354) and
// exportxy_rfaults (kind RELAX_FAULTS_XY, :1139-1206) of n sources in the
// internal convention; the GMT file adds the origin x0, y0
extern "C" int relax_write_faults(int kind, int n, const relax_source *src, double x0, double y0,
                                  const char *filename)
{
    if (!filename || n < 0 || (n > 0 && !src)) return fail(RELAX_ERR_ARG, "null argument");
    if (kind != RELAX_FAULTS_VTP && kind != RELAX_FAULTS_XY) return fail(RELAX_ERR_ARG, "unknown fault export %d", kind);
    FILE *fp = fopen(filename, "w");
    if (!fp) return fail(RELAX_ERR_ARG, "could not open %s for export", filename);
    if (kind == RELAX_FAULTS_VTP) fputs(XML_HEAD, fp);
    else fprintf(fp, "> # east, north\n");
    const int sgn[4][2] = {{-1, -1}, {-1, 1}, {1, 1}, {1, -1}};
    for (int k = 0; k < n; k++) {
        const relax_source &q = src[k];
        const Frame f(q.strike, q.dip);
        if (kind == RELAX_FAULTS_XY) {
            const double x[3] = {q.x + x0, q.y + y0, q.z};
            fprintf(fp, "> -Z%s\n", es(std::fabs(q.slip), 11, 2, 0).c_str());
            for (const auto &c4 : sgn) {
                double c[3];
                corner(f, x, q.length, q.width, 0.0, c4[0], c4[1], 0, c);
                fprintf(fp, "%s\n", row_es({c[1], c[0]}, 11, 2, 0).c_str());
            }
            continue;
        }
        const double x[3] = {q.x, q.y, q.z};
        std::vector<double> v;
        for (const auto &c4 : sgn) {
            double c[3];
            corner(f, x, q.length, q.width, 0.0, c4[0], c4[1], 0, c);
            v.insert(v.end(), c, c + 3);
        }
        vtp_points(fp, 4, 1, "Fault Patch", row_es(v, 11, 2, 0));
        vtp_polys(fp, "0 1 2 3", 3, "          4", 4, 4);
        fprintf(fp, "      <CellData Normals=\"slip\">\n");
        const double cr = std::cos(q.rake), sr = std::sin(q.rake);
        vtp_array(fp, "Float32", "slip", 3, "");
        fprintf(fp, "%s\n        </DataArray>\n",
                row_es({(f.s[0] * cr + f.d[0] * sr) * q.slip, (f.s[1] * cr + f.d[1] * sr) * q.slip,
                        (f.s[2] * cr + f.d[2] * sr) * q.slip}, 11, 2, 0).c_str());
        vtp_array(fp, "Float32", "opening", 3, "");
        fprintf(fp, "%s\n        </DataArray>\n      </CellData>\n    </Piece>\n",
                row_es({f.n[0] * q.opening, f.n[1] * q.opening, f.n[2] * q.opening}, 11, 2, 0).c_str());
    }
    if (kind == RELAX_FAULTS_VTP) fputs(XML_TAIL, fp);
    return closed(fp, filename);
}

// exportcoulombstress, src/export.f90:1893-2005
extern "C" int relax_write_coulomb(int n, const relax_segment *sop, const relax_tensor *sig, double time,
                                   const char *wdir, int isnew)
{
    if (!wdir || n < 0 || (n > 0 && (!sop || !sig))) return fail(RELAX_ERR_ARG, "null argument");
    for (int k = 0; k < n; k++) {
        const std::string file = std::string(wdir) + "/cfaults-sigma-" + iw(k + 1, 4, 4) + ".txt";
        FILE *fp = fopen(file.c_str(), isnew ? "w" : "a");
        if (!fp) return fail(RELAX_ERR_ARG, "could not open %s for writing", file.c_str());
        const relax_segment &g = sop[k];
        if (isnew) {
            fprintf(fp, "# center position (north, east, down): %s\n", row({g.x, g.y, g.z}, 9, 2, 0).c_str());
            fprintf(fp, "#         t        s11        s12        s13        s22        s23        s33       taus"
                        "       taud        tau       taun    Coulomb\n");
        }
        const SegStress r = resolve(g, &sig[k], nullptr);
        fprintf(fp, "%s\n",
                row({time, r.sig.s11, r.sig.s12, r.sig.s13, r.sig.s22, r.sig.s23, r.sig.s33, r.taustrike, r.taudip,
                     r.taus, r.taun, r.taucoulomb},
                    11, 3, 2)
                    .c_str());
        if (fclose(fp) != 0) return fail(RELAX_ERR_ARG, "writing %s failed", file.c_str());
    }
    return RELAX_OK;
}

// shiftedindex, src/elastic3d.f90:4063-4101, 0-based; sx3 is the number of
// planes (sx3/2 of the grid)
extern "C" int relax_shifted_index(double x1, double x2, double x3, int sx1, int sx2, int sx3, double dx1,
                                   double dx2, double dx3, int *i1, int *i2, int *i3)
{
    if (!i1 || !i2 || !i3) return fail(RELAX_ERR_ARG, "null argument");
    if (x1 > (double)(sx1 / 2 - 1) * dx1 || x1 < -(double)(sx1 / 2) * dx1)
        return fail(RELAX_ERR_ARG, "x1=%g outside the box", x1);
    if (x2 > (double)(sx2 / 2 - 1) * dx2 || x2 < -(double)(sx2 / 2) * dx2)
        return fail(RELAX_ERR_ARG, "x2=%g outside the box", x2);
    if (x3 > (double)(sx3 - 1) * dx3 || x3 < 0) return fail(RELAX_ERR_ARG, "x3=%g outside the box", x3);
    *i1 = (sx1 + fix(x1 / dx1)) % sx1;
    *i2 = (sx2 + fix(x2 / dx2)) % sx2;
    *i3 = fix(x3 / dx3);
    return RELAX_OK;
}

// exportpoints, src/util.f90:59-170: for each observation point (x1, x2,
// x3 in the computational frame) one line of wdir/<name>.ned, time,
// displacement rotated back to the user frame and stress (a new file with
// its header when isnew), and, when rot != 0, time and the unrotated
// displacement in wdir/<name>.c.txt.
extern "C" int relax_export_points(relax_ctx *ctx, int n, const double *x, const char *const *names, double time,
                                   double rot, const char *wdir, int isnew)
{
    int sx[3];
    double dx[3];
    if (!ctx || n < 0 || (n > 0 && (!x || !names)) || !wdir) return fail(RELAX_ERR_ARG, "null argument");
    if (n == 0) return RELAX_OK;
    int rc = relax_get_grid(ctx, sx, dx);
    if (rc != RELAX_OK) return rc;
    std::vector<int> idx(3 * (size_t)n);
    for (int k = 0; k < n; k++) {
        rc = relax_shifted_index(x[3 * k], x[3 * k + 1], x[3 * k + 2], sx[0], sx[1], sx[2] / 2, dx[0], dx[1], dx[2],
                                 &idx[3 * k], &idx[3 * k + 1], &idx[3 * k + 2]);
        if (rc != RELAX_OK) return rc;
    }
    std::vector<double> u(3 * (size_t)n);
    std::vector<relax_tensor> sig(n);
    rc = relax_get_points(ctx, n, idx.data(), u.data(), sig.data());
    if (rc != RELAX_OK) return rc;
    for (int k = 0; k < n; k++) {
        if (!names[k]) return fail(RELAX_ERR_ARG, "point %d has no name", k);
        const std::string base = std::string(wdir) + "/" + names[k];
        double v[3] = {u[3 * k], u[3 * k + 1], u[3 * k + 2]};
        rotation(v[0], v[1], -rot);
        FILE *fp = fopen((base + ".ned").c_str(), isnew ? "w" : "a");
        if (!fp) return fail(RELAX_ERR_ARG, "could not open %s.ned for writing", base.c_str());
        if (isnew) fprintf(fp, "%s\n", NED_HEADER);
        fprintf(fp, "%s\n", ned_row(time, v, sig[k]).c_str());
        if (fclose(fp) != 0) return fail(RELAX_ERR_ARG, "writing %s.ned failed", base.c_str());
        if (rot != 0.0) {
            fp = fopen((base + ".c.txt").c_str(), isnew ? "w" : "a");
            if (!fp) return fail(RELAX_ERR_ARG, "could not open %s.c.txt for writing", base.c_str());
            if (isnew) fprintf(fp, "#         t         u1         u2         u3\n");
            std::string r = es(time, 11, 3, 2);
            for (int j = 0; j < 3; j++) r += es(u[3 * k + j], 11, 3, 2);
            fprintf(fp, "%s\n", r.c_str());
            if (fclose(fp) != 0) return fail(RELAX_ERR_ARG, "writing %s.c.txt failed", base.c_str());
        }
    }
    return RELAX_OK;
}

// The step log line, formats 1100-1103 of src/relax.f90:1102-1105: "*" after
// the step number on output steps; the transient form adds the Maxwell times
// of the linear and nonlinear transient mechanisms.
extern "C" int relax_format_log(const relax_step_log *log, double interval, int transient, char *buf, size_t size)
{
    if (!log) return fail(RELAX_ERR_ARG, "null argument");
    std::string s = iw(log->i, 3, 3) + (log->output ? "*" : " ");
    s += es(log->dt, 9, 2, 2);
    s += es(log->tm_ve, 9, 2, 2) + es(log->tm_pl, 9, 2, 2) + es(log->tm_as, 9, 2, 2);
    if (transient) s += es(log->tm_tl, 9, 2, 2) + es(log->tm_tnl, 9, 2, 2);
    s += es(log->t, 9, 2, 2) + "/" + es(interval, 7, 2, 1);
    s += es(log->power, 9, 2, 2) + es(log->cei, 9, 2, 2);
    return copy_out(s, buf, size);
}

// The column header, formats 0990/0991 of src/relax.f90:1100-1101
extern "C" const char *relax_log_header(int transient)
{
    return transient ? " I  |   Dt   | tm(ve) | tm(pl) | tm(as) | tm(kl) | tm(kn) |     t/tmax     | power  |  C:E^i | "
                     : " I  |   Dt   | tm(ve) | tm(pl) | tm(as) |     t/tmax     | power  |  C:E^i | ";
}

// one row of a .ned file (format 14ES16.8E2, src/util.f90:120)
extern "C" int relax_format_ned(double time, const double *u, const relax_tensor *sig, char *buf, size_t size)
{
    if (!u || !sig) return fail(RELAX_ERR_ARG, "null argument");
    return copy_out(ned_row(time, u, *sig), buf, size);
}

extern "C" const char *relax_ned_header(void) { return NED_HEADER; }

// Fortran ESw.dEe of one value
extern "C" int relax_es_format(double v, int w, int d, int e, char *buf, size_t size)
{
    if (w < 1 || w > 60 || d < 0 || d > 40 || e < 0 || e > 4) return fail(RELAX_ERR_ARG, "format");
    return copy_out(es(v, w, d, e), buf, size);
}
