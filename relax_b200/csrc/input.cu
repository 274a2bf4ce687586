// input.cu -- RELAX's input file (subroutine init, src/input.f90:43-1767)
// read into a relax_config.
//
// The file is a sequence of data lines; lines whose first non-blank
// character is '#' are comments (getdata, src/getdata.f:1-24).  Each data
// line is read the way Fortran list-directed input reads a record: values
// separated by blanks or commas, a '/' ends the record, r*value repeats,
// D exponents are accepted and values beyond those asked for are ignored.
// The sections come in init's order; the geometry of faults, planes and
// weak zones goes through wangconvention and the observation points,
// dilatation sources and loads through the rotation, as init does.  With
// RELAX_INPUT_ECHO the values are printed back with init's formats.
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/relax_b200.h"

extern "C" __attribute__((visibility("hidden"))) int relax_noalloc_fail(int code, const char *msg);

namespace {

const double DEG2RAD = 0.01745329251994329547437168059786927;

typedef relax_obsplane ObsPlane;
typedef relax_segment Segment;

// ---------------------------------------------------------------------------
// Fortran edit descriptors used by the echo
// ---------------------------------------------------------------------------
std::string es(double v, int w, int d, int e)
{
    char buf[64];
    snprintf(buf, sizeof buf, "%.*E", d, v);
    std::string s(buf);
    const size_t p = s.find('E');
    if (p == std::string::npos) return std::string(w, '*');
    const int ex = atoi(s.c_str() + p + 1), ax = ex < 0 ? -ex : ex;
    int lim = 1;
    for (int k = 0; k < e; k++) lim *= 10;
    if (ax >= lim) return std::string(w, '*');
    char eb[16];
    snprintf(eb, sizeof eb, "E%c%0*d", ex < 0 ? '-' : '+', e, ax);
    const std::string out = s.substr(0, p) + eb;
    if ((int)out.size() > w) return std::string(w, '*');
    return std::string(w - out.size(), ' ') + out;
}

std::string iw(long v, int w, int m = 1)
{
    char buf[48];
    if (v < 0) snprintf(buf, sizeof buf, "-%0*ld", m, -v);
    else snprintf(buf, sizeof buf, "%0*ld", m, v);
    if ((int)strlen(buf) > w) return std::string(w, '*');
    return std::string(w - strlen(buf), ' ') + buf;
}

std::string fw(double v, int w, int d)
{
    char buf[64];
    snprintf(buf, sizeof buf, "%*.*f", w, d, v);
    if ((int)strlen(buf) > w) return std::string(w, '*');
    return buf;
}

std::string esn(const double *v, int n, int w, int d, int e)
{
    std::string s;
    for (int k = 0; k < n; k++) s += es(v[k], w, d, e);
    return s;
}

const char RULE[] = "# ----------------------------------------------------------------------------";

// ---------------------------------------------------------------------------
// wangconvention and rotation, src/input.f90:1780-1822
// ---------------------------------------------------------------------------
void rotation(double &x, double &y, double rot)
{
    const double a = rot * DEG2RAD, xx = x, yy = y;
    x = +xx * cos(a) + yy * sin(a);
    y = -xx * sin(a) + yy * cos(a);
}

void wang(double &slip, double &x, double &y, double &z, double length, double width, double &strike, double &dip,
          double &rake, double x0, double y0, double rot)
{
    slip = -slip;
    strike = -90.0 - strike;
    dip = 90.0 - dip;
    strike *= DEG2RAD;
    dip *= DEG2RAD;
    rake *= DEG2RAD;
    x = x - x0 - length / 2.0 * sin(strike) + width / 2.0 * sin(dip) * cos(strike);
    y = y - y0 - length / 2.0 * cos(strike) - width / 2.0 * sin(dip) * sin(strike);
    z = z + width / 2.0 * cos(dip);
    rotation(x, y, rot);
    strike = strike + rot * DEG2RAD;
}

// antialiasingfilter, src/input.f90:1836-1856
void antialias(double &slip, double &length, double &width, double dx1, double dx2, double dx3, double nyquist)
{
    const double dx = std::fmin(dx1, std::fmin(dx2, dx3)) * nyquist;
    if (length < dx) {
        slip = slip * length / dx;
        length = dx;
    }
    if (width < dx) {
        slip = slip * width / dx;
        width = dx;
    }
}

// fix, src/elastic3d.f90:70-83
int fix(double x)
{
    const double f = floor(x), c = ceil(x);
    return (x - f) > 0.5 ? (int)c : (int)f;
}

// ---------------------------------------------------------------------------
// list-directed records
// ---------------------------------------------------------------------------
struct ParseError {
    int code;
    std::string msg;
};

[[noreturn]] void perr(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw ParseError{RELAX_ERR_ARG, buf};
}

struct Record {
    std::vector<std::string> items;
    size_t pos = 0;
    int line = 0;
    std::string text;

    bool more() const { return pos < items.size(); }

    const std::string &next(const char *what)
    {
        if (pos >= items.size()) perr("input line %d: %s missing in \"%s\"", line, what, text.c_str());
        return items[pos++];
    }
    double real(const char *what)
    {
        std::string s = next(what);
        for (char &ch : s)
            if (ch == 'd' || ch == 'D' || ch == 'q' || ch == 'Q') ch = 'e';
        char *end = nullptr;
        errno = 0;
        const double v = strtod(s.c_str(), &end);
        if (end == s.c_str() || *end != '\0' || errno == ERANGE)
            perr("input line %d: %s: \"%s\" is not a number", line, what, items[pos - 1].c_str());
        return v;
    }
    int integer(const char *what)
    {
        const std::string &s = next(what);
        char *end = nullptr;
        errno = 0;
        const long v = strtol(s.c_str(), &end, 10);
        if (end == s.c_str() || *end != '\0' || errno == ERANGE || v > 2147483647L || v < -2147483647L)
            perr("input line %d: %s: \"%s\" is not an integer", line, what, s.c_str());
        return (int)v;
    }
};

struct Reader {
    const char *p;
    int line = 0;

    // getdata: the next line whose first non-blank character is not '#'
    // (blank lines are skipped too)
    std::string data(const char *what)
    {
        while (*p) {
            const char *e = strchr(p, '\n');
            std::string l = e ? std::string(p, e - p) : std::string(p);
            p = e ? e + 1 : p + strlen(p);
            line++;
            if (!l.empty() && l.back() == '\r') l.pop_back();
            const size_t f = l.find_first_not_of(" \t");
            if (f == std::string::npos || l[f] == '#') continue;
            return l;
        }
        perr("input ends before %s", what);
    }

    Record record(const char *what)
    {
        Record r;
        r.text = data(what);
        r.line = line;
        const std::string &s = r.text;
        size_t i = 0;
        while (i < s.size()) {
            const char ch = s[i];
            if (ch == ' ' || ch == '\t' || ch == ',') {
                i++;
                continue;
            }
            if (ch == '/') break;
            std::string tok;
            if (ch == '\'' || ch == '"') {
                const size_t j = s.find(ch, i + 1);
                tok = s.substr(i + 1, j == std::string::npos ? std::string::npos : j - i - 1);
                i = j == std::string::npos ? s.size() : j + 1;
            } else {
                size_t j = i;
                while (j < s.size() && s[j] != ' ' && s[j] != '\t' && s[j] != ',' && s[j] != '/') j++;
                tok = s.substr(i, j - i);
                i = j;
            }
            // r*value repeats a value r times
            const size_t star = tok.find('*');
            if (star != std::string::npos && star > 0 && tok.find_first_not_of("0123456789") == star &&
                star + 1 < tok.size()) {
                const int n = atoi(tok.substr(0, star).c_str());
                for (int k = 0; k < n; k++) r.items.push_back(tok.substr(star + 1));
            } else {
                r.items.push_back(tok);
            }
        }
        return r;
    }
};

}  // namespace

struct relax_input {
    relax_config cfg{};
    int flags = 0;
    std::string wdir;
    double x0 = 0, y0 = 0, rot = 0, oz = 0, ozs = 0;
    std::vector<double> pts;                 // 3 per point, computational frame
    std::vector<std::string> ptsname;
    std::vector<const char *> ptsname_c;
    std::vector<ObsPlane> op;
    std::vector<Segment> sop;
    std::vector<relax_tensor_layer> stresslayer, stressstruc;
    std::vector<relax_layer> layers[5], struc[5];    // linear, nonlinear, l/nl transient, fault creep
    std::vector<relax_weakzone> wz[4];
    std::vector<float> dg[4];
    std::vector<relax_plane> planes;
    std::vector<std::vector<relax_source>> es, ets, em, el;
    std::vector<std::vector<relax_weakzone>> ecub;        // cuboid eigenstrain sources
    std::vector<std::vector<relax_tetrahedron>> etet;     // tetrahedral ones
    std::vector<std::vector<double>> evert;               // their vertices
    std::vector<relax_event> events;
    std::vector<relax_source> is, its;
    int ncuboid = 0, ntetra = 0;      // totals over the events
    double minlength = 0, minwidth = 0;
};

namespace {

enum { L_LIN = 0, L_NON = 1, L_LT = 2, L_NLT = 3, L_FC = 4 };

struct Echo {
    bool on;
    void line(const std::string &s) const
    {
        if (on) printf("%s\n", s.c_str());
    }
    void text(const char *s) const
    {
        if (on) printf("%s\n", s);
    }
};

// the weak zones of one mechanism, src/input.f90:555-600
void read_weakzones(Reader &rd, relax_input &in, int m, const Echo &echo, const char *title, bool i5)
{
    echo.text(title);
    Record r = rd.record("the number of weak zones");
    const int n = r.integer("number of weak zones");
    echo.line(iw(n, 5));
    if (n < 0) perr("input line %d: negative number of weak zones", r.line);
    if (n == 0) return;
    echo.text(RULE);
    echo.text(i5 ? "#   n dgammadot0     x1       x2       x3  length   width thickn. strike   dip"
                 : "#  n dgammadot0     x1       x2       x3  length   width thickn. strike   dip");
    echo.text(RULE);
    for (int k = 1; k <= n; k++) {
        Record z = rd.record("a weak zone");
        const int i = z.integer("index");
        relax_weakzone w{};
        w.dgammadot0 = z.real("dgammadot0");
        w.x = z.real("x1"); w.y = z.real("x2"); w.z = z.real("x3");
        w.length = z.real("length"); w.width = z.real("width"); w.thickness = z.real("thickness");
        w.strike = z.real("strike"); w.dip = z.real("dip");
        const double v4[4] = {w.dgammadot0, w.x, w.y, w.z}, v3[3] = {w.length, w.width, w.thickness};
        echo.line(iw(k, i5 ? 5 : 4, i5 ? 5 : 4) + esn(v4, 4, 9, 2, 1) + esn(v3, 3, 8, 2, 1) + fw(w.strike, 7, 1) +
                  fw(w.dip, 6, 1));
        if (i != k) perr("input line %d: source index misfit (%d, expected %d)", z.line, i, k);
        double dummy = 0, rake = 0;
        wang(dummy, w.x, w.y, w.z, w.length, w.width, w.strike, w.dip, rake, in.x0, in.y0, in.rot);
        in.wz[m].push_back(w);
    }
}

// a viscous interface list, src/input.f90:480-540 and the like
void read_layers(Reader &rd, relax_input &in, int m, const Echo &echo, const char *title, const char *header,
                 int nval)
{
    echo.text(title);
    Record r = rd.record("the number of interfaces");
    const int n = r.integer("number of interfaces");
    echo.line(iw(n, 5));
    if (n < 0) perr("input line %d: negative number of interfaces", r.line);
    if (n == 0) return;
    echo.text(RULE);
    echo.text(header);
    echo.text(RULE);
    for (int k = 1; k <= n; k++) {
        Record l = rd.record("an interface");
        const int i = l.integer("index");
        relax_layer y{};
        y.z = l.real("depth");
        y.gammadot0 = l.real("gammadot0");
        switch (m) {
        case L_LIN:   // depth, gammadot0, cohesion; n = 1
            y.cohesion = l.real("cohesion");
            y.stressexponent = 1;
            break;
        case L_NON:   // depth, gammadot0, power, cohesion
            y.stressexponent = l.real("power");
            y.cohesion = l.real("cohesion");
            break;
        case L_LT:    // depth, gammadot0, Gk; n = 1
            y.Gk = l.real("Gk");
            y.stressexponent = 1;
            break;
        case L_NLT:   // depth, gammadot0, power, Gk
            y.stressexponent = l.real("power");
            y.Gk = l.real("Gk");
            break;
        default:      // depth, V0, (a-b)sigma, friction, cohesion
            y.stressexponent = l.real("(a-b)sigma");
            y.friction = l.real("friction");
            y.cohesion = l.real("cohesion");
            break;
        }
        std::string s = iw(i, 3, 3);
        if (m == L_FC) {
            const double v[5] = {y.z, y.gammadot0, y.stressexponent, y.friction, y.cohesion};
            s += esn(v, 5, 9, 2, 1);
        } else if (m == L_LIN) {
            const double v[3] = {y.z, y.gammadot0, y.cohesion};
            s += esn(v, 3, 10, 2, 2);
        } else if (m == L_LT) {
            const double v[3] = {y.z, y.gammadot0, y.Gk};
            s += esn(v, 3, 10, 2, 2);
        } else {
            const double v[4] = {y.z, y.gammadot0, y.stressexponent, m == L_NON ? y.cohesion : y.Gk};
            s += esn(v, 4, 10, 2, 2);
        }
        (void)nval;
        echo.line(s);
        if (y.gammadot0 < 0)
            perr("input line %d: %s must be positive", l.line, m == L_FC ? "slip rates" : "strain rates");
        if (i != k) perr("input line %d: index misfit (%d, expected %d)", l.line, i, k);
        in.layers[m].push_back(y);
    }
}

void parse(const char *text, relax_input &in)
{
    Reader rd{text};
    const Echo echo{(in.flags & RELAX_INPUT_ECHO) != 0};
    relax_config &c = in.cfg;

    echo.text("# grid dimension (sx1,sx2,sx3)");
    {
        Record r = rd.record("the grid dimension");
        c.sx1 = r.integer("sx1"); c.sx2 = r.integer("sx2"); c.sx3 = r.integer("sx3");
        echo.line(iw(c.sx1, 5) + iw(c.sx2, 5) + iw(c.sx3, 5));
    }
    echo.text("# sampling (dx1,dx2,dx3), smoothing (beta, nyquist)");
    {
        Record r = rd.record("the sampling");
        c.dx1 = r.real("dx1"); c.dx2 = r.real("dx2"); c.dx3 = r.real("dx3");
        c.beta = r.real("beta"); c.nyquist = r.real("nyquist");
        const double v[5] = {c.dx1, c.dx2, c.dx3, c.beta, c.nyquist};
        echo.line(esn(v, 5, 9, 2, 1));
    }
    echo.text("# origin position (x0,y0) and rotation");
    {
        Record r = rd.record("the origin");
        in.x0 = r.real("x0"); in.y0 = r.real("y0"); in.rot = r.real("rotation");
        const double v[3] = {in.x0, in.y0, in.rot};
        echo.line(esn(v, 3, 9, 2, 1));
    }
    echo.text("# observation depth (displacement and stress)");
    {
        Record r = rd.record("the observation depths");
        in.oz = r.real("oz"); in.ozs = r.real("ozs");
        const double v[2] = {in.oz, in.ozs};
        echo.line(esn(v, 2, 9, 2, 1));
    }
    echo.text("# output directory");
    {
        const std::string l = rd.data("the output directory");
        const size_t f = l.find_first_not_of(" \t");
        const size_t e = l.find_first_of(" \t", f);
        in.wdir = l.substr(f, e == std::string::npos ? std::string::npos : e - f);
        echo.line(" " + in.wdir + " (time report: " + in.wdir + "/time.txt)");
    }
    echo.text("# lambda, mu, gamma (gamma = (1 - nu) rho g / mu)");
    {
        Record r = rd.record("the elastic parameters");
        c.lambda = r.real("lambda"); c.mu = r.real("mu"); c.gam = r.real("gamma");
        const double v[3] = {c.lambda, c.mu, c.gam};
        echo.line(esn(v, 3, 10, 2, 2));
    }
    echo.text("# time interval, (positive time step) or (negative skip, scaling)");
    {
        Record r = rd.record("the time interval");
        {
            std::string t = r.text;
            while (!t.empty() && (t.back() == ' ' || t.back() == '\t')) t.pop_back();
            echo.line("  " + t);
        }
        c.interval = r.real("interval");
        c.odt = r.real("output time step");
        c.tscale = 1.0;
        if (c.odt < 0) {
            c.tscale = r.real("time-step scaling");
            c.skip = (int)ceil(-c.odt);
            echo.line("# output every " + iw(c.skip, 3, 3) + " steps, dt scaled by " + es(c.tscale, 7, 2, 1));
        } else {
            c.skip = 0;
            echo.line("# output every " + es(c.odt, 9, 2, 1) + " time unit");
        }
    }

    // observation planes, src/input.f90:321-356
    echo.text("# number of observation planes");
    {
        Record r = rd.record("the number of observation planes");
        const int n = r.integer("number of observation planes");
        echo.line(iw(n, 5));
        if (n > 0) {
            echo.text(RULE);
            echo.text("# n        x1       x2       x3   length    width strike    dip");
            echo.text(RULE);
        }
        for (int k = 1; k <= n; k++) {
            Record l = rd.record("an observation plane");
            const int i = l.integer("index");
            ObsPlane o{};
            o.x = l.real("x1"); o.y = l.real("x2"); o.z = l.real("x3");
            o.length = l.real("length"); o.width = l.real("width");
            o.strike = l.real("strike"); o.dip = l.real("dip");
            const double v[5] = {o.x, o.y, o.z, o.length, o.width};
            echo.line(iw(k, 3, 3) + " " + esn(v, 5, 9, 2, 1) + fw(o.strike, 7, 1) + fw(o.dip, 7, 1));
            if (i != k) perr("input line %d: plane index misfit (%d, expected %d)", l.line, i, k);
            double dummy = 0, rake = 0;
            wang(dummy, o.x, o.y, o.z, o.length, o.width, o.strike, o.dip, rake, in.x0, in.y0, in.rot);
            in.op.push_back(o);
        }
    }
    // observation points, src/input.f90:358-397
    echo.text("# number of observation points");
    {
        Record r = rd.record("the number of observation points");
        const int n = r.integer("number of observation points");
        echo.line(iw(n, 5));
        if (n > 0) {
            echo.text(RULE);
            echo.text("# n name       x1       x2       x3 (name is a 4-character string)");
            echo.text(RULE);
        }
        for (int k = 1; k <= n; k++) {
            Record l = rd.record("an observation point");
            const int i = l.integer("index");
            std::string name = l.next("name");
            // CHARACTER(LEN=4): truncated or blank-padded to 4 characters
            name = name.substr(0, 4);
            name.resize(4, ' ');
            double x1 = l.real("x1"), x2 = l.real("x2"), x3 = l.real("x3");
            const double v[3] = {x1, x2, x3};
            echo.line(iw(i, 3, 3) + " " + name + esn(v, 3, 9, 2, 1));
            x1 -= in.x0;
            x2 -= in.y0;
            rotation(x1, x2, in.rot);
            if (i != k) perr("input line %d: points index misfit (%d, expected %d)", l.line, i, k);
            in.pts.insert(in.pts.end(), {x1, x2, x3});
            in.ptsname.push_back(name);
        }
    }
    // stress observation segments, src/input.f90:399-451
    echo.text("# number of stress observation segments");
    {
        Record r = rd.record("the number of stress observation segments");
        const int n = r.integer("number of segments");
        echo.line(iw(n, 5));
        if (n > 0) {
            echo.text(RULE);
            echo.text("# n        xs       ys       zs  length   width strike   dip friction");
            echo.text(RULE);
        }
        for (int k = 1; k <= n; k++) {
            Record l = rd.record("a stress observation segment");
            const int i = l.integer("index");
            Segment g{};
            g.x = l.real("x1"); g.y = l.real("x2"); g.z = l.real("x3");
            g.length = l.real("length"); g.width = l.real("width");
            g.strike = l.real("strike"); g.dip = l.real("dip"); g.friction = l.real("friction");
            const double v3[3] = {g.x, g.y, g.z}, v2[2] = {g.length, g.width};
            echo.line(iw(i, 4, 4) + esn(v3, 3, 9, 2, 1) + esn(v2, 2, 8, 2, 1) + fw(g.strike, 7, 1) +
                      fw(g.dip, 6, 1) + fw(g.friction, 7, 1));
            if (i != k) perr("input line %d: source index misfit (%d, expected %d)", l.line, i, k);
            if (std::fmax(g.length, g.width) <= 0) perr("input line %d: length and width must be positive", l.line);
            double dummy = 0, rake = 0;
            wang(dummy, g.x, g.y, g.z, g.length, g.width, g.strike, g.dip, rake, in.x0, in.y0, in.rot);
            in.sop.push_back(g);
        }
    }
    // prestress, src/input.f90:453-496
    echo.text("# number of prestress interfaces");
    {
        Record r = rd.record("the number of prestress interfaces");
        const int n = r.integer("number of prestress interfaces");
        echo.line(iw(n, 5));
        if (n > 0) {
            echo.text(RULE);
            echo.text("# n    depth  sigma11  sigma12  sigma13  sigma22  sigma23  sigma33");
            echo.text(RULE);
        }
        for (int k = 1; k <= n; k++) {
            Record l = rd.record("a prestress interface");
            const int i = l.integer("index");
            relax_tensor_layer t{};
            double v[7];
            for (int j = 0; j < 7; j++) v[j] = l.real(j == 0 ? "depth" : "stress component");
            t.z = (float)v[0];
            t.t.s11 = (float)v[1]; t.t.s12 = (float)v[2]; t.t.s13 = (float)v[3];
            t.t.s22 = (float)v[4]; t.t.s23 = (float)v[5]; t.t.s33 = (float)v[6];
            const double vf[7] = {t.z, t.t.s11, t.t.s12, t.t.s13, t.t.s22, t.t.s23, t.t.s33};
            echo.line(iw(i, 3, 3) + esn(vf, 7, 9, 2, 1));
            if (i != k) perr("input line %d: index misfit (%d, expected %d)", l.line, i, k);
            in.stresslayer.push_back(t);
        }
    }
    // linear and nonlinear viscous interfaces and their weak zones
    read_layers(rd, in, L_LIN, echo, "# number of linear viscous interfaces", "# n     depth    gamma0  cohesion", 3);
    if (!in.layers[L_LIN].empty())
        read_weakzones(rd, in, 0, echo, "# number of linear weak zones", false);
    read_layers(rd, in, L_NON, echo, "# number of nonlinear viscous interfaces",
                "# n     depth    gamma0     power  cohesion", 4);
    if (!in.layers[L_NON].empty())
        read_weakzones(rd, in, 1, echo, "# number of nonlinear weak zones", true);
    if (in.flags & RELAX_INPUT_TRANSIENT) {
        read_layers(rd, in, L_LT, echo, "# number of linear transient interfaces", "# n     depth    gamma0        Gk", 3);
        if (!in.layers[L_LT].empty())
            read_weakzones(rd, in, 2, echo, "# number of transient weak zones", false);
        read_layers(rd, in, L_NLT, echo, "# number of nonlinear transient interfaces",
                    "# n     depth    gamma0     power        Gk", 4);
        if (!in.layers[L_NLT].empty())
            read_weakzones(rd, in, 3, echo, "# number of transient weak zones", false);
    }
    // fault creep and afterslip planes, src/input.f90:1000-1101
    read_layers(rd, in, L_FC, echo, "# number of fault creep interfaces",
                "# n    depth   gamma0 (a-b)sig friction cohesion", 5);
    if (!in.layers[L_FC].empty()) {
        echo.text("# number of afterslip planes");
        Record r = rd.record("the number of afterslip planes");
        const int n = r.integer("number of afterslip planes");
        echo.line(iw(n, 5));
        if (n > 0) {
            echo.text(RULE);
            echo.text("# n        x1       x2       x3   length    width strike    dip   rake");
            echo.text(RULE);
        }
        for (int k = 1; k <= n; k++) {
            Record l = rd.record("an afterslip plane");
            const int i = l.integer("index");
            relax_plane p{};
            p.x = l.real("x1"); p.y = l.real("x2"); p.z = l.real("x3");
            p.length = l.real("length"); p.width = l.real("width");
            p.strike = l.real("strike"); p.dip = l.real("dip"); p.rake = l.real("rake");
            const double v[5] = {p.x, p.y, p.z, p.length, p.width};
            echo.line(iw(i, 3, 3) + " " + esn(v, 5, 9, 2, 1) + fw(p.strike, 7, 1) + fw(p.dip, 7, 1) +
                      fw(p.rake, 7, 1));
            if (i != k) perr("input line %d: plane index misfit (%d, expected %d)", l.line, i, k);
            // the rake of the afterslip planes is reversed
            p.rake = p.rake >= 0.0 ? p.rake - 180.0 : p.rake + 180.0;
            double dummy = 0;
            wang(dummy, p.x, p.y, p.z, p.length, p.width, p.strike, p.dip, p.rake, in.x0, in.y0, in.rot);
            p.px2 = fix(p.length / c.dx2);
            p.px3 = fix(p.width / c.dx3);
            in.planes.push_back(p);
        }
    }

    in.minlength = c.sx1 * c.dx1 + c.sx2 * c.dx2;
    in.minwidth = c.sx3 * c.dx3;
    auto track = [&](double length, double width) {
        in.minlength = std::fmin(in.minlength, length);
        in.minwidth = std::fmin(in.minwidth, width);
    };

    // interseismic loading, src/input.f90:1107-1245
    echo.text("# number of inter-seismic strike-slip segments");
    {
        Record r = rd.record("the number of interseismic strike-slip segments");
        const int n = r.integer("number of segments");
        echo.line(iw(n, 5));
        if (n > 0) {
            echo.text(RULE);
            echo.text("#  n  slip/time  xs ys zs  length width  strike dip rake");
            echo.text(RULE);
        }
        for (int k = 1; k <= n; k++) {
            Record l = rd.record("an interseismic segment");
            const int i = l.integer("index");
            relax_source s{};
            s.slip = l.real("slip rate");
            s.x = l.real("x1"); s.y = l.real("x2"); s.z = l.real("x3");
            s.length = l.real("length"); s.width = l.real("width");
            s.strike = l.real("strike"); s.dip = l.real("dip"); s.rake = l.real("rake");
            s.beta = c.beta;
            const double v4[4] = {s.slip, s.x, s.y, s.z}, v2[2] = {s.length, s.width};
            echo.line(iw(i, 4, 4) + esn(v4, 4, 9, 2, 1) + esn(v2, 2, 8, 2, 1) + fw(s.strike, 7, 1) +
                      fw(s.dip, 6, 1) + fw(s.rake, 7, 1));
            if (i != k) perr("input line %d: source index misfit (%d, expected %d)", l.line, i, k);
            if (std::fmax(s.length, s.width) <= 0) perr("input line %d: lengths must be positive", l.line);
            track(s.length, s.width);
            antialias(s.slip, s.length, s.width, c.dx1, c.dx2, c.dx3, c.nyquist);
            wang(s.slip, s.x, s.y, s.z, s.length, s.width, s.strike, s.dip, s.rake, in.x0, in.y0, in.rot);
            in.is.push_back(s);
        }
        if (n > 0) echo.text(RULE);
    }
    echo.text("# number of inter-seismic tensile segments");
    {
        Record r = rd.record("the number of interseismic tensile segments");
        const int n = r.integer("number of segments");
        echo.line(iw(n, 5));
        if (n > 0) {
            echo.text(RULE);
            echo.text("#  n  opening       xs       ys       zs  length   width strike   dip");
            echo.text(RULE);
        }
        for (int k = 1; k <= n; k++) {
            Record l = rd.record("an interseismic tensile segment");
            const int i = l.integer("index");
            relax_source s{};
            s.opening = l.real("opening rate");
            s.x = l.real("x1"); s.y = l.real("x2"); s.z = l.real("x3");
            s.length = l.real("length"); s.width = l.real("width");
            s.strike = l.real("strike"); s.dip = l.real("dip");
            s.beta = c.beta;
            const double v4[4] = {s.opening, s.x, s.y, s.z}, v2[2] = {s.length, s.width};
            echo.line(iw(i, 4, 4) + esn(v4, 4, 9, 2, 1) + esn(v2, 2, 8, 2, 1) + fw(s.strike, 7, 1) +
                      fw(s.dip, 6, 1));
            if (i != k) perr("input line %d: tensile source index misfit (%d, expected %d)", l.line, i, k);
            if (std::fmax(s.length, s.width) <= 0) perr("input line %d: lengths must be positive", l.line);
            track(s.length, s.width);
            // slip = 0 goes through the filter: only the dimensions change
            s.slip = 0;
            antialias(s.slip, s.length, s.width, c.dx1, c.dx2, c.dx3, c.nyquist);
            double rake = 0;
            wang(s.slip, s.x, s.y, s.z, s.length, s.width, s.strike, s.dip, rake, in.x0, in.y0, in.rot);
            in.its.push_back(s);
        }
        if (n > 0) echo.text(RULE);
    }

    // coseismic events, src/input.f90:1247-1750
    echo.text("# number of events");
    int ne;
    {
        Record r = rd.record("the number of events");
        ne = r.integer("number of events");
        echo.line(iw(ne, 5));
        if (ne < 0) perr("input line %d: negative number of events", r.line);
    }
    in.es.resize(ne); in.ets.resize(ne); in.em.resize(ne); in.el.resize(ne);
    in.ecub.resize(ne); in.etet.resize(ne); in.evert.resize(ne);
    in.events.assign(ne, relax_event{});
    for (int e = 0; e < ne; e++) {
        relax_event &ev = in.events[e];
        if (e > 0) {
            echo.text("# time of next event");
            Record r = rd.record("the time of the event");
            ev.time = r.real("event time");
            // event times are multiples of the output time step
            if (c.skip == 0) ev.time = std::round(ev.time / c.odt) * c.odt;   // NINT
            echo.line(es(ev.time, 9, 2, 1) + " (multiple of " + es(c.odt, 9, 2, 1) + ")");
            if (ev.time <= in.events[e - 1].time)
                perr("input line %d: coseismic source time must increase", r.line);
        }
        echo.text("# number of coseismic strike-slip segments");
        {
            Record r = rd.record("the number of coseismic strike-slip segments");
            const int n = r.integer("number of segments");
            echo.line(iw(n, 5));
            if (n > 0) {
                echo.text(RULE);
                echo.text("#  n     slip       xs       ys       zs  length   width strike   dip   rake");
                echo.text(RULE);
            }
            for (int k = 1; k <= n; k++) {
                Record l = rd.record("a coseismic segment");
                const int i = l.integer("index");
                relax_source s{};
                s.slip = l.real("slip");
                s.x = l.real("x1"); s.y = l.real("x2"); s.z = l.real("x3");
                s.length = l.real("length"); s.width = l.real("width");
                s.strike = l.real("strike"); s.dip = l.real("dip"); s.rake = l.real("rake");
                // the smoothing parameter is optional
                const bool hasbeta = l.more();
                s.beta = hasbeta ? l.real("beta") : c.beta;
                if (hasbeta && s.beta > 0.5e8) perr("input line %d: invalid smoothing parameter (beta)", l.line);
                const double v4[4] = {s.slip, s.x, s.y, s.z}, v2[2] = {s.length, s.width};
                std::string o = iw(i, 4, 4) + esn(v4, 4, 9, 2, 1) + esn(v2, 2, 8, 2, 1) + fw(s.strike, 7, 1) +
                                fw(s.dip, 6, 1) + fw(s.rake, 7, 1);
                if (hasbeta) o += fw(s.beta, 6, 1);
                echo.line(o);
                if (i != k) perr("input line %d: source index misfit (%d, expected %d)", l.line, i, k);
                if (std::fmax(s.length, s.width) <= 0) perr("input line %d: lengths must be positive", l.line);
                track(s.length, s.width);
                wang(s.slip, s.x, s.y, s.z, s.length, s.width, s.strike, s.dip, s.rake, in.x0, in.y0, in.rot);
                in.es[e].push_back(s);
            }
            if (n > 0) echo.text(RULE);
        }
        echo.text("# number of coseismic tensile segments");
        {
            Record r = rd.record("the number of coseismic tensile segments");
            const int n = r.integer("number of segments");
            echo.line(iw(n, 5));
            if (n > 0) {
                echo.text(RULE);
                echo.text("#  n  opening       xs       ys       zs  length   width strike   dip");
                echo.text(RULE);
            }
            for (int k = 1; k <= n; k++) {
                Record l = rd.record("a tensile segment");
                const int i = l.integer("index");
                relax_source s{};
                s.opening = l.real("opening");
                s.x = l.real("x1"); s.y = l.real("x2"); s.z = l.real("x3");
                s.length = l.real("length"); s.width = l.real("width");
                s.strike = l.real("strike"); s.dip = l.real("dip");
                s.slip = s.opening;
                s.beta = c.beta;
                const double v4[4] = {s.opening, s.x, s.y, s.z}, v2[2] = {s.length, s.width};
                echo.line(iw(k, 4, 4) + esn(v4, 4, 9, 2, 1) + esn(v2, 2, 8, 2, 1) + fw(s.strike, 7, 1) +
                          fw(s.dip, 6, 1));
                if (i != k) perr("input line %d: source index misfit (%d, expected %d)", l.line, i, k);
                track(s.length, s.width);
                double rake = 0;
                wang(s.slip, s.x, s.y, s.z, s.length, s.width, s.strike, s.dip, rake, in.x0, in.y0, in.rot);
                in.ets[e].push_back(s);
            }
            if (n > 0) echo.text(RULE);
        }
        echo.text("# number of dilatation point sources");
        {
            Record r = rd.record("the number of dilatation point sources");
            const int n = r.integer("number of point sources");
            echo.line(iw(n, 5));
            if (n > 0) {
                echo.text(RULE);
                echo.text("#  n strain (positive for extension) xs ys zs");
                echo.text(RULE);
            }
            for (int k = 1; k <= n; k++) {
                Record l = rd.record("a dilatation point source");
                const int i = l.integer("index");
                relax_source s{};
                s.slip = l.real("strain");
                s.x = l.real("x1"); s.y = l.real("x2"); s.z = l.real("x3");
                s.beta = c.beta;
                const double v4[4] = {s.slip, s.x, s.y, s.z};
                echo.line(iw(k, 4, 4) + esn(v4, 4, 9, 2, 1));
                if (i != k) perr("input line %d: source index misfit (%d, expected %d)", l.line, i, k);
                rotation(s.x, s.y, in.rot);
                in.em[e].push_back(s);
            }
            if (n > 0) echo.text(RULE);
        }
        if (in.flags & RELAX_INPUT_EIGENSTRAIN) {
            echo.text("# number of cuboid eigenstrain sources");
            Record r = rd.record("the number of cuboid eigenstrain sources");
            const int n = r.integer("number of cuboids");
            echo.line(iw(n, 5));
            if (n < 0) perr("input line %d: negative number of cuboids", r.line);
            if (n > 0) {
                echo.text(RULE);
                echo.text("#  n       e11       e12       e13       e22       e23       e33       x1       x2       "
                          "x3  length   width thickness strike dip");
                echo.text(RULE);
            }
            for (int k = 1; k <= n; k++) {
                // src/input.f90:1510-1560: the strain, then the geometry of a weak zone
                Record q = rd.record("a cuboid");
                const int i = q.integer("index");
                relax_weakzone w{};
                const char *en[6] = {"e11", "e12", "e13", "e22", "e23", "e33"};
                float *ep[6] = {&w.e.s11, &w.e.s12, &w.e.s13, &w.e.s22, &w.e.s23, &w.e.s33};
                double ev[6];
                for (int j = 0; j < 6; j++) {
                    ev[j] = q.real(en[j]);
                    *ep[j] = (float)ev[j];
                }
                w.x = q.real("x1"); w.y = q.real("x2"); w.z = q.real("x3");
                w.length = q.real("length"); w.width = q.real("width"); w.thickness = q.real("thickness");
                w.strike = q.real("strike"); w.dip = q.real("dip");
                // echoed from the stored REAL*4 strain, as the reference prints its copy
                const double v9[9] = {w.e.s11, w.e.s12, w.e.s13, w.e.s22, w.e.s23, w.e.s33, w.x, w.y, w.z};
                const double v3[3] = {w.length, w.width, w.thickness}, v2[2] = {w.strike, w.dip};
                echo.line(iw(k, 4, 4) + esn(v9, 9, 10, 2, 2) + esn(v3, 3, 8, 2, 1) + esn(v2, 2, 9, 2, 1));
                if (i != k) perr("input line %d: source index misfit (%d, expected %d)", q.line, i, k);
                double dummy = 0, rake = 0;
                wang(dummy, w.x, w.y, w.z, w.length, w.width, w.strike, w.dip, rake, in.x0, in.y0, in.rot);
                in.ecub[e].push_back(w);
            }
            if (n > 0) echo.text(RULE);
            in.ncuboid += n;
            if (in.flags & RELAX_INPUT_CURVILINEAR) {
                echo.text("# number of distributed tetrahedral eigenstrain sources");
                Record t = rd.record("the number of tetrahedra");
                const int nt = t.integer("number of tetrahedra");
                echo.line(iw(nt, 5));
                if (nt < 0) perr("input line %d: negative number of tetrahedra", t.line);
                if (nt > 0) {
                    echo.text(RULE);
                    echo.text("#  n       e11       e12       e13       e22       e23       e33       i1       i2       "
                              "i3       i4");
                    echo.text(RULE);
                    for (int k = 1; k <= nt; k++) {
                        Record q = rd.record("a tetrahedron");
                        const int i = q.integer("index");
                        relax_tetrahedron tt{};
                        const char *en[6] = {"e11", "e12", "e13", "e22", "e23", "e33"};
                        float *ep[6] = {&tt.e.s11, &tt.e.s12, &tt.e.s13, &tt.e.s22, &tt.e.s23, &tt.e.s33};
                        for (int j = 0; j < 6; j++) *ep[j] = (float)q.real(en[j]);
                        tt.i1 = q.integer("i1"); tt.i2 = q.integer("i2");
                        tt.i3 = q.integer("i3"); tt.i4 = q.integer("i4");
                        const double v6[6] = {tt.e.s11, tt.e.s12, tt.e.s13, tt.e.s22, tt.e.s23, tt.e.s33};
                        echo.line(iw(k, 4, 4) + esn(v6, 6, 10, 2, 2) + " " + iw(tt.i1, 8) + " " + iw(tt.i2, 8) +
                                  " " + iw(tt.i3, 8) + " " + iw(tt.i4, 8));
                        if (i != k) perr("input line %d: source index misfit (%d, expected %d)", q.line, i, k);
                        in.etet[e].push_back(tt);
                    }
                    echo.text("# number of tetrahedron vertices");
                    Record v = rd.record("the number of tetrahedron vertices");
                    const int nv = v.integer("number of vertices");
                    echo.line(iw(nv, 5));
                    echo.text(RULE);
                    echo.text("#  n        x1        x2        x3");
                    echo.text(RULE);
                    if (nv <= 0) perr("input line %d: must provide tetrahedra vertices", v.line);
                    for (int k = 1; k <= nv; k++) {
                        Record q = rd.record("a vertex");
                        const int i = q.integer("index");
                        const double xyz[3] = {q.real("x1"), q.real("x2"), q.real("x3")};
                        echo.line(iw(k, 4, 4) + esn(xyz, 3, 10, 2, 2));
                        if (i != k) perr("input line %d: source index misfit (%d, expected %d)", q.line, i, k);
                        for (int j = 0; j < 3; j++) in.evert[e].push_back(xyz[j]);
                    }
                    for (const auto &tt : in.etet[e])
                        for (int vi : {tt.i1, tt.i2, tt.i3, tt.i4})
                            if (vi < 1 || vi > nv) perr("tetrahedron vertex %d out of range (1..%d)", vi, nv);
                }
                in.ntetra += nt;
            }
        }
        echo.text("# number of surface loads");
        {
            Record r = rd.record("the number of surface loads");
            const int n = r.integer("number of surface loads");
            echo.line(iw(n, 5));
            if (n > 0) {
                echo.text(RULE);
                echo.text("# t3 in units of force/surface, positive down");
                echo.text("# T>0 for t3 sin(2pi/T+phi), T<=0 for t3 H(t)");
                echo.text("#  n       xs       ys   length    width       t3        T      phi");
                echo.text(RULE);
            }
            for (int k = 1; k <= n; k++) {
                Record l = rd.record("a surface load");
                const int i = l.integer("index");
                relax_source s{};
                s.x = l.real("x1"); s.y = l.real("x2");
                s.length = l.real("length"); s.width = l.real("width");
                s.slip = l.real("t3"); s.period = l.real("period"); s.phase = l.real("phase");
                const bool hasbeta = l.more();
                s.beta = hasbeta ? l.real("beta") : c.beta;
                if (hasbeta && s.beta > 0.5e8) perr("input line %d: invalid smoothing parameter beta", l.line);
                const double v[8] = {s.x, s.y, s.length, s.width, s.slip, s.period, s.phase, s.beta};
                echo.line(iw(k, 4, 4) + esn(v, hasbeta ? 8 : 7, 9, 2, 1));
                if (i != k) perr("input line %d: source index misfit (%d, expected %d)", l.line, i, k);
                rotation(s.x, s.y, in.rot);
                in.el[e].push_back(s);
            }
            if (n > 0) echo.text(RULE);
        }
    }
    if (ne == 0) perr("input: at least one event is required");
    const relax_event &e0 = in.events[0];
    if (in.es[0].empty() && in.ets[0].empty() && in.em[0].empty() && in.el[0].empty() && in.ncuboid == 0 &&
        in.ntetra == 0 && c.interval <= 0)
        perr("input: no input dislocations or dilatation point sources or surface tractions for first event");
    (void)e0;
    if (echo.on) printf("# max sampling size (hor.,vert.):%s%s\n", es(in.minlength / 2.5, 8, 2, 1).c_str(),
                        es(in.minwidth / 2.5, 8, 2, 1).c_str());
}

// depth structures and the pointers of the configuration
int finish(relax_input &in)
{
    relax_config &c = in.cfg;
    if (c.sx3 < 2) return relax_noalloc_fail(RELAX_ERR_ARG, "input: sx3 must be at least 2");
    const int nz = c.sx3 / 2;
    const relax_layer **dst[5] = {&c.linearstruc, &c.nonlinearstruc, &c.ltransientstruc, &c.nltransientstruc,
                                  &c.faultcreepstruc};
    for (int m = 0; m < 5; m++) {
        *dst[m] = nullptr;
        if (in.layers[m].empty()) continue;
        in.struc[m].assign(nz, relax_layer{});
        const int rc = relax_viscoelastic_structure(in.layers[m].data(), (int)in.layers[m].size(), c.dx3, nz,
                                                    in.struc[m].data());
        if (rc != RELAX_OK) return rc;
        *dst[m] = in.struc[m].data();
    }
    c.stressstruc = nullptr;
    if (!in.stresslayer.empty()) {
        in.stressstruc.assign(nz, relax_tensor_layer{});
        const int rc = relax_tensor_structure(in.stresslayer.data(), (int)in.stresslayer.size(), c.dx3, nz,
                                              in.stressstruc.data());
        if (rc != RELAX_OK) return rc;
        c.stressstruc = in.stressstruc.data();
    }
    c.np = (int)in.planes.size();
    c.planes = in.planes.empty() ? nullptr : in.planes.data();
    for (size_t e = 0; e < in.events.size(); e++) {
        relax_event &ev = in.events[e];
        ev.ns = (int)in.es[e].size(); ev.s = ev.ns ? in.es[e].data() : nullptr;
        ev.nt = (int)in.ets[e].size(); ev.ts = ev.nt ? in.ets[e].data() : nullptr;
        ev.nm = (int)in.em[e].size(); ev.m = ev.nm ? in.em[e].data() : nullptr;
        ev.nl = (int)in.el[e].size(); ev.l = ev.nl ? in.el[e].data() : nullptr;
        ev.nc = (int)in.ecub[e].size(); ev.c = ev.nc ? in.ecub[e].data() : nullptr;
        ev.ntet = (int)in.etet[e].size(); ev.tet = ev.ntet ? in.etet[e].data() : nullptr;
        ev.nvert = (int)(in.evert[e].size() / 3); ev.vert = ev.nvert ? in.evert[e].data() : nullptr;
    }
    c.ne = (int)in.events.size();
    c.events = in.events.data();
    c.inter = relax_event{};
    c.inter.ns = (int)in.is.size(); c.inter.s = in.is.empty() ? nullptr : in.is.data();
    c.inter.nt = (int)in.its.size(); c.inter.ts = in.its.empty() ? nullptr : in.its.data();
    c.x0 = in.x0; c.y0 = in.y0; c.rot = in.rot;
    c.lineardgammadot0 = c.nonlineardgammadot0 = nullptr;
    c.ltransientdgammadot0 = c.nltransientdgammadot0 = nullptr;
    in.ptsname_c.clear();
    for (const auto &s : in.ptsname) in.ptsname_c.push_back(s.c_str());
    return RELAX_OK;
}

}  // namespace

extern "C" int relax_input_parse(const char *text, int flags, relax_input **out)
{
    if (!text || !out) return relax_noalloc_fail(RELAX_ERR_ARG, "null argument");
    *out = nullptr;
    relax_input *in = new relax_input;
    in->flags = flags;
    try {
        parse(text, *in);
    } catch (const ParseError &e) {
        delete in;
        return relax_noalloc_fail(e.code, e.msg.c_str());
    }
    const int rc = finish(*in);
    if (rc != RELAX_OK) {
        delete in;
        return rc;
    }
    *out = in;
    return RELAX_OK;
}

extern "C" int relax_input_read(const char *path, int flags, relax_input **out)
{
    FILE *fp = path ? fopen(path, "rb") : stdin;
    if (!fp) {
        char msg[512];
        snprintf(msg, sizeof msg, "cannot open %s: %s", path, strerror(errno));
        return relax_noalloc_fail(RELAX_ERR_ARG, msg);
    }
    std::string text;
    char buf[65536];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, n);
    if (path) fclose(fp);
    return relax_input_parse(text.c_str(), flags, out);
}

extern "C" void relax_input_free(relax_input *in) { delete in; }

extern "C" const relax_config *relax_input_config(const relax_input *in) { return in ? &in->cfg : nullptr; }

extern "C" int relax_input_get_info(const relax_input *in, relax_input_info *info)
{
    if (!in || !info) return relax_noalloc_fail(RELAX_ERR_ARG, "null argument");
    info->wdir = in->wdir.c_str();
    info->x0 = in->x0; info->y0 = in->y0; info->rot = in->rot;
    info->oz = in->oz; info->ozs = in->ozs;
    info->npts = (int)in->ptsname.size();
    info->pts = in->pts.empty() ? nullptr : in->pts.data();
    info->ptsname = in->ptsname_c.empty() ? nullptr : in->ptsname_c.data();
    info->nop = (int)in->op.size();
    info->nsop = (int)in->sop.size();
    for (int m = 0; m < 4; m++) info->nwz[m] = (int)in->wz[m].size();
    info->minlength = in->minlength;
    info->minwidth = in->minwidth;
    return RELAX_OK;
}

// The geometry files of init (src/input.f90:296-1452), in the order init
// writes them.  The reference's own names are kept, including two of its
// quirks: the linear transient weak zones go to weakzone-nl-KKK.xy and
// weakzones-nonlinear.vtp (the nonlinear zones' names), and rdykes-EEE.*
// hold the event's shear sources (exportvtk_rfaults / exportxy_rfaults read
// the shear list).  The linear transient .vtp takes that mechanism's own
// zone count, where the reference passes the nonlinear count.
extern "C" int relax_input_export_geometry(const relax_input *in, int vtk)
{
    if (!in) return relax_noalloc_fail(RELAX_ERR_ARG, "null input");
    const relax_config &c = in->cfg;
    const std::string w = in->wdir;
    auto name = [&](const char *stem, int k, int digits, const char *ext) {
        char b[96];
        snprintf(b, sizeof b, "/%s%0*d%s", stem, digits, k, ext);
        return w + b;
    };
    int rc = RELAX_OK;
    if (vtk) rc = relax_write_vtk_grid(c.sx1, c.sx2, c.sx3, c.dx1, c.dx2, c.dx3, (w + "/cgrid.vtp").c_str());
    // viscous and transient interfaces (a horizontal rectangle over the box)
    // and their weak zones
    struct Mech {
        int layer, zones;
        const char *lname, *xyname, *vtpname;
    };
    const Mech mech[4] = {{0, 0, "linearlayer-", "weakzone-", "/weakzones-linear.vtp"},
                          {1, 1, "nonlinearlayer-", "weakzone-nl-", "/weakzones-nonlinear.vtp"},
                          {2, 2, "ltransientlayer-", "weakzone-nl-", "/weakzones-nonlinear.vtp"},
                          {3, 3, "nltransientlayer-", "weakzone-nltr-", "/weakzones-nonlinear-transient.vtp"}};
    for (int m = 0; m < 4 && rc == RELAX_OK; m++) {
        if (m >= 2 && !(in->flags & RELAX_INPUT_TRANSIENT)) break;
        const auto &layers = in->layers[mech[m].layer];
        for (size_t k = 0; k < layers.size() && vtk && rc == RELAX_OK; k++)
            rc = relax_write_vtk_rectangle(0.0, 0.0, layers[k].z, (double)c.sx2 * c.dx2, (double)c.sx1 * c.dx1, 0.0,
                                           1.5708, name(mech[m].lname, (int)k + 1, 3, ".vtp").c_str());
        const auto &zones = in->wz[mech[m].zones];
        if (layers.empty() || zones.empty()) continue;
        for (size_t k = 0; k < zones.size() && rc == RELAX_OK; k++)
            rc = relax_write_xy_brick(&zones[k], name(mech[m].xyname, (int)k + 1, 3, ".xy").c_str());
        if (vtk && rc == RELAX_OK)
            rc = relax_write_vtk_bricks((int)zones.size(), zones.data(), (w + mech[m].vtpname).c_str());
    }
    // afterslip planes
    for (size_t k = 0; k < in->planes.size() && vtk && rc == RELAX_OK; k++) {
        const relax_plane &p = in->planes[k];
        rc = relax_write_vtk_rectangle(p.x, p.y, p.z, p.length, p.width, p.strike, p.dip,
                                       name("aplane-", (int)k + 1, 4, ".vtp").c_str());
    }
    // each event's shear faults and tensile dykes
    for (size_t e = 0; e < in->es.size() && rc == RELAX_OK; e++) {
        const auto &s = in->es[e];
        const relax_source *sp = s.empty() ? nullptr : s.data();
        const char *stems[2] = {"rfaults-", "rdykes-"};
        const bool has[2] = {!s.empty(), !in->ets[e].empty()};
        for (int q = 0; q < 2 && rc == RELAX_OK; q++) {
            if (!has[q]) continue;
            if (vtk) rc = relax_write_faults(RELAX_FAULTS_VTP, (int)s.size(), sp, 0.0, 0.0,
                                             name(stems[q], (int)e + 1, 3, ".vtp").c_str());
            if (rc == RELAX_OK)
                rc = relax_write_faults(RELAX_FAULTS_XY, (int)s.size(), sp, in->x0, in->y0,
                                        name(stems[q], (int)e + 1, 3, ".xy").c_str());
        }
    }
    return rc;
}

extern "C" int relax_input_obsplanes(const relax_input *in, const relax_obsplane **op, int *n)
{
    if (!in || !op || !n) return relax_noalloc_fail(RELAX_ERR_ARG, "null argument");
    *n = (int)in->op.size();
    *op = in->op.empty() ? nullptr : in->op.data();
    return RELAX_OK;
}

extern "C" int relax_input_segments(const relax_input *in, const relax_segment **sop, int *n)
{
    if (!in || !sop || !n) return relax_noalloc_fail(RELAX_ERR_ARG, "null argument");
    *n = (int)in->sop.size();
    *sop = in->sop.empty() ? nullptr : in->sop.data();
    return RELAX_OK;
}

extern "C" int relax_input_weakzones(const relax_input *in, int mechanism, const relax_weakzone **zones, int *n)
{
    if (!in || !zones || !n || mechanism < 0 || mechanism > 3) return relax_noalloc_fail(RELAX_ERR_ARG, "argument");
    *n = (int)in->wz[mechanism].size();
    *zones = in->wz[mechanism].empty() ? nullptr : in->wz[mechanism].data();
    return RELAX_OK;
}

// builddgammadot0 of each mechanism with weak zones (src/relax.f90:487-541),
// evaluated on `device` and kept in the input for relax_create
extern "C" int relax_input_build_weakzones(relax_input *in, int device)
{
    if (!in) return relax_noalloc_fail(RELAX_ERR_ARG, "null input");
    relax_config &c = in->cfg;
    const float **dst[4] = {&c.lineardgammadot0, &c.nonlineardgammadot0, &c.ltransientdgammadot0,
                            &c.nltransientdgammadot0};
    const size_t nh = (size_t)c.sx1 * c.sx2 * (c.sx3 / 2);
    for (int m = 0; m < 4; m++) {
        *dst[m] = nullptr;
        if (in->wz[m].empty()) continue;
        if (cudaSetDevice(device) != cudaSuccess) return relax_noalloc_fail(RELAX_ERR_CUDA, "cudaSetDevice failed");
        float *d = nullptr;
        if (cudaMalloc(&d, nh * sizeof(float)) != cudaSuccess)
            return relax_noalloc_fail(RELAX_ERR_NOMEM, "weak-zone field allocation failed");
        int rc = relax_op_dgammadot0(in->wz[m].data(), (int)in->wz[m].size(), c.sx1, c.sx2, c.sx3 / 2, c.dx1, c.dx2,
                                     c.dx3, 0.0, d, nullptr);
        in->dg[m].assign(nh, 0.f);
        if (rc == RELAX_OK &&
            cudaMemcpy(in->dg[m].data(), d, nh * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = relax_noalloc_fail(RELAX_ERR_CUDA, "weak-zone field copy failed");
        cudaFree(d);
        if (rc != RELAX_OK) return rc;
        *dst[m] = in->dg[m].data();
    }
    return RELAX_OK;
}
