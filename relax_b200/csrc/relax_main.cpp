// relax -- the command-line program of RELAX (src/relax.f90:1-1100 with the
// options of src/input.f90:64-185) on the B200 library: reads the input
// file (an argument or standard input), runs the coseismic solve of the
// first event and the relaxation loop on one GPU, writes the point time
// series every step and the map-view grids, VTK fields, afterslip planes,
// observation planes, stress segments and the time report on output steps,
// and prints the step log.
//
// GPU: RELAX_DEVICE (default 0).
#include <getopt.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/relax_b200.h"

namespace {

struct Options {
    bool grd = true, relax = true, stress = true, txt = true, vtk = true, vtkrelax = false, xyz = true;
    bool eigenstrain = false, transient = false, curvilinear = false, dryrun = false, help = false,
         version = false;
};

const char RULE[] = "# ----------------------------------------------------------------------------";

void usage()
{
    printf("usage:\n\n");
    printf("relax [-h] [--dry-run] [--help] [--no-grd-output] [--no-relax-output]\n");
    printf("      [--no-stress-output] [--no-txt-output] [--no-vtk-output]\n");
    printf("      [--no-xyz-output] [--with-eigenstrain] [--with-vtk-output]\n");
    printf("      [--with-vtk-relax-output] [--with-transient] [input file]\n\n");
    printf("options:\n");
    printf("   -h                      prints this message and aborts calculation\n");
    printf("   --dry-run               abort calculation, only output geometry\n");
    printf("   --help                  prints this message and aborts calculation\n");
    printf("   --no-grd-output         cancel output in GMT grd binary format\n");
    printf("   --no-relax-output       cancel output of the postseismic contribution\n");
    printf("   --no-stress-output      cancel output of stress tensor in any format\n");
    printf("   --no-txt-output         cancel output in text format\n");
    printf("   --no-vtk-output         cancel output in Paraview VTK format\n");
    printf("   --no-xyz-output         cancel output in GMT xyz format\n");
    printf("   --version               print version number and exit\n");
    printf("   --with-eigenstrain      includes eigenstrain sources\n");
    printf("   --with-stress-output    export stress tensor\n");
    printf("   --with-vtk-output       export output in Paraview VTK format\n");
    printf("   --with-vtk-relax-output export relaxation to VTK format\n");
    printf("   --with-transient        include the transient rheology\n\n");
    printf("description:\n");
    printf("   Evaluates the deformation due to fault slip, surface loading\n");
    printf("   or inflation and the time series of postseismic relaxation\n");
    printf("   that follows due to fault creep or viscoelastic flow.\n\n");
}

int check(int rc, const char *what)
{
    if (rc != RELAX_OK) fprintf(stderr, "relax: %s: %s\n", what, relax_last_error());
    return rc;
}

// reporttime, src/export.f90:42-65
int reporttime(const std::string &wdir, int append, double t)
{
    const std::string f = wdir + "/time.txt";
    FILE *fp = fopen(f.c_str(), append ? "a" : "w");
    if (!fp) {
        fprintf(stderr, "relax: could not open %s for export\n", f.c_str());
        return RELAX_ERR_ARG;
    }
    char b[32];
    relax_es_format(t, 11, 3, 2, b, sizeof b);
    fprintf(fp, "%s\n", b);
    fclose(fp);
    return RELAX_OK;
}

// exportoptsdat, src/export.f90:264-282
void exportoptsdat(const relax_input_info &info)
{
    if (info.npts <= 0) return;
    const std::string f = std::string(info.wdir) + "/opts.dat";
    FILE *fp = fopen(f.c_str(), "w");
    if (!fp) return;
    fprintf(fp, "# x1(north) x2(east) x3(down) name(4-char)\n");
    for (int k = 0; k < info.npts; k++) {
        char a[3][32];
        for (int j = 0; j < 3; j++) relax_es_format(info.pts[3 * k + j], 11, 4, 1, a[j], sizeof a[j]);
        fprintf(fp, "%s%s%s %s\n", a[0], a[1], a[2], info.ptsname[k]);
    }
    fclose(fp);
}

// wdir/<stem>-NNNN<ext>, the names of the segment exports
std::string name4(const std::string &wdir, const char *stem, int i, const char *ext)
{
    char b[96];
    snprintf(b, sizeof b, "/%s-%04d%s", stem, i, ext);
    return wdir + b;
}

std::string name3(const std::string &wdir, const char *stem, int i, int digits)
{
    char b[64];
    snprintf(b, sizeof b, "/%s-%0*d.vtk", stem, digits, i);
    return wdir + b;
}

}  // namespace

int main(int argc, char **argv)
{
    Options o;
    static const struct option longopts[] = {
        {"no-relax-output", no_argument, nullptr, 21}, {"no-txt-output", no_argument, nullptr, 22},
        {"no-vtk-output", no_argument, nullptr, 23},   {"no-grd-output", no_argument, nullptr, 24},
        {"no-xyz-output", no_argument, nullptr, 25},   {"no-stress-output", no_argument, nullptr, 26},
        {"version", no_argument, nullptr, 27},         {"with-eigenstrain", no_argument, nullptr, 28},
        {"with-stress-output", no_argument, nullptr, 29}, {"with-vtk-output", no_argument, nullptr, 30},
        {"with-vtk-relax-output", no_argument, nullptr, 31}, {"with-transient", no_argument, nullptr, 32},
        {"with-curvilinear", no_argument, nullptr, 33}, {"dry-run", no_argument, nullptr, 34},
        {"help", no_argument, nullptr, 'h'},           {nullptr, 0, nullptr, 0}};
    int ch;
    while ((ch = getopt_long(argc, argv, "h", longopts, nullptr)) != -1) {
        switch (ch) {
        case 21: o.relax = false; break;
        case 22: o.txt = false; break;
        case 23: o.vtk = false; break;
        case 24: o.grd = false; break;
        case 25: o.xyz = false; break;
        case 26: o.stress = false; break;
        case 27: o.version = true; break;
        case 28: o.eigenstrain = true; break;
        case 29: o.stress = true; break;
        case 30: o.vtk = true; break;
        case 31: o.vtkrelax = true; break;
        case 32: o.transient = true; break;
        case 33: o.curvilinear = true; break;
        case 34: o.dryrun = true; break;
        default: o.help = true; break;
        }
    }
    if (o.version) {
        printf("relax version 1.0.7 (%s), compiled on %s\n\n", relax_version(), __DATE__);
        return 0;
    }
    if (o.help) {
        usage();
        return 0;
    }
    printf("%s\n", RULE);
    printf("# RELAX: nonlinear postseismic relaxation with Fourier-domain Green's function\n");
    printf("#     * B200 (sm_100a) implementation of the Green's function and the time step\n");
    printf(o.vtk ? "#     * export to VTK format\n"
                 : "#     * export to VTK format cancelled                     (--no-vtk-output)\n");
    if (o.vtkrelax) printf("#     * export relaxation component to VTK format   (--with-vtk-relax-output)\n");
    printf("%s\n", RULE);
    fflush(stdout);

    const int flags = RELAX_INPUT_ECHO | (o.transient ? RELAX_INPUT_TRANSIENT : 0) |
                      (o.eigenstrain ? RELAX_INPUT_EIGENSTRAIN : 0) | (o.curvilinear ? RELAX_INPUT_CURVILINEAR : 0);
    relax_input *in = nullptr;
    const char *path = optind < argc ? argv[optind] : nullptr;
    int rc = relax_input_read(path, flags, &in);
    fflush(stdout);
    if (check(rc, "input") != RELAX_OK) return 1;
    relax_input_info info;
    relax_input_get_info(in, &info);
    const relax_config *cfg = relax_input_config(in);
    const std::string wdir = info.wdir;
    {
        // the write-permission test of init
        const std::string f = wdir + "/report.txt";
        FILE *fp = fopen(f.c_str(), "a");
        if (!fp) {
            fprintf(stderr, "relax: unable to access %s/time.txt\n", wdir.c_str());
            relax_input_free(in);
            return 1;
        }
        fclose(fp);
    }
    exportoptsdat(info);
    // the geometry files of init (grid, interfaces, weak zones, planes, faults)
    if (check(relax_input_export_geometry(in, o.vtk ? 1 : 0), "geometry files") != RELAX_OK) {
        relax_input_free(in);
        return 1;
    }
    if (o.dryrun) {
        printf("dry run: abort calculation\n");
        relax_input_free(in);
        return 0;
    }
    const char *dev = getenv("RELAX_DEVICE");
    const int device = dev ? atoi(dev) : 0;
    relax_ctx *ctx = nullptr;
    if (check(relax_input_build_weakzones(in, device), "weak zones") != RELAX_OK ||
        check(relax_create(cfg, device, &ctx), "relax_create") != RELAX_OK) {
        relax_input_free(in);
        return 1;
    }
    const int sx3h = cfg->sx3 / 2;
    const int slice = (int)(info.oz / cfg->dx3);
    const bool track_slice = o.grd && o.relax && slice >= 0 && slice < sx3h;
    rc = relax_track_relaxation(ctx, o.vtk ? sx3h : 0, o.vtkrelax ? sx3h : 0, track_slice ? slice : -1);
    const bool transient = cfg->ltransientstruc || cfg->nltransientstruc;
    char line[256];
    int e = 1, oi = 1;
    relax_step_log log{};

    // observation planes and stress observation segments (src/relax.f90:
    // 330-333, 425-466 after the coseismic step; 939-942, 993-1025 at output
    // steps); sig0 is the segments' stress after the coseismic step
    // (export_rfaults_stress_init, src/export.f90:1364-1394)
    const relax_obsplane *op = nullptr;
    const relax_segment *sop = nullptr;
    int nop = 0, nsop = 0;
    relax_input_obsplanes(in, &op, &nop);
    relax_input_segments(in, &sop, &nsop);
    std::vector<relax_tensor> sig0(nsop), sigs(nsop);
    auto planes_and_segments = [&](int index, double t, bool first) -> int {
        int r = RELAX_OK;
        if (o.eigenstrain && nop > 0)
            r = relax_export_plane_stress(ctx, RELAX_FIELD_GAMMA, nop, op, info.x0, info.y0, wdir.c_str(), index);
        if (r == RELAX_OK && nop > 0)
            r = relax_export_plane_stress(ctx, RELAX_FIELD_SIG, nop, op, info.x0, info.y0, wdir.c_str(), index);
        if (r != RELAX_OK || nsop == 0) return r;
        if ((r = relax_segment_stress(ctx, nsop, sop, sigs.data())) != RELAX_OK) return r;
        if (first) sig0 = sigs;
        const relax_tensor *s = sigs.data(), *ds = first ? nullptr : sigs.data(), *s0 = first ? nullptr : sig0.data();
        r = relax_write_segments(RELAX_SEG_VTP, nsop, sop, s, nullptr,
                                 name4(wdir, "rfaults-sigma", index, ".vtp").c_str());
        if (r == RELAX_OK)
            r = relax_write_segments(RELAX_SEG_VTP, nsop, sop, ds, s0,
                                     name4(wdir, "rfaults-dsigma", index, ".vtp").c_str());
        if (r == RELAX_OK)
            r = relax_write_segments(RELAX_SEG_GMT, nsop, sop, s, nullptr,
                                     name4(wdir, "rfaults-sigma", index, ".xy").c_str());
        if (r == RELAX_OK && first)
            r = relax_write_segments(RELAX_SEG_TRACTION, nsop, sop, s, nullptr,
                                     name4(wdir, "rfaults-traction", index, ".dat").c_str());
        if (r == RELAX_OK)
            r = relax_write_segments(RELAX_SEG_GMT, nsop, sop, ds, s0,
                                     name4(wdir, "rfaults-dsigma", index, ".xy").c_str());
        if (r == RELAX_OK) r = relax_write_coulomb(nsop, sop, s, t, wdir.c_str(), first ? 1 : 0);
        return r;
    };

    auto exports = [&](int index, double t, bool first) -> int {
        int r = RELAX_OK;
        // the afterslip planes, at output steps only (src/relax.f90:910-918)
        const int creep = (o.txt ? RELAX_CREEP_TXT : 0) | (o.grd ? RELAX_CREEP_GRD : 0) | (o.vtk ? RELAX_CREEP_VTK : 0);
        if (!first && creep)
            r = check(relax_export_creep(ctx, wdir.c_str(), index, creep), "afterslip planes");
        if (!first && transient && o.grd && r == RELAX_OK)
            r = check(relax_export_grd(ctx, RELAX_FIELD_EPS, info.ozs, info.x0, info.y0, wdir.c_str(), index),
                      "transient strain grids");
        if (o.grd) {
            if (track_slice && r == RELAX_OK)
                r = check(relax_export_grd(ctx, RELAX_FIELD_UR, info.oz, info.x0, info.y0, wdir.c_str(), index),
                          "postseismic grids");
            if (r == RELAX_OK)
                r = check(relax_export_grd(ctx, RELAX_FIELD_U, info.oz, info.x0, info.y0, wdir.c_str(), index),
                          "displacement grids");
        }
        if (o.vtk && r == RELAX_OK) {
            if (first) {
                r = check(relax_export_vtk(ctx, RELAX_FIELD_U, sx3h, 4, 4, 8, name3(wdir, "disp", 0, 3).c_str(),
                                           "coseismic displacement vector field", "displacement"),
                          "vtk");
            } else {
                r = check(relax_export_vtk(ctx, RELAX_FIELD_U, cfg->sx3 / 4, 4, 4, 8,
                                           name3(wdir, "disp", index, 3).c_str(),
                                           "cumulative displacement vector field", "displacement"),
                          "vtk");
                if (r == RELAX_OK)
                    r = check(relax_export_vtk(ctx, RELAX_FIELD_V, sx3h, 8, 8, 16, name3(wdir, "vel", index, 3).c_str(),
                                               "instantaneous velocity vector field", "velocity"),
                              "vtk");
            }
        }
        if (o.vtkrelax && r == RELAX_OK)
            r = check(relax_export_vtk(ctx, RELAX_FIELD_UR, first ? sx3h : cfg->sx3 / 4, 4, 4, 8,
                                       name3(wdir, "disp-relax", index, 4).c_str(),
                                       "postseismic displacement vector field", "displacement"),
                      "vtk");
        if (first && info.npts > 0 && r == RELAX_OK)
            r = check(relax_export_points(ctx, info.npts, info.pts, info.ptsname, t, info.rot, wdir.c_str(), 1),
                      "points");
        if (o.grd && o.stress && r == RELAX_OK)
            r = check(relax_export_grd(ctx, RELAX_FIELD_SIG, info.ozs, info.x0, info.y0, wdir.c_str(), index),
                      "stress grids");
        if (o.vtk && o.stress && r == RELAX_OK)
            r = check(relax_export_vtk(ctx, RELAX_FIELD_SIG, sx3h, 4, 4, 8, name3(wdir, "sigma", index, 4).c_str(),
                                       "stress tensor field", "stress"),
                      "vtk");
        if (r == RELAX_OK) r = check(planes_and_segments(index, t, first), "observation planes and segments");
        if (r == RELAX_OK) r = reporttime(wdir, first ? 0 : 1, t);
        return r;
    };

    printf("# event %03d\n", e);
    printf("%s\n", relax_log_header(transient));
    if (check(rc, "tracking") != RELAX_OK || check(relax_coseismic(ctx, 0, &log), "coseismic") != RELAX_OK ||
        exports(0, 0.0, true) != RELAX_OK) {
        relax_destroy(ctx);
        relax_input_free(in);
        return 1;
    }
    log.i = 0;
    relax_format_log(&log, cfg->interval, transient, line, sizeof line);
    printf("%s\n", line);
    fflush(stdout);
    int status = 0;
    while (cfg->interval > 0) {
        if (check(relax_step(ctx, nullptr, &log), "step") != RELAX_OK) {
            status = 1;
            break;
        }
        if (log.i == 0) break;      // t reached the interval
        if (log.event) {
            e++;
            printf("coseismic event %03d\n", e);
            printf("%s\n", relax_log_header(transient));
        }
        // points are exported at all time steps
        if (info.npts > 0 &&
            check(relax_export_points(ctx, info.npts, info.pts, info.ptsname, log.t, info.rot, wdir.c_str(), 0),
                  "points") != RELAX_OK) {
            status = 1;
            break;
        }
        if (log.output) {
            if (exports(oi, log.t, false) != RELAX_OK) {
                status = 1;
                break;
            }
            oi++;
        }
        relax_format_log(&log, cfg->interval, transient, line, sizeof line);
        printf("%s\n", line);
        fflush(stdout);
    }
    relax_destroy(ctx);
    relax_input_free(in);
    return status;
}
