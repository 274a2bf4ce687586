/*
 * relax_b200.h -- C ABI of the B200 (sm_100a) implementation of RELAX's
 * per-time-step relaxation loop.
 *
 * Two layers are exported:
 *
 *  1. A context API (relax_*): explicit handle, int status on every call,
 *     stream-ordered work on one CUDA device.  This is what a new host
 *     (C, C++, Fortran via iso_c_binding, Python via ctypes) binds.
 *
 *  2. A compatibility shim (cu*_ symbols, gfortran naming: lower case and a
 *     trailing underscore, scalars by value, arrays by reference) that
 *     replaces the reference CUDA layer symbol for symbol, so that the
 *     reference Fortran GPU driver links unchanged.  Each declaration below
 *     cites the reference function it replaces.
 *
 * Field layouts at the boundary are RELAX's: Fortran column-major, i1
 * fastest.  Vector fields are padded to sx1+2 in x1 (in-place real FFT
 * layout of src/relax.f90:250-252), tensors are arrays of 6-float structs
 * (TENSOR, src/types.f90:41-44), the physical half-space holds sx3/2 layers.
 * Inside the library the fields are kept in a structure-of-arrays layout.
 */
#ifndef RELAX_B200_H
#define RELAX_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* status codes                                                       */
/* ------------------------------------------------------------------ */
#define RELAX_OK               0
#define RELAX_ERR_ARG          1   /* invalid argument / size            */
#define RELAX_ERR_CUDA         2   /* CUDA runtime error                 */
#define RELAX_ERR_NOMEM        3   /* device or host allocation failed   */
#define RELAX_ERR_UNSUPPORTED  4   /* grid/feature not implemented       */
#define RELAX_ERR_STATE        5   /* call out of order / no context     */
#define RELAX_ERR_FRICTION     6   /* tau/((a-b)sigma) > 20, the abort of
                                      src/friction3d.f90:204-215         */
#define RELAX_ERR_POWER        7   /* stress exponent < 0.999999, the abort
                                      of src/viscoelastic3d.f90:262-267   */

/* ------------------------------------------------------------------ */
/* data types (binary compatible with the reference)                   */
/* ------------------------------------------------------------------ */

/* TENSOR, src/types.f90:41-44 (C mirror src/cuinclude.h:204-212) */
typedef struct relax_tensor {
    float s11, s12, s13, s22, s23, s33;
} relax_tensor;

/* TENSOR_LAYER_STRUCT, src/types.f90:52-56 */
typedef struct relax_tensor_layer {
    float z, dum;
    relax_tensor t;
} relax_tensor_layer;

/* LAYER_STRUCT, src/types.f90:31-34.  For fault-creep structures the
 * fields are reused as: gammadot0 = V0, stressexponent = (a-b)sigma,
 * friction = mu_f, cohesion = c (src/friction3d.f90:131-134). */
typedef struct relax_layer {
    double z, gammadot0, stressexponent, cohesion, friction, Gk;
} relax_layer;

/* SOURCE_STRUCT, src/types.f90:26-29, in the internal convention
 * (after wangconvention, src/input.f90:1780-1800): centre coordinates,
 * strike/dip/rake in radians, slip sign flipped. */
typedef struct relax_source {
    double slip, x, y, z, width, length, strike, dip, rake,
           period, phase, beta, opening;
} relax_source;

/* PLANE_STRUCT without its patch array, src/types.f90:92-97 */
typedef struct relax_plane {
    double x, y, z, width, length, strike, dip, rake;
    int px2, px3;
} relax_plane;

/* SLIPPATCH_STRUCT, src/types.f90:76-90 */
typedef struct relax_slippatch {
    double x1, x2, x3, lx, lz, slip, ss, ds, v, vss, vds, taus;
    relax_tensor sig;
} relax_slippatch;

/* WEAK_STRUCT, src/types.f90:46-50: a ductile (weak) zone in the internal
 * convention (after wangconvention, src/input.f90:574-583).  Negative
 * dimensions select spherical / cylindrical zones (src/viscoelastic3d.f90:
 * 403-430). */
typedef struct relax_weakzone {
    double dgammadot0, x, y, z, width, length, thickness, strike, dip;
    relax_tensor e;
} relax_weakzone;

/* An observation plane (the geometry of PLANE_STRUCT, src/types.f90:92-97)
 * in the internal convention: centre after wangconvention and the rotation,
 * strike and dip in radians (src/input.f90:321-356). */
typedef struct relax_obsplane {
    double x, y, z, length, width, strike, dip;
} relax_obsplane;

/* SEGMENT_STRUCT, src/types.f90:58-62 without sig0 (the stress at the
 * coseismic step, kept by the caller): a stress observation segment in the
 * internal convention (src/input.f90:399-451). */
typedef struct relax_segment {
    double x, y, z, length, width, strike, dip, friction;
} relax_segment;

/* TETRAHEDRON_STRUCT, src/types.f90:70-74: an eigenstrain e in the
 * tetrahedron of four vertices of the event's vertex list (1-based). */
typedef struct relax_tetrahedron {
    relax_tensor e;
    int i1, i2, i3, i4;
} relax_tetrahedron;

/* EVENT_STRUC, src/types.f90:99-106: shear, tensile, point and load
 * sources, and (input flag --with-eigenstrain, src/input.f90:1496-1660)
 * cuboid eigenstrain sources (WEAK_STRUCT: e and the geometry after
 * wangconvention; dgammadot0 unused) and, with --with-curvilinear,
 * tetrahedral ones over a vertex list (3 doubles per vertex). */
typedef struct relax_event {
    double time;
    int ns, nt, nm, nl;
    const relax_source *s;    /* shear dislocations                    */
    const relax_source *ts;   /* tensile cracks                        */
    const relax_source *m;    /* dilatation point sources              */
    const relax_source *l;    /* surface loads                         */
    int nc, ntet, nvert;      /* cuboids, tetrahedra, vertices         */
    const relax_weakzone *c;  /* cuboid eigenstrain sources            */
    const relax_tetrahedron *tet;
    const double *vert;       /* x1, x2, x3 of each vertex             */
} relax_event;

/* The part of SIMULATION_STRUCT (src/types.f90:118-266) that the time
 * loop reads.  Depth structures are per physical layer (sx3/2 entries),
 * i.e. already expanded by relax_viscoelastic_structure /
 * relax_tensor_structure.  A NULL structure means "mechanism absent"
 * (Fortran .NOT.ALLOCATED). */
typedef struct relax_config {
    int sx1, sx2, sx3;                  /* FFT box                     */
    double dx1, dx2, dx3, beta, nyquist;
    double lambda, mu, gam;             /* Lame parameters, gravity    */
    double interval, odt, tscale;       /* time-step policy            */
    int skip;                           /* >0: adaptive, skip mode     */
    const relax_tensor_layer *stressstruc;  /* prestress, NULL = zero  */
    const relax_layer *linearstruc;
    const relax_layer *nonlinearstruc;
    const relax_layer *faultcreepstruc;
    const float *lineardgammadot0;      /* optional weak-zone fields,  */
    const float *nonlineardgammadot0;   /* sx1*sx2*(sx3/2), or NULL    */
    int np;                             /* afterslip planes            */
    const relax_plane *planes;
    int ne;                             /* coseismic events            */
    const relax_event *events;
    relax_event inter;                  /* interseismic loading rates  */
    /* transient (Burgers) rheology, src/viscoelastic3d.f90:123-202 (the
     * reference's --with-transient): linear and nonlinear per-layer
     * structures (gammadot0, stressexponent, Gk; nz = sx3/2 entries) and
     * optional weak-zone fields, or NULL */
    const relax_layer *ltransientstruc;
    const relax_layer *nltransientstruc;
    const float *ltransientdgammadot0;
    const float *nltransientdgammadot0;
    /* origin and rotation of the input file (src/input.f90:238-241).  The
     * sources of event 0 smaller than nyquist*min(dx) get the space-domain
     * solution of Okada (1992) added to the coseismic displacement
     * (dislocations_disp, src/relax.f90:355-360, :1298-1349), which the
     * reference evaluates with the sources' input-file coordinates. */
    double x0, y0, rot;
} relax_config;

/* One line of RELAX's step log (src/relax.f90:1027-1047, format 1100):
 * I, Dt, tm(ve), tm(pl), tm(as), t, power, C:E^i; with the transient
 * rheology (formats 1102/1103) also the Maxwell times of the linear and
 * nonlinear transient mechanisms.  `output` is isoutput of the step
 * (src/relax.f90:907): the reference then prints format 1101/1103 ("*")
 * and writes its output files. */
typedef struct relax_step_log {
    int i;
    int event;         /* 1 when a coseismic event fired after the step */
    double dt, tm_ve, tm_pl, tm_as, t, power, cei;
    double tm_tl, tm_tnl;
    int output;
} relax_step_log;

/* field selectors for relax_get_field / relax_set_field / relax_get_plane */
#define RELAX_FIELD_U       1   /* 3 x float (sx1+2, sx2, sx3/2)         */
#define RELAX_FIELD_SIG     2   /* relax_tensor (sx1, sx2, sx3/2)        */
#define RELAX_FIELD_TAU     3   /* relax_tensor (sx1, sx2, sx3/2)        */
#define RELAX_FIELD_MOMENT  4   /* relax_tensor (sx1, sx2, sx3/2)        */
#define RELAX_FIELD_GAMMA   5   /* float (sx1+2, sx2, sx3/2)             */
#define RELAX_FIELD_EPS     6   /* relax_tensor (sx1, sx2, sx3/2): the
                                   transient strain epsilonik            */
#define RELAX_FIELD_V       7   /* planes only: the corrector's velocity  */
#define RELAX_FIELD_UR      8   /* planes only: postseismic displacement  */

/* ------------------------------------------------------------------ */
/* host helpers (no device work)                                      */
/* ------------------------------------------------------------------ */

/* viscoelasticstructure, src/elastic3d.f90:732-829: expand interface
 * list -> per-layer structure (nz = sx3/2 entries). */
int relax_viscoelastic_structure(const relax_layer *layers, int nlayers,
                                 double dx3, int nz, relax_layer *out);

/* tensorstructure, src/elastic3d.f90:630-702 */
int relax_tensor_structure(const relax_tensor_layer *layers, int nlayers,
                           double dx3, int nz, relax_tensor_layer *out);

/* wangconvention, src/input.f90:1780-1800 (+ rotation :1802-1815) */
void relax_wang_convention(double *slip, double *x, double *y, double *z,
                           double length, double width, double *strike,
                           double *dip, double *rake, double x0, double y0,
                           double rot);

/* ------------------------------------------------------------------ */
/* context API                                                        */
/* ------------------------------------------------------------------ */
typedef struct relax_ctx relax_ctx;

const char *relax_version(void);
const char *relax_last_error(void);     /* thread-local message        */

/* Allocates all device state for one RELAX instance on `device`.  The
 * configuration is deep-copied.  Replaces cuinflags_/cuinit_
 * (src/cuelastic.cu:736, :476).  Grids: sx1 >= 8 and a multiple of 4,
 * sx2 >= 2, even sx3 with sx3/2 >= 5, FFT lengths sx1/2, sx2, sx3
 * products of 2 and 3 (RELAX_ERR_UNSUPPORTED otherwise); the x1 and x2
 * derivatives take the 7-point FIR filter of src/kernel7.inc for
 * 5 <= sx <= 14 as optimalfilter (src/elastic3d.f90:846-907) does. */
int relax_create(const relax_config *cfg, int device, relax_ctx **out);
/* Replaces cudeinit_ (src/cuelastic.cu:1344).  The context's device
 * memory goes back to the library's own memory pool on that device, which
 * keeps it for the next context (creating a context then allocates nothing
 * from the device); relax_release_cached_memory returns it to the device. */
int relax_destroy(relax_ctx *ctx);
/* Returns the device memory that the library's pool on `device` holds but
 * no live context, batch or operator uses (cudaMemPoolTrimTo after a device
 * synchronisation).  Call it after destroying contexts when other code of
 * the process needs the memory.  No counterpart in the reference, whose
 * cudeinit_ frees with cudaFree. */
int relax_release_cached_memory(int device);

/* Precision of the time step's Green's functions.  RELAX_PRECISION_FP32
 * (the default) runs every FFT butterfly in FP32 as the reference does
 * (fft3, src/fourier.f90:177-201).  RELAX_PRECISION_MIXED runs the x3
 * transform's length-64 DFT sub-transforms as tensor-core products
 * (tcgen05, split BF16 hi/lo operands, FP32 accumulation; elastic response,
 * surface traction and Cerruti correction unchanged); boxes 128 deep only
 * (RELAX_ERR_UNSUPPORTED otherwise).  A mode of this library with no
 * counterpart in the reference. */
#define RELAX_PRECISION_FP32  0
#define RELAX_PRECISION_MIXED 1
int relax_set_precision(relax_ctx *ctx, int mode);

/* Stream the context's work is ordered on (cudaStream_t as void*). */
int relax_get_stream(relax_ctx *ctx, void **stream);

/* Coseismic solve of event `e` (0-based) at the current time:
 * dislocations -> greenfunctioncowling -> u (+)= v, tau update, then
 * sig = -tau + C:E(u)  (src/relax.f90:318-371 for e=0, :858-890 later). */
int relax_coseismic(relax_ctx *ctx, int e, relax_step_log *log0);

/* One RK2 predictor/corrector step (src/relax.f90:555-890).  If
 * dt_override is non-NULL its value replaces the adaptive Dt of
 * integrationstep (dt-schedule replay).  Returns RELAX_OK with
 * log->i == 0 when t >= interval (nothing done). */
int relax_step(relax_ctx *ctx, const double *dt_override, relax_step_log *log);

/* Runs the coseismic solve of event 0 and up to max_steps steps, stopping
 * at t >= interval; events are fired as the reference does.  logs has
 * room for max_steps+1 entries (entry 0 = coseismic line). */
int relax_run(relax_ctx *ctx, int max_steps, const double *dt_schedule,
              relax_step_log *logs, int *nsteps_done);

/* Host <-> device field copies in the reference layout (see
 * RELAX_FIELD_*); `bytes` must equal the field size. */
int relax_get_field(relax_ctx *ctx, int which, void *host, size_t bytes);
int relax_set_field(relax_ctx *ctx, int which, const void *host, size_t bytes);
/* Number of afterslip planes, and the patch grid (px2 x px3) of plane k. */
int relax_num_planes(relax_ctx *ctx, int *np);
int relax_get_plane_shape(relax_ctx *ctx, int k, int *px2, int *px3);
/* Afterslip patch state of plane k (px2*px3 entries, j2 fastest). */
int relax_get_patches(relax_ctx *ctx, int k, relax_slippatch *host, size_t n);
/* Current time, step counter, event index. */
int relax_get_time(relax_ctx *ctx, double *t, int *i, int *e);
/* Grid sizes (sx1, sx2, sx3) and sampling (dx1, dx2, dx3); either may be NULL. */
int relax_get_grid(relax_ctx *ctx, int *sx, double *dx);
/* One x3-plane i3 (0-based, < sx3/2) of a field: its components one after
 * the other (3 for U, 1 for GAMMA, 6 for the tensor fields in the order
 * s11 s12 s13 s22 s23 s33), each sx1 x sx2 floats, x1 fastest, unpadded.
 * The read-back of cuexportspatial_ (src/cuelastic.cu:1629). */
int relax_get_plane(relax_ctx *ctx, int which, int i3, float *host, size_t bytes);
/* Keeps, from the next step on, the corrector's velocity field v
 * (src/relax.f90:829) for planes i3 < vel_planes and the postseismic
 * displacement sum Dt v (src/relax.f90:839-850) for planes i3 < ur_planes
 * and for plane inter_i3 (-1: none), readable with relax_get_plane as
 * RELAX_FIELD_V / RELAX_FIELD_UR.  Costs 12 bytes per kept point and step.
 * Calling it again restarts the sums.  Not for batch members. */
int relax_track_relaxation(relax_ctx *ctx, int vel_planes, int ur_planes,
                           int inter_i3);
/* Displacement and stress at n grid points given as 0-based (i1, i2, i3)
 * triples: cuexportpoints_ (src/cuelastic.cu:1652) for many points. */
int relax_get_points(relax_ctx *ctx, int n, const int *index, double *u,
                     relax_tensor *sig);
/* monitorstressfield / monitorfield (src/elastic3d.f90:3404-3762): the
 * stress (RELAX_FIELD_SIG, into patch.sig) or the scalar RELAX_FIELD_GAMMA
 * (into patch.slip) sampled with the sinc-weighted 5x5x5 window on the
 * (px2+1) x (px3+1) points of plane `op` (tapered by beta), px2 + 1 fastest;
 * x1..x3 the point, lx / lz its along-strike / down-dip coordinates; points
 * outside the box read zero.  *px2, *px3 are set; `out` may be NULL to size
 * the grid, else it holds n >= (px2+1)(px3+1) patches. */
int relax_monitor_plane(relax_ctx *ctx, int which, const relax_obsplane *op,
                        double beta, relax_slippatch *out, size_t n,
                        int *px2, int *px3);
/* The stress at the centres of n stress observation segments (the nearest
 * grid node, shiftedindex with the full sx3 as in src/export.f90:1364-1394);
 * a centre below the stored half of the grid is an error. */
int relax_segment_stress(relax_ctx *ctx, int n, const relax_segment *sop,
                         relax_tensor *sig);

/* ------------------------------------------------------------------ */
/* the input file (subroutine init, src/input.f90:43-1767)            */
/*                                                                    */
/* The text of a RELAX input file, in init's order and with its        */
/* conventions (comment lines start with '#', Fortran list-directed   */
/* records, wangconvention for faults, planes and weak zones, rotation */
/* of points, dilatation sources and loads), is read into a           */
/* relax_config ready for relax_create.  Errors (index misfits,       */
/* negative rates, missing values) return RELAX_ERR_ARG with the line */
/* number in relax_last_error.  Cuboid eigenstrain sources (flag      */
/* RELAX_INPUT_EIGENSTRAIN) and tetrahedral ones (with                */
/* RELAX_INPUT_CURVILINEAR) are read into the events' nc/c and        */
/* ntet/tet/nvert/vert.                                               */
/* ------------------------------------------------------------------ */
typedef struct relax_input relax_input;

#define RELAX_INPUT_TRANSIENT    1   /* --with-transient: transient sections  */
#define RELAX_INPUT_EIGENSTRAIN  2   /* --with-eigenstrain: cuboid sections   */
#define RELAX_INPUT_CURVILINEAR  4   /* --with-curvilinear: tetrahedra        */
#define RELAX_INPUT_ECHO         8   /* print the values back as init does    */

typedef struct relax_input_info {
    const char *wdir;                /* output directory                      */
    double x0, y0, rot, oz, ozs;     /* origin, rotation, observation depths  */
    int npts;                        /* observation points: 3 * npts coords   */
    const double *pts;               /* in the computational frame            */
    const char *const *ptsname;      /* 4-character names                     */
    int nop, nsop;                   /* observation planes, stress segments   */
    int nwz[4];                      /* weak zones: linear, nonlinear, linear
                                        and nonlinear transient              */
    double minlength, minwidth;      /* smallest source dimensions            */
} relax_input_info;

int relax_input_parse(const char *text, int flags, relax_input **out);
/* path NULL: standard input */
int relax_input_read(const char *path, int flags, relax_input **out);
void relax_input_free(relax_input *in);
/* owned by the input; valid until relax_input_free */
const relax_config *relax_input_config(const relax_input *in);
int relax_input_get_info(const relax_input *in, relax_input_info *info);
/* weak zones of mechanism 0..3 in the internal convention */
/* observation planes and stress observation segments of the input */
int relax_input_obsplanes(const relax_input *in, const relax_obsplane **op,
                          int *n);
int relax_input_segments(const relax_input *in, const relax_segment **sop,
                         int *n);
int relax_input_weakzones(const relax_input *in, int mechanism,
                          const relax_weakzone **zones, int *n);
/* builddgammadot0 (src/viscoelastic3d.f90:320-435) of every mechanism with
 * weak zones, evaluated on `device`; sets the *dgammadot0 fields of the
 * configuration. */
int relax_input_build_weakzones(relax_input *in, int device);

/* ------------------------------------------------------------------ */
/* output files (host code, fed from the device fields)               */
/* ------------------------------------------------------------------ */

/* writegrd / writeNetcdf, src/exportnetcdf.f90:17-127: a GMT grid in the
 * netCDF classic format, pixel registration; z: nx x ny floats, x fastest;
 * x_i = x0 + i dx, y_j = y0 + j dy. */
int relax_write_grd(const float *z, int nx, int ny, double x0, double y0,
                    double dx, double dy, const char *title,
                    const char *filename);
/* exportgrd, src/export.f90:917-1057: three unpadded (sx1, sx2) planes ->
 * wdir/NNN-<suffix>.grd with the suffixes of `convention` (1 north/east/up,
 * 2 relax-*, 3 eqbf-*, 4 s11/s12/s13, 5 s22/s23/s33, 6 e11/e12/e13,
 * 7 e22/e23/e33); the third component is negated for 1..3 (positive up). */
int relax_write_grd3(const float *c1, const float *c2, const float *c3,
                     int sx1, int sx2, double dx1, double dx2, double origx,
                     double origy, const char *wdir, int index,
                     int convention);
/* The grids of a context's field: RELAX_FIELD_U at plane int(oz/dx3)
 * (exportgrd, convention 1), RELAX_FIELD_UR there as NNN-relax-*.grd
 * (convention 2), RELAX_FIELD_SIG / RELAX_FIELD_EPS at plane fix(oz/dx3)
 * (exportstressgrd, src/export.f90:860-908: 4/5, 6/7). */
int relax_export_grd(relax_ctx *ctx, int which, double oz, double origx,
                     double origy, const char *wdir, int index);
/* exportvtk_vectors_legacy / exportvtk_tensors_legacy (src/writevtk.c:72,
 * :151): VTK legacy binary structured points, big-endian floats.  comp:
 * 3 vector or 6 tensor component arrays of sx1 x sx2 x sx3 floats. */
int relax_write_vtk(const float *const *comp, int ncomp, int sx1, int sx2,
                    int sx3, double dx1, double dx2, double dx3, int j1,
                    int j2, int j3, const char *filename, const char *title,
                    const char *name);
/* The same for a context's U or tensor field over its first sx3 planes. */
int relax_export_vtk(relax_ctx *ctx, int which, int sx3, int j1, int j2,
                     int j3, const char *filename, const char *title,
                     const char *name);
/* exportcreep_asc / exportcreep_grd / exportcreep_vtk (src/export.f90:
 * 563-849): the patches of every afterslip plane as wdir/NNN.sKKKKK.creep.dat
 * (every third patch, RELAX_CREEP_TXT), as GMT grids of slip and slip rate
 * (RELAX_CREEP_GRD) and as VTK polydata wdir/creep-KKKKKs-NNN.vtk
 * (RELAX_CREEP_VTK). */
#define RELAX_CREEP_TXT 1
#define RELAX_CREEP_GRD 2
#define RELAX_CREEP_VTK 4
int relax_export_creep(relax_ctx *ctx, const char *wdir, int index,
                       int formats);
/* exportplanestress (src/export.f90:308-397): the stress on observation
 * plane k sampled by relax_monitor_plane, as the grids
 * wdir/NNN.opKKK-s11.grd ... -s33.grd; exporteigenstrain (:423-512) with
 * which = RELAX_FIELD_GAMMA: wdir/NNN.sKKKKK.estrain.grd.  x0, y0: origin
 * added to the sample points. */
int relax_export_plane_stress(relax_ctx *ctx, int which, int nop,
                              const relax_obsplane *op, double x0, double y0,
                              const char *wdir, int index);
/* The stress observation segments (src/export.f90:1403-2005), from the
 * stress at their centres (sig; NULL: zero) less sig0 when sig0 is given
 * (convention 1 of the reference):
 *   RELAX_SEG_GMT      exportgmt_rfaults_stress, one "> -Z" polygon each;
 *   RELAX_SEG_TRACTION exportgmt_rfaults_traction, position, shear traction
 *                      and normal vector;
 *   RELAX_SEG_VTP      exportvtk_rfaults_stress, VTK PolyData XML.
 * `filename` is the file written. */
#define RELAX_SEG_GMT 1
#define RELAX_SEG_TRACTION 2
#define RELAX_SEG_VTP 3
int relax_write_segments(int kind, int n, const relax_segment *sop,
                         const relax_tensor *sig, const relax_tensor *sig0,
                         const char *filename);
/* The geometry files of the input reader (VTK PolyData XML and GMT .xy):
 * exportvtk_grid (src/export.f90:1068-1127), the box of the grid;
 * exportvtk_rectangle (:2014-2093), a rectangle of centre x, length L along
 * strike, width W down dip (radians); exportxy_brick (:2101-2153) and
 * exportvtk_allbricks (:2295-2599), weak zones; exportvtk_rfaults
 * (RELAX_FAULTS_VTP, :1216-1354) and exportxy_rfaults (RELAX_FAULTS_XY,
 * :1139-1206, origin x0, y0 added), the sources of an event. */
#define RELAX_FAULTS_VTP 1
#define RELAX_FAULTS_XY 2
int relax_write_vtk_grid(int sx1, int sx2, int sx3, double dx1, double dx2,
                         double dx3, const char *filename);
int relax_write_vtk_rectangle(double x1, double x2, double x3, double L,
                              double W, double strike, double dip,
                              const char *filename);
int relax_write_xy_brick(const relax_weakzone *zone, const char *filename);
int relax_write_vtk_bricks(int n, const relax_weakzone *zones,
                           const char *filename);
int relax_write_faults(int kind, int n, const relax_source *src, double x0,
                       double y0, const char *filename);
/* All the geometry files that the input reader (init, src/input.f90:
 * 296-1452) writes into the input's output directory: with vtk the .vtp
 * files (grid, viscous and transient interfaces, weak zones, afterslip
 * planes, each event's faults), always the GMT .xy files (weak zones, each
 * event's faults). */
int relax_input_export_geometry(const relax_input *in, int vtk);
/* exportcoulombstress (src/export.f90:1893-2005): one line of time, stress
 * and shear, normal and Coulomb stress per segment appended to
 * wdir/cfaults-sigma-KKKK.txt (a new file with its header when isnew). */
int relax_write_coulomb(int n, const relax_segment *sop,
                        const relax_tensor *sig, double time,
                        const char *wdir, int isnew);
/* shiftedindex, src/elastic3d.f90:4063-4101, 0-based indices; sx3 is the
 * number of x3-planes held (sx3/2 of the grid). */
int relax_shifted_index(double x1, double x2, double x3, int sx1, int sx2,
                        int sx3, double dx1, double dx2, double dx3,
                        int *i1, int *i2, int *i3);
/* exportpoints, src/util.f90:59-170: x holds n (x1, x2, x3) observation
 * points in the computational frame; appends one line to each
 * wdir/<name>.ned (creates it with its header when isnew) and, when
 * rot != 0, to wdir/<name>.c.txt. */
int relax_export_points(relax_ctx *ctx, int n, const double *x,
                        const char *const *names, double time, double rot,
                        const char *wdir, int isnew);
/* The step log line, formats 1100-1103 (src/relax.f90:1102-1105), and the
 * column headers 0990/0991. */
int relax_format_log(const relax_step_log *log, double interval,
                     int transient, char *buf, size_t size);
const char *relax_log_header(int transient);
/* One .ned row (14ES16.8E2) and the .ned header line. */
int relax_format_ned(double time, const double *u, const relax_tensor *sig,
                     char *buf, size_t size);
const char *relax_ned_header(void);
/* Fortran ESw.dEe of one value; e = 0 gives ESw.d. */
int relax_es_format(double v, int w, int d, int e, char *buf, size_t size);

/* Checkpoint (no counterpart in the reference, which cannot restart a
 * run): relax_checkpoint_save writes the state a step reads -- u, tau,
 * moment, sig, gamma, the transient strain, the afterslip patches, the
 * tracked relaxation fields, time, counters and the step state -- to a raw
 * file with a checksum; relax_checkpoint_load restores it into a context
 * created from the same configuration (and the same
 * relax_track_relaxation), which then continues bit for bit. */
int relax_checkpoint_save(relax_ctx *ctx, const char *path);
int relax_checkpoint_load(relax_ctx *ctx, const char *path);

/* Waits for the context's stream. */
int relax_synchronize(relax_ctx *ctx);

/* Per-stage device timing: while enabled, every kernel the context launches
 * is bracketed by CUDA events on its stream; relax_profile_read sums the
 * durations of one stage (name: the kernel).  Enabling clears the record.
 * relax_launch_count counts this context's kernel launches (always on). */
int relax_profile(relax_ctx *ctx, int enable);
int relax_profile_stages(void);
int relax_profile_read(relax_ctx *ctx, int stage, double *total_ms,
                       int *launches, const char **name);
int relax_launch_count(relax_ctx *ctx, long long *n);

/* ------------------------------------------------------------------ */
/* batches (ensembles)                                                */
/*                                                                    */
/* No reference counterpart: RELAX runs one simulation per process.   */
/* A batch holds members that share the grid (sx, dx), the elastic    */
/* constants (lambda, mu, gam) and the number of afterslip planes;    */
/* they differ in events, rheology, prestress, weak zones and plane   */
/* geometry.  relax_batch_step advances every member by one RK2 step  */
/* (each with its own adaptive Dt) with one launch per stage for all  */
/* members and one host synchronisation; members whose time reached   */
/* the interval stay put and report i = 0.  Grids without the         */
/* register-resident passes (lengths other than 64/128/256 along x1    */
/* and x3, 64..512 along x2) step the members in turn.  Otherwise the  */
/* batch tunes itself on its first six steps: three batched (the third */
/* timed), three with the members in turn (the sixth timed), and the   */
/* faster form from then on (relax_batch_tuning); both forms give the  */
/* same results.  Events with surface loads are rejected              */
/* (RELAX_ERR_UNSUPPORTED).  Each member is a relax_ctx owned by the   */
/* batch (relax_batch_member) for field and patch access; do not      */
/* destroy or step it directly.                                       */
/* ------------------------------------------------------------------ */
typedef struct relax_batch relax_batch;

int relax_batch_create(const relax_config *members, int n, int device, relax_batch **batch);
int relax_batch_destroy(relax_batch *batch);
int relax_batch_size(relax_batch *batch, int *n);
int relax_batch_member(relax_batch *batch, int k, relax_ctx **member);
/* coseismic solve of event 0 of every member; logs: n entries or NULL */
int relax_batch_coseismic(relax_batch *batch, relax_step_log *logs);
/* logs: n entries */
int relax_batch_step(relax_batch *batch, relax_step_log *logs);
int relax_batch_launch_count(relax_batch *batch, long long *n);
int relax_batch_get_stream(relax_batch *batch, void **stream);
/* The tuner's state: mode 0 while measuring, 1 batched launches, 2 the
 * members in turn; the measured step times in ms (-1 until measured). */
int relax_batch_tuning(relax_batch *batch, int *mode, double *batched_ms,
                       double *in_turn_ms);

/* An ensemble of members with uneven grids (no reference counterpart).
 * The members are grouped by shape (grid, spacing, elastic constants,
 * number of afterslip planes) into batches, each with its own stream and
 * its own tuning; relax_ensemble_step queues every group's step, each
 * behind the previous group's (run concurrently, the groups competed for
 * L2 and took longer), and then waits once per group.  Members keep their
 * order: logs[k] and relax_ensemble_member(k) are member k of `members`.
 * Members stepped in an ensemble equal the same decks stepped alone, bit
 * for bit. */
typedef struct relax_ensemble relax_ensemble;

int relax_ensemble_create(const relax_config *members, int n, int device, relax_ensemble **ensemble);
int relax_ensemble_destroy(relax_ensemble *ensemble);
/* n: members, ngroups: shape groups (either may be NULL) */
int relax_ensemble_size(relax_ensemble *ensemble, int *n, int *ngroups);
int relax_ensemble_member(relax_ensemble *ensemble, int k, relax_ctx **member);
int relax_ensemble_coseismic(relax_ensemble *ensemble, relax_step_log *logs);
int relax_ensemble_step(relax_ensemble *ensemble, relax_step_log *logs);
int relax_ensemble_launch_count(relax_ensemble *ensemble, long long *n);
/* Group `group`'s grid (sx: 3 ints), member count and tuner state as
 * relax_batch_tuning reports it (any output may be NULL). */
int relax_ensemble_tuning(relax_ensemble *ensemble, int group, int *sx,
                          int *nmembers, int *mode, double *batched_ms,
                          double *in_turn_ms);

/* ------------------------------------------------------------------ */
/* stateless operators on device buffers (reference layout)           */
/*                                                                    */
/* Each takes device pointers in RELAX's layout and a CUDA stream      */
/* (NULL = legacy default stream); the work is enqueued, not waited   */
/* for.  They are the unit under the per-kernel parity tests.         */
/* ------------------------------------------------------------------ */

/* stressupdate, src/elastic3d.f90:956-1180: sig += C:E(u).
 * u1..u3: (sx1+2, sx2, sx3h) float; sig: (sx1, sx2, sx3h) relax_tensor. */
int relax_op_stressupdate(const float *u1, const float *u2, const float *u3,
                          double lambda, double mu, double dx1, double dx2,
                          double dx3, int sx1, int sx2, int sx3h,
                          relax_tensor *sig, void *stream);

/* equivalentbodyforce, src/elastic3d.f90:1214-1506:
 * c_i -= div(sig)_i on the first sx3h layers, t_i += sig_i3(x3=0).
 * c1..c3: (sx1+2, sx2, >=sx3h) float; t1..t3: (sx1+2, sx2) float. */
int relax_op_bodyforce(const relax_tensor *sig, double dx1, double dx2,
                       double dx3, int sx1, int sx2, int sx3h,
                       float *c1, float *c2, float *c3,
                       float *t1, float *t2, float *t3, void *stream);

/* viscouseigenstress, src/viscoelastic3d.f90:217-314.
 * structure/prestress: sx3h entries on the HOST (uploaded internally).
 * moment += ...; *maxwelltime = min(*maxwelltime, min 1/gammadot) when
 * maxwelltime != NULL; gamma (sx1+2, sx2, sx3h), written where active,
 * when non-NULL; dgammadot0 optional (sx1, sx2, sx3h).  Synchronous when
 * maxwelltime is requested. */
int relax_op_viscouseigenstress(double mu, const relax_layer *structure,
                                const relax_tensor_layer *prestress,
                                const relax_tensor *sig, int sx1, int sx2,
                                int sx3h, relax_tensor *moment,
                                double *maxwelltime, float *gamma,
                                const float *dgammadot0, void *stream);

/* transienteigenstress, src/viscoelastic3d.f90:123-202: moment +=
 * 2 gammadot Q and epsilonikdot = gammadot/mu Q with Q = s' - 2 Gk
 * epsilonik, per layer of `structure` (gammadot0, stressexponent, Gk; sx3h
 * entries); epsilonik and epsilonikdot may be the same buffer (the
 * reference's corrector call).  dgammadot0 optional (sx1, sx2, sx3h).
 * *maxwelltime = min(*maxwelltime, min 1/gammadot) when non-NULL
 * (synchronous then). */
int relax_op_transienteigenstress(double mu, const relax_layer *structure, const relax_tensor *sig,
                                  const relax_tensor *epsilonik, int sx1, int sx2, int sx3h,
                                  relax_tensor *moment, relax_tensor *epsilonikdot,
                                  double *maxwelltime, const float *dgammadot0, void *stream);

/* grnfct_okada, src/okada/green_space.f90:114-144: u += the displacement
 * of n rectangular dislocations in the half-space (Okada, 1992) at the
 * physical points, u1..u3 (sx1+2, sx2, sx3h) float on the device.  The
 * sources are in the input-file convention: top-edge reference point
 * (x = north, y = east, z = depth), strike, dip and rake in degrees, slip
 * and opening (tensile cracks). */
int relax_op_okada(const relax_source *sources, int n, double lambda, double mu,
                   int sx1, int sx2, int sx3h, double dx1, double dx2,
                   double dx3, float *u1, float *u2, float *u3, void *stream);
/* The same at one receiver (north, east, depth >= 0), on the host. */
int relax_okada_point(const relax_source *source, double lambda, double mu,
                      double x1, double x2, double x3, double *disp);

/* builddgammadot0, src/viscoelastic3d.f90:320-435: the fluidity
 * perturbation of `nz` weak zones (host array) at the physical points,
 * out (sx1, sx2, sx3h) on the device.  RELAX builds with beta = 0
 * (src/relax.f90:487-541). */
int relax_op_dgammadot0(const relax_weakzone *zones, int nz, int sx1, int sx2, int sx3h,
                        double dx1, double dx2, double dx3, double beta, float *out, void *stream);

/* frictioneigenstress, src/friction3d.f90:82-241 for one afterslip plane
 * (x..rake in the internal convention; L = plane width, W = plane length
 * as the reference call sites pass them).  Synchronous when maxwelltime
 * is requested. */
int relax_op_frictioneigenstress(double x, double y, double z, double L,
                                 double W, double strike, double dip,
                                 double rake, double beta,
                                 const relax_tensor *sig, double mu,
                                 const relax_layer *structure, int sx1,
                                 int sx2, int sx3h, double dx1, double dx2,
                                 double dx3, relax_tensor *moment,
                                 double *maxwelltime, void *stream);

/* greenfunctioncowling, src/green.f90:1008-1129: c1..c3 (sx1+2, sx2, sx3)
 * body forces in, displacements out (all sx3 layers); t1..t3 (sx1+2, sx2)
 * surface tractions are consumed (their content is undefined after the
 * call).  Replaces calfftnelasic_ (src/cugreen.cu:1453). */
int relax_op_green(float *c1, float *c2, float *c3, float *t1, float *t2,
                   float *t3, int sx1, int sx2, int sx3, double dx1,
                   double dx2, double dx3, double lambda, double mu,
                   double gam, void *stream);

/* greenfunctioncowling in the mixed-precision form of
 * RELAX_PRECISION_MIXED, on a 128-deep box (sx3 = 128), pruned as in the
 * time step (src/relax.f90:681): the body force's lower half (layers
 * sx3/2 .. sx3-1) must be zero, and only the upper sx3/2 layers of
 * c1..c3 receive the displacement (the lower half is left as it was).
 * Replaces calfftnelasic_ (src/cugreen.cu:1453) in that setting. */
int relax_op_green_mixed(float *c1, float *c2, float *c3, float *t1,
                         float *t2, float *t3, int sx1, int sx2, int sx3,
                         double dx1, double dx2, double dx3, double lambda,
                         double mu, double gam, void *stream);

/* The tensor-core DFT of relax_op_green_mixed on its own: `in` holds 128
 * vectors of 64 complex values (interleaved FP32 pairs, 128 x 64 x 2
 * floats), `out` receives their forward (inverse = 0, sign -1) or inverse
 * (inverse = 1, sign +1, unnormalised) DFT, each 64 x 2 floats.  For tests
 * of the split-precision product; synchronous.  No counterpart in the
 * reference (its FFT is FFTW / cuFFT). */
int relax_op_dft64_tc(const float *in, float *out, int inverse, void *stream);

/* greenfunctioncowling like relax_op_green, for callers that cannot
 * allocate device memory (a host whose pool allocator owns the device, or
 * code where cudaMalloc/cudaFree are not allowed): no allocation at all.
 * It has no counterpart in the reference.  Its scratch is one fixed 16 MiB
 * device array per device (held while the library is loaded), so grids
 * whose spectrum and twiddle tables exceed 16 MiB (3*(sx3+1)*sx2*(sx1/2+1)*8
 * + (sx1/2 + sx1 + sx2 + sx3)*8 bytes, e.g. above 128 x 128 x 64) return
 * RELAX_ERR_ARG.  The first call on each device looks the array up
 * (cudaGetSymbolAddress) and sets kernel attributes: make that first call
 * before any stream capture.  All calls share the array; calls that overlap
 * on the GPU race on it, so order them on one stream.  Grid rules: sx1 >= 8
 * and a multiple of 4, even sx3 >= 4, sx2 >= 2, FFT lengths sx1/2, sx2, sx3
 * products of 2 and 3.  relax_op_green asks in addition what a context
 * needs (sx3/2 >= 5, where the step's differentiators stop), so this entry
 * point also takes shallower grids. */
int relax_op_green_noalloc(float *c1, float *c2, float *c3, float *t1,
                           float *t2, float *t3, int sx1, int sx2, int sx3,
                           double dx1, double dx2, double dx3, double lambda,
                           double mu, double gam, void *stream);

/* 3-D real<->complex FFT in place on a (sx1+2, sx2, sx3) array with
 * RELAX's normalisation (src/fourier.f90:177-201): direction -1 forward
 * (x dx1 dx2 dx3), +1 inverse (/ (sx1 dx1 sx2 dx2 sx3 dx3)). */
int relax_op_fft3(float *data, int sx1, int sx2, int sx3, double dx1,
                  double dx2, double dx3, int direction, void *stream);

/* tensoramplitude, src/elastic3d.f90:446-466 (synchronous). */
int relax_op_tensoramplitude(const relax_tensor *t, int sx1, int sx2,
                             int sx3h, double dx1, double dx2, double dx3,
                             double *amp, void *stream);

/* ------------------------------------------------------------------ */
/* compatibility shim: the reference CUDA layer, symbol for symbol     */
/* (src/cuelastic.cu, src/cugreen.cu).  One implicit default context,  */
/* single thread, synchronous, as the reference.                      */
/* ------------------------------------------------------------------ */
typedef relax_tensor ST_TENSOR_C;

/* src/cuelastic.cu:736 */
void cuinflags_(int *istransient, int *nlwz, int *nnlwz, int *nltwz,
                int *nnltwz, int islinear, int isnonlinear,
                int isltransient, int isnltransient, int *iRet);
/* src/cuelastic.cu:476 */
void cuinit_(int sx1, int sx2, int sx3, double dx1, double dx2, double dx3,
             int *iRet);
/* src/cuelastic.cu:1344 */
void cudeinit_(void);
/* src/cuelastic.cu:1493 -- v = 0, t = 0 */
void curesetvectors_(void);
/* src/cuelastic.cu:1596 -- E_TENSOR_TYPE 1: sig, 2: moment, 3: tau <- 0 */
void cutensormemset_(int eType);
/* src/cuelastic.cu:1572 -- dir 0: device->host, 1: host->device */
void copytau_(ST_TENSOR_C *host, int sx1, int sx2, int sx3h, int dir);
/* src/cuelastic.cu:1330 -- t3 device -> host */
void cucopytraction_(float *t3, int sx1, int sx2, int *iRet);
/* src/cuelastic.cu:1483 -- u = v (first sx3h layers) */
void cufieldrep_(int sx1p2, int sx2, int sx3h);
/* src/cuelastic.cu:1412 -- 1: u = c1 u + c2 v, 2: v = c1 v + c2 u */
void cufieldadd_(int eType, float *a, float *b, float *c, float *d,
                 float *e, float *f, int sx1p2, int sx2, int sx3h,
                 float c1, float c2);
/* src/cuelastic.cu:1216 -- enum E_TENSOR_FIELD (src/cuinclude.h:100-111) */
void cutensorfieldadd_(int eField, int sx1, int sx2, int sx3h, float c1,
                       float c2);
/* src/cuelastic.cu:786 -- 1: sig += C:E(u), 2: sig += C:E(v) */
void custressupdatewrapper_(int eType, double lambda, double mu, double dx1,
                            double dx2, double dx3, int sx1, int sx2,
                            int sx3h, float *u1, float *u2, float *u3,
                            ST_TENSOR_C *sig);
/* src/cuelastic.cu:838 -- 1: div(sig), 2: div(moment) -> v, t */
void cubodyforceswrapper_(int eType, double dx1, double dx2, double dx3,
                          int sx1, int sx2, int sx3h, float *v1, float *v2,
                          float *v3, float *t1, float *t2, float *t3);
/* src/cugreen.cu:1453 -- Green's function on the context's v, t */
void calfftnelasic_(float *c1, float *c2, float *c3, float *t1, float *t2,
                    float *t3, int sx1, int sx2, int sx3, double dx1,
                    double dx2, double dx3, double lambda, double mu,
                    double gam, float *p1, float *p2, float *p3, int *iRet);
/* src/cuelastic.cu:1122 -- moment += viscous eigenstress of sig */
void cuviscouseigen_(relax_layer *structure, relax_tensor_layer *prestress,
                     double mu, int sx1, int sx2, int sx3h, double dx1,
                     double dx2, double dx3, int bMaxwell, double *tm,
                     int gammadot0type);
/* src/cuelastic.cu:1762 */
void cufrictioneigenstress_(double x, double y, double z, double L, double W,
                            double strike, double dip, double rake,
                            double beta, double mu, relax_layer *structure,
                            int sx1, int sx2, int sx3h, double dx1,
                            double dx2, double dx3, int bPresent, float *tm,
                            ST_TENSOR_C *moment, ST_TENSOR_C *sig);
/* src/cuelastic.cu:1350 -- 1: moment, 2: tau; sum of norms (no dV) */
void cutensoramp_(int eType, int sx1, int sx2, int sx3h, double *amp);
/* src/cuelastic.cu:874 -- body force + traction of one shear source */
void cusource_(double mu, double s, double x, double y, double z, double L,
               double W, double strike, double dip, double rake,
               double beta, int sx1, int sx2, int sx3, double dx1,
               double dx2, double dx3, float *f1, float *f2, float *f3,
               float *t1, float *t2, float *t3);
/* src/cuelastic.cu:1085 -- transient eigenstress on epsilonik (eType 4) or,
 * in place, on epsilonikdot (eType 5); bgammadot 3/4 = transient weak zones */
void cutransienteigenwrapper_(int eType, relax_layer *structure, double mu,
                              int sx1, int sx2, int sx3h, double dx1,
                              double dx2, double dx3, int bMaxwell,
                              double *dMaxwell, int bgammadot);
/* src/cuelastic.cu:1689 -- weak-zone fluidity field of one mechanism
 * (gammadotType 1..4: linear, nonlinear, linear / nonlinear transient) */
void cubuildgammadot_(int sx1, int sx2, int sx3h, double dx1, double dx2,
                      double dx3, int nz, relax_weakzone *zones,
                      int gammadotType);
/* src/cuelastic.cu:1629 -- one x3-plane of the padded displacement */
void cuexportspatial_(float *u1, float *u2, float *u3, int i3);
/* src/cuelastic.cu:1652 -- displacement and stress at one point (0-based) */
void cuexportpoints_(double *u1, double *u2, double *u3, ST_TENSOR_C *sig,
                     int i1, int i2, int i3);

#ifdef __cplusplus
}
#endif

#endif /* RELAX_B200_H */
