// common.cuh -- shared types of the B200 relaxation-loop library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/relax_b200.h"
#include "fft.cuh"

namespace relax {

// Sizes of one RELAX grid.  sx3 is the FFT box depth; the physical
// half-space (tensors, displacement) holds sx3h = sx3/2 layers
// (src/relax.f90:250-253).
struct Grid {
    int sx1, sx2, sx3, sx3h;
    int M;        // sx1/2: length of the packed complex transform along x1
    int K1;       // sx1/2 + 1 retained x1 wavenumbers
    double dx1, dx2, dx3;
    size_t nh;    // sx1*sx2*sx3h points of a physical field component
    size_t plane; // sx1*sx2
};

// Spectrum buffer: float2 [3][sx3+1][sx2][K1]; plane sx3 carries the 2-D
// surface traction transform.
__host__ __device__ __forceinline__ size_t sidx(const Grid &g, int c, int p, int i2, int k1)
{
    return (((size_t)c * (g.sx3 + 1) + p) * g.sx2 + i2) * g.K1 + k1;
}

// Per-depth rheology of one viscous mechanism, precomputed on the host
// (src/viscoelastic3d.f90:245-266): fluidity, stress exponent, cohesion and
// (taup/mu)^(n-1) of the deviatoric prestress taup.
struct DepthVisc {
    float g0, power, cohesion, tpow;
};

// Device-resident time-step state (src/relax.f90:555-890 host scalars).
struct StepState {
    double t, Dt, tm;          // time, current step, combined Maxwell time
    double maxwell[5];         // tm(ve), tm(pl), tm(as), transient linear / nonlinear
    double power, cei;         // log amplitudes of the last step
    float tmin[4];             // Maxwell-time minima of the last stress pass (viscous 2, transient 2)
    double dt_raw;             // the step chosen by k_dt before validation
    int fire;                  // t + Dt reaches the next event
    double dt_override;        // used when use_override != 0
    int use_override;
    int i, e, oi;
    int error;                 // device-side error flags (RELAX_ERR_*)
};

// Static description of the time-step policy, read by the dt kernel.
struct DtPolicy {
    double interval, odt, tscale, next_event_time;
    int skip, has_next_event, has_inter;
    int mech[5];               // linear, nonlinear, fault creep, transient linear / nonlinear present
};

#define RELAX_NTHREADS 256

// one layer of a transient (Burgers) structure: gammadot0, stress exponent
// and REAL(2 Gk) (src/viscoelastic3d.f90:171-181)
struct TransLayer {
    float g0, power, gk2, pad;
};

}  // namespace relax
