// Free-surface kernels' argument blocks and launchers (fs.cu).
#pragma once
#include "ow3d_internal.h"

namespace ow3d {

struct FsArgs {
    int Nxg, Nyg, Nzg;
    int three, nonlinear;
    int per;            // periodic in x: image columns instead of ghost layers
    double g;
    const double* SX;   // [2][Nxg][7]
    const double* SY;   // [2][Nyg][7]
    const double* SZ;   // [2][Nzg][7]
    const double* h;
    // the constant-flux current (IncWaveType 4): u = Q/h at the west and east
    // walls (OceanWave3DT0Setup.f90:325-326), 0 without one
    double Ul, Ur;
    // the flux wavemaker (IncWaveType 3): per row, the west wall's flux
    // FAC u (Uneumann) and eta_x source of the last k_paddle; null without one
    const double* Uw;
    const double* Es;
};

// The flux wavemaker's signal on the device (waveGenerationFromPaddleSignal.f90).
struct PaddleDev {
    int nt, Nyg, j0, j1;     // time levels; rows; interior rows j0..j1 (1-based)
    double dt, ramp;
    const double* F;         // nt x Nyg: the flux interpolated onto the rows
    const double* X;         // nt x Nyg: eta_x = -u_t / g likewise
    double *Uw, *Es;         // Nyg each: the values at the last RK time
};


// The time level on the device: the simulation time at the start of the
// current step and the step number (1 for the first step). The kernels whose
// work depends on them read this instead of taking the values as launch
// parameters, so that a captured step replays correctly at every step.
struct StepDev {
    double time;
    long long tstep;
};

// The wavemaker's values at RK time (device time) + off.
void fs_paddle(const PaddleDev& d, const StepDev* sd, double off, cudaStream_t st);

// One relaxation zone on the device (PreprocessRelaxationZones.f90).
struct RelaxZoneDev {
    int i0, i1, j0, j1;      // 1-based, ghost-inclusive box
    int xdir;                // gamma varies along x (XorY == 'X') or y
    int wavegen, phion;
    const double* gam;       // gamma along the relaxation direction
    int tmode, nt;           // target table (see ow3d_set_relax_target)
    double tdt;
    const double* eta;       // [nt][box]
    const double* phis;
};

// Savitzky-Golay filter coefficients (FilterInit.f90) as FILTERING.f90 reads them.
struct FilterDev {
    int alpha;
    const double* fc;        // 2*alpha+1 centred weights (offset -alpha..alpha)
    const double* F2;        // (2*alpha+1) x alpha boundary weights, column-major
};

// The pressure-damping zone of a 2-D deck (funPressureTerm.f90:218-311).
struct PDampDev {
    int type, i1, nd, rank;  // i1: 1-based first point of the zone, nd points
    const double* gamPhi;    // Nxg
    const double* gamEta;    // Nxg
    const double* D1;        // nd x rank first-derivative weights (type 0)
    const double* Linv;      // nd x nd inverse of the zone matrix, row-major (type 0)
    double *f, *r, *x;       // nd each: gamma * phi_x, the zone right-hand side, its solution
    double *NuD, *Pd;        // Nxg each: the kinematic and dynamic damping terms
    double Ur;               // the current's velocity at the east wall (0 without one)
};

// The roller breaking model of an x flume (DetectBreaking.f90). Columns are
// 1-based in thick and eta_x (nfx + 1 entries), 0-based elsewhere.
struct BreakDev {
    int nfx;                 // Nxg
    int cap;                 // roller records held (nfx)
    int dynamics;            // i_breaking == 1: Qr_x enters the kinematic condition
    double dx, dx_inv, g, del_fac, dt, T_half;
    double tan_b, tan_0;     // tan(phi_b), tan(phi_0)
    double* tan_phi;         // nfx: the roller angle, carried from step to step
    double* tan_old;         // nfx: its value at the start of the call
    double* eta_x;           // nfx + 1
    double* thick;           // nfx + 1: roller thickness
    double* Qr_x;            // nfx: the term the next fs_stage subtracts
    int* n_rollers;          // rollers found by the last update call
    int *npts, *toe;         // cap each: points covered, toe column (1-based)
    double *xr, *sr;         // cap each: toe position (x = (j-1) dx) and elevation
    double *r_thick, *r_tan; // cap each: thickness behind the toe, tan(phi) at the toe
};

// Rollers of the surface E and Qr_x; update: also the roller-angle update and
// the roller records (the call after the step).
void fs_breaking(const BreakDev& b, const double* E, int update, cudaStream_t st);

// Local smoothing by the surface's vertical acceleration (LocalSmoothing2D.f90,
// LocalSmoothing3D.f90), after each step.
struct SmoothDev {
    double tol;              // accel_tol_fact * g
    double dt_inv;
    const double* z;         // Nzg sigma levels
    const double *hx, *hy;
    double* WH[3];           // W after step t is filed in WH[t % 3]
    double* Wt;              // C: the surface dw/dt of the last step
    int* flag;               // C: -dw/dt reached the limit at a point i = 6..Nxg-5
    int* any;                // some point of the step did
    double *sE, *sP;         // C each: the filtered fields before the copy back
};

// From the third step on: dw/dt, the flags, and the filter of E and P where
// they call for it; every step: W filed in the history ring.
int fs_local_smoothing(const FsArgs& a, const SmoothDev& s, const double* phi, double* E, double* P,
                       const double* Ex, const double* Ey, const double* W, double* const* kE, const StepDev* sd,
                       cudaStream_t st);

// NuD and Pd of the state (E, P): the damping terms the next fs_stage adds.
void fs_pdamp(const FsArgs& a, const PDampDev& d, const double* E, const double* P, cudaStream_t st);
// NuD and Pd may be null (no pressure damping), Qr_x likewise (no breaking).
void fs_stage(const FsArgs& a, const double* E, const double* P, const double* W, const double* Ex, const double* Px,
              const double* Ey, const double* Py, const double* E0, const double* P0, double c, double* kE,
              double* kP, double* tE, double* tP, const double* NuD, const double* Pd, const double* Qr_x,
              cudaStream_t st);
void fs_rk_final(const FsArgs& a, double* E, double* P, double* const* kE, double* const* kP, double dt,
                 cudaStream_t st);
// Relaxation at RK time = (device time) + off.
void fs_relax(const FsArgs& a, const RelaxZoneDev* zones, int nz, double* E, double* P, const StepDev* sd, double off,
              double transient, cudaStream_t st);
// Start of a step: tstep += 1. End of a step: time += dt.
void fs_step_begin(StepDev* sd, cudaStream_t st);
void fs_step_end(StepDev* sd, double dt, cudaStream_t st);
// src: the ghost sources of the surface derivatives. 0 at set-up, where the
// reference's sources are still zero (OceanWave3DT0Setup.f90:444); 1 in the
// RK stages, whose fields carry the current's flux in the potential's source
// (Runge_Kutta_4.f90:85-88); 2 at the end of a step, whose field also carries
// the flux wavemaker's west-wall flux and eta_x (waveGenerationFromPaddleSignal.f90:
// 107-110 writes them to the step's own field only).
void fs_derivs(const FsArgs& a, double* E, double* P, double* Ex, double* Exx, double* Px, double* Ey, double* Eyy,
               double* Py, int src, cudaStream_t st);
void fs_wvel(const FsArgs& a, const double* phi, const double* E, double* W, cudaStream_t st);
// Periodic x: copy the distinct columns into the image columns of a field
// with nz values per column (1 <- Nxg-2, Nxg-1 <- 2, Nxg <- 3), or zero them.
void fs_images(const FsArgs& a, double* v, int nz, int zero, cudaStream_t st);
void fs_set_rhs(const FsArgs& a, const double* P, double* rhs, cudaStream_t st);
// stage3: the stage-3 form, applied only from the second step on (sd->tstep > 1).
void fs_extrap(double* phi, const double* lnew, const double* llast, int64_t n, int stage3, const StepDev* sd,
               cudaStream_t st);
// every > 0: filter only when sd->tstep is a multiple of `every` (U unchanged otherwise).
void fs_filter(const FsArgs& a, const FilterDev& f, double* U, double* tmp, const StepDev* sd, int every,
               cudaStream_t st);
void fs_unstable(const FsArgs& a, const double* E, double hmax10, int* flag, cudaStream_t st);

}  // namespace ow3d
