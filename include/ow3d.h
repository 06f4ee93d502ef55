/*
 * ow3d.h -- C ABI of the B200-native OceanWave3D hot path.
 *
 * The library replaces two call sites of the reference Fortran program:
 *
 *   (1) the per-stage Laplace solve
 *         CALL iterative_solution(RHS, n_rows, BuildLinearSystem, PHI, FineGrid)
 *       (src/wrappers/iterative_solution.f90:1-136, called from
 *        src/timeintegration/Runge_Kutta_4.f90:129,216,309,419)
 *       -> ow3d_solve / ow3d_solve_device
 *
 *   (2) the whole RK4 free-surface time step
 *         CALL timeintegration_fsbc   (src/timeintegration/timeintegration_fsbc.f90:1-45)
 *       -> ow3d_step
 *
 * The set-up half of the reference (OceanWave3DT0Setup, src/main/OceanWave3DT0Setup.f90)
 * maps to ow3d_read_deck + ow3d_create.
 *
 * Conventions shared with the reference:
 *   - All arrays are caller-owned, column-major Fortran arrays with ghost points
 *     included:  3-D fields are PHI(k,i,j), k (sigma) fastest, size
 *     Nzg*Nxg*Nyg with Nzg = Nz+GhostGridZ, Nxg = Nx+2*GhostGridX,
 *     Nyg = Ny+2*GhostGridY (src/initialization/InitializeVariables.f90:24);
 *     2-D free-surface fields are E(i,j), size Nxg*Nyg.
 *   - Pointers are only read or written during the call; nothing is retained.
 *   - Every function returns an int status: 0 = OK, > 0 = warning, < 0 = error.
 *     No function calls exit() or aborts the process.
 *   - One handle per host thread; calls on one handle are not thread-safe.
 */
#ifndef OW3D_H
#define OW3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define OW3D_OK                 0
#define OW3D_NOT_CONVERGED      1   /* GMRES hit its matvec limit; solution kept
                                       (the reference accepts this silently,
                                       iterative_solution.f90:117-134)          */
#define OW3D_ERR_BAD_INPUT     -1
#define OW3D_ERR_CUDA          -2
#define OW3D_ERR_OOM           -3   /* device allocation failed / admission denied */
#define OW3D_ERR_UNSTABLE      -4   /* max|eta| > 10 max h (OceanWave3DTakeATimeStep.f90:54) */
#define OW3D_ERR_TIMEOUT       -5
#define OW3D_ERR_NO_DEVICE     -6
#define OW3D_ERR_IO            -7
#define OW3D_ERR_UNSUPPORTED   -8

/* ------------------------------------------------------- build-only knobs */
#define OW3D_PREC_FP64          0   /* everything FP64 ("plain" form)                 */
#define OW3D_PREC_MIXED         1   /* MG hierarchy + smoother FP32, Krylov/RK4 FP64  */

#define OW3D_KRYLOV_FGMRES      0   /* right-preconditioned flexible GMRES (default)   */
#define OW3D_KRYLOV_LGMRES      1   /* left-preconditioned GMRES, stopping test on the
                                       preconditioned residual (SPARSKIT2 semantics
                                       used by iterative_solution.f90:23-24)            */

#define OW3D_SMOOTHER_MULTICOLOUR     0   /* multicolour column Gauss-Seidel (default)  */
#define OW3D_SMOOTHER_LEXICOGRAPHIC   1   /* the reference's row order (GaussSeidel.f90) */

#define OW3D_MAX_ZONES          8
#define OW3D_MAX_KIN_FILES     20   /* kinematics output slices (ReadInputFileParameters.f90:305) */

/* One relaxation zone: deck line 13 continuation
 * "x1 x2 y1 y2 ftype param XorY WavegenONOFF XorYgen degrees"
 * (src/IO/ReadInputFileParameters.f90:505-517,
 *  src/initialization/PreprocessRelaxationZones.f90). */
typedef struct ow3d_zone {
    double x1, x2, y1, y2;
    int    ftype;        /* +/-9 (sponge 1->0), +/-10 (3rd-order 0->1), 11..14  */
    double param;
    char   XorY;         /* 'X' or 'Y' */
    int    WavegenONOFF; /* 0: absorption (sponge), 1: generation              */
    char   XorYgen;
    double degrees;
    int    PhiOnOff;     /* sponge relaxes phi too when 1 (default 1)          */
} ow3d_zone;

/* Parameters of the positional input deck (src/IO/ReadInputFileParameters.f90),
 * restricted to the fields the hot path reads, plus build-only knobs. */
typedef struct ow3d_params {
    /* line 2 */
    int    IC, IncWaveType;       /* ow3d_read_deck reads 4 as 1 with current_flag = 1
                                     (see current_Q) and 5 as 3 with current_flag = 1 */
    /* line 3 */
    double Lx, Ly, Lz;
    int    Nx, Ny, Nz;
    int    GridX, GridY, GridZ;
    int    GhostGridX, GhostGridY, GhostGridZ;
    /* line 4 */
    int    alpha, beta, gamma;
    int    alphaprecond, betaprecond, gammaprecond;
    /* line 5 */
    int    Nsteps;
    double dt;
    int    timemethod;
    double CFL;
    int    extrapolationONOFF;
    double time0;
    /* line 6 */
    double g;
    /* line 7 */
    int    solver;                /* 1 = GMRES (0 = defect correction: unsupported) */
    int    Precond;               /* 3 = multigrid, 0 = none                         */
    int    MGCoarseningStrategy;  /* 0 (default), 1, 2                               */
    int    GMRESmaxiterations;
    double reltol, abstol;
    int    maxit;                 /* V-cycles per preconditioner application         */
    char   cyclet;                /* 'V' (W/F: unsupported)                          */
    int    nu1, nu2;
    int    MGmaxgrids;
    /* line 10 */
    int    LinearONOFF;           /* 1 = nonlinear, 0 = linear (reference naming)    */
    int    PressureTermOnOff;     /* must be 0                                       */
    /* line 11 */
    int    filteringONOFF, filterALPHA, filterORDER;
    double sigma_filt[3];
    /* line 13 */
    int    relaxONOFF;
    double relaxTransientTime;
    int    relaxNo;
    char   relaxXorY;
    double relaxDegrees;
    ow3d_zone zones[OW3D_MAX_ZONES];
    /* build-only knobs (not part of the deck; defaults from ow3d_default_params) */
    int    precision;             /* OW3D_PREC_*   */
    int    krylov;                /* OW3D_KRYLOV_* */
    int    device;                /* CUDA device ordinal */
    /* line 9 (after the build-only knobs, so the layout above is unchanged) */
    int    StoreDataONOFF;        /* >0: EP_#####.bin every n steps, <0: fort.NNN every -n steps, 0: none */
    int    formattype;            /* EP file form (1 and the default both write unformatted records);
                                     20 / 21: kinematics output to Kinematics<nn>.bin / one
                                     Kinematics_<nn>_<it>.bin per output time (22: point
                                     output, parsed but not supported) */
    /* line 9, formattype 20-22 (ReadInputFileParameters.f90:300-405) */
    int    iKinematics;           /* nonzero: kinematics output */
    int    nOutFiles;             /* output slices, at most OW3D_MAX_KIN_FILES (10 for 21, 22) */
    int    kinematics[OW3D_MAX_KIN_FILES][9];  /* per slice: xbeg xend xstride ybeg yend ystride
                                     tbeg tend tstride (interior indices and time levels, 1-based;
                                     formattype 22 keeps tbeg tend tstride only) */
    /* the incident linear wave of IncWaveType 2, the deck line after the
     * curvilinear line (ReadInputFileParameters.f90:591-647) */
    int    ispec;                 /* -1 mono-chromatic, 0 PM, 1 and 3 JONSWAP, 2 from a file,
                                     |ispec| >= 30 directional */
    int    seed, seed2;           /* random-wave seeds, made negative as the reference does */
    double Tp, Hs, h0;            /* period (peak period), height (significant height), depth */
    double kh_max, x0, y0;        /* spectrum cut-off; origin of the wave's phase */
    double gamma_jonswap, beta0, s0;  /* JONSWAP gamma (3.3 unless ispec 3 / >= 30), heading, spreading */
    /* line 8, the stream-function wave of IncWaveType 1 (ReadInputFileParameters.f90:291-293) */
    double sf_H, sf_h, sf_L, sf_T;    /* height, depth, wavelength, period */
    double sf_uEorS;                  /* mean current (Eulerian or Stokes) */
    int    sf_wavel_or_per;           /* 0: the wavelength is given, 1: the period */
    int    sf_euler_or_stokes;        /* 0: Eulerian current, 1: Stokes drift */
    int    sf_nsteps;                 /* height steps of the solver */
    int    sf_nmodes;                 /* Fourier modes */
    /* line 3 with Lz <= 0: the bathymetry file named after the ghost flags */
    char   bathymetry_file[256];
    /* deck features outside this library's path, kept so that ow3d_create
     * can refuse a deck that needs them instead of running without them */
    double accel_tol_fact;            /* line 2: local filtering by acceleration, on for (0, 100] (1e30 when absent) */
    int    i_breaking;                /* line 12: breaking model (see T_half below) */
    int    PDampingONOFF;             /* pressure-damping zones on */
    int    swenseONOFF;               /* SWENSE on */
    int    curvilinearONOFF;          /* curvilinear grid on */
    /* the pressure-damping line and its zone (ReadInputFileParameters.f90:534-545;
     * the reference runs one zone, PreprocessPDampingZones.f90) */
    int    NDampZones;
    int    pd_type;                   /* 0: damp the velocity through p_d (a 1-D solve over the zone), else phi */
    double pd_x0, pd_x1, pd_y0, pd_y1;/* zone box BBox(1:4) */
    double pd_g0Phi, pd_g0Eta;        /* strengths: gamma = 2 pi g0 exp(-((x - x1)/(x1 - x0))^2 / 0.125) */
    /* 1 when ow3d_read_deck read accel_tol_fact from line 2: the reference
     * then smooths locally for every value up to 100 g, 0 and negative values
     * included (LocalSmoothing2D.f90:37); 0 for parameters built by a caller,
     * where accel_tol_fact = 0 means no local smoothing */
    int    accel_from_deck;
    /* build-only knob, no counterpart in the reference (whose lateral rows
     * are walls, BuildLinearSystem.f90:149-216): 1 = periodic in x. The Nx
     * points span one period including both ends, x_1 = 0 and x_Nx = Lx,
     * which hold the same value; the Nx - 1 distinct columns are coupled
     * cyclically in every stencil, the ghost columns are unused. */
    int    periodic_x;
    /* line 12, the roller breaking model of x flumes (DetectBreaking.f90;
     * ReadInputFileParameters.f90:478-479), after i_breaking above: 1 = rollers
     * found and their flux slope Qr_x subtracted from the kinematic condition
     * at every RK stage, 2 (or any other positive value) = rollers found and
     * reported only. Applied when Ny = 1, as in the reference; ignored in 3-D. */
    double T_half;                    /* s over which tan(phi) relaxes to tan(phi_0); > 0 */
    double phi_b, phi_0;              /* breaking and terminal roller angles, degrees */
    double del_fac;                   /* roller thickness factor f_delta */
    double cel_fac, gamma_break;      /* read and kept; the reference computes nothing from them */
    /* the constant-flux current of IncWaveType 4 (ReadInputFileParameters.f90:42-49,
     * 655-690): ow3d_read_deck reads IncWaveType 4 as 1 (the stream-function
     * wave) with current_flag = 1 and the flux Q from the line after the
     * curvilinear line. The lateral Neumann rows then carry u = Q/h at the
     * west and east walls (Runge_Kutta_4.f90:112,207,291,412) and the surface
     * potential's ghost points the same flux (:85-88). */
    int    current_flag;
    double current_Q;                 /* m^2/s */
    /* the flux wavemaker of IncWaveType 3 (and 5): the deck line after the
     * curvilinear line (ReadInputFileParameters.f90:579-589). The paddle
     * signal itself is read with ow3d_read_paddle_signal and installed with
     * ow3d_set_paddle_signal before the first step. */
    double flux_ramp;                 /* ramp time of the boundary flux, s */
    int    flux_order;                /* points of the interpolation in y (1..10) */
    char   flux_file[256];            /* paddle-signal file named by the deck */
} ow3d_params;

typedef struct ow3d_handle ow3d_handle;

/* Solver statistics: the counters of OceanWave3DTakeATimeStep.f90:76-122 plus
 * device timings. Iterations are counted as matvec requests, including the
 * initial residual, exactly as iterative_solution.f90:58-60 counts them. */
typedef struct ow3d_stats {
    int64_t solves;
    int64_t total_iterations;
    int     min_iterations, max_iterations;
    int     last_iterations;
    int64_t not_converged;
    double  last_residual;        /* final residual estimate of the last solve */
    double  time;                 /* simulation time                           */
    int64_t tstep;                /* number of completed time steps            */
    double  last_initial_residual;/* |rhs - A phi0| of the last solve (FGMRES; the
                                     preconditioned residual for left GMRES)     */
    double  last_tolerance;       /* its stopping threshold reltol*|r0| + abstol
                                     (iterative_solution.f90:24,44-45)          */
} ow3d_stats;

/* ------------------------------------------------------------- set-up */

/* Fill *p with the defaults the reference uses when a deck omits optional
 * fields, plus precision = FP64, krylov = FGMRES, device = 0. */
int ow3d_default_params(ow3d_params* p);

/* Parse a positional OceanWave3D input deck (ReadInputFileParameters.f90:18-747)
 * into *p. Fields beyond line 13 that the hot path does not use are skipped.
 * Replaces: ReadInputFileParameters (src/IO/ReadInputFileParameters.f90:1). */
int ow3d_read_deck(const char* path, ow3d_params* p);

/* Create a simulation on the device: grid, stencils, sigma levels, multigrid
 * hierarchy and workspaces. h..hyy are the bathymetry and its derivatives,
 * Nxg*Nyg each, ghosts included (SetupInitialConditions.f90:51-111).
 * Replaces: the device-relevant part of OceanWave3DT0Setup
 * (OceanWave3DT0Setup.f90:35-444: SetupCompDomain, PreProcessDiffStencils,
 *  ConstructTableCrossDerivatives, MGPreProcess, FilterInit,
 *  PreprocessRelaxationZones). */
int ow3d_create(const ow3d_params* p,
                const double* h, const double* hx, const double* hxx,
                const double* hy, const double* hyy,
                ow3d_handle** out);

int ow3d_destroy(ow3d_handle* h);

/* Grid dimensions including ghosts and the device bytes the handle holds. */
int ow3d_dims(const ow3d_handle* h, int* Nxg, int* Nyg, int* Nzg, size_t* device_bytes);

/* Estimated device bytes a handle with parameters *p would allocate
 * (used by the serving loop's admission gate). */
int ow3d_estimate_bytes(const ow3d_params* p, size_t* bytes);

/* ------------------------------------------------- the Laplace solve */

/* One Laplace solve A(eta) phi = rhs with the 6th-order sigma-transformed
 * operator, preconditioned by the low-order multigrid V-cycle.
 *   rhs       : Nzg*Nxg*Nyg, host, read
 *   phi_inout : Nzg*Nxg*Nyg, host, initial guess in, solution out
 *   E,Ex,Exx,Ey,Eyy : the free-surface elevation and its horizontal
 *               derivatives (Nxg*Nyg each, host) that define the sigma
 *               coefficients (DetermineTransformationConstantsArray.f90);
 *               Ey/Eyy may be NULL in 2-D.
 *   iterations: out, matvec count as iterative_solution.f90:58-60 counts it.
 * Replaces: iterative_solution(rhss, n_rows, BuildLinearSystem, sol, FineGrid)
 *   (src/wrappers/iterative_solution.f90:1, matvec callback
 *    src/functions/BuildLinearSystem.f90:1). */
int ow3d_solve(ow3d_handle* h, const double* rhs, double* phi_inout,
               const double* E, const double* Ex, const double* Exx,
               const double* Ey, const double* Eyy, int* iterations);

/* Same, with all pointers in device memory of the handle's device. Runs on the
 * handle's stream; returns after the solve completed. */
int ow3d_solve_device(ow3d_handle* h, const double* d_rhs, double* d_phi_inout,
                      const double* d_E, const double* d_Ex, const double* d_Exx,
                      const double* d_Ey, const double* d_Eyy, int* iterations);

/* y = A phi with the high-order operator (BuildLinearSystem.f90:1-290) for the
 * surface state (E..Eyy). Host pointers. Probe/unit-test entry point. */
int ow3d_matvec(ow3d_handle* h, const double* phi, double* y,
                const double* E, const double* Ex, const double* Exx,
                const double* Ey, const double* Eyy);

/* Allocation-free residual check -- no counterpart in the reference, which
 * has no device. d_res = d_rhs - A(eta) d_phi with the high-order operator
 * and *norm2 = ||d_res||_2 (host scalar). Every array is caller-owned DEVICE
 * memory of the handle's device (d_Ey, d_Eyy may be NULL in 2-D; the surface
 * is ignored for a linear run). The call allocates nothing: its only scratch
 * is a fixed file-scope device array (1024 partial sums) whose address is
 * looked up once per device on the first call on that device; that first
 * call should come before any stream capture begins. Vectors longer than
 * 2^31-1 elements are rejected with OW3D_ERR_UNSUPPORTED. Calls that overlap
 * in time on one device share that scratch and must be serialised by the
 * caller. Runs on the handle's stream and synchronises it: it returns after
 * the norm is on the host. */
int ow3d_residual_device_noalloc(ow3d_handle* h, const double* d_rhs, const double* d_phi,
                                 const double* d_E, const double* d_Ex, const double* d_Exx,
                                 const double* d_Ey, const double* d_Eyy,
                                 double* d_res, double* norm2);

/* u = M^{-1} r: maxit V-cycles of the low-order multigrid preconditioner from
 * u = 0 (MultiGridSolveLinearSystem.f90:1-95). Host pointers. */
int ow3d_precondition(ow3d_handle* h, const double* r, double* u);

/* ------------------------------------------------- the time step */

/* Set the free-surface state: E, P (surface potential) and W (vertical surface
 * velocity), Nxg*Nyg each, and the 3-D potential phi (may be NULL: zero), at
 * simulation time t. Mirrors the state OceanWave3DT0Setup leaves behind. */
int ow3d_set_state(ow3d_handle* h, const double* E, const double* P,
                   const double* W, const double* phi, double t);

/* Overwrite the surface elevation E and surface potential P (Nxg*Nyg, host)
 * between time steps without touching phi, W or the extrapolation history,
 * e.g. when a coupled host modifies the surface (the reference's global
 * Wavefield%E, Wavefield%P). Recomputes the surface derivatives. */
int ow3d_put_surface(ow3d_handle* h, const double* E, const double* P);

/* Read back E, P, W (Nxg*Nyg) and phi (Nzg*Nxg*Nyg); any pointer may be NULL. */
int ow3d_get_state(ow3d_handle* h, double* E, double* P, double* W,
                   double* phi, double* t);

/* Geometry and initial surface of the deck's IC where the reference builds
 * them from formulas (SetupInitialConditions.f90): 0 (Lz > 0: flat, still
 * water), 1 (deep-water nonlinear standing wave, nonlinearstandingwave1D.f90),
 * 3 (the Whalin shoal, bottomWhalin.f90), 4 and 5 (flat deep / shallow water,
 * a cosine surface), 7 (flat,
 * the stream-function wave over the basin at time0 when relaxation is on,
 * the non-generating zones' weights then applied three times as the
 * reference does). h..hyy, E, P: Nxg*Nyg, ghosts included, for ow3d_create
 * and ow3d_set_state (which takes the surface derivatives itself). Other ICs
 * return OW3D_ERR_UNSUPPORTED (IC -1: ow3d_read_init_file; Lz <= 0:
 * ow3d_read_bathymetry). hx..hyy may be NULL. Host-only. */
int ow3d_initial_condition(const ow3d_params* p, double* h, double* hx, double* hxx, double* hy, double* hyy,
                           double* E, double* P);

/* The bathymetry file of a deck with Lz <= 0 (its name is p->bathymetry_file,
 * relative to where the deck's run starts), as SetupInitialConditions.f90:51-111
 * reads it: a header line, the gradient flag (0: each record holds h, h_x,
 * h_xx, h_y, h_yy; 1: h only, the derivatives then taken with the 7-point x
 * and y stencils as OceanWave3DT0Setup.f90:346-364 does), one record per
 * interior point, x fastest. Outputs are Nxg*Nyg (ghosts take the values of
 * the adjacent interior points), ready for ow3d_create; hx..hyy and flag may
 * be NULL. The reference then sets Lz to h at the first point. Host-only. */
int ow3d_read_bathymetry(const ow3d_params* p, const char* path, double* h, double* hx, double* hxx,
                         double* hy, double* hyy, int* flag);

/* The stream-function wave of the deck's line 8 (IncWaveType 1): Fenton's
 * Fourier solution as stream_func_set_up / stream_func_coeffs compute it
 * (src/utilities/stream_func_set_up.f90:1-59, stream_func_coeffs.f:1-153),
 * evaluated as stream_func_wave_finite (stream_func_wave_finite.f:3-71):
 * eta and the surface potential phiS at the n positions x (m, in the frame
 * where the crest is at x = 0 at t = 0) at time t (s); eta / phis may be
 * NULL. info (4 doubles, may be NULL): wavenumber, wavelength, period and
 * phase speed. Host-only. For relaxation targets sample every RK stage time
 * and pass the series with ow3d_set_relax_target mode 1; for an initial
 * condition evaluate at t = 0. */
int ow3d_stream_function_wave(const ow3d_params* p, int n, const double* x, double t, double* eta,
                              double* phis, double* info);

/* The incident wave of IncWaveType 2 on generation zone `zone` (0-based), as
 * OceanWave3DT0Setup.f90:176-255 builds RandomWave(zone)%eta and %Phis
 * before the time loop: nt samples every dt, on the zone's box (i fastest,
 * then j; the x-directed wave repeated on every row), ready for
 * ow3d_set_relax_target(h, zone, 0, nt, dt, eta, phis). box (5 ints, may be
 * NULL) receives the ghost-inclusive 1-based bounds i0 i1 j0 j1 and the
 * number of samples the reference builds (Nsteps for ispec -1, else the
 * power of two at or above Nsteps); eta and phis may be NULL to query box
 * only. Host-only (no handle, no device). Supported: ispec -1 (mono-chromatic
 * from t = time0, random_wave_signal.f90:151-172), 0 (Pierson-Moskowitz), 1
 * and 3 (JONSWAP) long-crested random waves from t = 0 with the reference's
 * random phases (RAN1_b seeded with seed2), spectra, kh_max truncation and
 * wavenumbers (fdwvnum.f90); -30, 30 and 31, the same waves at heading beta0
 * on every point of the zone (random_wave_signal_3D.f90, zones with
 * degrees = 0); 33 and 34, JONSWAP seas with normal (build_coeff_3D.f90)
 * and cos^(2 s0) (spreading.f90) spreading, each component on its own
 * heading drawn as the reference draws it; for random waves nt is at most
 * the reference's sample count. Waves from a file (ispec 2) return
 * OW3D_ERR_UNSUPPORTED. */
int ow3d_incident_wave(const ow3d_params* p, int zone, int nt, double* eta, double* phis, int* box);

/* The incident wave of IncWaveType 2 on generation zone `zone` (0-based),
 * synthesised on the device and installed as the zone's relaxation target
 * (mode 0: sampled every dt, mid-stage targets averaged), without the series
 * crossing the host: the same wave as ow3d_incident_wave followed by
 * ow3d_set_relax_target(h, zone, 0, nt, dt, ...), to rounding. The
 * amplitudes, wavenumbers and headings (the reference's sequential random
 * generator, a few thousand numbers) are set up on the host; every sample at
 * every point of the zone is formed on the device -- the mono-chromatic wave
 * in closed form, random waves as the sum over their modes that the
 * reference's inverse real transform evaluates (random_wave_signal.f90:48-172,
 * random_wave_signal_3D.f90). nt: the samples to build, at most the count
 * ow3d_incident_wave reports in box[4] for random waves. Replaces: the
 * RandomWave(i)%eta, %Phis set-up of OceanWave3DT0Setup.f90:176-255. */
int ow3d_incident_wave_device(ow3d_handle* h, int zone, int nt);

/* Relaxation-zone target signal for generation zone `zone` (0-based):
 * nt samples of eta and surface phi on the zone rectangle (i fastest, then j,
 * ghost-inclusive index box of the zone), sampled every dt_sample from t=0.
 * mode 0: dt_sample = dt and mid-stage targets are the average of the two
 *         neighbouring samples (AnalyticWaveMaker2D.f90:26-33, IncWaveType 2);
 * mode 1: dt_sample = dt/2, every RK stage time is a sample (IncWaveType 1). */
int ow3d_set_relax_target(ow3d_handle* h, int zone, int mode, int nt,
                          double dt_sample, const double* eta, const double* phis);

/* Advance nsteps RK4 steps (Runge_Kutta_4.f90:1-429 with rhsFreeSurface3D or
 * rhsLinearFreeSurface3D, relaxation, SG filtering), device resident.
 * Replaces: timeintegration_fsbc (timeintegration_fsbc.f90:1-45) called from
 * OceanWave3DTakeATimeStep.f90:27. Returns OW3D_ERR_UNSTABLE on the
 * reference's instability test; OW3D_NOT_CONVERGED if any solve hit the limit. */
int ow3d_step(ow3d_handle* h, int nsteps);

/* The paddle-signal file of the flux wavemaker (setupWavePaddle.f90:43-67): a
 * header line, `dt nt n2`, the n2 y positions of the signal points, then nt
 * records `time flux(1..n2)`. Call with y = flux = NULL (or cap too small)
 * to get dt, nt and n2; then with y (n2) and flux (nt * n2, time-major) of
 * at least cap = nt * n2 values. Host-only. */
int ow3d_read_paddle_signal(const char* path, int cap, double* dt, int* nt, int* n2, double* y, double* flux);

/* Install the flux wavemaker's signal on a handle of IncWaveType 3 (or 5):
 * the boundary flux u(t, y) at the n2 points y (uniformly spaced from dy/2)
 * every dt, and eta_x = -u_t / g from its 5-point time derivative
 * (setupWavePaddle.f90:89-122). Each RK stage then imposes, on the west
 * wall, the flux ramped over flux_ramp and interpolated linearly in time and
 * with flux_order points in y (waveGenerationFromPaddleSignal.f90:43-111):
 * in the Neumann rows of every level above the bottom, and in the ghost
 * points of the surface potential and elevation at the end of each step.
 * Replaces: setupWavePaddle. Required before the first ow3d_step of such a
 * handle; OW3D_ERR_BAD_INPUT for unevenly spaced points or a signal shorter
 * than Nsteps * dt. */
int ow3d_set_paddle_signal(ow3d_handle* h, int nt, int n2, double dt, const double* y, const double* flux);

/* on = 1: the coarse levels of every V-cycle run in one thread-block
 * cluster of 16 SMs (8 where 16 cannot be resident) instead of a cooperative
 * grid over every SM -- no counterpart in the reference. For handles stepped
 * together (ow3d_step_batch): the coarse cycles of different simulations then
 * overlap, where a grid-wide cycle takes the whole device for its duration.
 * Measured on a B200 over a stream of the serving configuration's sizes: 1.55x
 * the batched throughput and half the step latency; a handle stepped alone is
 * 10-30% slower with it, so the default is off. Results are bitwise the same
 * either way. Drops the handle's captured graphs. */
int ow3d_set_coarse_cluster(ow3d_handle* h, int on);

/* Row order of the multigrid smoother's Gauss-Seidel steps.
 * OW3D_SMOOTHER_MULTICOLOUR (default): interior columns in 2 or 4 colour
 * classes, each column bottom to top with the ghost and bottom rows it
 * borders -- a different ordering of the same relaxations, with about the
 * reference's smoothing per step, that runs in parallel.
 * OW3D_SMOOTHER_LEXICOGRAPHIC: the reference's order on every level, which
 * gives the reference's iterates up to rounding: the special rows (bottom and
 * lateral ghost rows, MGPreProcess.f90:376-439), then per smoothing step a
 * sweep over all rows in index order and the special rows again
 * (GaussSeidel.f90:15-26, GaussSeidelSpecialPoints.f90:43-53,
 * MultiGridSolver.f90:118-126,174-181), run as wavefronts in one thread block
 * per sweep; the V cycle then descends to the coarsest level's inverse on
 * every application (no fused coarse cycle, no dense sub-cycle operator).
 * Together with krylov = OW3D_KRYLOV_LGMRES this is the reference's
 * preconditioned solver. Many times slower than the default: meant for
 * checking results against the reference, not for production runs. Drops the
 * handle's captured graphs. Replaces: the smoother choice of
 * MultiGridSolver.f90 (the reference has only the lexicographic order). */
int ow3d_set_smoother_order(ow3d_handle* h, int order);

/* The rollers of the roller breaking model (i_breaking > 0, Ny = 1) after
 * the last completed step, as the reference writes them to roller.dat each
 * step (DetectBreaking.f90:205-211): *n_rollers receives their number (0
 * when the model is off), and for the first min(n, cap) rollers, in the
 * order found (from the right end of the flume): npts = grid points the
 * roller covers, toe = the 1-based, ghost-inclusive column just ahead of the
 * toe, x = the toe's position measured as the reference does, (j - 1) dx
 * from the ghost column, eta = the elevation at the toe, thickness = the
 * roller thickness one column behind the toe, tan_phi = tan(phi) at the toe
 * column after the step's update. Any array may be NULL. The reference
 * holds at most Nxg / 10 rollers; this library holds all. Synchronises the
 * handle's stream. Replaces: the roller.dat record of detect_breaking. */
int ow3d_rollers(ow3d_handle* h, int cap, int* n_rollers, int* npts, int* toe, double* x, double* eta,
                 double* thickness, double* tan_phi);

/* ow3d_step, plus the device time of the steps measured with CUDA events on
 * the handle's stream (milliseconds). */
int ow3d_step_timed(ow3d_handle* h, int nsteps, double* device_ms);

/* Advance n independent simulations together -- no counterpart in the
 * reference, which runs one simulation per process. Handle i takes nsteps[i]
 * RK4 steps, each simulation at its own pace, driven by the calling thread:
 * every handle with steps left has its next step in flight as its step
 * graph on its own stream (see ow3d_set_graphs), and as soon as one
 * completes the thread launches that handle's next step (handles that
 * cannot use graphs step directly in between). The simulations' kernels so
 * overlap on the device. status[i] and wall_ms[i] (either may be NULL)
 * receive each handle's ow3d_step status and the host time in milliseconds
 * from the call's start to the end of its last step. The handles must be
 * distinct. Returns the most severe status. Each result is the same as
 * ow3d_step on that handle alone (handles share no state). */
int ow3d_step_batch(ow3d_handle* const* hs, int n, const int* nsteps, int* status, double* wall_ms);

int ow3d_get_stats(const ow3d_handle* h, ow3d_stats* s);
int ow3d_reset_stats(ow3d_handle* h);

/* 1 (the default): with the multigrid preconditioner (FGMRES or left GMRES),
 * from the second RK4 step on every step is one CUDA graph launch (one graph per
 * parity of the step number, captured on first use): each of its four
 * solves is the initial residual, one conditional node per Arnoldi step --
 * enabled on the device by the previous step's stopping test -- and the
 * solution update, so the host waits once per step. Before that (and in
 * ow3d_solve), from the handle's second solve on, each Arnoldi step is one
 * graph launch. 0: kernels are launched one by one. Decks with a
 * pressure-damping zone always launch directly;
 * ow3d_set_relax_target drops the step graphs (they hold the target table).
 * Results are bitwise the same either way. */
int ow3d_set_graphs(ow3d_handle* h, int on);

/* Zone-box of relaxation zone `zone` in 1-based ghost-inclusive indices. */
int ow3d_zone_box(const ow3d_handle* h, int zone, int* i0, int* i1, int* j0, int* j1);

/* ------------------------------------------------------------- files
 * The reference's result and hot-start files (io.cpp). The *_file functions
 * work on host arrays only (no device, no handle); the handle forms copy the
 * state off the device first. Messages of the *_file functions are in
 * ow3d_io_last_error(). */

/* EP_#####.bin as StoreData writes it (src/IO/StoreData.f90:11-29): three
 * Fortran unformatted records (32-bit length markers, little-endian):
 * nx ny | x(nx*ny) y(nx*ny) | E(nx*ny) P(nx*ny), x fastest, ghosts included. */
int ow3d_write_ep_file(const char* path, int nx, int ny, const double* x, const double* y,
                       const double* E, const double* P);
/* fort.NNN as StoreDataAscii writes it (src/IO/StoreDataAscii.f90:21-31):
 * "x y E P" per point in 4e16.6e3, an empty line after each row. */
int ow3d_write_ascii_file(const char* path, int nx, int ny, const double* x, const double* y,
                          const double* E, const double* P);
/* OceanWave3D.end (OceanWave3DTakeATimeStep.f90:146-162): header line,
 * "Lx Ly Nx Ny time", then "E P" at the Nx*Ny interior points, x fastest. */
int ow3d_write_end_file(const char* path, double xtank, double ytank, int Nx, int Ny, double time,
                        const double* E, const double* P);
/* Read a hot-start file OceanWave3D.init in that format
 * (ReadInputFileParameters.f90:113-125, SetupInitialConditions.f90:18-27);
 * its Nx, Ny must equal the given ones. E, P: Nx*Ny interior values. */
int ow3d_read_init_file(const char* path, int Nx, int Ny, double* E, double* P, double* time);
const char* ow3d_io_last_error(void);

/* Handle forms: the current state into dir ("" = working directory).
 * fields 0 = E, P; 1 = h, hx (the reference's bathymetry file, nr 99999 /
 * 899). ow3d_store_data applies the deck's StoreDataONOFF schedule at the
 * handle's current step, as OceanWave3DT0Setup.f90:531-548 (step 0) and
 * OceanWave3DTakeATimeStep.f90:131-187 do; *files = number written. */
int ow3d_write_ep(ow3d_handle* h, const char* dir, int nr, int fields);
int ow3d_write_ascii(ow3d_handle* h, const char* dir, int nr, int fields);
int ow3d_write_end(ow3d_handle* h, const char* path);
int ow3d_store_data(ow3d_handle* h, const char* dir, int* files);

/* Fluid kinematics of the current state on the whole grid, ghost points
 * included (Nzg*Nxg*Nyg values each, k fastest), as StoreKinematicData
 * computes them (src/IO/StoreKinematicData.f90:256-460):
 *   u = phi_x + s_x phi_s, v = phi_y + s_y phi_s, w = phi_s / d,
 * with phi_s the sigma derivative, d = h + eta and s_x = ((1 - z) h_x -
 * z eta_x) / d (the s_x, s_y terms only when LinearONOFF is nonzero);
 * grads (9 consecutive fields, may be NULL), in the reference's order and
 * meaning: D_s(phi_s)/d, D_x(phi_s)+s_x D_s(phi_s), D_y(phi_s)+s_y D_s(phi_s),
 * D_s(u)/d, D_x(u)+s_x D_s(u), D_y(u)+s_y D_s(u), and the same three for v.
 * Any of u, v, w may be NULL. Computed on the device from the handle's phi,
 * eta and eta derivatives after the last step (or ow3d_set_state). */
int ow3d_kinematics(ow3d_handle* h, double* u, double* v, double* w, double* grads);

/* Kinematics output of the deck's line 9 (formattype 20 or 21, iKinematics
 * nonzero) at the handle's current step, as OceanWave3DT0Setup.f90:551-590
 * and OceanWave3DTakeATimeStep.f90:193-204 call StoreKinematicData: at step
 * 0 the header records of every slice, then, for each slice whose time range
 * holds level L = step + 1 and with step a multiple of tstride, the 16
 * records of level L. formattype 20 appends to dir/Kinematics<nn>.bin (the
 * header truncates it); 21 writes dir/Kinematics_<nn>_<L>.bin per call (the
 * header into ..._00000.bin). Records are Fortran unformatted (32-bit length
 * markers): header (xbeg, xend, xstride, ybeg, yend, ystride, tbeg, tend,
 * tstride as int32, dt as double, Nzg as int32), (x, y, h, hx, hy) per point
 * of the slice, z(1:Nzg); per level: eta, eta_x, eta_y on the slice, then
 * phi, u, v, w and the 9 gradient fields on the slice's columns (k fastest).
 * *files = number of files written or appended to. */
int ow3d_store_kinematics(ow3d_handle* h, const char* dir, int* files);

const char* ow3d_strerror(int status);
/* Message of the last failing call on this host thread (empty if none). */
const char* ow3d_last_error(void);
const char* ow3d_version(void);

/* ------------------------------------------------------ measurement */

/* The multigrid hierarchy of a handle (MGPreProcess.f90:95-215): the number
 * of levels, and level `level`'s interior sizes (0 = coarsest) and the
 * colours of its Gauss-Seidel smoother (2, or 4 with mixed-derivative terms). */
int ow3d_level_count(const ow3d_handle* h);
int ow3d_level_dims(const ow3d_handle* h, int level, int* Nx, int* Ny, int* Nz, int* ncolor);

/* Number of kernels this library has launched since it was loaded, over all
 * handles and threads (the cooperative coarse-grid kernel counts as one). */
unsigned long long ow3d_launch_count(void);

/* Device time of `reps` launches of one kernel on this handle's stream,
 * measured with CUDA events around each launch; before each launch a write of
 * the Krylov basis (larger than L2) evicts the inputs from L2, outside the
 * timed interval. which 0 = high-order operator, 1 = one preconditioner
 * application (V-cycle), 2 = one colour pass of the finest multigrid level
 * (FP64 handles). Returns the total milliseconds of the launches. */
int ow3d_bench_kernel(ow3d_handle* h, int which, int reps, double* ms_total);

#ifdef __cplusplus
}
#endif
#endif /* OW3D_H */
