// Host-side set-up of one simulation: grid, stencils, multigrid hierarchy,
// relaxation zones and filter coefficients (the device-relevant half of
// OceanWave3DT0Setup, src/main/OceanWave3DT0Setup.f90:35-444).
#pragma once
#include <complex>
#include <string>
#include <vector>
#include "../../include/ow3d.h"

namespace ow3d {

constexpr int kMaxNzgHost = 64;      // sigma levels incl. the ghost level
constexpr int kMaxLevelsHost = 16;   // multigrid levels

// Per-position stencils of half width a: w[((order-1)*n + pos)*rank + m].
struct Stencil {
    int n = 0, rank = 0;
    std::vector<double> w;
    double at(int order, int pos, int m) const { return w[((size_t)(order - 1) * n + pos) * rank + m]; }
};

struct LevelHost {
    int Nx = 1, Ny = 1, Nz = 1, Nxg = 1, Nyg = 1, Nzg = 1;
    int xc = 0, yc = 0, zc = 0;     // coarsened w.r.t. the next finer level
    int ncolor = 2;
    std::vector<double> x, y, z, zs;
    std::vector<double> h, hx, hxx, hy, hyy;
    Stencil SX, SY, SZ;             // half width 1
};

struct GridHost {
    int Nx, Ny, Nz, gx, gy, gz, Nxg, Nyg, Nzg;
    int64_t N, C;
    int three;
    int per = 0;                    // periodic in x
    std::vector<double> x, y, z, zs;
    std::vector<double> h, hx, hxx, hy, hyy;
    Stencil SX, SY, SZ;             // half width 3
    std::vector<LevelHost> levels;  // levels[0] coarsest
};

struct ZoneHost {
    int i0, i1, j0, j1;
    int xdir, wavegen, phion;
    std::vector<double> gam;
};

void fd_weights(double z, const double* x, int n, int order, double* w);
Stencil stencils_xy(const std::vector<double>& x, int a);
Stencil stencils_periodic(const std::vector<double>& x, int a);
Stencil stencils_z(const std::vector<double>& z, int Nz, int gz, int g);

// Returns 0 or an OW3D_ERR_* code with a message in *err.
// Parameter checks that need no geometry (grid sizes, stencil widths, knobs).
int check_params(const ow3d_params& p, std::string* err);
// Deck features outside the path (breaking, pressure damping, SWENSE, ...):
// 0, or OW3D_ERR_UNSUPPORTED with a message.
int check_supported(const ow3d_params& p, std::string* err);
// The roller breaking model runs: i_breaking > 0 on an x flume (Ny = 1),
// where the reference calls detect_breaking (Runge_Kutta_4.f90:55).
bool breaking_on(const ow3d_params& p);
// Local smoothing by the vertical acceleration runs (LocalSmoothing2D.f90:37):
// every acceleration limit up to 100 g that a deck gives (decks write 1000 to
// turn it off), or a limit in (0, 100] that a caller sets (0, the value of a
// zero-initialised ow3d_params, counts as off).
bool smoothing_on(const ow3d_params& p);

// The flux wavemaker's paddle signal (setupWavePaddle.f90): flux time-major, nt x n2.
struct PaddleSignal {
    double dt = 0;
    int nt = 0, n2 = 0;
    std::vector<double> y, flux;
};
int read_paddle_signal(const char* path, PaddleSignal& ps, std::string* err);
int paddle_tables(const ow3d_params& p, const GridHost& G, const PaddleSignal& ps, std::vector<double>& F,
                  std::vector<double>& X, std::string* err);

int build_grid(const ow3d_params& p, const double* h, const double* hx, const double* hxx, const double* hy,
               const double* hyy, GridHost& G, std::string* err);
std::vector<ZoneHost> build_zones(const ow3d_params& p, const GridHost& G);

// The pressure-damping zone of a 2-D deck (PreprocessPDampingZones.f90:24-70,
// BuildPDampMatrices.f90:17-86). gamPhi and gamEta span the Nxg points of
// the row; type 0 adds the first-derivative weights over the zone's nd
// points (DfDx_1D_Uneven: 2a+1 weights per point from node start[i]) and
// the zone's Dirichlet-Laplacian-Neumann matrix L (nd x nd, row-major) with
// its inverse, which the device applies in place of the reference's sparse
// LU solve.
struct PDampHost {
    int type = 0, i1 = 0, nd = 0, rank = 0;   // i1: 1-based first point of the zone
    std::vector<double> gamPhi, gamEta;
    std::vector<double> D1;                  // nd x rank
    std::vector<int> start;                  // nd
    std::vector<double> L, Linv;             // nd x nd
};
int build_pdamp(const ow3d_params& p, const GridHost& G, PDampHost& d, std::string* err);
void filter_coeffs(const ow3d_params& p, std::vector<double>& fc, std::vector<double>& F2);

int default_params(ow3d_params* p);
double fd_wavenumber(double hb, double omega, double grav);
struct Ran1 {
    int iv[32] = {0};
    int iy = 0;
    float next(int& idum);
};
int incident_wave_samples(const ow3d_params& p);
int read_bathymetry(const ow3d_params& p, const char* path, double* h, double* hx, double* hxx, double* hy,
                    double* hyy, int* flag_out, std::string* err);

// Stream-function wave of the deck's line 8 (sfwave.cpp): the solution
// vector z (1-based, 2N+10 unknowns), the elevation coefficients y (1..N),
// wavenumber, wavelength, period, phase speed and gravity.
struct SFWave {
    int n = 0;
    double k = 0, L = 0, T = 0, c = 0, g = 0;
    std::vector<double> z, y;
};
int stream_function_solve(const ow3d_params& p, SFWave& w, std::string* err);
void stream_function_eval(const SFWave& w, int nx, const double* x, double t, double* eta, double* phis);
int initial_condition(const ow3d_params& p, double* h, double* hx, double* hxx, double* hy, double* hyy, double* E,
                      double* P, std::string* err);
int incident_wave(const ow3d_params& p, int zone, int nt, double* eta, double* phis, int* box, std::string* err);

// The incident wave of a generation zone as its components, shared by the
// host synthesis (incident_wave) and the device kernels (incwave.cu). The
// series is evaluated on the zone box's points: long-crested waves on one x
// line (ny_eval = 1, repeated on the rows), waves at a heading on every row.
// The point (i, j) lies at dx[i], dy[j] from the wave's origin; the
// mono-chromatic wave is amp cos(nu d - omega t) with d = cosb dx + sinb dy
// and t = t0 + n dt; a random wave is, at sample n,
//   sum_{k=1}^{kmax-1} Re(c_k e^(i nu_k d_k) e^(-2 pi i k n / N)),
// d_k = kcos_k dx + ksin_k dy for spread seas (kcos non-empty), else d, and
// its surface potential likewise with (g / (k domega)) (-i) c_k.
struct IncidentWave {
    int bx = 0, by = 0, nt = 0, ny_eval = 1, N = 0, kmax = 0;
    bool heading = false, mono = false;
    double cosb = 1, sinb = 0, g = 9.81;
    double omega = 0, nu = 0, amp = 0, phifact = 0, t0 = 0, dt = 0;   // mono-chromatic
    double domega = 0;
    std::vector<double> dx, dy;
    std::vector<std::complex<double>> c;   // [kmax]
    std::vector<double> nus, kcos, ksin;   // [kmax] ([N/2] for kcos, ksin)
};
// With query_only non-null the call only fills box (any deck) and sets *query_only.
int incident_wave_setup(const ow3d_params& p, int zone, int nt, IncidentWave& w, int* box, bool* query_only,
                        std::string* err);
int read_deck(const char* path, ow3d_params* p, std::string* err);

}  // namespace ow3d
