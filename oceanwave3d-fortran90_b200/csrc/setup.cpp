// Host-side set-up: deck parsing, grid, finite-difference stencils, the
// multigrid hierarchy metadata, relaxation zones and Savitzky-Golay filter
// coefficients. Everything here runs once per simulation; the per-step work
// is on the device.
#include "setup.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace ow3d {

// ------------------------------------------------------------- stencils
// Finite-difference weights on arbitrary nodes by Fornberg's recurrence
// (B. Fornberg, Math. Comp. 51 (1988) 699-706), the algorithm of the
// reference's `weights` routine (src/utilities/stream_func_wave_finite.f:128-168).
// Returns the weights of derivative `order` at z on nodes x[0..n].
void fd_weights(double z, const double* x, int n, int order, double* w) {
    const int M = order;
    std::vector<double> c((size_t)(n + 1) * (M + 1), 0.0);
    auto C = [&](int j, int k) -> double& { return c[(size_t)j * (M + 1) + k]; };
    double c1 = 1.0, c4 = x[0] - z;
    C(0, 0) = 1.0;
    for (int i = 1; i <= n; ++i) {
        const int mn = std::min(i, M);
        double c2 = 1.0;
        const double c5 = c4;
        c4 = x[i] - z;
        for (int j = 0; j < i; ++j) {
            const double c3 = x[i] - x[j];
            c2 *= c3;
            if (j == i - 1) {
                for (int k = mn; k >= 1; --k) C(i, k) = c1 * (k * C(i - 1, k - 1) - c5 * C(i - 1, k)) / c2;
                C(i, 0) = -c1 * c5 * C(i - 1, 0) / c2;
            }
            for (int k = mn; k >= 1; --k) C(j, k) = (c4 * C(j, k) - k * C(j, k - 1)) / c3;
            C(j, 0) = c4 * C(j, 0) / c3;
        }
        c1 = c2;
    }
    for (int j = 0; j <= n; ++j) w[j] = C(j, M);
}

// x / y stencils: window of 2a+1 nodes centred on the point, shifted inwards at
// the first and last a points (BuildStencilsGridX.f90:162-196). The grids are
// uniform, so the nodes are taken at their exact offsets q*dx from the point
// (q an integer): every row with the same window shift gets bitwise the same
// weights, which lets the device keep one centred stencil for all interior
// points. The reference forms the offsets from absolute coordinates, which
// perturbs the weights row by row at the level of rounding only (about 1e-13
// relative at x ~ 50 m). A grid that is not uniform to 1e-12 takes the
// absolute coordinates.
Stencil stencils_xy(const std::vector<double>& x, int a) {
    Stencil s;
    s.n = (int)x.size();
    s.rank = 2 * a + 1;
    s.w.assign((size_t)2 * s.n * s.rank, 0.0);
    if (s.n == 1 || a == 0) return s;
    const double dx = (x[(size_t)s.n - 1] - x[0]) / (double)(s.n - 1);
    bool uniform = dx > 0.0;
    for (int i = 0; i < s.n && uniform; ++i)
        uniform = std::fabs(x[(size_t)i] - (x[0] + dx * i)) <= 1e-12 * std::fabs(dx) * s.n;
    std::vector<double> nodes(s.rank), w(s.rank);
    for (int order = 1; order <= 2; ++order)
        for (int i = 1; i <= s.n; ++i) {
            const int shift = (i - 1 < a) ? a - i + 1 : (i >= s.n - a + 1 ? (s.n - a) - i : 0);
            for (int m = 0; m < s.rank; ++m)
                nodes[m] = uniform ? (double)(m - a + shift) * dx : x[(size_t)(i + m - a + shift - 1)];
            fd_weights(uniform ? 0.0 : x[i - 1], nodes.data(), s.rank - 1, order, w.data());
            std::copy(w.begin(), w.end(), s.w.begin() + ((size_t)(order - 1) * s.n + (i - 1)) * s.rank);
        }
    return s;
}

// Periodic direction (no counterpart in the reference): every position takes
// the centred stencil of half width a, from the exact offsets q*dx.
Stencil stencils_periodic(const std::vector<double>& x, int a) {
    Stencil s;
    s.n = (int)x.size();
    s.rank = 2 * a + 1;
    s.w.assign((size_t)2 * s.n * s.rank, 0.0);
    const double dx = (x[(size_t)s.n - 1] - x[0]) / (double)(s.n - 1);
    std::vector<double> nodes(s.rank), w(s.rank);
    for (int m = 0; m < s.rank; ++m) nodes[m] = (double)(m - a) * dx;
    for (int order = 1; order <= 2; ++order) {
        fd_weights(0.0, nodes.data(), s.rank - 1, order, w.data());
        for (int i = 0; i < s.n; ++i) std::copy(w.begin(), w.end(), s.w.begin() + ((size_t)(order - 1) * s.n + i) * s.rank);
    }
    return s;
}

// sigma stencils, one-sided near the free surface and the bottom ghost
// (PreProcessDiffStencils.f90:108-132).
Stencil stencils_z(const std::vector<double>& z, int Nz, int gz, int g) {
    Stencil s;
    const int Nzp = Nz + gz;
    s.n = Nzp;
    s.rank = 2 * g + 1;
    s.w.assign((size_t)2 * s.n * s.rank, 0.0);
    std::vector<double> nodes(s.rank), w(s.rank);
    for (int order = 1; order <= 2; ++order)
        for (int i = 1; i <= Nzp; ++i) {
            int left, off;  // expansion node index within the window, window offset
            if (i - 1 < g) { const int d = g - i + 1; left = g - d; off = d; }
            else if (i >= Nz - g + 1) { const int d = i - (Nzp - g); left = g + d; off = -d; }
            else { left = g; off = 0; }
            for (int m = 0; m < s.rank; ++m) nodes[m] = z[(size_t)(i + m - g + off - 1)];
            fd_weights(nodes[left], nodes.data(), s.rank - 1, order, w.data());
            std::copy(w.begin(), w.end(), s.w.begin() + ((size_t)(order - 1) * s.n + (i - 1)) * s.rank);
        }
    return s;
}

// ------------------------------------------------------------- hierarchy
// Level count: NINT(log2(max(Nx,Ny,Nz)-1)) in single precision (MGPreProcess.f90:449-458).
static int level_count(int nx, int ny, int nz) {
    const float nmax = (float)std::max(nx, std::max(ny, nz));
    return (int)std::lround(std::log10(nmax - 1.0f) / std::log10(2.0f));
}

static void coarsen_flags(int strategy, int nx, int ny, int nz, int& xc, int& yc, int& zc) {
    xc = yc = zc = 0;
    if (strategy == 1) {
        if (nx == ny && nx == nz) xc = yc = zc = 1;
        else if (nx > ny && nx > nz) xc = 1;
        else if (ny > nx && ny > nz) yc = 1;
        else if (nz > nx && nz > ny) zc = 1;
        else if (nx == ny && nx > nz) xc = yc = 1;
        else if (nx == nz && nx > ny) xc = zc = 1;
        else if (ny == nz && ny > nx) yc = zc = 1;
    } else if (strategy == 2) {
        xc = nx > 3; yc = ny > 3; zc = nz > 3;
    } else {  // MGPreProcess.f90:140-178
        if (nx == 1) { yc = 1; zc = (ny == nz); }
        else if (ny == 1) { xc = 1; zc = (nx == nz); }
        else if (nx == ny && nx == nz) xc = yc = zc = 1;
        else { xc = nx > nz; yc = ny > nz; zc = (nx < nz && ny < nz); }
    }
}

static void level_sigma(LevelHost& L) {
    L.zs = L.z;
    L.zs[0] = 0.0;  // DetermineTransformationConstantsArray.f90:59 (sigma = 0 below the bottom)
}

static void level_colours(LevelHost& L) {
    double m = 0;
    for (size_t c = 0; c < L.hx.size(); ++c) m = std::max(m, std::max(std::fabs(L.hx[c]), std::fabs(L.hy[c])));
    // Mixed-derivative terms couple diagonal neighbour columns; without them a
    // red-black colouring of the columns is a proper colouring.
    L.ncolor = (L.Nxg > 1 && L.Nyg > 1 && m > 0) ? 4 : 2;
}

bool breaking_on(const ow3d_params& p) { return p.i_breaking > 0 && p.Ny == 1 && p.Nx > 1; }

bool smoothing_on(const ow3d_params& p) {
    return p.accel_from_deck ? p.accel_tol_fact <= 100.0 : (p.accel_tol_fact > 0.0 && p.accel_tol_fact <= 100.0);
}

// Deck features that change the physics but lie outside this library's path:
// a deck that turns one on is refused (OW3D_ERR_UNSUPPORTED) rather than run
// without it. A raw IncWaveType 4 or 5 is the deck's code for what the parser
// stores as 1 or 3 plus current_flag (ReadInputFileParameters.f90:42-49).
int check_supported(const ow3d_params& p, std::string* err) {
    auto no = [&](const char* m) { if (err) *err = m; return OW3D_ERR_UNSUPPORTED; };
    if (p.IncWaveType == 4 || p.IncWaveType == 5)
        return no("IncWaveType 4 / 5: give IncWaveType 1 / 3 with current_flag = 1, as ow3d_read_deck reads them");
    if (p.PDampingONOFF != 0) {
        // BuildPDampMatrices.f90:37-40 stops for Ny > 1; the friction form
        // (type != 0) spreads its gamma over y lines inconsistently there
        if (p.Ny > 1 || p.Nx < 2) return no("pressure damping is built for x-directed zones of 2-D decks (Ny = 1)");
        if (p.NDampZones != 1) return no("one pressure-damping zone per deck (the reference stops on more)");
    }
    if (p.swenseONOFF != 0) return no("SWENSE is not built");
    if (p.curvilinearONOFF != 0 && p.Nx > 1 && p.Ny > 1) return no("curvilinear grids are not built");
    return 0;
}

int check_params(const ow3d_params& p, std::string* err) {
    auto fail = [&](const char* m) { if (err) *err = m; return OW3D_ERR_BAD_INPUT; };
    if (p.Nx < 1 || p.Ny < 1 || p.Nz < 3) return fail("Nx, Ny >= 1 and Nz >= 3 required");
    if (p.Nx == 1) return fail("Nx == 1 (2-D in y) is not supported; orient the flume along x");
    if (p.GhostGridZ != 1) return fail("GhostGridZ must be 1 (ReadInputFileParameters.f90:283-285)");
    if (p.Nx > 1 && p.GhostGridX != 1) return fail("GhostGridX must be 1");
    if (p.Ny > 1 && p.GhostGridY != 1) return fail("GhostGridY must be 1");
    if (p.alpha != 3 || (p.Ny > 1 && p.beta != 3) || p.gamma != 3) return fail("alpha = beta = gamma = 3 required");
    if (p.alphaprecond != 1 || (p.Ny > 1 && p.betaprecond != 1) || p.gammaprecond != 1)
        return fail("alphaprecond = betaprecond = gammaprecond = 1 required");
    if (p.Nz + 1 > 34) return fail("Nz must be at most 33 (32 interior sigma rows per multigrid column)");
    const int Nxg = p.Nx + 2, Nyg = p.Ny + (p.Ny > 1 ? 2 : 0), Nzg = p.Nz + 1;
    if (Nxg < 8 || (p.Ny > 1 && Nyg < 8) || Nzg < 8) return fail("at least 7 points per direction (6th-order stencils)");
    if (p.filteringONOFF > 0) {
        const int NP = 2 * p.filterALPHA + 1;
        if (p.filterALPHA < 1 || p.filterALPHA > 6) return fail("filterALPHA must be 1..6 (FilterInit.f90 boundary filters)");
        if (Nxg < NP + 2 || (p.Ny > 1 && Nyg < NP + 2)) return fail("grid too small for the filter width");
    }
    if ((double)Nxg * (double)Nyg * (double)Nzg >= 2147483647.0)
        return fail("grid too large: at most 2^31-1 unknowns per simulation (32-bit point indices)");
    if (p.precision != OW3D_PREC_FP64 && p.precision != OW3D_PREC_MIXED) return fail("precision must be 0 or 1");
    if (p.krylov != OW3D_KRYLOV_FGMRES && p.krylov != OW3D_KRYLOV_LGMRES) return fail("krylov must be 0 or 1");
    if (p.GMRESmaxiterations < 1) return fail("GMRESmaxiterations must be >= 1");
    if (p.IncWaveType == 3) {
        if (p.periodic_x != 0) return fail("periodic_x: the flux wavemaker is the west wall's flux");
        if (p.flux_order < 1 || p.flux_order > 10) return fail("flux wavemaker: interpolation order 1..10 required");
    }
    if (p.current_flag != 0 && p.current_Q != 0.0 && p.periodic_x != 0)
        return fail("periodic_x: the constant-flux current enters through the walls");
    if (smoothing_on(p) && p.periodic_x != 0)
        return fail("periodic_x: local smoothing by the vertical acceleration is built for wall boundaries");
    if (breaking_on(p)) {
        // the roller-angle update divides by T_half (DetectBreaking.f90:181)
        if (!(p.T_half > 0.0)) return fail("breaking model: T_half > 0 required");
        if (!(p.del_fac >= 0.0)) return fail("breaking model: f_delta >= 0 required");
        if (p.periodic_x != 0) return fail("periodic_x: the breaking model is built for wall boundaries");
    }
    if (p.periodic_x != 0) {
        if (p.Nx < 9) return fail("periodic_x: at least 8 distinct points per period (Nx >= 9)");
        if (p.PDampingONOFF != 0) return fail("periodic_x: pressure-damping zones need the wall boundaries");
        if (p.iKinematics != 0) return fail("periodic_x: the kinematics output is built for wall boundaries");
    }
    return 0;
}

int build_grid(const ow3d_params& p, const double* h, const double* hx, const double* hxx, const double* hy,
               const double* hyy, GridHost& G, std::string* err) {
    auto fail = [&](const char* m) { if (err) *err = m; return OW3D_ERR_BAD_INPUT; };
    if (int r = check_params(p, err)) return r;
    G.Nx = p.Nx; G.Ny = p.Ny; G.Nz = p.Nz;
    G.gx = 1; G.gy = (p.Ny > 1) ? 1 : 0; G.gz = 1;
    G.Nxg = p.Nx + 2 * G.gx; G.Nyg = p.Ny + 2 * G.gy; G.Nzg = p.Nz + G.gz;
    G.C = (int64_t)G.Nxg * G.Nyg; G.N = G.C * G.Nzg;
    G.three = (p.Ny > 1) ? 1 : 0;
    if (G.Nxg < 8 || (G.three && G.Nyg < 8) || G.Nzg < 8) return fail("at least 7 points per direction (6th-order stencils)");
    // SetupCompDomain.f90:35-79
    if (p.filteringONOFF > 0) {
        const int NP = 2 * p.filterALPHA + 1;
        if (p.filterALPHA < 1 || p.filterALPHA > 6) return fail("filterALPHA must be 1..6 (FilterInit.f90 boundary filters)");
        if (G.Nxg < NP + 2 || (G.three && G.Nyg < NP + 2)) return fail("grid too small for the filter width");
    }
    G.x.assign(G.Nxg, 0.0); G.y.assign(G.Nyg, p.Ly); G.z.assign(G.Nzg, 0.0);
    for (int i = -G.gx; i <= p.Nx - 1 + G.gx; ++i) G.x[i + G.gx] = (double)i / (double)(p.Nx - 1) * p.Lx;
    if (p.Ny > 1)
        for (int j = -G.gy; j <= p.Ny - 1 + G.gy; ++j) G.y[j + G.gy] = (double)j / (double)(p.Ny - 1) * p.Ly;
    const double pi = 3.14159265358979323846;
    for (int k = 0; k <= p.Nz - 1; ++k)
        G.z[k + 1] = (p.GridZ == 0) ? (double)k / (double)(p.Nz - 1) * p.Lz
                                    : std::sin(pi * (double)k / (double)(2 * (p.Nz - 1)));
    G.z[0] = -G.z[2];
    G.zs = G.z; G.zs[0] = 0.0;
    const size_t C = (size_t)G.C;
    auto cp = [&](const double* s, std::vector<double>& d) { d.assign(C, 0.0); if (s) std::copy(s, s + C, d.begin()); };
    cp(h, G.h); cp(hx, G.hx); cp(hxx, G.hxx); cp(hy, G.hy); cp(hyy, G.hyy);
    if (!h) return fail("bathymetry h is required");
    for (size_t c = 0; c < C; ++c) if (!(G.h[c] > 0)) return fail("depth h must be positive everywhere (ghosts included)");
    if (p.periodic_x != 0)
        for (size_t c = 0; c < C; ++c)
            if (G.hx[c] != 0.0 || G.hy[c] != 0.0) {
                if (err) *err = "periodic_x: a flat bottom (h_x = h_y = 0) is required";
                return OW3D_ERR_UNSUPPORTED;
            }
    G.per = p.periodic_x != 0 ? 1 : 0;
    G.SX = G.per ? stencils_periodic(G.x, 3) : stencils_xy(G.x, 3);
    G.SY = stencils_xy(G.y, G.three ? 3 : 0);
    G.SZ = stencils_z(G.z, p.Nz, 1, 3);
    // multigrid hierarchy (MGPreProcess.f90:31-318)
    G.levels.clear();
    if (p.Precond != 3) return 0;
    int L = level_count(p.Nx, p.Ny, p.Nz);
    if (L > p.MGmaxgrids && p.MGmaxgrids > 0) L = p.MGmaxgrids;
    if (L < 1) L = 1;
    if (L > kMaxLevelsHost) return fail("too many multigrid levels");
    G.levels.assign(L, LevelHost());
    LevelHost& F = G.levels[L - 1];
    F.Nx = p.Nx; F.Ny = p.Ny; F.Nz = p.Nz; F.Nxg = G.Nxg; F.Nyg = G.Nyg; F.Nzg = G.Nzg;
    F.x = G.x; F.y = G.y; F.z = G.z;
    F.h = G.h; F.hx = G.hx; F.hxx = G.hxx; F.hy = G.hy; F.hyy = G.hyy;
    for (int l = L - 2; l >= 0; --l) {
        const LevelHost& f = G.levels[l + 1];
        LevelHost& c = G.levels[l];
        int xc, yc, zc;
        coarsen_flags(p.MGCoarseningStrategy, f.Nx, f.Ny, f.Nz, xc, yc, zc);
        if (xc && f.Nx % 2 == 0) return fail("cannot coarsen in x: Nx must be odd (MGPreProcess.f90:184)");
        if (yc && f.Ny % 2 == 0) return fail("cannot coarsen in y: Ny must be odd");
        c.Nx = xc ? (f.Nx - 1) / 2 + 1 : f.Nx;
        c.Ny = yc ? (f.Ny - 1) / 2 + 1 : f.Ny;
        c.Nz = zc ? (f.Nz - 1) / 2 + 1 : f.Nz;
        if (zc && c.Nz % 2 == 0) return fail("cannot coarsen in z: Nz must be odd");
        c.xc = xc; c.yc = yc; c.zc = zc;
        const int XF = xc ? 2 : 1, YF = yc ? 2 : 1, ZF = zc ? 2 : 1;
        c.Nxg = c.Nx + 2 * G.gx; c.Nyg = c.Ny + 2 * G.gy; c.Nzg = c.Nz + 1;
        c.x.assign(c.Nxg, 0.0);
        for (int i = 2; i <= c.Nxg - 1; ++i) c.x[i - 1] = f.x[(size_t)(2 + (i - 2) * XF - 1)];
        c.x[0] = c.x[1] - (c.x[2] - c.x[1]);
        c.x[c.Nxg - 1] = c.x[c.Nxg - 2] + (c.x[c.Nxg - 2] - c.x[c.Nxg - 3]);
        c.y.assign(c.Nyg, p.Ly);
        if (G.three) {
            for (int j = 2; j <= c.Nyg - 1; ++j) c.y[j - 1] = f.y[(size_t)(2 + (j - 2) * YF - 1)];
            c.y[0] = c.y[1] - (c.y[2] - c.y[1]);
            c.y[c.Nyg - 1] = c.y[c.Nyg - 2] + (c.y[c.Nyg - 2] - c.y[c.Nyg - 3]);
        }
        c.z.assign(c.Nzg, 0.0);
        c.z[0] = -f.z[(size_t)(2 + ZF - 1)];
        for (int k = 2; k <= c.Nzg; ++k) c.z[k - 1] = f.z[(size_t)(2 + (k - 2) * ZF - 1)];
        const size_t Cc = (size_t)c.Nxg * c.Nyg;
        c.h.assign(Cc, 0.0); c.hx.assign(Cc, 0.0); c.hxx.assign(Cc, 0.0); c.hy.assign(Cc, 0.0); c.hyy.assign(Cc, 0.0);
        for (int j = 1 + G.gy; j <= c.Nyg - G.gy; ++j)
            for (int i = 2; i <= c.Nxg - 1; ++i) {
                const int fi = 2 + (i - 2) * XF, fj = G.gy ? 2 + (j - 2) * YF : 1;
                const size_t cc = (size_t)(i - 1) + (size_t)c.Nxg * (j - 1);
                const size_t ff = (size_t)(fi - 1) + (size_t)f.Nxg * (fj - 1);
                c.h[cc] = f.h[ff]; c.hx[cc] = f.hx[ff]; c.hxx[cc] = f.hxx[ff]; c.hy[cc] = f.hy[ff]; c.hyy[cc] = f.hyy[ff];
            }
        // depth on the ghost points copied from the adjacent interior (MGPreProcess.f90:311-314)
        for (int j = 1; j <= c.Nyg; ++j) {
            c.h[(size_t)c.Nxg * (j - 1)] = c.h[1 + (size_t)c.Nxg * (j - 1)];
            c.h[(size_t)(c.Nxg - 1) + (size_t)c.Nxg * (j - 1)] = c.h[(size_t)(c.Nxg - 2) + (size_t)c.Nxg * (j - 1)];
        }
        for (int i = 1; i <= c.Nxg; ++i) {
            c.h[(size_t)(i - 1)] = c.h[(size_t)(i - 1) + (size_t)c.Nxg * (1 + G.gy - 1)];
            c.h[(size_t)(i - 1) + (size_t)c.Nxg * (c.Nyg - 1)] = c.h[(size_t)(i - 1) + (size_t)c.Nxg * (c.Nyg - G.gy - 1)];
        }
    }
    for (auto& Lv : G.levels) {
        level_sigma(Lv);
        level_colours(Lv);
        Lv.SX = G.per ? stencils_periodic(Lv.x, 1) : stencils_xy(Lv.x, 1);
        Lv.SY = stencils_xy(Lv.y, G.three ? 1 : 0);
        Lv.SZ = stencils_z(Lv.z, Lv.Nz, 1, 1);
        if (Lv.Nxg < 4 || (G.three && Lv.Nyg < 4) || Lv.Nzg < 4) return fail("multigrid level too small");
    }
    return 0;
}

// ------------------------------------------------------- relaxation zones
// PreprocessRelaxationZones.f90 (TracePosition) + GammaFunctions.f90:20-35.
static int trace_position(const std::vector<double>& x, double x0) {
    for (size_t i = 0; i < x.size(); ++i) if (x0 <= x[i]) return (int)i + 1;
    return (int)x.size();
}
static std::vector<double> gamma_fn(const double* x, int n, int dir, int ftype, double param) {
    std::vector<double> g(n), t(n);
    for (int i = 0; i < n; ++i) t[i] = (n > 1) ? (x[i] - x[0]) / (x[n - 1] - x[0]) : x[i];
    const double e1 = std::exp(1.0) - 1.0;
    for (int i = 0; i < n; ++i) {
        const double q = (n > 1) ? (x[i] - x[n - 1]) / (x[n - 1] - x[0]) : 0.0;
        switch (std::abs(ftype)) {
            case 9: g[i] = 1.0 - std::pow(t[i], param); break;
            case 10: g[i] = 3.0 * t[i] * t[i] - 2.0 * t[i] * t[i] * t[i]; break;
            case 11: g[i] = (std::exp(std::pow(t[i], param)) - 1.0) / e1; break;
            case 12: g[i] = std::exp(-q * q / (2.0 * param * param)); break;
            case 13: g[i] = 1.0 - std::exp(-q * q / (2.0 * param * param)); break;
            case 14: g[i] = 1.0 - (std::exp(std::pow(t[i], param)) - 1.0) / e1; break;
            default: g[i] = 1.0;
        }
    }
    if (dir == -1) std::reverse(g.begin(), g.end());
    return g;
}
// ------------------------------------------------- pressure-damping zone
// PreprocessPDampingZones.f90:24-70 and BuildPDampMatrices.f90:17-86 for the
// one zone of a 2-D deck.
int build_pdamp(const ow3d_params& p, const GridHost& G, PDampHost& d, std::string* err) {
    d = PDampHost{};
    if (p.PDampingONOFF == 0) return 0;
    auto bad = [&](const char* m) { if (err) *err = m; return OW3D_ERR_BAD_INPUT; };
    const int nx = (int)G.x.size();
    const int i1 = trace_position(G.x, p.pd_x0), i2 = trace_position(G.x, p.pd_x1);
    if (i2 < i1) return bad("pressure-damping zone: x1 < x0");
    const int nd = i2 - i1 + 1;
    d.type = p.pd_type; d.i1 = i1; d.nd = nd;
    // Gaussian gamma (GammaFunctions.f90 type 12, parameter 0.25): 1 at the
    // zone's last point
    const std::vector<double> gt = gamma_fn(&G.x[(size_t)i1 - 1], nd, 1, 12, 0.25);
    const double two_pi = 2.0 * M_PI;
    d.gamPhi.assign((size_t)nx, 0.0); d.gamEta.assign((size_t)nx, 0.0);
    for (int i = 0; i < nd; ++i) {
        d.gamPhi[(size_t)i1 - 1 + i] = two_pi * p.pd_g0Phi * gt[(size_t)i];
        d.gamEta[(size_t)i1 - 1 + i] = two_pi * p.pd_g0Eta * gt[(size_t)i];
    }
    if (d.type != 0) return 0;
    const int a = p.alpha, rank = 2 * a + 1;
    d.rank = rank;
    if (nd < rank) return bad("pressure-damping zone: a type-0 zone needs at least 2*alpha+1 points");
    // 1st and 2nd derivative weights on nd nodes: the reference takes the
    // first nd nodes of the row, x(1:nd) (BuildPDampMatrices.f90:25), which
    // on these uniform grids gives the weights of the zone's own nodes
    const Stencil s = stencils_xy(std::vector<double>(G.x.begin(), G.x.begin() + nd), a);
    auto w = [&](int order, int i, int m) { return s.w[((size_t)(order - 1) * nd + i) * rank + m]; };
    d.D1.resize((size_t)nd * rank); d.start.resize((size_t)nd);
    for (int i = 0; i < nd; ++i) {
        d.start[(size_t)i] = (i < a) ? 0 : (i >= nd - a ? nd - rank : i - a);
        for (int m = 0; m < rank; ++m) d.D1[(size_t)i * rank + m] = w(1, i, m);
    }
    // Dirichlet at the first point, the Laplacian inside, Neumann at the last
    d.L.assign((size_t)nd * nd, 0.0);
    d.L[0] = 1.0;
    for (int r = 1; r < nd; ++r)
        for (int m = 0; m < rank; ++m)
            d.L[(size_t)r * nd + d.start[(size_t)r] + m] = (r == nd - 1) ? w(1, r, m) : w(2, r, m);
    // its inverse: LU with partial pivoting confined to the band (kl below
    // the diagonal, kl + ku above after row exchanges), then nd solves
    int kl = 0, ku = 0;
    for (int r = 1; r < nd; ++r) {
        kl = std::max(kl, r - d.start[(size_t)r]);
        ku = std::max(ku, d.start[(size_t)r] + rank - 1 - r);
    }
    const int ub = kl + ku;
    std::vector<double> A = d.L;
    std::vector<int> piv((size_t)nd);
    for (int k = 0; k < nd; ++k) {
        const int rmax = std::min(nd - 1, k + kl), cmax = std::min(nd - 1, k + ub);
        int pr = k;
        for (int r = k + 1; r <= rmax; ++r)
            if (std::fabs(A[(size_t)r * nd + k]) > std::fabs(A[(size_t)pr * nd + k])) pr = r;
        piv[(size_t)k] = pr;
        if (A[(size_t)pr * nd + k] == 0.0) return bad("pressure-damping zone: the zone Laplacian is singular");
        if (pr != k)
            for (int c = k; c <= cmax; ++c) std::swap(A[(size_t)k * nd + c], A[(size_t)pr * nd + c]);
        const double pv = A[(size_t)k * nd + k];
        for (int r = k + 1; r <= rmax; ++r) {
            const double f = A[(size_t)r * nd + k] / pv;
            A[(size_t)r * nd + k] = f;
            if (f != 0.0)
                for (int c = k + 1; c <= cmax; ++c) A[(size_t)r * nd + c] -= f * A[(size_t)k * nd + c];
        }
    }
    d.Linv.assign((size_t)nd * nd, 0.0);
    std::vector<double> b((size_t)nd);
    for (int col = 0; col < nd; ++col) {
        std::fill(b.begin(), b.end(), 0.0);
        b[(size_t)col] = 1.0;
        for (int k = 0; k < nd; ++k) {
            std::swap(b[(size_t)k], b[(size_t)piv[(size_t)k]]);
            const double bk = b[(size_t)k];
            if (bk != 0.0)
                for (int r = k + 1; r <= std::min(nd - 1, k + kl); ++r) b[(size_t)r] -= A[(size_t)r * nd + k] * bk;
        }
        for (int k = nd - 1; k >= 0; --k) {
            double acc = b[(size_t)k];
            for (int c = k + 1; c <= std::min(nd - 1, k + ub); ++c) acc -= A[(size_t)k * nd + c] * b[(size_t)c];
            b[(size_t)k] = acc / A[(size_t)k * nd + k];
        }
        for (int r = 0; r < nd; ++r) d.Linv[(size_t)r * nd + col] = b[(size_t)r];
    }
    return 0;
}

std::vector<ZoneHost> build_zones(const ow3d_params& p, const GridHost& G) {
    std::vector<ZoneHost> out;
    if (p.relaxONOFF != 1) return out;
    for (int z = 0; z < p.relaxNo && z < OW3D_MAX_ZONES; ++z) {
        const ow3d_zone& d = p.zones[z];
        ZoneHost Z;
        Z.i0 = Z.i1 = Z.j0 = Z.j1 = 1;
        if (p.Nx > 1) { Z.i0 = trace_position(G.x, d.x1); Z.i1 = trace_position(G.x, d.x2); }
        if (p.Ny > 1) { Z.j0 = trace_position(G.y, d.y1); Z.j1 = trace_position(G.y, d.y2); }
        Z.xdir = (d.XorY == 'X' || d.XorY == 'x');
        Z.wavegen = d.WavegenONOFF;
        Z.phion = d.PhiOnOff;
        const int dir = d.ftype >= 0 ? 1 : -1;
        if (Z.xdir) Z.gam = gamma_fn(&G.x[(size_t)Z.i0 - 1], Z.i1 - Z.i0 + 1, dir, d.ftype, d.param);
        else Z.gam = gamma_fn(&G.y[(size_t)Z.j0 - 1], Z.j1 - Z.j0 + 1, dir, d.ftype, d.param);
        out.push_back(Z);
    }
    return out;
}

// ------------------------------------------------------ incident linear wave
// Finite-depth wavenumber of angular frequency omega in depth hb, with the
// steps of the reference's fdwvnum (src/utilities/fdwvnum.f90:14-45): an
// explicit first guess for the root of r tanh r = h (h = hb omega^2/g) and,
// for h <= 4.8, one correction; the shallow and deep limits outside
// 1e-5 < h < 1e5. Kept step for step so that the incident wave has the
// reference's wavenumber to the last bit.
double fd_wavenumber(double hb, double omega, double grav) {
    const double kinf = omega * omega / grav;
    const double h = hb * kinf;
    if (h < 1e-5) return omega / std::sqrt(grav * hb);
    if (h > 1e5) return kinf;
    const double hi = 1.0 / h, twoh = h + h, hh = h * h;
    const double e2h = std::exp(-std::min(twoh, 30.0));
    double r0h = (h <= 2.0) ? std::sqrt(h) * ((0.031 * h + 0.169) * h + 1.0) : h + h * e2h * (2.0 - 12.0 * e2h);
    if (h <= 4.8) {
        const double rh = hh - r0h * r0h;
        const double sh = 1.0 / (h - rh);
        const double fh = sh * (0.5 * std::log((r0h + h) / (r0h - h)) - r0h);
        r0h = r0h - fh * rh * (1.0 + fh * r0h * h * sh);
    }
    return r0h * hi * kinf;
}

// Park and Miller's minimal standard generator (x <- 16807 x mod 2^31-1, by
// Schrage's factorisation) with the Bays-Durham shuffle over 32 entries, in
// the form of the reference's RAN1_b (src/utilities/RAN1_b.f90:1-36): a
// non-positive idum (re)starts the sequence, the deviate is single precision
// and kept below 1. The state persists between calls like the routine's SAVE.
float Ran1::next(int& idum) {
    const int ia = 16807, im = 2147483647, iq = 127773, ir = 2836, ntab = 32, ndiv = 1 + (im - 1) / ntab;
    const float am = 1.0f / (float)im, rnmx = 1.0f - 1.2e-7f;
    if (idum <= 0 || iy == 0) {
        idum = std::max(-idum, 1);
        for (int j = ntab + 8; j >= 1; --j) {
            const int k = idum / iq;
            idum = ia * (idum - k * iq) - ir * k;
            if (idum < 0) idum += im;
            if (j <= ntab) iv[j - 1] = idum;
        }
        iy = iv[0];
    }
    const int k = idum / iq;
    idum = ia * (idum - k * iq) - ir * k;
    if (idum < 0) idum += im;
    const int j = 1 + iy / ndiv;
    iy = iv[j - 1];
    iv[j - 1] = idum;
    return std::min(am * (float)iy, rnmx);
}

namespace {
// PM_spectrum.f90:9-21 (T02 = 0.71 Tp with 0.71 a single-precision constant)
double pm_spectrum(double f, double Hs, double Tp) {
    const double pi = std::acos(-1.0);
    const double T02 = (double)0.71f * Tp;
    const double A = Hs * Hs / (4.0 * pi * std::pow(T02, 4)), B = 1.0 / (pi * std::pow(T02, 4));
    return f <= 0.0 ? 0.0 : A / std::pow(f, 5) * std::exp(-B / std::pow(f, 4));
}
// JONSWAP_spectrum.f90:8-29 (g = 9.82 there)
double jonswap_spectrum(double f, double Hs, double Tp, double gamma) {
    const double pi = std::acos(-1.0), grav = 9.82;
    const double fp = 1.0 / Tp;
    const double alpha = 3.32285 * Hs * Hs * std::pow(fp, 4);
    const double A = alpha * grav * grav / std::pow(2.0 * pi, 4), B = 5.0 / 4.0 * std::pow(fp, 4);
    if (f <= 0.0) return 0.0;
    const double sigma = f <= fp ? 0.07 : 0.09;
    const double a = std::exp(-0.5 * std::pow((f - fp) / (sigma * fp), 2));
    return A / std::pow(f, 5) * std::exp(-B / std::pow(f, 4)) * std::pow(gamma, a);
}
// Headings (radians) of the ncta frequency components of a cos^(2 s0)
// spread sea, drawn from the generator by the inverse of the tabulated
// cumulative distribution (spreading.f90:1-89). beta0 enters as the
// reference passes it (in degrees, used as radians there). A deviate above
// the table's last value takes the last heading (the reference reads past
// its table there).
std::vector<double> spread_headings(Ran1& rng, int& seed2, double s0, double beta0, int ncta) {
    const double pi = std::acos(-1.0);
    const double ipow = 2.0 * s0;
    const double ctamax = beta0 + 0.5 * pi, ctamin = beta0 - 0.5 * pi;
    const double dcta1 = (ctamax - ctamin) / (double)(float)(ncta - 1);
    double sum1 = 0.0;
    for (int i = 1; i <= ncta; ++i) {
        const double aaa = ctamin + (i - 1) * dcta1;
        sum1 = sum1 + std::pow(std::cos((aaa - beta0) / 2.0), ipow) * dcta1;
    }
    const double spm = 1.0 / sum1;
    std::vector<double> cta((size_t)ncta + 1), cosint((size_t)ncta + 1);
    double ds = 0.0;
    const double dcta = pi / (double)(float)ncta;
    for (int i = 1; i <= ncta; ++i) {
        cta[(size_t)i] = ctamin + (i - 1) * dcta;
        ds = ds + std::pow(std::cos((cta[(size_t)i] - beta0) / 2.0), ipow) * dcta;
        cosint[(size_t)i] = ds * spm;
    }
    std::vector<double> beta((size_t)ncta + 1, 0.0);
    for (int j = 1; j <= ncta; ++j) {
        const double ps = (double)rng.next(seed2);
        int i = 1;
        while (i <= ncta && !(cosint[(size_t)i] >= ps)) ++i;
        beta[(size_t)j] = cta[(size_t)std::min(i, ncta)];
    }
    return beta;   // 1-based
}

// erf^-1(p) for 0 <= p < 1: a first guess from the asymptotic form
// sqrt(-log(1-p)) blended with the series p sqrt(pi)/2, refined by Newton
// steps on erf(x) - p (the reference's InvErf, a rational approximation of
// Blair, Edwards and Johnson 1976, returns the same root to rounding).
double inverse_erf(double p) {
    if (p <= 0.0) return 0.0;
    const double spi = std::sqrt(std::acos(-1.0));
    double x = p < 0.7 ? 0.5 * spi * p * (1.0 + std::acos(-1.0) / 12.0 * p * p)
                       : std::sqrt(-std::log((1.0 - p) * spi)) ;
    for (int it = 0; it < 60; ++it) {
        const double f = std::erf(x) - p;
        const double d = 2.0 / spi * std::exp(-x * x);
        const double step = f / d;
        x -= step;
        if (std::fabs(step) <= 1e-16 * std::max(1.0, std::fabs(x))) break;
    }
    return x;
}

// In-place radix-2 transform X_j = sum_k Z_k exp(-2 pi i j k / n), n a power of two.
void fft_minus(std::vector<std::complex<double>>& Z) {
    const size_t n = Z.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(Z[i], Z[j]);
    }
    const double pi = std::acos(-1.0);
    for (size_t len = 2; len <= n; len <<= 1) {
        for (size_t i = 0; i < n; i += len)
            for (size_t q = 0; q < len / 2; ++q) {
                const double a = -2.0 * pi * (double)q / (double)len;
                const std::complex<double> w(std::cos(a), std::sin(a));
                const std::complex<double> u = Z[i + q], v = Z[i + q + len / 2] * w;
                Z[i + q] = u + v;
                Z[i + q + len / 2] = u - v;
            }
    }
}
}  // namespace

// Samples of the incident wave the reference builds: nt_ref = Nsteps for the
// mono-chromatic wave, else the power of two at or above Nsteps
// (OceanWave3DT0Setup.f90:178-191).
int incident_wave_samples(const ow3d_params& p) {
    if (p.ispec < 0) return p.Nsteps;
    int i = (int)std::lround(std::log((double)p.Nsteps) / std::log(2.0));
    if (std::pow(2.0, i) < p.Nsteps) ++i;
    return 1 << std::max(i, 1);
}

// The incident wave of IncWaveType 2 on the box of generation zone `zone`,
// the x-directed line replicated over the zone's rows as
// RelaxationModule_new.f90:104-112 applies it:
//  * ispec -1 (random_wave_signal.f90:151-172): eta = H/2 cos(nu (x - x0) -
//    omega t), phiS = g/omega H/2 sin(...), t = time0 + n dt;
//  * ispec 0 (P-M), 1 and 3 (JONSWAP) (build_coeff.f90:19-63,
//    random_wave_coefficients.f90:53-100, random_wave_signal.f90:48-150):
//    coefficients c_k = sqrt(2 S(f_k) df) e^(2 pi i psi_k), psi_k from the
//    generator above seeded with seed2 (the phase rounded to single precision
//    as CMPLX does), truncated at kh_max, moved to x by e^(i nu_k (x - x0)),
//    and summed over the N = nt_ref samples t = n dt as the inverse real
//    transform does: eta_n = sum_k Re(c_k e^(i nu_k d) e^(-2 pi i k n / N)),
//    phiS likewise with g/omega_k (-i) c_k.
int incident_wave_setup(const ow3d_params& p, int zone, int nt, IncidentWave& w, int* box, bool* query_only,
                        std::string* err) {
    auto fail = [&](const std::string& m, int code) { if (err) *err = m; return code; };
    if (query_only) *query_only = false;
    if (p.relaxONOFF != 1 || zone < 0 || zone >= p.relaxNo || zone >= OW3D_MAX_ZONES)
        return fail("incident_wave: no such relaxation zone", OW3D_ERR_BAD_INPUT);
    const ow3d_zone& d = p.zones[zone];
    if (!(d.XorYgen == 'X' || d.XorYgen == 'x') || d.WavegenONOFF != 1)
        return fail("incident_wave: zone " + std::to_string(zone) + " is not an x-directed generation zone",
                    OW3D_ERR_BAD_INPUT);
    int r = check_params(p, err);
    if (r) return r;
    GridHost G;
    const int Nxg = p.Nx + (p.Nx > 1 ? 2 : 0), Nyg = p.Ny + (p.Ny > 1 ? 2 : 0);
    std::vector<double> ones((size_t)Nxg * Nyg, 1.0), zeros(ones.size(), 0.0);
    r = build_grid(p, ones.data(), zeros.data(), zeros.data(), zeros.data(), zeros.data(), G, err);
    if (r) return r;
    const std::vector<ZoneHost> Z = build_zones(p, G);
    const ZoneHost& z = Z[(size_t)zone];
    const int nref = incident_wave_samples(p);
    if (box) { box[0] = z.i0; box[1] = z.i1; box[2] = z.j0; box[3] = z.j1; box[4] = nref; }
    if (query_only) { *query_only = true; return OW3D_OK; }
    if (p.IncWaveType != 2) return fail("incident_wave: the deck's IncWaveType is not 2", OW3D_ERR_BAD_INPUT);
    if (!(p.ispec == -1 || p.ispec == 0 || p.ispec == 1 || p.ispec == 3 || p.ispec == -30 || p.ispec == 30 ||
          p.ispec == 31 || p.ispec == 33 || p.ispec == 34))
        return fail("incident_wave: ispec " + std::to_string(p.ispec) +
                        " (waves from a file) is not supported; -1, 0, 1, 3, -30, 30, 31, 33 and 34 are",
                    OW3D_ERR_UNSUPPORTED);
    if (std::abs(p.ispec) >= 30 && d.degrees != 0.0)   // ReadInputFileParameters.f90:710-714
        return fail("incident_wave: waves at a heading need a zone with degrees = 0", OW3D_ERR_BAD_INPUT);
    if (nt < 1 || !(p.Tp > 0) || !(p.h0 > 0) || !(p.dt > 0) || p.Nsteps < 1)
        return fail("incident_wave: bad arguments", OW3D_ERR_BAD_INPUT);
    if (p.ispec >= 0 && nt > nref)
        return fail("incident_wave: a random wave has " + std::to_string(nref) + " samples", OW3D_ERR_BAD_INPUT);
    const double pi = std::acos(-1.0), two = 2.0, twopi = two * pi;
    w = IncidentWave{};
    w.bx = z.i1 - z.i0 + 1;
    w.by = z.j1 - z.j0 + 1;
    w.nt = nt;
    w.g = p.g;
    // long-crested along x (|ispec| < 30): one x line, repeated on the rows;
    // at heading beta0 (random_wave_signal_3D.f90): every point of the box
    w.heading = std::abs(p.ispec) >= 30;
    w.ny_eval = w.heading ? w.by : 1;
    w.cosb = w.heading ? std::cos(pi / 180.0 * p.beta0) : 1.0;
    w.sinb = w.heading ? std::sin(pi / 180.0 * p.beta0) : 0.0;
    w.dx.resize((size_t)w.bx);
    w.dy.assign((size_t)w.ny_eval, 0.0);
    for (int i = 0; i < w.bx; ++i) w.dx[(size_t)i] = G.x[(size_t)(z.i0 - 1 + i)] - p.x0;
    if (w.heading)
        for (int j = 0; j < w.ny_eval; ++j) w.dy[(size_t)j] = G.y[(size_t)(z.j0 - 1 + j)] - p.y0;
    if (p.ispec < 0) {
        w.mono = true;
        w.omega = twopi / p.Tp;
        w.nu = fd_wavenumber(p.h0, w.omega, p.g);
        w.amp = p.Hs / two;
        w.phifact = p.g / w.omega;
        w.t0 = p.time0;
        w.dt = p.dt;
        return OW3D_OK;
    }
    const int N = nref;
    w.N = N;
    const double df = 1.0 / (N * p.dt), cst = std::sqrt(df);
    w.domega = twopi / (N * p.dt);
    const bool pm = (p.ispec == 0 || p.ispec == 30);   // the others: JONSWAP
    std::vector<std::complex<double>> c((size_t)N / 2, 0.0);
    std::vector<double>& kcos = w.kcos;
    std::vector<double>& ksin = w.ksin;
    Ran1 rng;
    int seed2 = p.seed2;
    if (p.ispec == 34) {
        // build_coeff_3D_Cos.f90:38-52: the headings take the first N/2
        // deviates; converted to degrees and back for the phase
        const std::vector<double> b = spread_headings(rng, seed2, p.s0, p.beta0, N / 2);
        kcos.assign((size_t)N / 2, 0.0); ksin.assign((size_t)N / 2, 0.0);
        const double rad2deg = 1.0 / (pi / 180.0), deg2rad = pi / 180.0;
        for (int k = 1; k < N / 2; ++k) {
            const double deg = b[(size_t)(k + 1)] * rad2deg;   // beta(i) with i = k + 1
            kcos[(size_t)k] = std::cos(deg2rad * deg);
            ksin[(size_t)k] = std::sin(deg2rad * deg);
        }
    }
    for (int i = 2; i <= N / 2; ++i) {
        const double freq = (i - 1) * df;
        const double psi = (double)rng.next(seed2);
        const float cr = (float)std::cos(twopi * psi), ci = (float)std::sin(twopi * psi);
        const double spec = pm ? pm_spectrum(freq, p.Hs, p.Tp) : jonswap_spectrum(freq, p.Hs, p.Tp, p.gamma_jonswap);
        const double a = std::sqrt(two * spec) * cst;
        c[(size_t)(i - 1)] = std::complex<double>(a * (double)cr, a * (double)ci);
        if (p.ispec == 33) {
            // build_coeff_3D.f90:44-58: a normally spread heading from the
            // same deviate; the reference's InvErf returns -1 for a
            // negative argument (ErfReal.f90:406-409), kept as it is
            const double rad2deg = 180.0 / pi, fp = 1.0 / p.Tp;
            const double sigma = 0.2 * std::pow(freq / fp, 2.5);
            const double erf1 = std::erf(pi / (two * std::sqrt(two * sigma)));
            const double arg = (two * psi - 1.0) * erf1;
            const double erf2 = arg >= 0.0 ? inverse_erf(arg) : -1.0;
            const double deg = p.beta0 + rad2deg * std::sqrt(2.0 * sigma) * erf2;
            if (kcos.empty()) { kcos.assign((size_t)N / 2, 0.0); ksin.assign((size_t)N / 2, 0.0); }
            kcos[(size_t)(i - 1)] = std::cos(pi / 180.0 * deg);
            ksin[(size_t)(i - 1)] = std::sin(pi / 180.0 * deg);
        }
    }
    // truncation at kh_max (random_wave_coefficients.f90:92-100): the
    // coefficients from index n_cut - 1 on are zero
    const int n_cut = (int)std::lround(std::sqrt(p.g * p.kh_max / p.h0 * std::tanh(p.kh_max)) / w.domega) + 1;
    for (int k = std::max(n_cut - 1, 1); k < N / 2; ++k) c[(size_t)k] = 0.0;
    w.kmax = std::min(n_cut, N / 2);
    w.c.assign(c.begin(), c.begin() + std::max(w.kmax, 1));
    w.nus.assign((size_t)std::max(w.kmax, 1), 0.0);
    for (int k = 1; k < w.kmax; ++k) w.nus[(size_t)k] = fd_wavenumber(p.h0, k * w.domega, p.g);
    return OW3D_OK;
}

int incident_wave(const ow3d_params& p, int zone, int nt, double* eta, double* phis, int* box, std::string* err) {
    IncidentWave w;
    bool query = false;
    const int r = incident_wave_setup(p, zone, nt, w, box, (!eta && !phis) ? &query : nullptr, err);
    if (r || query) return r;   // the box query works for every deck
    const int bx = w.bx, by = w.by, ny_eval = w.ny_eval;
    std::vector<double> le((size_t)nt * bx * ny_eval), lp(le.size());   // [n][j][i]
    auto at = [&](int n, int j, int i) { return ((size_t)n * ny_eval + j) * bx + i; };
    auto dist_of = [&](int i, int j) { return w.cosb * w.dx[(size_t)i] + w.sinb * w.dy[(size_t)j]; };
    if (w.mono) {
        // random_wave_signal.f90:151-172
        for (int n = 0; n < nt; ++n) {
            const double t = w.t0 + n * w.dt;
            for (int j = 0; j < ny_eval; ++j)
                for (int i = 0; i < bx; ++i) {
                    const double dist = dist_of(i, j);
                    le[at(n, j, i)] = w.amp * std::cos(w.nu * dist - w.omega * t);
                    lp[at(n, j, i)] = w.phifact * w.amp * std::sin(w.nu * dist - w.omega * t);
                }
        }
    } else {
        const int N = w.N;
        std::vector<std::complex<double>> ZE((size_t)N), ZP((size_t)N);
        for (int j = 0; j < ny_eval; ++j)
            for (int i = 0; i < bx; ++i) {
                std::fill(ZE.begin(), ZE.end(), 0.0);
                std::fill(ZP.begin(), ZP.end(), 0.0);
                for (int k = 1; k < w.kmax; ++k) {
                    const double omega = k * w.domega, nu = w.nus[(size_t)k];
                    const double dist = w.kcos.empty() ? dist_of(i, j)
                                                       : w.kcos[(size_t)k] * w.dx[(size_t)i] + w.ksin[(size_t)k] * w.dy[(size_t)j];
                    const std::complex<double> e =
                        w.c[(size_t)k] * std::complex<double>(std::cos(nu * dist), std::sin(nu * dist));
                    const std::complex<double> v = (w.g / omega) * std::complex<double>(e.imag(), -e.real());
                    ZE[(size_t)k] = e; ZE[(size_t)(N - k)] = std::conj(e);
                    ZP[(size_t)k] = v; ZP[(size_t)(N - k)] = std::conj(v);
                }
                fft_minus(ZE);
                fft_minus(ZP);
                for (int n = 0; n < nt; ++n) {
                    le[at(n, j, i)] = 0.5 * ZE[(size_t)n].real();
                    lp[at(n, j, i)] = 0.5 * ZP[(size_t)n].real();
                }
            }
    }
    for (int n = 0; n < nt; ++n)
        for (int j = 0; j < by; ++j)
            for (int i = 0; i < bx; ++i) {
                const size_t q = (size_t)n * bx * by + (size_t)j * bx + i;
                const size_t src = at(n, w.heading ? j : 0, i);
                if (eta) eta[q] = le[src];
                if (phis) phis[q] = lp[src];
            }
    return OW3D_OK;
}

// -------------------------------------------------------------- filtering
// Savitzky-Golay smoothing weights: value at offset 0 of the least-squares
// polynomial of degree m through offsets -nl..nr (savgol.f90 with ld = 0).
static std::vector<double> savgol(int nl, int nr, int m) {
    const int M = m + 1;
    std::vector<double> A((size_t)M * M, 0.0), b(M, 0.0);
    // normal equations: A(a,b) = sum_k k^(a+b)
    for (int a = 0; a < M; ++a)
        for (int c = 0; c < M; ++c) {
            double s = 0;
            for (int k = -nl; k <= nr; ++k) s += (a + c == 0) ? 1.0 : std::pow((double)k, a + c);
            A[(size_t)a * M + c] = s;
        }
    b[0] = 1.0;
    for (int k = 0; k < M; ++k) {  // Gaussian elimination, partial pivoting
        int pr = k;
        for (int r = k + 1; r < M; ++r) if (std::fabs(A[(size_t)r * M + k]) > std::fabs(A[(size_t)pr * M + k])) pr = r;
        if (pr != k) { for (int c = 0; c < M; ++c) std::swap(A[(size_t)k * M + c], A[(size_t)pr * M + c]); std::swap(b[k], b[pr]); }
        for (int r = k + 1; r < M; ++r) {
            const double f = A[(size_t)r * M + k] / A[(size_t)k * M + k];
            for (int c = k; c < M; ++c) A[(size_t)r * M + c] -= f * A[(size_t)k * M + c];
            b[r] -= f * b[k];
        }
    }
    for (int r = M - 1; r >= 0; --r) {
        double t = b[r];
        for (int c = r + 1; c < M; ++c) t -= A[(size_t)r * M + c] * b[c];
        b[r] = t / A[(size_t)r * M + r];
    }
    std::vector<double> w(nl + nr + 1);
    for (int k = -nl; k <= nr; ++k) {
        double s = b[0], f = 1.0;
        for (int q = 1; q <= m; ++q) { f *= k; s += b[q] * f; }
        w[k + nl] = s;
    }
    return w;
}

// FilterInit.f90:29-231. fc: 2a+1 centred weights. F2: the boundary weights in
// the (2a+1) x a column-major view FILTERING.f90 uses on the reference's
// max(2a+1,13) x max(a,6) storage.
void filter_coeffs(const ow3d_params& p, std::vector<double>& fc, std::vector<double>& F2) {
    const int a = p.filterALPHA, NP = 2 * a + 1;
    fc = savgol(a, a, p.filterORDER);
    const int ld = std::max(NP, 13), nc = std::max(a, 6);
    std::vector<double> S((size_t)ld * nc, 0.0);
    auto at = [&](int r, int c) -> double& { return S[(size_t)(c - 1) * ld + (r - 1)]; };
    // Off-centred boundary filters of Berland et al. (J. Comput. Phys. 224,
    // 2007), the table FilterInit.f90:149-186 applies with weights sigma_filt.
    static const double b1[4] = {0.320882352941, -0.465, 0.179117647059, -0.035};
    static const double b2[7] = {-0.085777408970, 0.277628171524, -0.356848072173, 0.223119093072,
                                 -0.057347064865, -0.000747264596, -0.000027453993};
    static const double b3[11] = {0.052523901012, -0.206299133811, 0.353527998250, -0.348142394842,
                                  0.181481803619, 0.009440804370, -0.077675100452, 0.044887364863,
                                  -0.009971961849, 0.000113359420, 0.000113359420};
    at(1, 1) = 1.0; for (int r = 0; r < 4; ++r) at(r + 1, 1) -= p.sigma_filt[0] * b1[r];
    at(2, 2) = 1.0; for (int r = 0; r < 7; ++r) at(r + 1, 2) -= p.sigma_filt[1] * b2[r];
    at(3, 3) = 1.0; for (int r = 0; r < 11; ++r) at(r + 1, 3) -= p.sigma_filt[2] * b3[r];
    const int degree[3] = {5, 6, 8};
    for (int c = 4; c <= 6; ++c) {
        const int hw = c - 1;
        const std::vector<double> w = savgol(hw, hw, degree[c - 4]);
        for (int r = 1; r <= 2 * hw + 1; ++r) at(r, c) = w[(size_t)r - 1];
    }
    if (std::fabs(p.sigma_filt[0]) < 1e-12) {
        std::fill(S.begin(), S.end(), 0.0);
        for (int i = 1; i <= nc; ++i) at(i, i) = 1.0;
    }
    F2.assign(S.begin(), S.begin() + (size_t)NP * a);
}

// ------------------------------------------------------------- the deck
int default_params(ow3d_params* p) {
    if (!p) return OW3D_ERR_BAD_INPUT;
    std::memset(p, 0, sizeof(*p));
    p->IC = 0; p->IncWaveType = 0;
    p->Lx = p->Ly = p->Lz = 1.0;
    p->Nx = 17; p->Ny = 1; p->Nz = 9;
    p->GridZ = 1; p->GhostGridX = p->GhostGridY = p->GhostGridZ = 1;
    p->alpha = p->beta = p->gamma = 3;
    p->alphaprecond = p->betaprecond = p->gammaprecond = 1;
    p->Nsteps = 1; p->dt = 0.01; p->timemethod = 1; p->CFL = 0; p->extrapolationONOFF = 1;
    p->g = 9.81;
    p->solver = 1; p->Precond = 3; p->MGCoarseningStrategy = 0; p->GMRESmaxiterations = 23;
    p->reltol = 1e-8; p->abstol = 1e-6; p->maxit = 1; p->cyclet = 'V'; p->nu1 = 1; p->nu2 = 1; p->MGmaxgrids = 0;
    p->LinearONOFF = 1; p->PressureTermOnOff = 0;
    p->filteringONOFF = 0; p->filterALPHA = 6; p->filterORDER = 10;
    p->sigma_filt[0] = 0.08; p->sigma_filt[1] = 0.08; p->sigma_filt[2] = 0.4;
    p->relaxONOFF = 0; p->relaxXorY = 'X';
    for (auto& z : p->zones) { z.XorY = 'X'; z.XorYgen = 'X'; z.PhiOnOff = 1; }
    p->precision = OW3D_PREC_FP64; p->krylov = OW3D_KRYLOV_FGMRES; p->device = 0;
    p->StoreDataONOFF = 0; p->formattype = 0;
    p->iKinematics = 0; p->nOutFiles = 0;
    std::memset(p->kinematics, 0, sizeof(p->kinematics));
    p->ispec = -1; p->seed = 0; p->seed2 = 0;
    p->Tp = 0; p->Hs = 0; p->h0 = 0; p->kh_max = 0; p->x0 = 0; p->y0 = 0;
    p->gamma_jonswap = 3.3; p->beta0 = 0; p->s0 = 1.0;
    p->sf_H = p->sf_h = p->sf_L = p->sf_T = p->sf_uEorS = 0;
    p->sf_wavel_or_per = p->sf_euler_or_stokes = 0; p->sf_nsteps = 1; p->sf_nmodes = 0;
    std::memset(p->bathymetry_file, 0, sizeof p->bathymetry_file);
    p->accel_tol_fact = 1e30; p->i_breaking = 0; p->PDampingONOFF = 0; p->swenseONOFF = 0; p->curvilinearONOFF = 0;
    p->T_half = 0; p->phi_b = 0; p->phi_0 = 0; p->del_fac = 0; p->cel_fac = 0; p->gamma_break = 0;
    p->current_flag = 0; p->current_Q = 0;
    p->flux_ramp = 0; p->flux_order = 1; std::memset(p->flux_file, 0, sizeof p->flux_file);
    return OW3D_OK;
}

namespace {
// Fortran list-directed records: whitespace/comma separated items, D exponents.
struct Record {
    std::vector<std::string> t;
    bool num(size_t i) const {
        if (i >= t.size()) return false;
        std::string s = t[i];
        for (auto& ch : s) if (ch == 'd' || ch == 'D') ch = 'e';
        char* end = nullptr;
        std::strtod(s.c_str(), &end);
        return end && *end == 0 && !s.empty();
    }
    double d(size_t i) const {
        std::string s = t[i];
        for (auto& ch : s) if (ch == 'd' || ch == 'D') ch = 'e';
        return std::strtod(s.c_str(), nullptr);
    }
    int n(size_t i) const { return (int)std::lround(d(i)); }
    char c(size_t i) const {
        std::string s = t[i];
        for (char ch : s) if (ch != '\'' && ch != '"') return ch;
        return ' ';
    }
    size_t nnum() const { size_t k = 0; while (num(k)) ++k; return k; }
};
Record split(const std::string& line) {
    Record r;
    std::string cur;
    for (char ch : line) {
        if (std::isspace((unsigned char)ch) || ch == ',') { if (!cur.empty()) { r.t.push_back(cur); cur.clear(); } }
        else cur += ch;
    }
    if (!cur.empty()) r.t.push_back(cur);
    return r;
}
}  // namespace

// ReadInputFileParameters.f90:18-517 (lines 1-13 of the deck).
int read_deck(const char* path, ow3d_params* p, std::string* err) {
    auto fail = [&](const std::string& m) { if (err) *err = m; return OW3D_ERR_BAD_INPUT; };
    std::ifstream f(path);
    if (!f) { if (err) *err = std::string("cannot open ") + path; return OW3D_ERR_IO; }
    default_params(p);
    std::vector<std::string> lines;
    std::string s;
    while (std::getline(f, s)) lines.push_back(s);
    size_t li = 1;  // line 0 is the header
    // list-directed reads pass over blank records
    auto blank = [&](size_t i) { return lines[i].find_first_not_of(" \t\r") == std::string::npos; };
    auto next = [&]() -> Record {
        while (li < lines.size() && blank(li)) ++li;
        return li < lines.size() ? split(lines[li++]) : Record();
    };
    Record r = next();  // IC [IncWaveType [accel_tol_fact]]
    if (!r.num(0)) return fail("line 2: IC expected");
    p->IC = r.n(0);
    p->IncWaveType = r.num(1) ? r.n(1) : 0;
    // IncWaveType 4 and 5 are the stream-function wave and the flux
    // wavemaker on a constant-flux current (ReadInputFileParameters.f90:45-48)
    if (p->IncWaveType == 4) { p->IncWaveType = 1; p->current_flag = 1; }
    if (p->IncWaveType == 5) { p->IncWaveType = 3; p->current_flag = 1; }
    if (r.num(2)) { p->accel_tol_fact = r.d(2); p->accel_from_deck = 1; }
    r = next();  // Lx Ly Lz Nx Ny Nz GridX GridY GridZ GhostGridX GhostGridY GhostGridZ
    if (r.nnum() < 12) return fail("line 3: 12 grid values expected");
    p->Lx = r.d(0); p->Ly = r.d(1); p->Lz = r.d(2);
    p->Nx = r.n(3); p->Ny = r.n(4); p->Nz = r.n(5);
    p->GridX = r.n(6); p->GridY = r.n(7); p->GridZ = r.n(8);
    p->GhostGridX = r.n(9); p->GhostGridY = r.n(10); p->GhostGridZ = r.n(11);
    if (p->Nx == 1) p->GhostGridX = 0;
    if (p->Ny == 1) p->GhostGridY = 0;
    if (p->Lz <= 0.0) {   // the bathymetry comes from a file (ReadInputFileParameters.f90:61-69)
        if (r.t.size() < 13) return fail("line 3: Lz <= 0 needs a bathymetry file name");
        std::snprintf(p->bathymetry_file, sizeof p->bathymetry_file, "%s", r.t[12].c_str());
    }
    r = next();  // alpha beta gamma alphaprecond betaprecond gammaprecond
    if (r.nnum() < 6) return fail("line 4: 6 stencil values expected");
    p->alpha = r.n(0); p->beta = r.n(1); p->gamma = r.n(2);
    p->alphaprecond = r.n(3); p->betaprecond = r.n(4); p->gammaprecond = r.n(5);
    if (p->Nx == 1) { p->alpha = 0; p->alphaprecond = 0; }
    if (p->Ny == 1) { p->beta = 0; p->betaprecond = 0; }
    r = next();  // Nsteps dt timemethod CFL extrapolationONOFF [time0]
    if (r.nnum() < 5) return fail("line 5: Nsteps dt timemethod CFL extrapolationONOFF expected");
    p->Nsteps = r.n(0); p->dt = r.d(1); p->timemethod = r.n(2); p->CFL = r.d(3); p->extrapolationONOFF = r.n(4);
    p->time0 = r.num(5) ? r.d(5) : 0.0;
    if (p->CFL != 0.0) {
        const double dx = p->Lx / (p->Nx - 1.0), dy = p->Ny > 1 ? p->Ly / (p->Ny - 1.0) : dx;
        p->dt = p->CFL * (p->Nx == 1 ? dy : dx);
    }
    r = next();  // g [rho]
    if (!r.num(0)) return fail("line 6: g expected");
    p->g = r.d(0);
    r = next();  // [solver] Precond MGCoarseningStrategy GMRESmaxiterations reltol abstol maxit cyclet nu1 nu2 MGmaxgrids
    {
        const size_t k = r.nnum();
        size_t o;
        if (k >= 7 && r.t.size() >= 11 && !r.num(7)) { p->solver = r.n(0); o = 1; }
        else if (k >= 6 && r.t.size() >= 10 && !r.num(6)) { p->solver = 1; o = 0; }
        else return fail("line 7: solver line not recognised");
        p->Precond = r.n(o); p->MGCoarseningStrategy = r.n(o + 1); p->GMRESmaxiterations = r.n(o + 2);
        p->reltol = r.d(o + 3); p->abstol = r.d(o + 4); p->maxit = r.n(o + 5); p->cyclet = r.c(o + 6);
        p->nu1 = r.n(o + 7); p->nu2 = r.n(o + 8); p->MGmaxgrids = r.n(o + 9);
    }
    r = next();  // stream-function line H h L T WAVELorPER uEorS EorS nsteps nmodes (always present, :291-293)
    if (r.nnum() >= 9) {
        p->sf_H = r.d(0); p->sf_h = r.d(1); p->sf_L = r.d(2); p->sf_T = r.d(3); p->sf_wavel_or_per = r.n(4);
        p->sf_uEorS = r.d(5); p->sf_euler_or_stokes = r.n(6); p->sf_nsteps = r.n(7); p->sf_nmodes = r.n(8);
    }
    r = next();  // StoreDataONOFF formattype [iKinematics nOutFiles] (ReadInputFileParameters.f90:300-405)
    if (r.nnum() >= 1) p->StoreDataONOFF = r.n(0);
    if (r.nnum() >= 2) {
        const int ft = r.n(1);
        p->formattype = ft;
        if (ft == 20 || ft == 21 || ft == 22) {
            if (!r.num(2) || !r.num(3)) return fail("line 9: formattype 20-22 needs iKinematics and nOutFiles");
            p->iKinematics = r.n(2);
            const int nout = r.n(3);
            if (nout < 0 || nout > (ft == 20 ? OW3D_MAX_KIN_FILES : 10))
                return fail("line 9: too many kinematics output files");
            p->nOutFiles = nout;
            for (int i = 0; i < nout; ++i) {
                Record q = next();
                int* o = p->kinematics[i];
                if (ft == 22) {
                    // x y tbeg tend tstride: point output (kept: the time range only)
                    if (q.nnum() < 5) return fail("line 9: kinematics output line " + std::to_string(i + 1) + " unreadable");
                    o[6] = q.n(2); o[7] = q.n(3); o[8] = q.n(4);
                } else {
                    if (q.nnum() < 9) return fail("line 9: kinematics output line " + std::to_string(i + 1) + " unreadable");
                    for (int m = 0; m < 9; ++m) o[m] = q.n(m);
                    if (o[0] < 1 || o[1] > p->Nx || o[0] > o[1]) return fail("kinematics x coordinate range is invalid");
                    if (o[3] < 1 || o[4] > p->Ny || o[3] > o[4]) return fail("kinematics y coordinate range is invalid");
                    if (o[2] < 1 || o[5] < 1 || o[8] < 1) return fail("kinematics strides must be positive");
                }
                if (o[6] < 1 || o[7] > p->Nsteps || o[6] > o[7]) return fail("kinematics time range is invalid");
            }
        }
    }
    r = next();  // LinearONOFF PressureTermONOFF
    if (r.nnum() < 1) return fail("line 10: LinearONOFF expected");
    p->LinearONOFF = r.n(0); p->PressureTermOnOff = r.num(1) ? r.n(1) : 0;
    r = next();  // filteringONOFF filterALPHA filterORDER sigma_filt(1:3)
    if (r.nnum() < 3) return fail("line 11: filter line expected");
    p->filteringONOFF = r.n(0); p->filterALPHA = r.n(1); p->filterORDER = r.n(2);
    for (int q = 0; q < 3; ++q) p->sigma_filt[q] = r.num(3 + q) ? r.d(3 + q) : 0.0;
    r = next();  // optional breaking line (7 numbers), else the relaxation line
    if (r.nnum() >= 7) {
        // i_breaking, T_half, phi_b, phi_0, f_delta, f_cel, gamma_break
        p->i_breaking = r.n(0); p->T_half = r.d(1); p->phi_b = r.d(2); p->phi_0 = r.d(3);
        p->del_fac = r.d(4); p->cel_fac = r.d(5); p->gamma_break = r.d(6);
        r = next();
    }
    // relaxONOFF relaxTransientTime relaxNo relaxXorY relaxDegrees
    if (r.nnum() < 3) return fail("line 13: relaxation line expected");
    p->relaxONOFF = r.n(0); p->relaxTransientTime = r.d(1); p->relaxNo = r.n(2);
    p->relaxXorY = r.t.size() > 3 ? r.c(3) : 'X';
    p->relaxDegrees = (r.t.size() > 4 && r.num(4)) ? r.d(4) : 0.0;
    if (p->relaxONOFF == 1) {
        if (p->relaxNo > OW3D_MAX_ZONES) return fail("too many relaxation zones");
        for (int z = 0; z < p->relaxNo; ++z) {
            Record q = next();
            if (q.t.size() < 10) return fail("relaxation zone line: 10 items expected");
            ow3d_zone& Z = p->zones[z];
            Z.x1 = q.d(0); Z.x2 = q.d(1); Z.y1 = q.d(2); Z.y2 = q.d(3); Z.ftype = q.n(4); Z.param = q.d(5);
            Z.XorY = q.c(6); Z.WavegenONOFF = q.n(7); Z.XorYgen = q.c(8); Z.degrees = q.d(9); Z.PhiOnOff = 1;
        }
    }
    // ReadInputFileParameters.f90:534-653: an optional pressure-damping line
    // (two integers, then its zone lines when on), the SWENSE line, the
    // curvilinear line, then the incident-wave line of IncWaveType 2. Decks
    // that end earlier keep the defaults (the hot path does not need them).
    while (li < lines.size() && blank(li)) ++li;
    if (li >= lines.size()) return OW3D_OK;
    {
        Record q = next();
        auto integer = [&](size_t i) {
            if (!q.num(i)) return false;
            for (char ch : q.t[i]) if (!(std::isdigit((unsigned char)ch) || ch == '-' || ch == '+')) return false;
            return true;
        };
        if (integer(0) && integer(1)) {
            p->PDampingONOFF = q.n(0);
            p->NDampZones = q.n(1);
            // the zone lines x0 x1 y0 y1 g0Phi g0Eta type (:539-545); the
            // first is kept (the reference runs one zone)
            if (q.n(0) != 0)
                for (int z = 0; z < q.n(1); ++z) {
                    Record r = next();
                    if (r.nnum() < 7) { if (err) *err = "pressure-damping zone line: 7 numbers expected"; return OW3D_ERR_BAD_INPUT; }
                    if (z == 0) {
                        p->pd_x0 = r.d(0); p->pd_x1 = r.d(1); p->pd_y0 = r.d(2); p->pd_y1 = r.d(3);
                        p->pd_g0Phi = r.d(4); p->pd_g0Eta = r.d(5); p->pd_type = r.n(6);
                    }
                }
        } else {
            --li;   // not a pressure-damping line (the reference backspaces, :555-562)
        }
    }
    while (li < lines.size() && blank(li)) ++li;
    if (li >= lines.size()) return OW3D_OK;
    {
        Record q = next();  // SWENSE line
        if (q.num(0)) p->swenseONOFF = q.n(0);
    }
    while (li < lines.size() && blank(li)) ++li;
    if (li >= lines.size()) return OW3D_OK;
    {
        Record q = next();  // curvilinearONOFF
        if (q.num(0)) p->curvilinearONOFF = q.n(0);
    }
    if (p->IncWaveType == 3) {
        // ramp time, interpolation order, paddle-signal file (:579-589)
        Record q = next();
        if (q.nnum() < 2 || q.t.size() < 3) return fail("flux-wavemaker line: ramp time, order and file expected");
        p->flux_ramp = q.d(0); p->flux_order = q.n(1);
        std::snprintf(p->flux_file, sizeof p->flux_file, "%s", q.t[2].c_str());
    } else if (p->IncWaveType == 2) {
        Record q = next();
        if (q.nnum() < 1) return fail("incident-wave line expected for IncWaveType 2");
        p->ispec = q.n(0);
        if (q.nnum() < 9) return fail("incident-wave line: ispec Tp Hs h0 kh_max seed seed2 x0 y0 expected");
        p->Tp = q.d(1); p->Hs = q.d(2); p->h0 = q.d(3); p->kh_max = q.d(4);
        p->seed = q.n(5); p->seed2 = q.n(6); p->x0 = q.d(7); p->y0 = q.d(8);
        p->gamma_jonswap = 3.3; p->beta0 = 0.0; p->s0 = 1.0;
        if (p->ispec == 3) {
            if (q.nnum() < 10) return fail("incident-wave line: ispec 3 needs gamma");
            p->gamma_jonswap = q.d(9);
        } else if (std::abs(p->ispec) >= 30) {
            // ... x0 y0 inc_wave_file beta0 s0 gamma (the file name is the 10th item)
            if (q.t.size() < 13 || !q.num(10) || !q.num(11) || !q.num(12))
                return fail("incident-wave line: |ispec| >= 30 needs a file name, beta0, s0 and gamma");
            p->beta0 = q.d(10); p->s0 = q.d(11); p->gamma_jonswap = q.d(12);
        }
        if (p->seed >= 0) p->seed = -p->seed;     // :632-647
        if (p->seed2 >= 0) p->seed2 = -p->seed2;
    }
    if (p->current_flag) {
        // the current's flux Q (:655-665); a line that does not read as a
        // number turns the current off (Q = 0)
        while (li < lines.size() && blank(li)) ++li;
        if (li < lines.size()) {
            Record q = next();
            p->current_Q = q.num(0) ? q.d(0) : 0.0;
        }
    }
    return OW3D_OK;
}

// ------------------------------------------------------ paddle signal
// setupWavePaddle.f90:43-67: a header line, "dt nt n2", the n2 y positions,
// then nt records "time flux(1..n2)" (list-directed: a record may span lines).
int read_paddle_signal(const char* path, PaddleSignal& ps, std::string* err) {
    auto fail = [&](const std::string& m, int code) { if (err) *err = m; return code; };
    if (!path) return fail("read_paddle_signal: no file", OW3D_ERR_BAD_INPUT);
    std::ifstream f(path);
    if (!f) return fail(std::string("read_paddle_signal: cannot open ") + path, OW3D_ERR_IO);
    std::string header;
    if (!std::getline(f, header)) return fail("read_paddle_signal: no header line", OW3D_ERR_IO);
    std::vector<double> v;
    std::string tok;
    while (f >> tok) {
        for (char& ch : tok) if (ch == 'D' || ch == 'd') ch = 'e';
        char* end = nullptr;
        const double x = std::strtod(tok.c_str(), &end);
        if (end == tok.c_str()) break;
        v.push_back(x);
    }
    if (v.size() < 3) return fail("read_paddle_signal: dt nt n2 expected", OW3D_ERR_IO);
    ps.dt = v[0]; ps.nt = (int)v[1]; ps.n2 = (int)v[2];
    if (ps.nt < 5 || ps.n2 < 1) return fail("read_paddle_signal: at least 5 times and 1 point required", OW3D_ERR_BAD_INPUT);
    const size_t need = 3 + (size_t)ps.n2 + (size_t)ps.nt * (1 + (size_t)ps.n2);
    if (v.size() < need) return fail("read_paddle_signal: error reading wave flux data (file too short)", OW3D_ERR_IO);
    ps.y.assign(v.begin() + 3, v.begin() + 3 + ps.n2);
    ps.flux.resize((size_t)ps.nt * ps.n2);
    for (int i = 0; i < ps.nt; ++i)
        for (int j = 0; j < ps.n2; ++j) ps.flux[(size_t)i * ps.n2 + j] = v[3 + (size_t)ps.n2 + (size_t)i * (1 + ps.n2) + 1 + j];
    return OW3D_OK;
}

// Neville's algorithm: the value at x of the polynomial through (xa[i],
// ya[i]), i < n, built column by column of the difference tableau from the
// entry nearest x, the correction path kept as central as it can be -- the
// published algorithm of the reference's polint (polint.f90).
static double neville(const double* xa, const double* ya, int n, double x) {
    double c[10], d[10];
    int ns = 1;   // 1-based, as the path rule is written
    double dif = std::fabs(x - xa[0]);
    for (int i = 1; i <= n; ++i) {
        const double dift = std::fabs(x - xa[i - 1]);
        if (dift < dif) { ns = i; dif = dift; }
        c[i - 1] = ya[i - 1];
        d[i - 1] = ya[i - 1];
    }
    double y = ya[ns - 1];
    ns = ns - 1;
    for (int m = 1; m <= n - 1; ++m) {
        for (int i = 1; i <= n - m; ++i) {
            const double ho = xa[i - 1] - x, hp = xa[i + m - 1] - x;
            const double w = c[i] - d[i - 1];
            const double den = w / (ho - hp);
            d[i - 1] = hp * den;
            c[i - 1] = ho * den;
        }
        double dy;
        if (2 * ns < n - m) dy = c[ns];
        else { dy = d[ns - 1]; ns = ns - 1; }
        y = y + dy;
    }
    return y;
}

// The signal on the rows of the grid (setupWavePaddle.f90:77-122 and the
// y interpolation of waveGenerationFromPaddleSignal.f90:65-96, which does not
// depend on time): F[i * Nyg + j] = u and X[...] = eta_x = -u_t / g at time
// level i (0-based) and row j, interior rows only.
int paddle_tables(const ow3d_params& p, const GridHost& G, const PaddleSignal& ps, std::vector<double>& F,
                  std::vector<double>& X, std::string* err) {
    auto fail = [&](const std::string& m) { if (err) *err = m; return OW3D_ERR_BAD_INPUT; };
    const int nt = ps.nt, n2 = ps.n2, order = p.flux_order;
    if (order < 1 || order > 10 || order > n2) return fail("paddle signal: the interpolation order must be 1..min(10, n2)");
    const double dy_local = 2.0 * ps.y[0];
    for (int i = 2; i <= n2 - 1; ++i)
        if (std::fabs(ps.y[(size_t)i - 1] - (ps.y[(size_t)i - 2] + dy_local)) >= 1e-5)
            return fail("paddle signal: the points must be uniformly spaced from y = dy/2 to ymax - dy/2");
    if ((double)nt * ps.dt < (double)p.Nsteps * p.dt)
        return fail("paddle signal: the time series is shorter than Nsteps * dt");
    // eta_x = -1/g u_t, 5-point derivative weights at each of 5 uniform times
    double tt[5], w[5][5];
    for (int q = 0; q < 5; ++q) tt[q] = q * ps.dt;
    for (int q = 0; q < 5; ++q) fd_weights(tt[q], tt, 4, 1, w[q]);
    const double gfac = -1.0 / p.g;
    std::vector<double> ex((size_t)nt * n2);
    for (int j = 0; j < n2; ++j) {
        auto fl = [&](int i) { return ps.flux[(size_t)i * n2 + j]; };   // 0-based time
        for (int i = 0; i < nt; ++i) {
            int row, base;
            if (i < 2) { row = i; base = 0; }
            else if (i < nt - 2) { row = 2; base = i - 2; }
            else { row = 4 - (nt - 1 - i); base = nt - 5; }
            double acc = 0;
            for (int q = 0; q < 5; ++q) acc += w[row][q] * fl(base + q);
            ex[(size_t)i * n2 + j] = gfac * acc;
        }
    }
    const int Nyg = G.Nyg;
    F.assign((size_t)nt * Nyg, 0.0);
    X.assign((size_t)nt * Nyg, 0.0);
    for (int j = 1 + G.gy; j <= G.Ny + G.gy; ++j) {
        const double y0 = G.y[(size_t)j - 1];
        int nny = (int)std::lround(y0 / dy_local) + 1 - order / 2;   // NINT: half away from zero
        if (nny < 1) nny = 1;
        else if (nny + order - 1 > n2) nny = n2 - order + 1;
        std::vector<double> a((size_t)order), b((size_t)order);
        for (int i = 0; i < nt; ++i) {
            for (int q = 0; q < order; ++q) {
                a[(size_t)q] = ps.flux[(size_t)i * n2 + nny - 1 + q];
                b[(size_t)q] = ex[(size_t)i * n2 + nny - 1 + q];
            }
            F[(size_t)i * Nyg + j - 1] = neville(&ps.y[(size_t)nny - 1], a.data(), order, y0);
            X[(size_t)i * Nyg + j - 1] = neville(&ps.y[(size_t)nny - 1], b.data(), order, y0);
        }
    }
    return OW3D_OK;
}

// ------------------------------------------------------------- bathymetry
// The bathymetry file of a deck with Lz <= 0 (SetupInitialConditions.f90:51-111,
// OceanWave3DT0Setup.f90:346-364): a header line, the gradient flag, then one
// record per interior point (x fastest) holding h (flag 1) or h, h_x, h_xx,
// h_y, h_yy (flag 0). The ghost points take the values of the adjacent
// interior points; with flag 1 the derivatives are the 7-point DiffXEven /
// DiffYEven ones of the ghost-extended h. Outputs are Nxg*Nyg, ghosts included.
int read_bathymetry(const ow3d_params& p, const char* path, double* h, double* hx, double* hxx, double* hy,
                    double* hyy, int* flag_out, std::string* err) {
    auto fail = [&](const std::string& m, int code) { if (err) *err = m; return code; };
    if (!path || !h) return fail("read_bathymetry: bad arguments", OW3D_ERR_BAD_INPUT);
    std::ifstream f(path);
    if (!f) return fail(std::string("read_bathymetry: cannot open ") + path, OW3D_ERR_IO);
    std::vector<std::string> lines;
    std::string s;
    while (std::getline(f, s)) lines.push_back(s);
    size_t li = 1;   // line 0 is the header
    auto next = [&]() -> Record {
        while (li < lines.size() && lines[li].find_first_not_of(" \t\r") == std::string::npos) ++li;
        return li < lines.size() ? split(lines[li++]) : Record();
    };
    Record r = next();
    if (!r.num(0)) return fail("read_bathymetry: the gradient flag is missing", OW3D_ERR_BAD_INPUT);
    const int flag = r.n(0);
    if (flag != 0 && flag != 1) return fail("read_bathymetry: the gradient flag must be 0 or 1", OW3D_ERR_BAD_INPUT);
    const int gx = p.Nx > 1 ? 1 : 0, gy = p.Ny > 1 ? 1 : 0;
    const int Nxg = p.Nx + 2 * gx, Nyg = p.Ny + 2 * gy;
    std::vector<double> F[5];
    for (auto& v : F) v.assign((size_t)Nxg * Nyg, 0.0);
    for (int j = 1 + gy; j <= p.Ny + gy; ++j)
        for (int i = 1 + gx; i <= p.Nx + gx; ++i) {
            Record q = next();
            const size_t c = (size_t)(i - 1) + (size_t)Nxg * (j - 1);
            const int need = flag == 1 ? 1 : 5;
            if ((int)q.nnum() < need)
                return fail("read_bathymetry: record for point (" + std::to_string(i - gx) + ", " + std::to_string(j - gy) +
                                ") needs " + std::to_string(need) + " values",
                            OW3D_ERR_BAD_INPUT);
            for (int m = 0; m < need; ++m) F[m][c] = q.d(m);
        }
    auto at = [&](std::vector<double>& v, int i, int j) -> double& { return v[(size_t)(i - 1) + (size_t)Nxg * (j - 1)]; };
    for (auto& v : F) {   // ghost extension (SetupInitialConditions.f90:89-108)
        for (int j = 1; j <= Nyg; ++j) { at(v, 1, j) = at(v, 1 + gx, j); at(v, Nxg, j) = at(v, p.Nx + gx, j); }
        for (int i = 1; i <= Nxg; ++i) { at(v, i, 1) = at(v, i, 1 + gy); at(v, i, Nyg) = at(v, i, p.Ny + gy); }
    }
    if (flag == 1) {
        GridHost G;
        std::vector<double> ones((size_t)Nxg * Nyg, 1.0), zeros(ones.size(), 0.0);
        int rc = build_grid(p, ones.data(), zeros.data(), zeros.data(), zeros.data(), zeros.data(), G, err);
        if (rc) return rc;
        auto diff = [&](const Stencil& S, bool alongx, int order, std::vector<double>& out) {
            const int n = alongx ? Nxg : Nyg;
            for (int j = 1; j <= Nyg; ++j)
                for (int i = 1; i <= Nxg; ++i) {
                    const int pos = alongx ? i : j;
                    const int ws = pos <= 3 ? 1 : (pos <= n - 3 ? pos - 3 : n - 6);
                    double acc = 0.0;
                    for (int m = 0; m < 7; ++m)
                        acc += S.at(order, pos - 1, m) * (alongx ? at(F[0], ws + m, j) : at(F[0], i, ws + m));
                    at(out, i, j) = acc;
                }
        };
        if (p.Nx > 1) { diff(G.SX, true, 1, F[1]); diff(G.SX, true, 2, F[2]); }
        if (p.Ny > 1) { diff(G.SY, false, 1, F[3]); diff(G.SY, false, 2, F[4]); }
    }
    double* out[5] = {h, hx, hxx, hy, hyy};
    for (int m = 0; m < 5; ++m)
        if (out[m]) std::copy(F[m].begin(), F[m].end(), out[m]);
    if (flag_out) *flag_out = flag;
    return OW3D_OK;
}

}  // namespace ow3d
