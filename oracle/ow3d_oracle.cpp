// ORACLE -- test infrastructure only (see oracle_setup.hpp). CPU FP64
// restatement of the OceanWave3D hot path: the high-order sigma-transformed
// Laplace operator, the multigrid preconditioner assembled as the reference
// assembles it, GMRES, and the RK4 free-surface step. Two modes:
//
//   mode 0  "reference-faithful": lexicographic Gauss-Seidel with the special
//           point pass (GaussSeidel.f90, GaussSeidelSpecialPoints.f90) and
//           left-preconditioned GMRES with SPARSKIT2 semantics
//           (iterative_solution.f90:20-56); this is also the timed CPU
//           baseline of bench.py.
//   mode 1  "device-matched": the same operators, with the smoother ordering
//           the CUDA path uses (multicolour column Gauss-Seidel) and the Krylov
//           variant selected by params.krylov (right-preconditioned flexible
//           GMRES with classical Gram-Schmidt and conditional
//           re-orthogonalisation, or the left-preconditioned variant), so
//           that the CUDA results can be compared to 1e-10.
//
// The SPARSKIT2 routines the reference links (gmres, mgsro, amux, coocsr,
// clncsr) and the HSL MA41 coarse LU are not part of the reference tree; they
// are restated here from their published algorithms (dense partial-pivoting LU
// stands in for MA41).
#include "oracle_setup.hpp"
#include <cstdio>
#include <cstdlib>
#include <memory>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

struct Level {
    LevelGrid G;
    Stencil1D SX, SY, SZ;
    CSR A;
    vector<int> ighost;       // 1-based global row indices (MGPreProcess.f90:376-439)
    vector<double> LU; vector<int> piv;  // coarsest level dense LU
    int ncolor = 0;
    int cross = 0;            // mixed-derivative terms present (h_x or h_y nonzero)
    int per = 0;              // periodic in x
    // work vectors for the V-cycle
    vector<double> x, b, r;
};

struct Zone {
    int i0 = 1, i1 = 1, j0 = 1, j1 = 1;  // 1-based, ghost-inclusive
    char XorY = 'X', XorYgen = 'X';
    int wavegen = 0, phion = 1;
    vector<double> gam;                  // along the relaxation direction
    int tmode = -1, nt = 0; double tdt = 0;
    vector<double> eta, phis;            // [nt][box]
};

struct Sim {
    ow3d_params p;
    int mode = 0;
    int per = 0;                         // periodic in x (params.periodic_x)
    int gx, gy, gz, Nxg, Nyg, Nzg, N, C, dimcase;
    LevelGrid fine;                      // fine grid + bathymetry
    Stencil1D SX, SY, SZ;                // high-order stencils
    CrossTables T;                       // high-order cross tables (Precond==0 part)
    vector<Level> lev;                   // lev[0] coarsest ... lev[L-1] finest
    // state
    vector<double> E, P, W, Ex, Exx, Ey, Eyy, Px, Py;
    vector<double> tE, tP, tW, tEx, tExx, tEy, tEyy, tPx, tPy;
    vector<double> sEx, sPx, sEy, sPy;   // ghost source terms of Wavefield
    vector<double> tsEx, tsPx;           // those of Wavefield_tmp (the RK stages)
    // the flux wavemaker (IncWaveType 3; setupWavePaddle.f90)
    int pad = 0, pad_nt = 0, pad_n2 = 0;
    double pad_dt = 0;
    vector<double> pad_y, pad_flux, pad_etax;   // nt x n2, time-major
    vector<double> Uneu;                 // per row: the west wall's flux FAC u (Uneumann, k >= 2)
    vector<double> PHI, LASTPHI0, LASTPHI1, RHS;
    vector<double> dsig;                 // 5*N, dsigmanew(k,i,j,1..5) for the current stage
    double time = 0; int64_t tstep = 0;
    vector<Zone> zones;
    // pressure damping (PreprocessPDampingZones.f90, BuildPDampMatrices.f90)
    int pd_i1 = 0, pd_nd = 0;
    vector<double> gamPhi, gamEta, NuD, Pd;
    Stencil1D pdGrad;                    // BuildStencil_1D_Uneven over x(1:nd)
    vector<double> pdLU; vector<int> pdPiv;
    vector<double> fc, fc2;              // filter: centre (NP) and boundary view (NP*alpha)
    int NP = 0;
    // the roller breaking model of x flumes (DetectBreaking.f90)
    double Ul = 0, Ur = 0;               // constant-flux current at the west and east walls
    int brk = 0;                         // i_breaking > 0 and Ny == 1
    double tan_b = 0, tan_0 = 0;         // tan(phi_b), tan(phi_0)
    vector<double> tan_phi, Qr_x;        // per column: roller angle state, roller flux slope
    vector<int> r_npts, r_toe;           // rollers of the last completed step
    vector<double> r_x, r_eta, r_thick, r_tan;
    // local smoothing by the vertical acceleration (LocalSmoothing2D/3D.f90)
    int smooth = 0;
    vector<double> WHist[3], EtatHist1;  // W after the last three steps; eta_t of the last step
    vector<double> accel_Wt;             // the last call's Lagrangian dw/dt at the surface
    vector<int> accel_pts;               // columns (0-based) where it exceeded the limit
    // stats
    int64_t solves = 0, totit = 0, notconv = 0; int minit = 1 << 30, maxit = 0, lastit = 0;
    double lastres = 0;
};

static inline size_t gid(const Sim& s, int k, int i, int j) {  // 1-based -> 0-based
    return (size_t)(k - 1) + (size_t)s.Nzg * ((size_t)(i - 1) + (size_t)s.Nxg * (size_t)(j - 1));
}

// Periodic x: copy the distinct columns into the image columns of a field of
// nz values per column -- column 1 <- Nxg-2, Nxg-1 <- 2, Nxg <- 3.
static void images_x(const Sim& s, double* v, int nz) {
    const int Nx = s.Nxg;
    for (int j = 1; j <= s.Nyg; ++j) {
        double* r = v + (size_t)nz * Nx * (j - 1);
        for (int k = 0; k < nz; ++k) {
            r[(size_t)nz * 0 + k] = r[(size_t)nz * (Nx - 3) + k];
            r[(size_t)nz * (Nx - 2) + k] = r[(size_t)nz * 1 + k];
            r[(size_t)nz * (Nx - 1) + k] = r[(size_t)nz * 2 + k];
        }
    }
}
static void zero_images_x(const Sim& s, double* v, int nz) {
    const int Nx = s.Nxg;
    for (int j = 1; j <= s.Nyg; ++j) {
        double* r = v + (size_t)nz * Nx * (j - 1);
        for (int k = 0; k < nz; ++k) r[k] = r[(size_t)nz * (Nx - 2) + k] = r[(size_t)nz * (Nx - 1) + k] = 0.0;
    }
}

// ---------------------------------------------------------------- grids
// SetupCompDomain.f90:35-79
static void setup_fine_grid(Sim& s) {
    const ow3d_params& p = s.p;
    LevelGrid& G = s.fine;
    G.Nx = p.Nx; G.Ny = p.Ny; G.Nz = p.Nz; G.Nxg = s.Nxg; G.Nyg = s.Nyg; G.Nzg = s.Nzg;
    G.x.assign(s.Nxg, p.Lx); G.y.assign(s.Nyg, p.Ly); G.z.assign(s.Nzg, 0.0);
    if (p.Nx > 1)
        for (int i = -s.gx; i <= p.Nx - 1 + s.gx; ++i) G.x[i + s.gx] = (double)i / (double)(p.Nx - 1) * p.Lx;
    if (p.Ny > 1)
        for (int i = -s.gy; i <= p.Ny - 1 + s.gy; ++i) G.y[i + s.gy] = (double)i / (double)(p.Ny - 1) * p.Ly;
    const double pi = 3.14159265358979323846264338327950288;
    for (int i = 0; i <= p.Nz - 1; ++i) {
        if (p.GridZ == 0) G.z[i + s.gz] = (double)i / (double)(p.Nz - 1) * p.Lz;
        else G.z[i + s.gz] = std::sin(pi * (double)i / (double)(2 * (p.Nz - 1)));
    }
    if (s.gz == 1) G.z[0] = -G.z[2];
}

// MGPreProcess.f90:31,449-458: number of levels, single-precision log as the reference.
static int no_grids(int nx, int ny, int nz) {
    float Nmax = (float)std::max(nx, std::max(ny, nz));
    float tmp = std::log10(Nmax - 1.0f) / std::log10(2.0f);
    return (int)std::lround(tmp);
}

// MGPreProcess.f90:95-318: coarsening strategy and coarse grid geometry.
static int build_hierarchy(Sim& s) {
    const ow3d_params& p = s.p;
    int L = no_grids(p.Nx, p.Ny, p.Nz);
    if (L > p.MGmaxgrids && p.MGmaxgrids > 0) L = p.MGmaxgrids;
    if (L < 1) L = 1;
    s.lev.assign(L, Level());
    Level& F = s.lev[L - 1];
    F.G = s.fine;
    for (int k = L - 2; k >= 0; --k) {
        const LevelGrid& f = s.lev[k + 1].G;
        LevelGrid& c = s.lev[k].G;
        int NFx = f.Nx, NFy = f.Ny, NFz = f.Nz;
        int xc = 0, yc = 0, zc = 0;
        if (p.MGCoarseningStrategy == 1) {
            if (NFx == NFy && NFx == NFz) { xc = yc = zc = 1; }
            else if (NFx > NFy && NFx > NFz) xc = 1;
            else if (NFy > NFx && NFy > NFz) yc = 1;
            else if (NFz > NFx && NFz > NFy) zc = 1;
            else if (NFx == NFy && NFx > NFz) { xc = yc = 1; }
            else if (NFx == NFz && NFx > NFy) { xc = zc = 1; }
            else if (NFy == NFz && NFy > NFx) { yc = zc = 1; }
        } else if (p.MGCoarseningStrategy == 2) {
            if (NFx > 3) xc = 1; if (NFy > 3) yc = 1; if (NFz > 3) zc = 1;
        } else {
            if (NFx == 1) { if (NFy == NFz) { yc = zc = 1; } else yc = 1; }
            else if (NFy == 1) { if (NFx == NFz) { xc = zc = 1; } else xc = 1; }
            else {
                if (NFx == NFy && NFx == NFz) { xc = yc = zc = 1; }
                else {
                    if (NFx > NFz) xc = 1;
                    if (NFy > NFz) yc = 1;
                    if (NFx < NFz && NFy < NFz) zc = 1;
                }
            }
        }
        int XF = 1, YF = 1, ZF = 1;
        if (xc) { c.Nx = (f.Nx - 1) / 2 + 1; if (f.Nx % 2 == 0) return -1; XF = 2; } else c.Nx = f.Nx;
        if (yc) { c.Ny = (f.Ny - 1) / 2 + 1; if (f.Ny % 2 == 0) return -1; YF = 2; } else c.Ny = f.Ny;
        if (zc) { c.Nz = (f.Nz - 1) / 2 + 1; if (c.Nz % 2 == 0) return -1; ZF = 2; } else c.Nz = f.Nz;
        c.Nxg = c.Nx + 2 * s.gx; c.Nyg = c.Ny + 2 * s.gy; c.Nzg = c.Nz + s.gz;
        // x by injection, ghosts by extrapolation (:223-257)
        c.x.assign(c.Nxg, 0.0); c.y.assign(c.Nyg, p.Ly);
        if (c.Nxg > 1) {
            for (int i = 1 + s.gx; i <= c.Nxg - s.gx; ++i) c.x[i - 1] = f.x[(1 + s.gx) + (i - 1 - s.gx) * XF - 1];
            if (s.gx == 1) {
                c.x[0] = c.x[1] - (c.x[2] - c.x[1]);
                c.x[c.Nxg - 1] = c.x[c.Nxg - 2] + (c.x[c.Nxg - 2] - c.x[c.Nxg - 3]);
            }
        } else c.x[0] = f.x[0];
        if (c.Nyg > 1) {
            for (int j = 1 + s.gy; j <= c.Nyg - s.gy; ++j) c.y[j - 1] = f.y[(1 + s.gy) + (j - 1 - s.gy) * YF - 1];
            if (s.gy == 1) {
                c.y[0] = c.y[1] - (c.y[2] - c.y[1]);
                c.y[c.Nyg - 1] = c.y[c.Nyg - 2] + (c.y[c.Nyg - 2] - c.y[c.Nyg - 3]);
            }
        } else c.y[0] = f.y[0];
        // z (:299-306)
        c.z.assign(c.Nzg, 0.0);
        if (s.gz == 1) {
            c.z[0] = -f.z[(2 + ZF) - 1];
            for (int kk = 2; kk <= c.Nzg; ++kk) c.z[kk - 1] = f.z[2 + (kk - 2) * ZF - 1];
        } else {
            for (int kk = 1; kk <= c.Nzg; ++kk) c.z[kk - 1] = f.z[1 + (kk - 1) * ZF - 1];
        }
        // h, hx, hxx, hy, hyy by injection; h ghosts copied (:219-314)
        size_t Cc = (size_t)c.Nxg * c.Nyg;
        c.h.assign(Cc, 0.0); c.hx.assign(Cc, 0.0); c.hxx.assign(Cc, 0.0); c.hy.assign(Cc, 0.0); c.hyy.assign(Cc, 0.0);
        for (int j = 1 + s.gy; j <= c.Nyg - s.gy; ++j)
            for (int i = 1 + s.gx; i <= c.Nxg - s.gx; ++i) {
                int fi = (1 + s.gx) + (i - 1 - s.gx) * XF, fj = (1 + s.gy) + (j - 1 - s.gy) * YF;
                size_t cc = (size_t)(i - 1) + (size_t)c.Nxg * (j - 1), ff = (size_t)(fi - 1) + (size_t)f.Nxg * (fj - 1);
                c.h[cc] = f.h[ff]; c.hx[cc] = f.hx[ff]; c.hxx[cc] = f.hxx[ff]; c.hy[cc] = f.hy[ff]; c.hyy[cc] = f.hyy[ff];
            }
        for (int j = 1; j <= c.Nyg; ++j) {
            c.h[(size_t)c.Nxg * (j - 1)] = c.h[(size_t)(1 + s.gx - 1) + (size_t)c.Nxg * (j - 1)];
            c.h[(size_t)(c.Nxg - 1) + (size_t)c.Nxg * (j - 1)] = c.h[(size_t)(c.Nxg - s.gx - 1) + (size_t)c.Nxg * (j - 1)];
        }
        for (int i = 1; i <= c.Nxg; ++i) {
            c.h[(size_t)(i - 1)] = c.h[(size_t)(i - 1) + (size_t)c.Nxg * (1 + s.gy - 1)];
            c.h[(size_t)(i - 1) + (size_t)c.Nxg * (c.Nyg - 1)] = c.h[(size_t)(i - 1) + (size_t)c.Nxg * (c.Nyg - s.gy - 1)];
        }
    }
    return 0;
}

// ------------------------------------------------- low-order matrix assembly
// PreparePreconditioner.f90:77-111 -> PreProcessDiffStencils, PrepareFullOperatorStencils,
// DetermineTransformationConstantsArray (eta = 0), ConstructTableCrossDerivatives(...,1),
// BuildLinearSystemMatrix.f90:1-338, CleanSparseMatrixCOO (sum duplicates),
// CSRdiaREORDER (diagonal first).
static void assemble_level(const Sim& s, Level& Lv) {
    const ow3d_params& p = s.p;
    const LevelGrid& G = Lv.G;
    const int a = p.alphaprecond, b = p.betaprecond, g = p.gammaprecond;
    const int Nxg = G.Nxg, Nyg = G.Nyg, Nzg = G.Nzg;
    Lv.SX = s.per ? build_stencils_periodic(G.x, a) : build_stencils_xy(G.x, a);
    Lv.SY = build_stencils_xy(G.y, b);
    Lv.SZ = build_stencils_z(G.z, G.Nz, s.gz, g);
    CrossTables T = build_cross_tables(G, Lv.SX, Lv.SY, Lv.SZ, g, s.gx, s.gy, s.gz);
    auto L = [&](int k, int i, int j) -> int { return k + Nzg * (i - 1) + Nzg * Nxg * (j - 1); };  // 1-based
    auto inb = [&](int k, int i, int j) { return k >= 1 && k <= Nzg && i >= 1 && i <= Nxg && j >= 1 && j <= Nyg; };
    int dimc = (Nyg == 1) ? 1 : (Nxg == 1 ? 2 : 3);
    auto sig = [&](int k, int i, int j, double* o) {
        size_t c = (size_t)(i - 1) + (size_t)Nxg * (j - 1);
        double zk = (k == 1) ? 0.0 : G.z[k - 1];
        sigma_coeffs(dimc, zk, 0, 0, 0, 0, 0, G.h[c], G.hx[c], G.hxx[c], G.hy[c], G.hyy[c], o);
    };
    auto diff = [](int i, int al, int n) { return (i < al + 1) ? al + 1 - i : (i > n - al ? n - al - i : 0); };
    // Full-rank 1-D stencils of PrepareFullOperatorStencils, as (col,val) lists.
    auto DX = [&](int k, int i, int j, int order, double f, RowAcc& R) {
        if (Nxg == 1) return;
        if (s.per) {   // centred, cyclic
            for (int m = 0; m <= 2 * a; ++m) R.add(L(k, wrap_x(i + (m - a), Nxg), j), f * Lv.SX.at(order, i - 1, m));
            return;
        }
        int da = diff(i, a, Nxg);
        for (int m = 0; m <= 2 * a; ++m) R.add(L(k, i + (m - a) + da, j), f * Lv.SX.at(order, i - 1, m));
    };
    auto DY = [&](int k, int i, int j, int order, double f, RowAcc& R) {
        if (Nyg == 1) return;
        int db = diff(j, b, Nyg);
        for (int m = 0; m <= 2 * b; ++m) R.add(L(k, i, j + (m - b) + db), f * Lv.SY.at(order, j - 1, m));
    };
    auto DZ = [&](int k, int i, int j, int order, double f, RowAcc& R) {
        int dg = diff(k, g, Nzg);
        for (int m = 0; m <= 2 * g; ++m) R.add(L(k + (m - g) + dg, i, j), f * Lv.SZ.at(order, k - 1, m));
    };
    const int rank = 2 * g + 1;
    int ranka = Nxg > 1 ? rank : 1, rankb = Nyg > 1 ? rank : 1;
    // Cross derivative full-rank stencils of ConstructTableCrossDerivatives.f90:266-351.
    auto DXZ = [&](int k, int i, int j, double f, RowAcc& R) {
        vector<int> idxb(rankb);
        int db = (Nyg > 1) ? diff(j, g, Nyg) : 0;
        for (int m = 0; m < rankb; ++m) idxb[m] = (Nyg == 1) ? 1 : j + (m - g) + db;
        for (int jj = 0; jj < rankb; ++jj)
            for (int kk = 0; kk < rank; ++kk) {
                int Iz = T.IZ1[T.id(k, i, j, kk)]; double Sz = T.SZ1[T.id(k, i, j, kk)];
                for (int ii = 0; ii < ranka; ++ii) {
                    int Ix = T.IX[T.id(Iz, i, j, ii)]; double Sx = T.SX[T.id(Iz, i, j, ii)];
                    if (inb(Iz, Ix, idxb[jj])) R.add(L(Iz, Ix, idxb[jj]), f * (Sx * Sz));
                }
            }
    };
    auto DYZ = [&](int k, int i, int j, double f, RowAcc& R) {
        vector<int> idxa(ranka);
        int da = (Nxg > 1) ? diff(i, g, Nxg) : 0;
        for (int m = 0; m < ranka; ++m) idxa[m] = (Nxg == 1) ? 1 : i + (m - g) + da;
        for (int ii = 0; ii < ranka; ++ii)
            for (int kk = 0; kk < rank; ++kk) {
                int Iz = T.IZ2[T.id(k, i, j, kk)]; double Sz = T.SZ2[T.id(k, i, j, kk)];
                for (int jj = 0; jj < rankb; ++jj) {
                    int Iy = T.IY[T.id(Iz, i, j, jj)]; double Sy = T.SY[T.id(Iz, i, j, jj)];
                    if (inb(Iz, idxa[ii], Iy)) R.add(L(Iz, idxa[ii], Iy), f * (Sy * Sz));
                }
            }
    };
    const int n = Nxg * Nyg * Nzg;
    vector<RowAcc> rows(n);
    const int gx = s.gx, gy = s.gy;
    bool three = (Nxg - 2 * gx > 1) && (Nyg - 2 * gy > 1);
    bool xonly = !three && (Nxg - 2 * gx > 1);
    bool yonly = !three && !xonly && (Nyg - 2 * gy > 1);
    double sg[5];
    for (int j = 1 + gy; j <= Nyg - gy; ++j)
        for (int i = 1 + gx; i <= Nxg - gx; ++i)
            for (int k = 1; k <= Nzg; ++k) {
                RowAcc& R = rows[L(k, i, j) - 1];
                size_t c = (size_t)(i - 1) + (size_t)Nxg * (j - 1);
                if (k == Nzg) { R.add(L(k, i, j), 1.0); continue; }
                if (k == 1) {
                    sig(2, i, j, sg);
                    double hx = G.hx[c], hy = G.hy[c];
                    // the packed arrays are summed entry-wise first, then stored
                    RowAcc P;
                    if (Nxg > 1 && Nyg > 1) {
                        DZ(2, i, j, 1, sg[4] + hx * sg[1] + hy * sg[3], P);
                        DX(2, i, j, 1, hx, P); DY(2, i, j, 1, hy, P);
                    } else if (Nxg > 1) {
                        DZ(2, i, j, 1, sg[4] + hx * sg[1], P); DX(2, i, j, 1, hx, P);
                    } else if (Nyg > 1) {
                        DZ(2, i, j, 1, sg[4] + hy * sg[3], P); DY(2, i, j, 1, hy, P);
                    }
                    for (size_t t = 0; t < P.cols.size(); ++t) R.add(P.cols[t], P.vals[t]);
                    continue;
                }
                sig(k, i, j, sg);
                RowAcc P;
                if (three) {
                    DX(k, i, j, 2, 1.0, P); DY(k, i, j, 2, 1.0, P); DZ(k, i, j, 1, sg[2], P);
                    DZ(k, i, j, 2, sg[1] * sg[1] + sg[3] * sg[3] + sg[4] * sg[4], P);
                } else if (xonly) {
                    DX(k, i, j, 2, 1.0, P); DZ(k, i, j, 1, sg[2], P);
                    DZ(k, i, j, 2, sg[1] * sg[1] + sg[4] * sg[4], P);
                } else if (yonly) {
                    DY(k, i, j, 2, 1.0, P); DZ(k, i, j, 1, sg[2], P);
                    DZ(k, i, j, 2, sg[3] * sg[3] + sg[4] * sg[4], P);
                }
                for (size_t t = 0; t < P.cols.size(); ++t) R.add(P.cols[t], P.vals[t]);
                if (s.per) continue;   // periodic levels have no mixed-derivative terms (flat bottom)
                if (three || xonly) DXZ(k, i, j, 2.0 * sg[1], R);
                if (three || yonly) DYZ(k, i, j, 2.0 * sg[3], R);
            }
    if (gx == 1) {
        for (int j = 1 + gy; j <= Nyg - gy; ++j)
            for (int k = 1 + s.gz; k <= Nzg; ++k) {
                DX(k, 2, j, 1, 1.0, rows[L(k, 1, j) - 1]);
                DX(k, Nxg - 1, j, 1, 1.0, rows[L(k, Nxg, j) - 1]);
            }
    }
    if (gy == 1) {
        for (int i = 1 + gx; i <= Nxg - gx; ++i)
            for (int k = 1 + s.gz; k <= Nzg; ++k) {
                DY(k, i, 2, 1, 1.0, rows[L(k, i, 1) - 1]);
                DY(k, i, Nyg - 1, 1, 1.0, rows[L(k, i, Nyg) - 1]);
            }
    }
    auto ident = [&](int k, int i, int j) { rows[L(k, i, j) - 1].add(L(k, i, j), 1.0); };
    if (gx + gy == 2) {
        for (int k = 1; k <= Nzg; ++k) { ident(k, 1, 1); ident(k, Nxg, 1); ident(k, 1, Nyg); ident(k, Nxg, Nyg); }
        for (int i = 1 + gx; i <= Nxg - gx; ++i) { ident(1, i, 1); ident(1, i, Nyg); }
        for (int j = 1 + gy; j <= Nyg - gy; ++j) { ident(1, 1, j); ident(1, Nxg, j); }
    } else if (gx == 1 && Nyg == 1) {
        ident(1, 1, 1); ident(1, Nxg, 1);
    } else if (gy == 1 && Nxg == 1) {
        ident(1, 1, 1); ident(1, 1, Nyg);
    }
    if (s.per)   // ghost columns and the repeated column: identity rows
        for (int j = 1; j <= Nyg; ++j)
            for (int k = 1; k <= Nzg; ++k)
                for (int i : {1, Nxg - 1, Nxg}) { rows[L(k, i, j) - 1].clear(); ident(k, i, j); }
    // CSR, diagonal first
    CSR& A = Lv.A; A.n = n; A.rp.assign(n + 1, 0);
    for (int r = 0; r < n; ++r) A.rp[r + 1] = A.rp[r] + (int)rows[r].cols.size();
    A.ci.resize(A.rp[n]); A.v.resize(A.rp[n]);
    for (int r = 0; r < n; ++r) {
        int o = A.rp[r];
        for (size_t t = 0; t < rows[r].cols.size(); ++t) { A.ci[o + t] = rows[r].cols[t] - 1; A.v[o + t] = rows[r].vals[t]; }
        for (int t = A.rp[r]; t < A.rp[r + 1]; ++t)
            if (A.ci[t] == r) { std::swap(A.ci[t], A.ci[o]); std::swap(A.v[t], A.v[o]); break; }
    }
    // multicolour classes for the device-matched smoother: the row couples to
    // diagonal neighbour columns only through the cross terms.
    double hmax = 0; for (size_t c = 0; c < G.hx.size(); ++c) hmax = std::max(hmax, std::max(std::fabs(G.hx[c]), std::fabs(G.hy[c])));
    Lv.ncolor = (Nyg > 1 && Nxg > 1) ? (hmax > 0 ? 4 : 2) : 2;
    Lv.cross = hmax > 0 ? 1 : 0;
    Lv.per = s.per;
}

static void dense_lu(Level& Lv) {
    int n = Lv.A.n;
    Lv.LU.assign((size_t)n * n, 0.0); Lv.piv.assign(n, 0);
    for (int r = 0; r < n; ++r)
        for (int t = Lv.A.rp[r]; t < Lv.A.rp[r + 1]; ++t) Lv.LU[(size_t)r * n + Lv.A.ci[t]] += Lv.A.v[t];
    double* a = Lv.LU.data();
    for (int k = 0; k < n; ++k) {
        int pr = k; double mx = std::fabs(a[(size_t)k * n + k]);
        for (int r = k + 1; r < n; ++r) if (std::fabs(a[(size_t)r * n + k]) > mx) { mx = std::fabs(a[(size_t)r * n + k]); pr = r; }
        Lv.piv[k] = pr;
        if (pr != k) for (int c = 0; c < n; ++c) std::swap(a[(size_t)k * n + c], a[(size_t)pr * n + c]);
        double d = a[(size_t)k * n + k];
        for (int r = k + 1; r < n; ++r) {
            double f = a[(size_t)r * n + k] / d; a[(size_t)r * n + k] = f;
            for (int c = k + 1; c < n; ++c) a[(size_t)r * n + c] -= f * a[(size_t)k * n + c];
        }
    }
}
static void dense_solve(const Level& Lv, double* x) {
    int n = Lv.A.n; const double* a = Lv.LU.data();
    for (int k = 0; k < n; ++k) if (Lv.piv[k] != k) std::swap(x[k], x[Lv.piv[k]]);
    for (int r = 0; r < n; ++r) { double s = x[r]; for (int c = 0; c < r; ++c) s -= a[(size_t)r * n + c] * x[c]; x[r] = s; }
    for (int r = n - 1; r >= 0; --r) { double s = x[r]; for (int c = r + 1; c < n; ++c) s -= a[(size_t)r * n + c] * x[c]; x[r] = s / a[(size_t)r * n + r]; }
}

// MGPreProcess.f90:376-439
static void build_ighost(Level& Lv) {
    const LevelGrid& G = Lv.G; Lv.ighost.clear();
    int gidx = 0;
    for (int jj = 1; jj <= G.Nyg; ++jj)
        for (int ii = 1; ii <= G.Nxg; ++ii)
            for (int kk = 1; kk <= G.Nzg; ++kk) {
                ++gidx;
                bool sp = (G.Nyg > 1 && G.Nxg > 1) ? (kk == 1 || ii == 1 || ii == G.Nxg || jj == 1 || jj == G.Nyg)
                        : (G.Nxg > 1 ? (kk == 1 || ii == 1 || ii == G.Nxg) : (kk == 1 || jj == 1 || jj == G.Nyg));
                if (sp) Lv.ighost.push_back(gidx);
            }
}

// ------------------------------------------------------- MG components
static inline void gs_row(const CSR& A, int r, double* x, const double* b) {
    double s = 0;
    for (int t = A.rp[r] + 1; t < A.rp[r + 1]; ++t) s += x[A.ci[t]] * A.v[t];
    x[r] = (b[r] - s) / A.v[A.rp[r]];
}
// GaussSeidel.f90:15-26
static void gs_lex(const CSR& A, double* x, const double* b) { for (int r = 0; r < A.n; ++r) gs_row(A, r, x, b); }
// GaussSeidelSpecialPoints.f90:43-53
static void gs_special(const Level& Lv, double* x, const double* b) {
    for (int g1 : Lv.ighost) gs_row(Lv.A, g1 - 1, x, b);
}
// Device-matched smoother (mode 1). One smoothing step is one pass per colour
// over the interior columns of that colour (2 colours by (i+j) parity, or 4 by
// (i, j) parities when mixed-derivative terms couple diagonal columns). The
// task of one interior column (i, j), in this order:
//   1. identity corner columns diagonal to it (3-D; (2,2) owns (1,1), ...),
//   2. the lateral ghost columns it reads (i = 2 -> (1, j), i = Nxg-1 ->
//      (Nxg, j), likewise in j), relaxed from the current values,
//   3. its bottom row (k = 1, the kinematic bottom condition),
//   4. its rows k = 2..Nzg, bottom to top,
//   5. its bottom row again (consistent with the new column),
//   6. the lateral ghost columns whose Neumann stencil contains the column
//      (i = 2 or 3 -> (1, j); i = Nxg-1 or Nxg-2 -> (Nxg, j); likewise in j).
// Each ghost column is thus relaxed after each of its two interior neighbours
// and ends every smoothing step consistent with both, as the reference's
// trailing GaussSeidelSpecialPoints pass leaves it.
// On levels with mixed-derivative terms the row k = 2 of a column next to a
// ghost column reads level-1 values of the columns two to the side (the
// shifted stencil of ConstructTableCrossDerivatives at the ghost level): the
// bottom rows of same-colour interior columns and the (identity) level-1 rows
// of ghost columns other same-colour tasks relax. There all level-1 rows --
// interior bottoms and ghost identities -- are relaxed in a separate pass
// before the first and after every colour sweep instead (steps 3 and 5 and the
// ghosts' level-1 rows dropped from the colour passes), so that no task reads
// what another task of its pass writes.
static void dm_pass(const Level& Lv, int colour, double* x, const double* b) {
    const LevelGrid& G = Lv.G; const int Nzg = G.Nzg, Nxg = G.Nxg, Nyg = G.Nyg;
    const bool three = Nxg > 1 && Nyg > 1;
    const bool fuse_bottom = !Lv.cross;
    auto col_rows = [&](int i, int j, int k0, int k1) {
        for (int k = k0; k <= k1; ++k) gs_row(Lv.A, (k - 1) + Nzg * ((i - 1) + Nxg * (j - 1)), x, b);
    };
    const int j0 = three ? 2 : 1, j1 = three ? Nyg - 1 : 1;
    const bool per = Lv.per != 0;
    const int ilast = per ? Nxg - 2 : Nxg - 1;   // periodic: the distinct columns only
    // the tasks of one colour read nothing another task of the colour writes,
    // so rows of tasks run in parallel with the same result as in sequence
#pragma omp parallel for schedule(static) if (three)
    for (int j = j0; j <= j1; ++j)
        for (int i = 2; i <= ilast; ++i) {
            const int col = (Lv.ncolor == 4) ? ((i & 1) + 2 * (j & 1)) : ((i + j) & 1);
            if (col != colour) continue;
            if (per) {
                // no x ghost columns; the y ghost columns as usual
                const int g0 = fuse_bottom ? 1 : 2;
                if (three && j == 2) col_rows(i, 1, g0, Nzg);
                if (three && j == Nyg - 1) col_rows(i, Nyg, g0, Nzg);
                col_rows(i, j, fuse_bottom ? 1 : 2, Nzg);
                if (fuse_bottom) col_rows(i, j, 1, 1);
                if (three && (j == 2 || j == 3)) col_rows(i, 1, g0, Nzg);
                if (three && (j == Nyg - 1 || j == Nyg - 2)) col_rows(i, Nyg, g0, Nzg);
                continue;
            }
            if (three) {
                const int cis[2] = {i == 2 ? 1 : 0, i == Nxg - 1 ? Nxg : 0};
                const int cjs[2] = {j == 2 ? 1 : 0, j == Nyg - 1 ? Nyg : 0};
                for (int ci : cis) for (int cj : cjs) if (ci && cj) col_rows(ci, cj, 1, Nzg);
            }
            const int g0 = fuse_bottom ? 1 : 2;   // first ghost row this pass relaxes
            if (i == 2) col_rows(1, j, g0, Nzg);
            if (i == Nxg - 1) col_rows(Nxg, j, g0, Nzg);
            if (three && j == 2) col_rows(i, 1, g0, Nzg);
            if (three && j == Nyg - 1) col_rows(i, Nyg, g0, Nzg);
            col_rows(i, j, fuse_bottom ? 1 : 2, Nzg);
            if (fuse_bottom) col_rows(i, j, 1, 1);
            if (i == 2 || i == 3) col_rows(1, j, g0, Nzg);
            if (i == Nxg - 1 || i == Nxg - 2) col_rows(Nxg, j, g0, Nzg);
            if (three && (j == 2 || j == 3)) col_rows(i, 1, g0, Nzg);
            if (three && (j == Nyg - 1 || j == Nyg - 2)) col_rows(i, Nyg, g0, Nzg);
        }
}
// Level-1 rows: bottom rows of all interior columns (each reads only rows >= 2)
// and the identity rows of the lateral ghost columns (corners excluded).
static void dm_bottoms(const Level& Lv, double* x, const double* b) {
    const LevelGrid& G = Lv.G; const int Nzg = G.Nzg, Nxg = G.Nxg, Nyg = G.Nyg;
    const bool three = Nxg > 1 && Nyg > 1;
    const int j0 = three ? 2 : 1, j1 = three ? Nyg - 1 : 1;
    auto row1 = [&](int i, int j) { gs_row(Lv.A, Nzg * ((i - 1) + Nxg * (j - 1)), x, b); };
    for (int j = j0; j <= j1; ++j)
        for (int i = 2; i <= Nxg - 1; ++i) row1(i, j);
    for (int j = j0; j <= j1; ++j) { row1(1, j); row1(Nxg, j); }
    if (three)
        for (int i = 2; i <= Nxg - 1; ++i) { row1(i, 1); row1(i, Nyg); }
}
static void dm_smooth(const Level& Lv, double* x, const double* b, int nu) {
    if (Lv.cross) dm_bottoms(Lv, x, b);
    for (int s = 0; s < nu; ++s) {
        for (int c = 0; c < Lv.ncolor; ++c) dm_pass(Lv, c, x, b);
        if (Lv.cross) dm_bottoms(Lv, x, b);
    }
}
static void csr_mv(const CSR& A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int r = 0; r < A.n; ++r) { double s = 0; for (int t = A.rp[r]; t < A.rp[r + 1]; ++t) s += A.v[t] * x[A.ci[t]]; y[r] = s; }
}

// MGRestriction3DExplicit.f90:19-128
static void restrict_(const Sim& s, const Level& Fl, const Level& Cl, const double* rf, double* rc) {
    const LevelGrid &F = Fl.G, &Cg = Cl.G;
    int Nxf = F.Nxg - 2 * s.gx, Nxc = Cg.Nxg - 2 * s.gx, Nyf = F.Nyg - 2 * s.gy, Nyc = Cg.Nyg - 2 * s.gy;
    int Nzf = F.Nzg - s.gz, Nzc = Cg.Nzg - s.gz;
    int xc = Nxf > Nxc, yc = Nyf > Nyc, zc = Nzf > Nzc;
    vector<double> t(rf, rf + (size_t)F.Nxg * F.Nyg * F.Nzg);
    auto I = [&](int k, int i, int j) -> size_t { return (size_t)(k - 1) + (size_t)F.Nzg * ((size_t)(i - 1) + (size_t)F.Nxg * (j - 1)); };
    const double half = 0.5, one = 1.0;
    // each sweep writes the points of one parity from the other parity only
    if (xc) {
        // periodic x: the west neighbour of the first column is the last
        // distinct column (same spacing), and the repeated column is skipped
        const int ilast = s.per ? Nxf + s.gx - 1 : Nxf + s.gx;
#pragma omp parallel for schedule(static)
        for (int ifn = 1 + s.gx; ifn <= ilast; ifn += 2) {
            double dW = F.x[ifn - 1] - F.x[ifn - 2], dE = F.x[ifn] - F.x[ifn - 1];
            double dxc = one / (dW + dE);
            const int iw = s.per ? wrap_x(ifn - 1, F.Nxg) : ifn - 1;
            for (int kf = 1 + s.gz; kf <= Nzf + s.gz - 1; ++kf)
                for (int jf = 1 + s.gy; jf <= Nyf + s.gy; ++jf)
                    t[I(kf, ifn, jf)] = (half * dxc) * (dW * t[I(kf, iw, jf)] + (dW + dE) * t[I(kf, ifn, jf)] + dE * t[I(kf, ifn + 1, jf)]);
        }
    }
    if (yc) {
#pragma omp parallel for schedule(static)
        for (int jf = 1 + s.gy; jf <= Nyf + s.gy; jf += 2) {
            double dS = F.y[jf - 1] - F.y[jf - 2], dN = F.y[jf] - F.y[jf - 1];
            double dyc = one / (dS + dN);
            for (int kf = 1 + s.gz; kf <= Nzf + s.gz - 1; ++kf)
                for (int ifn = 1 + s.gx; ifn <= Nxf + s.gx; ifn += 1 + xc)
                    t[I(kf, ifn, jf)] = (half * dyc) * (dS * t[I(kf, ifn, jf - 1)] + (dN + dS) * t[I(kf, ifn, jf)] + dN * t[I(kf, ifn, jf + 1)]);
        }
    }
    if (zc) {
        for (int kf = 1 + s.gz; kf <= Nzf + s.gz - 1; kf += 2) {
            double dU = F.z[kf] - F.z[kf - 1], dD = F.z[kf - 1] - F.z[kf - 2];
            double dzc = one / (dD + dU);
#pragma omp parallel for schedule(static)
            for (int ifn = 1 + s.gx; ifn <= Nxf + s.gx; ifn += 1 + xc)
                for (int jf = 1 + s.gy; jf <= Nyf + s.gy; jf += 1 + yc)
                    t[I(kf, ifn, jf)] = (half * dzc) * (dD * t[I(kf - 1, ifn, jf)] + dU * t[I(kf + 1, ifn, jf)]) + half * t[I(kf, ifn, jf)];
        }
    }
    std::fill(rc, rc + (size_t)Cg.Nxg * Cg.Nyg * Cg.Nzg, 0.0);
#pragma omp parallel for schedule(static)
    for (int jc = 1 + s.gy; jc <= Nyc + s.gy; ++jc)
        for (int ic = 1 + s.gx; ic <= Nxc + s.gx; ++ic)
            for (int kc = 1 + s.gz; kc <= Nzc + s.gz; ++kc) {
                int kf = 1 + s.gz + (kc - 1 - s.gz) * (1 + zc), ifn = 1 + s.gx + (ic - 1 - s.gx) * (1 + xc), jf = 1 + s.gy + (jc - 1 - s.gy) * (1 + yc);
                rc[(size_t)(kc - 1) + (size_t)Cg.Nzg * ((size_t)(ic - 1) + (size_t)Cg.Nxg * (jc - 1))] =
                    (s.per && ic == Cg.Nxg - 1) ? 0.0 : t[I(kf, ifn, jf)];
            }
}

// MGProlongation3DExplicit.f90:19-110
static void prolong_(const Sim& s, const Level& Fl, const Level& Cl, double* pf, const double* pc) {
    const LevelGrid &F = Fl.G, &Cg = Cl.G;
    int Nxf = F.Nxg - 2 * s.gx, Nxc = Cg.Nxg - 2 * s.gx, Nyf = F.Nyg - 2 * s.gy, Nyc = Cg.Nyg - 2 * s.gy;
    int Nzf = F.Nzg - s.gz, Nzc = Cg.Nzg - s.gz;
    int XF = Nxf > Nxc ? 2 : 1, YF = Nyf > Nyc ? 2 : 1, ZF = Nzf > Nzc ? 2 : 1;
    auto I = [&](int k, int i, int j) -> size_t { return (size_t)(k - 1) + (size_t)F.Nzg * ((size_t)(i - 1) + (size_t)F.Nxg * (j - 1)); };
    auto Ic = [&](int k, int i, int j) -> size_t { return (size_t)(k - 1) + (size_t)Cg.Nzg * ((size_t)(i - 1) + (size_t)Cg.Nxg * (j - 1)); };
    std::fill(pf, pf + (size_t)F.Nxg * F.Nyg * F.Nzg, 0.0);
#pragma omp parallel for schedule(static)
    for (int jc = 1 + s.gy; jc <= Nyc + s.gy; ++jc)
        for (int ic = 1 + s.gx; ic <= Nxc + s.gx; ++ic)
            for (int kc = 1 + s.gz; kc <= Nzc + s.gz - 1; ++kc)
                pf[I(1 + s.gz + (kc - 1 - s.gz) * ZF, 1 + s.gx + (ic - 1 - s.gx) * XF, 1 + s.gy + (jc - 1 - s.gy) * YF)] = pc[Ic(kc, ic, jc)];
    const double one = 1.0;
    if (XF == 2) {
#pragma omp parallel for schedule(static)
        for (int jf = 1 + s.gy; jf <= Nyf + s.gy; jf += YF)
            for (int ifn = 2 + s.gx; ifn <= Nxf + s.gx; ifn += XF) {
                double dW = F.x[ifn - 1] - F.x[ifn - 2], dE = F.x[ifn] - F.x[ifn - 1], dxf = one / (dW + dE);
                // periodic x: the repeated column holds zero, its value is column 2's
                const int ie = (s.per && ifn + 1 == F.Nxg - 1) ? 2 : ifn + 1;
                for (int kf = 1 + s.gz; kf <= Nzf + s.gz - 1; kf += ZF)
                    pf[I(kf, ifn, jf)] = (dE * pf[I(kf, ifn - 1, jf)] + dW * pf[I(kf, ie, jf)]) * dxf;
            }
    }
    if (YF == 2) {
#pragma omp parallel for schedule(static)
        for (int ifn = 1 + s.gx; ifn <= Nxf + s.gx; ++ifn)
            for (int jf = 2 + s.gy; jf <= Nyf + s.gy; jf += YF) {
                double dS = F.y[jf - 1] - F.y[jf - 2], dN = F.y[jf] - F.y[jf - 1], dyf = one / (dS + dN);
                for (int kf = 1 + s.gz; kf <= Nzf + s.gz - 1; kf += ZF)
                    pf[I(kf, ifn, jf)] = (dN * pf[I(kf, ifn, jf - 1)] + dS * pf[I(kf, ifn, jf + 1)]) * dyf;
            }
    }
    if (ZF == 2) {
        for (int kf = 2 + s.gz; kf <= Nzf + s.gz - 1; kf += ZF) {
            double dD = F.z[kf - 1] - F.z[kf - 2], dU = F.z[kf] - F.z[kf - 1], dzf = one / (dD + dU);
#pragma omp parallel for schedule(static)
            for (int jf = 1 + s.gy; jf <= Nyf + s.gy; ++jf)
                for (int ifn = 1 + s.gx; ifn <= Nxf + s.gx; ++ifn)
                    pf[I(kf, ifn, jf)] = (dU * pf[I(kf - 1, ifn, jf)] + dD * pf[I(kf + 1, ifn, jf)]) * dzf;
        }
    }
}

// MultiGridSolver.f90:5-192 (V cycle)
static void mg_solver(Sim& s, int k, double* x, const double* b) {
    Level& Lv = s.lev[k];
    if (k == 0) {
        size_t n = Lv.A.n;
        for (size_t t = 0; t < n; ++t) x[t] = b[t];
        dense_solve(Lv, x);
        return;
    }
    auto smooth = [&](int nu) {
        if (s.mode == 0) { gs_special(Lv, x, b); for (int i = 0; i < nu; ++i) { gs_lex(Lv.A, x, b); gs_special(Lv, x, b); } }
        else dm_smooth(Lv, x, b, nu);
    };
    smooth(s.p.nu1);
    size_t n = Lv.A.n;
    vector<double> Ax(n), r(n);
    csr_mv(Lv.A, x, Ax.data());
#pragma omp parallel for schedule(static)
    for (long t = 0; t < (long)n; ++t) r[t] = b[t] - Ax[t];
    Level& Cl = s.lev[k - 1];
    vector<double> rc(Cl.A.n), dxc(Cl.A.n, 0.0), dxf(n);
    restrict_(s, Lv, Cl, r.data(), rc.data());
    mg_solver(s, k - 1, dxc.data(), rc.data());
    prolong_(s, Lv, Cl, dxf.data(), dxc.data());
#pragma omp parallel for schedule(static)
    for (long t = 0; t < (long)n; ++t) x[t] += dxf[t];
    smooth(s.p.nu2);
}

// MultiGridSolveLinearSystem.f90:26-91
static void precond(Sim& s, const double* r, double* u) {
    int L = (int)s.lev.size();
    if (L == 0) { std::copy(r, r + s.N, u); return; }
    std::fill(u, u + s.N, 0.0);
    for (int it = 1; it <= s.p.maxit; ++it) {
        if (L == 1 && it > 1) break;
        mg_solver(s, L - 1, u, r);
    }
}

// ------------------------------------------------- high-order operator
// DiffXEven.f90, DiffYEven.f90, DiffZArbitrary.f90 on a (Nz,Nx,Ny) array.
static void diff_x(const Sim& s, const double* v, double* o, int order, int Nz) {
    int a = s.p.alpha, rank = 2 * a + 1, Nx = s.Nxg, Ny = s.Nyg;
    if (s.per) {
        // centred stencils on the distinct columns, indices taken cyclically
        for (int j = 1; j <= Ny; ++j)
            for (int i = 2; i <= Nx - 2; ++i)
                for (int k = 1; k <= Nz; ++k) {
                    double acc = 0;
                    for (int m = 0; m < rank; ++m)
                        acc += s.SX.at(order, i - 1, m) * v[(size_t)(k - 1) + (size_t)Nz * ((size_t)(wrap_x(i - a + m, Nx) - 1) + (size_t)Nx * (j - 1))];
                    o[(size_t)(k - 1) + (size_t)Nz * ((size_t)(i - 1) + (size_t)Nx * (j - 1))] = acc;
                }
        images_x(s, o, Nz);
        return;
    }
#pragma omp parallel for schedule(static) if (Ny > 1)
    for (int j = 1; j <= Ny; ++j)
        for (int i = 1; i <= Nx; ++i) {
            int st = (i <= a) ? 1 : (i <= Nx - a ? i - a : Nx + 1 - rank);
            for (int k = 1; k <= Nz; ++k) {
                double acc = 0;
                for (int m = 0; m < rank; ++m) acc += s.SX.at(order, i - 1, m) * v[(size_t)(k - 1) + (size_t)Nz * ((size_t)(st + m - 1) + (size_t)Nx * (j - 1))];
                o[(size_t)(k - 1) + (size_t)Nz * ((size_t)(i - 1) + (size_t)Nx * (j - 1))] = acc;
            }
        }
}
static void diff_y(const Sim& s, const double* v, double* o, int order, int Nz) {
    int b = s.p.beta, rank = 2 * b + 1, Nx = s.Nxg, Ny = s.Nyg;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= Ny; ++j) {
        int st = (j <= b) ? 1 : (j <= Ny - b ? j - b : Ny + 1 - rank);
        for (int i = 1; i <= Nx; ++i)
            for (int k = 1; k <= Nz; ++k) {
                double acc = 0;
                for (int m = 0; m < rank; ++m) acc += s.SY.at(order, j - 1, m) * v[(size_t)(k - 1) + (size_t)Nz * ((size_t)(i - 1) + (size_t)Nx * (st + m - 1))];
                o[(size_t)(k - 1) + (size_t)Nz * ((size_t)(i - 1) + (size_t)Nx * (j - 1))] = acc;
            }
    }
}
static void diff_z(const Sim& s, const double* v, double* o, int order) {
    int g = s.p.gamma, rank = 2 * g + 1, Nz = s.Nzg;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < s.C; ++c)
        for (int k = 1; k <= Nz; ++k) {
            int st = (k <= g) ? 1 : (k <= Nz - g ? k - g : Nz + 1 - rank);
            double acc = 0;
            for (int m = 0; m < rank; ++m) acc += s.SZ.at(order, k - 1, m) * v[(size_t)c * Nz + st + m - 1];
            o[(size_t)c * Nz + k - 1] = acc;
        }
}

// BuildLinearSystem.f90:1-290 with DiffXEven_CD / DiffZArbitrary_CD tables.
static void matvec_ho(Sim& s, const double* phi, double* out) {
    const int Nx = s.Nxg, Ny = s.Nyg, Nz = s.Nzg, rank = s.T.rank;
    const size_t N = s.N;
    vector<double> dpdx(N, 0), ddpdxx(N, 0), dpdy(N, 0), ddpdyy(N, 0), dpds(N), ddpdss(N), tmp(N), ddpdsdx(N, 0), ddpdsdy(N, 0);
    const double* dsg = s.dsig.data();
    auto DS = [&](int k, int i, int j, int c) { return dsg[gid(s, k, i, j) * 5 + (c - 1)]; };
    if (Nx > 1 && s.per) {
        // no lateral walls: the mixed derivative is D_sigma(D_x phi) with the
        // centred x stencil at every level (no shifted windows)
        diff_x(s, phi, dpdx.data(), 1, Nz); diff_x(s, phi, ddpdxx.data(), 2, Nz);
        diff_z(s, dpdx.data(), ddpdsdx.data(), 1);
    } else if (Nx > 1) {
        diff_x(s, phi, dpdx.data(), 1, Nz); diff_x(s, phi, ddpdxx.data(), 2, Nz);
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= Ny; ++j) for (int i = 1; i <= Nx; ++i) for (int k = 1; k <= Nz; ++k) {
            double acc = 0;
            for (int m = 0; m < rank; ++m) acc += s.T.SX[s.T.id(k, i, j, m)] * phi[gid(s, k, s.T.IX[s.T.id(k, i, j, m)], j)];
            tmp[gid(s, k, i, j)] = acc;
        }
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= Ny; ++j) for (int i = 1; i <= Nx; ++i) for (int k = 1; k <= Nz; ++k) {
            double acc = 0;
            for (int m = 0; m < rank; ++m) acc += s.T.SZ1[s.T.id(k, i, j, m)] * tmp[gid(s, s.T.IZ1[s.T.id(k, i, j, m)], i, j)];
            ddpdsdx[gid(s, k, i, j)] = acc;
        }
    }
    if (Ny > 1) {
        diff_y(s, phi, dpdy.data(), 1, Nz); diff_y(s, phi, ddpdyy.data(), 2, Nz);
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= Ny; ++j) for (int i = 1; i <= Nx; ++i) for (int k = 1; k <= Nz; ++k) {
            double acc = 0;
            for (int m = 0; m < rank; ++m) acc += s.T.SY[s.T.id(k, i, j, m)] * phi[gid(s, k, i, s.T.IY[s.T.id(k, i, j, m)])];
            tmp[gid(s, k, i, j)] = acc;
        }
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= Ny; ++j) for (int i = 1; i <= Nx; ++i) for (int k = 1; k <= Nz; ++k) {
            double acc = 0;
            for (int m = 0; m < rank; ++m) acc += s.T.SZ2[s.T.id(k, i, j, m)] * tmp[gid(s, s.T.IZ2[s.T.id(k, i, j, m)], i, j)];
            ddpdsdy[gid(s, k, i, j)] = acc;
        }
    }
    diff_z(s, phi, dpds.data(), 1); diff_z(s, phi, ddpdss.data(), 2);
    std::fill(out, out + N, 0.0);
    const int gx = s.gx, gy = s.gy, gz = s.gz;
    const double two = 2.0;
    if (Nx == 1) {
        for (int j = 1 + gy; j <= Ny - gy; ++j) for (int k = 1; k <= Nz; ++k) {
            size_t G = gid(s, k, 1, j); double hy = s.fine.hy[(size_t)Nx * (j - 1)];
            if (k == Nz) out[G] = phi[G];
            else if (k == 1) out[G] = (DS(k + gz, 1, j, 5) + hy * DS(k + gz, 1, j, 4)) * dpds[G + gz] + hy * dpdy[G + gz];
            else out[G] = ddpdyy[G] + DS(k, 1, j, 3) * dpds[G] + two * (DS(k, 1, j, 4) * ddpdsdy[G]) +
                          (DS(k, 1, j, 4) * DS(k, 1, j, 4) + DS(k, 1, j, 5) * DS(k, 1, j, 5)) * ddpdss[G];
        }
    } else if (Ny == 1) {
        for (int i = 1 + gx; i <= Nx - gx; ++i) for (int k = 1; k <= Nz; ++k) {
            size_t G = gid(s, k, i, 1); double hx = s.fine.hx[i - 1];
            if (k == Nz) out[G] = phi[G];
            else if (k == 1) out[G] = hx * dpdx[G + gz] + (DS(k + gz, i, 1, 5) + hx * DS(k + gz, i, 1, 2)) * dpds[G + gz];
            else out[G] = ddpdxx[G] + two * DS(k, i, 1, 2) * ddpdsdx[G] +
                          (DS(k, i, 1, 2) * DS(k, i, 1, 2) + DS(k, i, 1, 5) * DS(k, i, 1, 5)) * ddpdss[G] + DS(k, i, 1, 3) * dpds[G];
        }
    } else {
#pragma omp parallel for schedule(static)
        for (int j = 1 + gy; j <= Ny - gy; ++j) for (int i = 1 + gx; i <= Nx - gx; ++i) for (int k = 1; k <= Nz; ++k) {
            size_t G = gid(s, k, i, j); size_t c = (size_t)(i - 1) + (size_t)Nx * (j - 1);
            double hx = s.fine.hx[c], hy = s.fine.hy[c];
            if (k == Nz) out[G] = phi[G];
            else if (k == 1)
                out[G] = (DS(k + gz, i, j, 5) + hx * DS(k + gz, i, j, 2) + hy * DS(k + gz, i, j, 4)) * dpds[G + gz] +
                         hx * dpdx[G + gz] + hy * dpdy[G + gz];
            else
                out[G] = ddpdxx[G] + ddpdyy[G] + DS(k, i, j, 3) * dpds[G] +
                         two * (DS(k, i, j, 2) * ddpdsdx[G] + DS(k, i, j, 4) * ddpdsdy[G]) +
                         (DS(k, i, j, 2) * DS(k, i, j, 2) + DS(k, i, j, 4) * DS(k, i, j, 4) + DS(k, i, j, 5) * DS(k, i, j, 5)) * ddpdss[G];
        }
    }
    if (gx == 1) {
        for (int j = 1 + gy; j <= Ny - gy; ++j) for (int k = 1; k <= Nz; ++k) {
            out[gid(s, k, 1, j)] = dpdx[gid(s, k, 2, j)];
            out[gid(s, k, Nx, j)] = dpdx[gid(s, k, Nx - 1, j)];
        }
    }
    if (gy == 1) {
        for (int i = 1 + gx; i <= Nx - gx; ++i) for (int k = 1; k <= Nz; ++k) {
            out[gid(s, k, i, 1)] = dpdy[gid(s, k, i, 2)];
            out[gid(s, k, i, Ny)] = dpdy[gid(s, k, i, Ny - 1)];
        }
    }
    auto id_ = [&](int k, int i, int j) { size_t G = gid(s, k, i, j); out[G] = phi[G]; };
    if (gx + gy == 2) {
        for (int k = 1; k <= Nz; ++k) { id_(k, 1, 1); id_(k, Nx, 1); id_(k, 1, Ny); id_(k, Nx, Ny); }
        for (int i = 1; i <= Nx; ++i) { id_(1, i, 1); id_(1, i, Ny); }
        for (int j = 1; j <= Ny; ++j) { id_(1, 1, j); id_(1, Nx, j); }
    }
    if (gx == 1 && Ny == 1) { id_(1, 1, 1); id_(1, Nx, 1); }
    if (gy == 1 && Nx == 1) { id_(1, 1, 1); id_(1, 1, Ny); }
    if (s.per)   // the ghost columns and the repeated column are identity rows
        for (int j = 1; j <= Ny; ++j)
            for (int k = 1; k <= Nz; ++k) { id_(k, 1, j); id_(k, Nx - 1, j); id_(k, Nx, j); }
}

// DetermineTransformationConstantsArray for the surface state (E..Eyy).
static void update_sigma(Sim& s, const double* E, const double* Ex, const double* Exx, const double* Ey, const double* Eyy) {
    s.dsig.assign((size_t)5 * s.N, 0.0);
    const LevelGrid& G = s.fine;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < s.C; ++c) {
        double e = E ? E[c] : 0, ex = (Ex && s.Nxg > 1) ? Ex[c] : 0, exx = (Exx && s.Nxg > 1) ? Exx[c] : 0;
        double ey = (Ey && s.Nyg > 1) ? Ey[c] : 0, eyy = (Eyy && s.Nyg > 1) ? Eyy[c] : 0;
        for (int k = 1; k <= s.Nzg; ++k) {
            double zk = (k == 1) ? 0.0 : G.z[k - 1];
            sigma_coeffs(s.dimcase, zk, e, ex, exx, ey, eyy, G.h[c], G.hx[c], G.hxx[c], G.hy[c], G.hyy[c],
                         &s.dsig[((size_t)c * s.Nzg + k - 1) * 5]);
        }
    }
}

// ---------------------------------------------------------------- GMRES
static double dot(const double* a, const double* b, size_t n) {
    double acc = 0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (long t = 0; t < (long)n; ++t) acc += a[t] * b[t];
    return acc;
}

// Plane rotation [c s; -s c] that maps (x, y) to (r, 0), r = sqrt(x^2 + y^2)
// (the role of SPARSKIT2 `givens` in gmres).
static void givens(double& x, double& y, double& c, double& sn) {
    double r = std::sqrt(x * x + y * y);
    if (r == 0.0) { c = 1.0; sn = 0.0; return; }
    c = x / r; sn = y / r; x = r; y = 0.0;
}

// Left-preconditioned GMRES with the reverse-communication semantics of
// iterative_solution.f90:20-56 (restated from SPARSKIT2 gmres/mgsro).
static int solve_lgmres(Sim& s, const double* rhs, double* sol, int& iters, double& resid) {
    const size_t n = s.N; const int m = std::max(2, s.p.GMRESmaxiterations);
    const int maxmv = m;
    vector<vector<double>> V(m + 1, vector<double>(n));
    vector<double> w(n), u(n), H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1);
    int mv = 0; double tol = 0; bool first = true;
    iters = 0;
    for (;;) {
        matvec_ho(s, sol, w.data()); ++mv;
        for (size_t t = 0; t < n; ++t) w[t] = rhs[t] - w[t];
        precond(s, w.data(), V[0].data());
        double beta = std::sqrt(dot(V[0].data(), V[0].data(), n));
        if (first) { tol = s.p.reltol * beta + s.p.abstol; first = false; }
        resid = beta;
        if (beta <= tol) { iters = mv; return OW3D_OK; }
        for (size_t t = 0; t < n; ++t) V[0][t] /= beta;
        std::fill(g.begin(), g.end(), 0.0); g[0] = beta;
        int k = 0;
        for (;;) {
            ++k;
            matvec_ho(s, V[k - 1].data(), w.data()); ++mv;
            precond(s, w.data(), u.data());
            // mgsro (MGS with selective re-orthogonalisation, reorth = 0.98)
            double nrm0 = dot(u.data(), u.data(), n), thr = nrm0 * 0.98;
            double* hc = &H[(size_t)(k - 1) * (m + 1)];
            for (int i = 0; i < k; ++i) {
                double fct = dot(u.data(), V[i].data(), n); hc[i] = fct;
                for (size_t t = 0; t < n; ++t) u[t] -= fct * V[i][t];
                if (fct * fct > thr) {
                    fct = dot(u.data(), V[i].data(), n); hc[i] += fct;
                    for (size_t t = 0; t < n; ++t) u[t] -= fct * V[i][t];
                }
                nrm0 -= hc[i] * hc[i]; if (nrm0 < 0) nrm0 = 0; thr = nrm0 * 0.98;
            }
            double nrm1 = std::sqrt(dot(u.data(), u.data(), n));
            hc[k] = nrm1;
            if (nrm1 > 0) for (size_t t = 0; t < n; ++t) V[k][t] = u[t] / nrm1;
            for (int i = 0; i < k - 1; ++i) {
                double a0 = hc[i];
                hc[i] = cs[i] * a0 + sn[i] * hc[i + 1];
                hc[i + 1] = cs[i] * hc[i + 1] - sn[i] * a0;
            }
            double c, sg; givens(hc[k - 1], hc[k], c, sg); cs[k - 1] = c; sn[k - 1] = sg;
            double al = -sg * g[k - 1]; g[k - 1] = c * g[k - 1]; g[k] = al;
            resid = std::fabs(al);
            if (k < m && !(resid <= tol) && mv < maxmv && nrm1 > 0) continue;
            break;
        }
        // back substitution and update sol += V y
        int kk = k;
        while (kk > 0 && H[(size_t)(kk - 1) * (m + 1) + kk - 1] == 0.0) --kk;
        vector<double> y(kk);
        for (int i = kk - 1; i >= 0; --i) {
            double t = g[i];
            for (int j = i + 1; j < kk; ++j) t -= H[(size_t)j * (m + 1) + i] * y[j];
            y[i] = t / H[(size_t)i * (m + 1) + i];
        }
        for (int i = 0; i < kk; ++i) for (size_t t = 0; t < n; ++t) sol[t] += y[i] * V[i][t];
        if (resid <= tol) { iters = mv; return OW3D_OK; }
        if (mv >= maxmv) { iters = mv; return OW3D_NOT_CONVERGED; }
    }
}

// Right-preconditioned flexible GMRES as the device path runs it: classical
// Gram-Schmidt, one re-orthogonalisation pass when the norm drops below
// 1/sqrt(2) of its value before projection (Daniel-Gragg-Kaufman-Stewart).
// Right-preconditioned flexible GMRES (device mode, krylov = FGMRES) with
// delayed classical Gram-Schmidt with reorthogonalisation (DCGS2: Swirydowicz,
// Langou, Ananthan, Yang, Thomas, "Low synchronization Gram-Schmidt and
// generalized minimal residual algorithms", NLAA 2021). Step j:
//   z_j = M^{-1} (s_j V_j), W = A z_j;
//   one reduction: a_i = <V_i, V_j> (i < j), alpha = <V_j, V_j>, b_i = <V_i, W> (i <= j);
//   the second Gram-Schmidt pass of V_j, lagged by one step: sigma_i = s_i a_i,
//   nu = sqrt(alpha - sum sigma_i^2), q_j = (V_j - sum sigma_i s_i V_i) / nu, which
//   completes Hessenberg column j-1 (H[j-1][i] += sigma_i, H[j-1][j] = nu) and
//   its Givens rotation;
//   column j: h_i = s_i b_i (i < j), h_j = (b_j - sum sigma_i s_i b_i) / nu;
//   one update: V_j <- nu q_j, W <- W - sum_i h_i q_i, |W| gives H[j][j+1];
//   the Givens rotation of column j and the stopping test use that norm (the
//   next step's reorthogonalisation of W refines the column and its rotation).
// Vectors are stored unnormalised with s_i = 1/|V_i| as on the device.
static int solve_fgmres(Sim& s, const double* rhs, double* sol, int& iters, double& resid) {
    const size_t n = s.N; const int m = std::max(2, s.p.GMRESmaxiterations);
    const int maxmv = m;
    vector<vector<double>> V(m + 1, vector<double>(n)), Z(m, vector<double>(n));
    vector<double> W(n), vin(n), sc(m + 2), Hr((size_t)(m + 1) * (m + 1), 0.0), R((size_t)(m + 1) * (m + 1), 0.0);
    vector<double> cs(m + 1), sn(m + 1), g(m + 2), gsave(m + 1), a(m + 1), bb(m + 1), sig(m + 1), hq(m + 1);
    auto HR = [&](int col, int row) -> double& { return Hr[(size_t)col * (m + 1) + row]; };
    auto RR = [&](int col, int row) -> double& { return R[(size_t)col * (m + 1) + row]; };
    // rotate raw column col with the rotations 0..col-1, form rotation col and update g
    auto rotate = [&](int col) {
        for (int r = 0; r <= col + 1; ++r) RR(col, r) = HR(col, r);
        for (int i = 0; i < col; ++i) {
            const double a0 = RR(col, i);
            RR(col, i) = cs[i] * a0 + sn[i] * RR(col, i + 1);
            RR(col, i + 1) = cs[i] * RR(col, i + 1) - sn[i] * a0;
        }
        double c, sg;
        givens(RR(col, col), RR(col, col + 1), c, sg);
        cs[col] = c; sn[col] = sg;
        g[col] = gsave[col];
        const double al = -sg * g[col];
        g[col] = c * g[col];
        g[col + 1] = al;
        return std::fabs(al);
    };
    int mv = 0; double tol = 0; bool first = true;
    for (;;) {
        matvec_ho(s, sol, W.data()); ++mv;
        for (size_t t = 0; t < n; ++t) V[0][t] = rhs[t] - W[t];
        double beta = std::sqrt(dot(V[0].data(), V[0].data(), n));
        if (first) { tol = s.p.reltol * beta + s.p.abstol; first = false; }
        resid = beta;
        if (beta <= tol) { iters = mv; return OW3D_OK; }
        sc[0] = 1.0 / beta;
        std::fill(g.begin(), g.end(), 0.0); g[0] = beta;
        std::fill(Hr.begin(), Hr.end(), 0.0);
        int k = 0;
        for (int j = 0;; ++j) {
#pragma omp parallel for schedule(static)
            for (long t = 0; t < (long)n; ++t) vin[t] = V[j][t] * sc[j];
            precond(s, vin.data(), Z[j].data());
            matvec_ho(s, Z[j].data(), W.data()); ++mv;
            for (int i = 0; i < j; ++i) a[i] = dot(V[i].data(), V[j].data(), n);
            const double alpha = dot(V[j].data(), V[j].data(), n);
            for (int i = 0; i <= j; ++i) bb[i] = dot(V[i].data(), W.data(), n);
            if (j >= 1) {
                double ss = 0;
                for (int i = 0; i < j; ++i) { sig[i] = sc[i] * a[i]; ss += sig[i] * sig[i]; }
                const double nu = std::sqrt(std::max(alpha - ss, 0.0));
                for (int i = 0; i < j; ++i) HR(j - 1, i) += sig[i];
                HR(j - 1, j) = nu;
                sc[j] = nu > 0 ? 1.0 / nu : 0.0;
                resid = rotate(j - 1);
            }
            double corr = 0;
            for (int i = 0; i < j; ++i) { hq[i] = sc[i] * bb[i]; corr += sig[i] * hq[i]; }
            const double hj = (j >= 1) ? (bb[j] - corr) * sc[j] : sc[j] * bb[j];
            for (int i = 0; i < j; ++i) HR(j, i) = hq[i];
            HR(j, j) = hj;
            // update: V_j <- V_j - sum sigma_i s_i V_i ; W <- W - sum h_i s_i V_i - h_j s_j V_j(new)
            double ww = 0;
#pragma omp parallel for reduction(+ : ww) schedule(static)
            for (long t = 0; t < (long)n; ++t) {
                double vj = V[j][t], w = W[t];
                for (int i = 0; i < j; ++i) { vj -= sig[i] * sc[i] * V[i][t]; w -= hq[i] * sc[i] * V[i][t]; }
                w -= hj * sc[j] * vj;
                V[j][t] = vj; W[t] = w;
                ww += w * w;
            }
            const double nrm = std::sqrt(ww);
            V[j + 1] = W;
            HR(j, j + 1) = nrm;
            sc[j + 1] = nrm > 0 ? 1.0 / nrm : 0.0;
            gsave[j] = g[j];
            resid = rotate(j);
            k = j + 1;
            if (k < m && !(resid <= tol) && mv < maxmv && nrm > 0) continue;
            break;
        }
        int kk = k;
        while (kk > 0 && RR(kk - 1, kk - 1) == 0.0) --kk;
        vector<double> y(kk);
        for (int i = kk - 1; i >= 0; --i) {
            double t = g[i];
            for (int j = i + 1; j < kk; ++j) t -= RR(j, i) * y[j];
            y[i] = t / RR(i, i);
        }
#pragma omp parallel for schedule(static)
        for (long t = 0; t < (long)n; ++t) { double acc = sol[t]; for (int i = 0; i < kk; ++i) acc += y[i] * Z[i][t]; sol[t] = acc; }
        if (resid <= tol) { iters = mv; return OW3D_OK; }
        if (mv >= maxmv) { iters = mv; return OW3D_NOT_CONVERGED; }
    }
}

static int solve(Sim& s, const double* rhs, double* sol, int& iters, double& resid) {
    bool left = (s.mode == 0) || (s.p.krylov == OW3D_KRYLOV_LGMRES);
    int st = left ? solve_lgmres(s, rhs, sol, iters, resid) : solve_fgmres(s, rhs, sol, iters, resid);
    ++s.solves; s.totit += iters; s.lastit = iters; s.lastres = resid;
    s.minit = std::min(s.minit, iters); s.maxit = std::max(s.maxit, iters);
    if (st == OW3D_NOT_CONVERGED) ++s.notconv;
    return st;
}

// ------------------------------------------------- free-surface operators
// 2-D x/y differentiation of a (Nxg,Nyg) field: DiffXEven with Nz = 1.
static void dx2(const Sim& s, const double* v, double* o, int order) { diff_x(s, v, o, order, 1); }
static void dy2(const Sim& s, const double* v, double* o, int order) { diff_y(s, v, o, order, 1); }

// UpdateGhostLayerX.f90:15-20, UpdateGhostLayerY.f90
static void ghost_x(const Sim& s, double* v, const double* S) {
    int a = s.p.alpha, rank = 2 * a + 1, Nx = s.Nxg;
    for (int j = 1 + s.gy; j <= s.Nyg - s.gy; ++j) {
        double* r = v + (size_t)Nx * (j - 1); const double* Sr = S + (size_t)Nx * (j - 1);
        double acc = 0;
        for (int m = 1; m < rank; ++m) acc += s.SX.at(1, 1 + s.gx - 1, m) * r[m];
        r[0] = (Sr[1 + s.gx - 1] - acc) / s.SX.at(1, 1 + s.gx - 1, 0);
        acc = 0;
        for (int m = 0; m < rank - 1; ++m) acc += s.SX.at(1, Nx - s.gx - 1, m) * r[Nx - rank + m];
        r[Nx - 1] = (Sr[Nx - s.gx - 1] - acc) / s.SX.at(1, Nx - s.gx - 1, rank - 1);
    }
}
static void ghost_y(const Sim& s, double* v, const double* S) {
    int b = s.p.beta, rank = 2 * b + 1, Nx = s.Nxg, Ny = s.Nyg;
    for (int i = 1 + s.gx; i <= Nx - s.gx; ++i) {
        double acc = 0;
        for (int m = 1; m < rank; ++m) acc += s.SY.at(1, 1 + s.gy - 1, m) * v[(size_t)(i - 1) + (size_t)Nx * m];
        v[(size_t)(i - 1)] = (S[(size_t)(i - 1) + (size_t)Nx * (1 + s.gy - 1)] - acc) / s.SY.at(1, 1 + s.gy - 1, 0);
        acc = 0;
        for (int m = 0; m < rank - 1; ++m) acc += s.SY.at(1, Ny - s.gy - 1, m) * v[(size_t)(i - 1) + (size_t)Nx * (Ny - rank + m)];
        v[(size_t)(i - 1) + (size_t)Nx * (Ny - 1)] = (S[(size_t)(i - 1) + (size_t)Nx * (Ny - s.gy - 1)] - acc) / s.SY.at(1, Ny - s.gy - 1, rank - 1);
    }
}
// DifferentiationsFreeSurfacePlane.f90:13-32 (Cartesian branch)
// tmp: the RK stages' field (Wavefield_tmp), whose x sources are its own
static void fs_derivs(Sim& s, vector<double>& E, vector<double>& P, vector<double>& Ex, vector<double>& Exx,
                      vector<double>& Px, vector<double>& Ey, vector<double>& Eyy, vector<double>& Py, bool tmp = false) {
    if (s.per) {
        // periodic x: image columns in place of the ghost-layer update
        images_x(s, E.data(), 1); dx2(s, E.data(), Ex.data(), 1); dx2(s, E.data(), Exx.data(), 2);
        images_x(s, P.data(), 1); dx2(s, P.data(), Px.data(), 1);
    } else if (s.p.Nx > 1) {
        ghost_x(s, E.data(), tmp ? s.tsEx.data() : s.sEx.data()); dx2(s, E.data(), Ex.data(), 1); dx2(s, E.data(), Exx.data(), 2);
        ghost_x(s, P.data(), tmp ? s.tsPx.data() : s.sPx.data()); dx2(s, P.data(), Px.data(), 1);
    }
    if (s.p.Ny > 1) {
        ghost_y(s, E.data(), s.sEy.data()); dy2(s, E.data(), Ey.data(), 1); dy2(s, E.data(), Eyy.data(), 2);
        ghost_y(s, P.data(), s.sPy.data()); dy2(s, P.data(), Py.data(), 1);
    }
}
// VerticalFreeSurfaceVelocity.f90:17
static void vertical_velocity(Sim& s, vector<double>& W) {
    int g = s.p.gamma, rank = 2 * g + 1, Nz = s.Nzg;
    for (int c = 0; c < s.C; ++c) {
        double acc = 0;
        for (int m = 0; m < rank; ++m) acc += s.SZ.at(1, Nz - 1, m) * s.PHI[(size_t)c * Nz + (Nz - 2 * g + m) - 1];
        W[c] = s.dsig[((size_t)c * Nz + Nz - 1) * 5 + 4] * acc;
    }
    if (s.per) images_x(s, W.data(), 1);
}
// rhsFreeSurface3D.f90:12-28, rhsLinearFreeSurface3D.f90
static void fs_rhs(const Sim& s, const vector<double>& E, const vector<double>& P, const vector<double>& W,
                   const vector<double>& Ex, const vector<double>& Px, const vector<double>& Ey, const vector<double>& Py,
                   vector<double>& kE, vector<double>& kP) {
    const double g = s.p.g, one = 1.0, half = 0.5;
    for (int c = 0; c < s.C; ++c) {
        if (s.p.LinearONOFF == 0) { kE[c] = W[c]; kP[c] = -g * E[c]; continue; }
        if (s.p.Nx == 1) {
            kE[c] = -Ey[c] * Py[c] + W[c] * (one + Ey[c] * Ey[c]);
            kP[c] = -g * E[c] - half * (Py[c] * Py[c] - W[c] * W[c] * (one + Ey[c] * Ey[c]));
        } else if (s.p.Ny == 1) {
            kE[c] = -Ex[c] * Px[c] + W[c] * (one + Ex[c] * Ex[c]) - s.Qr_x[c];
            kP[c] = -g * E[c] - half * (Px[c] * Px[c] - W[c] * W[c] * (one + Ex[c] * Ex[c]));
        } else {
            kE[c] = -Ex[c] * Px[c] - Ey[c] * Py[c] + W[c] * (one + Ex[c] * Ex[c] + Ey[c] * Ey[c]);
            kP[c] = -g * E[c] - half * (Px[c] * Px[c] + Py[c] * Py[c] - W[c] * W[c] * (one + Ex[c] * Ex[c] + Ey[c] * Ey[c]));
        }
    }
    for (int c = 0; c < s.C; ++c) { kE[c] += s.NuD[c]; kP[c] += s.Pd[c]; }   // rhsFreeSurface3D.f90:27-28
    if (s.gx + s.gy == 2) {  // Zero_Corners.f90
        int Nx = s.Nxg, Ny = s.Nyg;
        size_t cs4[4] = {0, (size_t)Nx - 1, (size_t)Nx * (Ny - 1), (size_t)Nx * Ny - 1};
        for (size_t c : cs4) { kE[c] = 0; kP[c] = 0; }
    }
}

// RelaxationModule_new.f90:1-276 (X/X and Y/Y zones) with AnalyticWaveMaker2D.f90:21-34.
static void relax(Sim& s, vector<double>& E, vector<double>& P, double RKtime, double time) {
    if (s.p.relaxONOFF != 1) return;
    double FAC = (RKtime < s.p.relaxTransientTime) ? RKtime / s.p.relaxTransientTime : 1.0;
    int Nx = s.Nxg;
    for (Zone& z : s.zones) {
        int bx = z.i1 - z.i0 + 1, by = z.j1 - z.j0 + 1;
        const double* te = nullptr; const double* tp = nullptr; vector<double> ae, ap;
        if (z.wavegen) {
            if (z.tmode < 0 || z.nt == 0) continue;
            size_t box = (size_t)bx * by;
            if (z.tmode == 1) {
                long it = std::lround(RKtime / z.tdt); it = std::max(0L, std::min(it, (long)z.nt - 1));
                te = &z.eta[(size_t)it * box]; tp = &z.phis[(size_t)it * box];
            } else {
                double diff = (RKtime - time) / z.tdt, tol = 10e-14;
                if (diff < tol || std::fabs(1.0 - diff) < tol) {
                    long it = std::lround(RKtime / z.tdt); it = std::max(0L, std::min(it, (long)z.nt - 1));
                    te = &z.eta[(size_t)it * box]; tp = &z.phis[(size_t)it * box];
                } else {
                    long it = std::lround(time / z.tdt); it = std::max(0L, std::min(it, (long)z.nt - 2));
                    ae.resize(box); ap.resize(box);
                    for (size_t t = 0; t < box; ++t) {
                        ae[t] = 0.5 * (z.eta[(size_t)it * box + t] + z.eta[(size_t)(it + 1) * box + t]);
                        ap[t] = 0.5 * (z.phis[(size_t)it * box + t] + z.phis[(size_t)(it + 1) * box + t]);
                    }
                    te = ae.data(); tp = ap.data();
                }
            }
        }
        for (int j = z.j0; j <= z.j1; ++j)
            for (int i = z.i0; i <= z.i1; ++i) {
                double gm = (z.XorY == 'X') ? z.gam[i - z.i0] : z.gam[j - z.j0];
                size_t c = (size_t)(i - 1) + (size_t)Nx * (j - 1), t = (size_t)(i - z.i0) + (size_t)bx * (j - z.j0);
                if (!z.wavegen) {
                    E[c] = E[c] * gm;
                    if (z.phion) P[c] = P[c] * gm;
                } else {
                    E[c] = E[c] * gm + FAC * te[t] * (1.0 - gm);
                    P[c] = P[c] * gm + FAC * tp[t] * (1.0 - gm);
                }
            }
    }
}

// FILTERING.f90:17-57
static void filter(Sim& s, vector<double>& U) {
    int Nx = s.Nxg, Ny = s.Nyg, al = s.p.filterALPHA, NP = s.NP, gx = s.gx, gy = s.gy;
    auto F2 = [&](int m, int i) { return s.fc2[(size_t)(i - 1) * NP + (m - 1)]; };  // (NP x alpha) view
    if (Nx > 1 && s.per) {
        // periodic x: the centred filter on every distinct column, cyclic
        vector<double> t = U;
        for (int j = 1 + gy; j <= Ny - gy; ++j)
            for (int i = 2; i <= Nx - 2; ++i) {
                double a = 0;
                for (int m = 1; m <= NP; ++m) a += t[(size_t)(wrap_x(i - al + m - 1, Nx) - 1) + (size_t)Nx * (j - 1)] * s.fc[m - 1];
                U[(size_t)(i - 1) + (size_t)Nx * (j - 1)] = a;
            }
        images_x(s, U.data(), 1);
    } else if (Nx > 1) {
        vector<double> t = U;
        for (int j = 1 + gy; j <= Ny - gy; ++j) {
            auto T = [&](int i) { return t[(size_t)(i - 1) + (size_t)Nx * (j - 1)]; };
            auto Uw = [&](int i) -> double& { return U[(size_t)(i - 1) + (size_t)Nx * (j - 1)]; };
            for (int i = 1; i <= al; ++i) { double a = 0; for (int m = 1; m <= NP; ++m) a += T(gx + m) * F2(m, i); Uw(i + gx) = a; }
            for (int i = 1 + gx + al; i <= Nx - gx - al; ++i) { double a = 0; for (int m = 1; m <= NP; ++m) a += T(i - al + m - 1) * s.fc[m - 1]; Uw(i) = a; }
            for (int i = 1; i <= al; ++i) { double a = 0; for (int m = 1; m <= NP; ++m) a += T(Nx - gx - NP + m) * F2(NP + 1 - m, al + 1 - i); Uw(Nx - gx - al + i) = a; }
        }
    }
    if (Ny > 1) {
        vector<double> t = U;
        for (int i = 1 + gx; i <= Nx - gx; ++i) {
            auto T = [&](int j) { return t[(size_t)(i - 1) + (size_t)Nx * (j - 1)]; };
            auto Uw = [&](int j) -> double& { return U[(size_t)(i - 1) + (size_t)Nx * (j - 1)]; };
            for (int j = 1; j <= al; ++j) { double a = 0; for (int m = 1; m <= NP; ++m) a += T(gy + m) * F2(m, j); Uw(j + gy) = a; }
            for (int j = 1 + gy + al; j <= Ny - gy - al; ++j) { double a = 0; for (int m = 1; m <= NP; ++m) a += T(j - al + m - 1) * s.fc[m - 1]; Uw(j) = a; }
            for (int j = 1; j <= al; ++j) { double a = 0; for (int m = 1; m <= NP; ++m) a += T(Ny - gy - NP + m) * F2(NP + 1 - m, al + 1 - j); Uw(Ny - gy - al + j) = a; }
        }
    }
}

// Savitzky-Golay smoothing weights (savgol.f90, Numerical Recipes formulation):
// least-squares polynomial of degree m on offsets -nl..nr, value at 0 (ld = 0).
// c[k+nl] is the weight of offset k.
static vector<double> sg_weights(int nl, int nr, int m) {
    int M = m + 1;
    vector<double> A((size_t)M * M, 0.0), bb(M, 0.0);
    for (int ipj = 0; ipj <= 2 * m; ++ipj) {
        double sm = (ipj == 0) ? 1.0 : 0.0;
        for (int k = 1; k <= nr; ++k) sm += std::pow((double)k, ipj);
        for (int k = 1; k <= nl; ++k) sm += std::pow((double)-k, ipj);
        int mm = std::min(ipj, 2 * m - ipj);
        for (int imj = -mm; imj <= mm; imj += 2) A[(size_t)((ipj + imj) / 2) * M + (ipj - imj) / 2] = sm;
    }
    bb[0] = 1.0;
    // Gaussian elimination with partial pivoting
    vector<int> pv(M);
    for (int k = 0; k < M; ++k) {
        int pr = k; for (int r = k + 1; r < M; ++r) if (std::fabs(A[(size_t)r * M + k]) > std::fabs(A[(size_t)pr * M + k])) pr = r;
        if (pr != k) { for (int c = 0; c < M; ++c) std::swap(A[(size_t)k * M + c], A[(size_t)pr * M + c]); std::swap(bb[k], bb[pr]); }
        for (int r = k + 1; r < M; ++r) { double f = A[(size_t)r * M + k] / A[(size_t)k * M + k]; for (int c = k; c < M; ++c) A[(size_t)r * M + c] -= f * A[(size_t)k * M + c]; bb[r] -= f * bb[k]; }
    }
    for (int r = M - 1; r >= 0; --r) { double t = bb[r]; for (int c = r + 1; c < M; ++c) t -= A[(size_t)r * M + c] * bb[c]; bb[r] = t / A[(size_t)r * M + r]; }
    vector<double> c(nl + nr + 1);
    for (int k = -nl; k <= nr; ++k) { double sm = bb[0], fac = 1.0; for (int q = 1; q <= m; ++q) { fac *= k; sm += bb[q] * fac; } c[k + nl] = sm; }
    return c;
}

// FilterInit.f90:29-231 -> centre coefficients and the (NP x alpha) view of the
// boundary coefficient array exactly as FILTERING.f90 addresses it.
static void filter_init(Sim& s) {
    int al = s.p.filterALPHA, NP = 2 * al + 1; s.NP = NP;
    vector<double> c = sg_weights(al, al, s.p.filterORDER);
    s.fc = c;  // offsets -al..al
    int ld = std::max(NP, 13), nc = std::max(al, 6);
    vector<double> F((size_t)ld * nc, 0.0);
    auto at = [&](int r, int col) -> double& { return F[(size_t)(col - 1) * ld + (r - 1)]; };
    const double t1[4] = {0.320882352941, -0.465, 0.179117647059, -0.035};
    const double t2[7] = {-0.085777408970, 0.277628171524, -0.356848072173, 0.223119093072, -0.057347064865, -0.000747264596, -0.000027453993};
    const double t3[11] = {0.052523901012, -0.206299133811, 0.353527998250, -0.348142394842, 0.181481803619, 0.009440804370,
                           -0.077675100452, 0.044887364863, -0.009971961849, 0.000113359420, 0.000113359420};
    at(1, 1) = 1.0; for (int r = 0; r < 4; ++r) at(r + 1, 1) -= s.p.sigma_filt[0] * t1[r];
    at(2, 2) = 1.0; for (int r = 0; r < 7; ++r) at(r + 1, 2) -= s.p.sigma_filt[1] * t2[r];
    at(3, 3) = 1.0; for (int r = 0; r < 11; ++r) at(r + 1, 3) -= s.p.sigma_filt[2] * t3[r];
    for (int col = 4; col <= 6; ++col) {
        int h = col - 1, n = 2 * h + 1, ord = (col == 4) ? 5 : (col == 5 ? 6 : 8);
        vector<double> w = sg_weights(h, h, ord);
        for (int r = 1; r <= n; ++r) at(r, col) = w[r - 1];
    }
    if (std::fabs(s.p.sigma_filt[0]) < 1e-12) {
        std::fill(F.begin(), F.end(), 0.0);
        for (int i = 1; i <= nc; ++i) at(i, i) = 1.0;
    }
    s.fc2.assign((size_t)NP * al, 0.0);
    for (size_t f = 0; f < s.fc2.size(); ++f) s.fc2[f] = F[f];
}

// PreprocessRelaxationZones.f90 + GammaFunctions.f90
static vector<double> gamma_fn(const double* x, int n, int dir, int ftype, double param) {
    vector<double> t(n), g(n);
    for (int i = 0; i < n; ++i) t[i] = (n > 1) ? (x[i] - x[0]) / (x[n - 1] - x[0]) : x[i];
    for (int i = 0; i < n; ++i) {
        switch (std::abs(ftype)) {
            case 9: g[i] = 1.0 - std::pow(t[i], param); break;
            case 10: g[i] = 3.0 * t[i] * t[i] - 2.0 * t[i] * t[i] * t[i]; break;
            case 11: g[i] = (std::exp(std::pow(t[i], param)) - 1) / (std::exp(1.0) - 1.0); break;
            case 12: { double q = (x[i] - x[n - 1]) / (x[n - 1] - x[0]); g[i] = std::exp(-q * q / (2 * param * param)); break; }
            case 13: { double q = (x[i] - x[n - 1]) / (x[n - 1] - x[0]); g[i] = 1 - std::exp(-q * q / (2 * param * param)); break; }
            case 14: g[i] = 1 - (std::exp(std::pow(t[i], param)) - 1) / (std::exp(1.0) - 1.0); break;
            default: g[i] = 1.0;
        }
    }
    if (dir == -1) std::reverse(g.begin(), g.end());
    return g;
}
static int trace(const vector<double>& x, double x0) {
    for (size_t i = 0; i < x.size(); ++i) if (x0 <= x[i]) return (int)i + 1;
    return (int)x.size();
}
// PreprocessPDampingZones.f90:24-70 and BuildPDampMatrices.f90:17-86 (one
// x-directed zone, 2-D).
static void setup_pdamp(Sim& s) {
    s.NuD.assign(s.C, 0.0); s.Pd.assign(s.C, 0.0);
    if (s.p.PDampingONOFF == 0) return;
    const int nx = s.Nxg;
    int i1 = trace(s.fine.x, s.p.pd_x0), i2 = trace(s.fine.x, s.p.pd_x1), nd = i2 - i1 + 1;
    s.pd_i1 = i1; s.pd_nd = nd;
    vector<double> gt = gamma_fn(&s.fine.x[i1 - 1], nd, 1, 12, 0.25);
    s.gamPhi.assign(nx, 0.0); s.gamEta.assign(nx, 0.0);
    for (int i = 1; i <= nd; ++i) {
        s.gamPhi[i1 + i - 2] = 2.0 * M_PI * s.p.pd_g0Phi * gt[i - 1];
        s.gamEta[i1 + i - 2] = 2.0 * M_PI * s.p.pd_g0Eta * gt[i - 1];
    }
    if (s.p.pd_type != 0) return;
    const int a = s.p.alpha, rank = 2 * a + 1;
    s.pdGrad = orc::build_stencils_xy(vector<double>(s.fine.x.begin(), s.fine.x.begin() + nd), a);
    const Stencil1D& G = s.pdGrad;
    vector<double>& A = s.pdLU;
    A.assign((size_t)nd * nd, 0.0);
    auto put = [&](int i, int col, double v) { A[(size_t)(i - 1) * nd + (col - 1)] = v; };   // 1-based
    put(1, 1, 1.0);
    for (int i = 2; i <= a; ++i)
        for (int m = 1; m <= rank; ++m) put(i, m, G.at(2, i - 1, m - 1));
    for (int i = a + 1; i <= nd - a; ++i)
        for (int m = 1; m <= rank; ++m) put(i, i - a - 1 + m, G.at(2, i - 1, m - 1));
    for (int i = nd - a + 1; i <= nd - 1; ++i)
        for (int m = 1; m <= rank; ++m) put(i, nd - rank + m, G.at(2, i - 1, m - 1));
    for (int m = 1; m <= rank; ++m) put(nd, nd - rank + m, G.at(1, nd - 1, m - 1));
    // dense LU with partial pivoting in place of the reference's MA41
    s.pdPiv.assign(nd, 0);
    for (int k = 0; k < nd; ++k) {
        int pr = k;
        for (int r = k + 1; r < nd; ++r) if (std::fabs(A[(size_t)r * nd + k]) > std::fabs(A[(size_t)pr * nd + k])) pr = r;
        s.pdPiv[k] = pr;
        if (pr != k) for (int c = 0; c < nd; ++c) std::swap(A[(size_t)k * nd + c], A[(size_t)pr * nd + c]);
        for (int r = k + 1; r < nd; ++r) {
            double f = A[(size_t)r * nd + k] / A[(size_t)k * nd + k];
            A[(size_t)r * nd + k] = f;
            if (f != 0.0) for (int c = k + 1; c < nd; ++c) A[(size_t)r * nd + c] -= f * A[(size_t)k * nd + c];
        }
    }
}
// DfDx_1D_Uneven.f90:17-29
static void pd_dfdx(const Sim& s, const vector<double>& f, vector<double>& fx) {
    const int nd = s.pd_nd, a = s.p.alpha, rank = 2 * a + 1;
    for (int i = 1; i <= nd; ++i) {
        int lo = (i <= a) ? 1 : (i <= nd - a ? i - a : nd - rank + 1);
        double acc = 0.0;
        for (int m = 1; m <= rank; ++m) acc += f[lo + m - 2] * s.pdGrad.at(1, i - 1, m - 1);
        fx[i - 1] = acc;
    }
}
// funPressureTerm.f90:218-311: NuD and Pd of the state (E, P) at time t > 0;
// they keep their values otherwise.
static void pressure_term(Sim& s, const vector<double>& E, const vector<double>& P, double t) {
    if (s.p.PDampingONOFF == 0 || !(t > 0)) return;
    const int nx = s.Nxg;
    if (s.p.pd_type == 0) {
        const int nd = s.pd_nd, id0 = s.pd_i1;
        vector<double> tmp(nd), rhs(nd);
        for (int i = 1; i <= nd; ++i) tmp[i - 1] = P[id0 + i - 2];
        pd_dfdx(s, tmp, rhs);
        for (int i = 1; i <= nd; ++i) tmp[i - 1] = s.gamPhi[id0 + i - 2] * (rhs[i - 1] - s.Ur);   // relative to the current
        pd_dfdx(s, tmp, rhs);
        rhs[0] = P[id0 - 1]; rhs[nd - 1] = 0.0;
        const double* A = s.pdLU.data();
        for (int k = 0; k < nd; ++k) if (s.pdPiv[k] != k) std::swap(rhs[k], rhs[s.pdPiv[k]]);
        for (int r = 0; r < nd; ++r) { double v = rhs[r]; for (int c = 0; c < r; ++c) v -= A[(size_t)r * nd + c] * rhs[c]; rhs[r] = v; }
        for (int r = nd - 1; r >= 0; --r) {
            double v = rhs[r];
            for (int c = r + 1; c < nd; ++c) v -= A[(size_t)r * nd + c] * rhs[c];
            rhs[r] = v / A[(size_t)r * nd + r];
        }
        for (int i = 1; i <= nx; ++i) s.NuD[i - 1] = -s.gamEta[i - 1] * E[i - 1];
        std::fill(s.Pd.begin(), s.Pd.end(), 0.0);
        for (int i = 1; i <= nd; ++i) s.Pd[id0 + i - 2] = -(rhs[i - 1] - rhs[0]);
    } else {
        for (int j = 1; j <= s.Nyg; ++j)
            for (int i = 1; i <= nx; ++i) {
                size_t k = (size_t)(j - 1) * nx + (i - 1);
                s.NuD[k] = -s.gamEta[k] * E[k];
                s.Pd[k] = -s.gamPhi[k] * P[k];
            }
    }
}

static void setup_zones(Sim& s) {
    s.zones.clear();
    if (s.p.relaxONOFF != 1) return;
    for (int z = 0; z < s.p.relaxNo && z < OW3D_MAX_ZONES; ++z) {
        const ow3d_zone& Zd = s.p.zones[z]; Zone Z;
        int dir = Zd.ftype >= 0 ? 1 : -1;
        if (s.p.Nx > 1) { Z.i0 = trace(s.fine.x, Zd.x1); Z.i1 = trace(s.fine.x, Zd.x2); }
        if (s.p.Ny > 1) { Z.j0 = trace(s.fine.y, Zd.y1); Z.j1 = trace(s.fine.y, Zd.y2); }
        Z.XorY = Zd.XorY; Z.XorYgen = Zd.XorYgen; Z.wavegen = Zd.WavegenONOFF; Z.phion = Zd.PhiOnOff;
        if (Z.XorY == 'X') Z.gam = gamma_fn(&s.fine.x[Z.i0 - 1], Z.i1 - Z.i0 + 1, dir, Zd.ftype, Zd.param);
        else Z.gam = gamma_fn(&s.fine.y[Z.j0 - 1], Z.j1 - Z.j0 + 1, dir, Zd.ftype, Zd.param);
        s.zones.push_back(Z);
    }
}

// ------------------------------------------------------------- breaking
// DetectBreaking.f90:72-211 on the surface elevation E of an x flume (1-based
// column j, nfx = Nxg columns). Rollers are searched from the right end: a
// toe lies between j-1 and j where the slope eta_x (forward differences at
// j+1/2) crosses -tan(phi(j)) and no roller covers j yet; its sub-grid
// position comes from the local quadratic, and the roller extends back while
// the surface stays above the tangent line from the toe, with thickness
// del_fac times that height (capped at eta - eta_toe). Qr_x, the 1-2-1
// smoothed g * thickness, enters the kinematic condition when i_breaking is 1
// (rhsFreeSurface3D.f90:17). With update (the call after the step, :175-186)
// tan(phi) returns to tan(phi_b) everywhere except from three points ahead of
// each toe to the back of its roller, where it moves linearly toward
// tan(phi_0) by dt / T_half of the way from the toe's previous value, and the
// rollers are recorded as the reference writes them to roller.dat
// (:205-211). Rollers are not capped at nfx/10 (the reference's arrays) and
// angle updates past the last column are dropped (the reference writes
// them out of bounds).
static void detect_breaking(Sim& s, const vector<double>& E, bool update) {
    const int nfx = s.Nxg;
    const double half = 0.5, two = 2.0, quart = 0.25, g = s.p.g;
    const double dx = s.p.Lx / ((double)s.p.Nx - 1.0), dx_inv = 1.0 / dx;
    auto et = [&](int j) { return E[(size_t)j - 1]; };
    vector<double> tan_old(s.tan_phi), thick(nfx + 1, 0.0), eta_x(nfx + 1, 0.0), Qr(nfx + 1, 0.0);
    std::fill(s.Qr_x.begin(), s.Qr_x.end(), 0.0);
    for (int j = 2; j <= nfx - 2; ++j) eta_x[j] = dx_inv * (et(j + 1) - et(j));
    vector<int> npts, toe; vector<double> xr_l, sr_l;
    for (int j = nfx - 2; j >= 3; --j) {
        const double tphib = s.tan_phi[(size_t)j - 1];
        if (!(eta_x[j - 1] < -tphib && eta_x[j] >= -tphib && thick[j] <= 0.0)) continue;
        const double a = half * dx_inv * (eta_x[j] - eta_x[j - 1]);
        const double b = half * (eta_x[j] + eta_x[j - 1]);
        const double c = et(j);
        const double dxr = -(tphib + b) / (two * a);
        const double xr = (double)(j - 1) * dx + dxr;
        const int jr = (int)(xr * dx_inv) + 2;
        const double sr = a * dxr * dxr + b * dxr + c;
        int n = 0;
        for (int i = jr - 1; i >= 3; --i) {
            double d = s.p.del_fac * (et(i) - (sr + tphib * (xr - (double)(i - 1) * dx)));
            if (d < 0.0) break;
            if (d > et(i) - sr) d = et(i) - sr;
            thick[i] = d; ++n;
            Qr[i] = g * thick[i];
        }
        npts.push_back(n); toe.push_back(jr); xr_l.push_back(xr); sr_l.push_back(sr);
    }
    const int nr = (int)npts.size();
    if (update) {
        std::fill(s.tan_phi.begin(), s.tan_phi.end(), s.tan_b);
        for (int r = 0; r < nr; ++r) {
            const double tphib = tan_old[(size_t)toe[r] - 1];
            for (int i = 1; i <= npts[r] + 3; ++i) {
                const int idx = toe[r] + 4 - i;
                if (idx >= 1 && idx <= nfx) s.tan_phi[(size_t)idx - 1] = tphib + s.p.dt / s.p.T_half * (s.tan_0 - tphib);
            }
        }
        s.r_npts = npts; s.r_toe = toe; s.r_x = xr_l; s.r_eta = sr_l;
        s.r_thick.assign(nr, 0.0); s.r_tan.assign(nr, 0.0);
        for (int r = 0; r < nr; ++r) { s.r_thick[r] = thick[toe[r] - 1]; s.r_tan[r] = s.tan_phi[(size_t)toe[r] - 1]; }
    }
    if (nr > 0 && s.p.i_breaking == 1)
        for (int j = 3; j <= nfx - 2; ++j) s.Qr_x[(size_t)j - 1] = quart * Qr[j + 1] + half * Qr[j] + quart * Qr[j - 1];
}

// --------------------------------------------------- local smoothing
// LocalSmoothing2D.f90:37-145 (x flumes) and LocalSmoothing3D.f90 (3-D),
// called after each step from OceanWave3DTakeATimeStep.f90:33-39 with the
// step number: from the third step on, the Lagrangian vertical acceleration
// of the surface, dw/dt = (3 W^n - 4 W^(n-1) + W^(n-2)) / (2 dt) - w_z eta_t
// + u w_x (+ v w_y) + w w_z, is formed from the last solution (the velocity
// and its gradients in physical space by the sigma chain rule, as the
// reference takes them on the whole grid); where -dw/dt >= accel_tol_fact g
// at a point i = 6..Nxg-5 of a row, the points i-5..i+5 of that row get the
// weight 1/4, and if any point did, eta and the surface potential of every
// row are filtered with [a, 1-2a, a] over i = 2..Nxg-1. As in the reference
// the 3-D v takes the x derivative of phi (DiffXEven called with beta).
static void local_smoothing(Sim& s) {
    if (!s.smooth || s.tstep < 3) return;
    const int Nx = s.Nxg, Ny = s.Nyg, Nz = s.Nzg;
    const size_t N = s.N, C = s.C;
    const bool three = s.dimcase == 3;
    const double one = 1.0, half = 0.5, two = 2.0, three_ = 3.0, four = 4.0;
    const vector<double>& z = s.fine.z;
    vector<double> d(C), U(N), V(three ? N : 0), W(N), Wz(N), Wx(N), Wy(three ? N : 0);
    for (size_t c = 0; c < C; ++c) d[c] = s.fine.h[c] + s.E[c];
    diff_x(s, s.PHI.data(), U.data(), 1, Nz);
    if (three) diff_x(s, s.PHI.data(), V.data(), 1, Nz);
    diff_z(s, s.PHI.data(), W.data(), 1);
    for (size_t c = 0; c < C; ++c)
        for (int k = 1; k <= Nz; ++k) {
            const size_t q = c * Nz + (size_t)k - 1;
            W[q] = W[q] / d[c];
            U[q] = U[q] + ((one - z[k - 1]) * s.fine.hx[c] - z[k - 1] * s.Ex[c]) * W[q];
            if (three) V[q] = V[q] + ((one - z[k - 1]) * s.fine.hy[c] - z[k - 1] * s.Ey[c]) * W[q];
        }
    diff_z(s, W.data(), Wz.data(), 1);
    diff_x(s, W.data(), Wx.data(), 1, Nz);
    if (three) diff_y(s, W.data(), Wy.data(), 1, Nz);
    for (size_t c = 0; c < C; ++c)
        for (int k = 1; k <= Nz; ++k) {
            const size_t q = c * Nz + (size_t)k - 1;
            Wz[q] = Wz[q] / d[c];
            Wx[q] = Wx[q] + ((one - z[k - 1]) * s.fine.hx[c] - z[k - 1] * s.Ex[c]) * Wz[q];
            if (three) Wy[q] = Wy[q] + ((one - z[k - 1]) * s.fine.hy[c] - z[k - 1] * s.Ey[c]) * Wz[q];
        }
    const double dt_inv = one / s.p.dt;
    vector<double>& Wt = s.accel_Wt;
    Wt.assign(C, 0.0);
    for (size_t c = 0; c < C; ++c) {
        const size_t q = c * Nz + (size_t)Nz - 1;
        Wt[c] = half * dt_inv * (three_ * s.WHist[0][c] - four * s.WHist[1][c] + s.WHist[2][c]) - Wz[q] * s.EtatHist1[c];
        if (three) Wt[c] = Wt[c] + U[q] * Wx[q] + V[q] * Wy[q] + W[q] * Wz[q];
        else Wt[c] = Wt[c] + U[q] * Wx[q] + W[q] * Wz[q];
    }
    const double accel_tol = s.p.accel_tol_fact * s.p.g;
    vector<double> alpha_s(C, 0.0);
    s.accel_pts.clear();
    for (int j = 1; j <= Ny; ++j)
        for (int i = 6; i <= Nx - 5; ++i) {
            const size_t c = (size_t)(i - 1) + (size_t)Nx * (j - 1);
            if (-Wt[c] >= accel_tol) {
                s.accel_pts.push_back((int)c);
                for (int ii = i - 5; ii <= i + 5; ++ii) alpha_s[(size_t)(ii - 1) + (size_t)Nx * (j - 1)] = 0.25;
            }
        }
    if (s.accel_pts.empty()) return;
    const vector<double> et(s.E), ph(s.P);
    for (int j = 1; j <= Ny; ++j)
        for (int i = 2; i <= Nx - 1; ++i) {
            const size_t c = (size_t)(i - 1) + (size_t)Nx * (j - 1);
            const double a = alpha_s[c];
            s.E[c] = a * et[c - 1] + (one - two * a) * et[c] + a * et[c + 1];
            s.P[c] = a * ph[c - 1] + (one - two * a) * ph[c] + a * ph[c + 1];
        }
}

// ------------------------------------------------------- flux wavemaker
// polint.f90 (Neville's algorithm, the published method): the value at x of
// the polynomial through (xa[i], ya[i]), i < n.
static double polint(const double* xa, const double* ya, int n, double x) {
    vector<double> c(ya, ya + n), d(ya, ya + n);
    int ns = 1;
    double dif = std::fabs(x - xa[0]);
    for (int i = 1; i <= n; ++i) {
        double dift = std::fabs(x - xa[i - 1]);
        if (dift < dif) { ns = i; dif = dift; }
    }
    double y = ya[ns - 1];
    ns = ns - 1;
    for (int m = 1; m <= n - 1; ++m) {
        for (int i = 1; i <= n - m; ++i) {
            double ho = xa[i - 1] - x, hp = xa[i + m - 1] - x;
            double w = c[i] - d[i - 1];
            double den = ho - hp;
            den = w / den;
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

// waveGenerationFromPaddleSignal.f90:43-111 at RKtime: the flux and eta_x of
// the two signal levels around it (itime = floor(RKtime / dt) + 1, kept
// inside the table), interpolated in y with `order` points, linearly in time,
// the flux ramped; Uneumann per row, and the west-wall sources of Wavefield.
static void paddle_signal(Sim& s, double RKtime) {
    const int n2 = s.pad_n2, order = s.p.flux_order, Nx = s.Nxg;
    int itime = (int)std::floor(RKtime / s.pad_dt) + 1;
    if (itime < 1) itime = 1;
    if (itime > s.pad_nt - 1) itime = s.pad_nt - 1;
    double dl1 = RKtime - (itime - 1) * s.pad_dt, dl2 = itime * s.pad_dt - RKtime;
    double tw1 = dl2 / (dl1 + dl2), tw2 = dl1 / (dl1 + dl2);
    const double r = s.p.flux_ramp;
    double FAC = 1.0;
    if (RKtime < r) FAC = -2.0 / (r * r * r) * (RKtime * RKtime * RKtime) + 3.0 / (r * r) * (RKtime * RKtime);
    const double dy_local = s.pad_y[0] * 2;
    for (int j = 1 + s.gy; j <= s.p.Ny + s.gy; ++j) {
        double y0 = s.fine.y[(size_t)j - 1];
        int NNY = (int)std::lround(y0 / dy_local) + 1 - order / 2;
        if (NNY < 1) NNY = 1;
        else if (NNY + order - 1 > n2) NNY = n2 - order + 1;
        auto at = [&](const vector<double>& tab, int it) {
            vector<double> v((size_t)order);
            for (int q = 0; q < order; ++q) v[(size_t)q] = tab[(size_t)(it - 1) * n2 + NNY - 1 + q];
            return polint(&s.pad_y[(size_t)NNY - 1], v.data(), order, y0);
        };
        double flux0 = at(s.pad_flux, itime), etax0 = at(s.pad_etax, itime);
        double flux1 = at(s.pad_flux, itime + 1), etax1 = at(s.pad_etax, itime + 1);
        double flux = tw1 * flux0 + tw2 * flux1;
        double etax = tw1 * etax0 + tw2 * etax1;
        s.Uneu[(size_t)j - 1] = FAC * flux;
        s.sPx[(size_t)(1 + s.gx - 1) + (size_t)Nx * (j - 1)] = FAC * flux;
        s.sEx[(size_t)(1 + s.gx - 1) + (size_t)Nx * (j - 1)] = etax;
    }
}

// ------------------------------------------------------------- RK4 step
// Runge_Kutta_4.f90:1-429 (nonlinear or linear FSBC, no SWENSE, no pressure).
static int rk4_step(Sim& s) {
    ++s.tstep;
    const int64_t tstep = s.tstep;
    const double dt = s.p.dt, half = 0.5, time = s.time;
    const size_t C = s.C;
    vector<double> k1E(C), k1P(C), k2E(C), k2P(C), k3E(C), k3P(C), k4E(C), k4P(C);
    vector<double>& LPnew = (tstep - 1) % 2 == 0 ? s.LASTPHI0 : s.LASTPHI1;
    vector<double>& LPlast = (tstep % 2) == 0 ? s.LASTPHI0 : s.LASTPHI1;
    LPnew = s.PHI;
    int status = OW3D_OK;
    auto set_rhs = [&](const vector<double>& Pf) {
        const int Nz = s.Nzg;
        for (int j = 1 + s.gy; j <= s.Nyg - s.gy; ++j)
            for (int i = 1 + s.gx; i <= s.Nxg - s.gx; ++i) s.RHS[gid(s, Nz, i, j)] = Pf[(size_t)(i - 1) + (size_t)s.Nxg * (j - 1)];
        if (s.gx == 1)   // Runge_Kutta_4.f90:108-113: Uneumann (the wavemaker's flux above the bottom row) + the current
            for (int j = 1 + s.gy; j <= s.Nyg - s.gy; ++j)
                for (int k = 1; k <= Nz; ++k) {
                    const double un = (s.pad && k >= 1 + s.gz) ? s.Uneu[(size_t)j - 1] : 0.0;
                    s.RHS[gid(s, k, 1, j)] = un + s.Ul;
                    s.RHS[gid(s, k, s.Nxg, j)] = s.Ur;
                }
        if (s.per) zero_images_x(s, s.RHS.data(), Nz);   // identity rows of the image columns
    };
    auto sigma_for = [&](const vector<double>& E, const vector<double>& Ex, const vector<double>& Exx,
                         const vector<double>& Ey, const vector<double>& Eyy) {
        if (s.p.LinearONOFF == 1) update_sigma(s, E.data(), Ex.data(), Exx.data(), Ey.data(), Eyy.data());
    };
    auto do_solve = [&]() {
        int it; double res;
        int st = solve(s, s.RHS.data(), s.PHI.data(), it, res);
        if (st == OW3D_NOT_CONVERGED) status = OW3D_NOT_CONVERGED;
    };
    // Runge_Kutta_4.f90:80-88 (and :261-268, :382-389): the potential's ghost
    // source of the stage's field set to zero, the flux wavemaker called at
    // RK time (it writes Uneumann and the sources of Wavefield, whichever
    // field the stage uses, waveGenerationFromPaddleSignal.f90:107-110), then
    // the constant-flux current added at the west and east boundary columns
    auto zero_src = [&](bool tmp, double RKt) {
        vector<double>& px = tmp ? s.tsPx : s.sPx;
        std::fill(px.begin(), px.end(), 0.0);
        if (s.pad) paddle_signal(s, RKt);
        if (s.gx == 1)
            for (int j = 1; j <= s.Nyg; ++j) {
                px[(size_t)(1 + s.gx - 1) + (size_t)s.Nxg * (j - 1)] += s.Ul;
                px[(size_t)(s.p.Nx + s.gx - 1) + (size_t)s.Nxg * (j - 1)] += s.Ur;
            }
    };
    auto breaking = [&](const vector<double>& Ef) { if (s.brk && s.p.i_breaking == 1) detect_breaking(s, Ef, false); };
    // stage 1
    pressure_term(s, s.E, s.P, time);
    breaking(s.E);
    fs_rhs(s, s.E, s.P, s.W, s.Ex, s.Px, s.Ey, s.Py, k1E, k1P);
    for (size_t c = 0; c < C; ++c) { s.tE[c] = s.E[c] + half * dt * k1E[c]; s.tP[c] = s.P[c] + half * dt * k1P[c]; }
    double RKtime = time + half * dt;
    relax(s, s.tE, s.tP, RKtime, time);
    zero_src(true, RKtime);
    fs_derivs(s, s.tE, s.tP, s.tEx, s.tExx, s.tPx, s.tEy, s.tEyy, s.tPy, true);
    sigma_for(s.tE, s.tEx, s.tExx, s.tEy, s.tEyy);
    set_rhs(s.tP);
    if (s.p.extrapolationONOFF == 1)
        for (size_t t = 0; t < (size_t)s.N; ++t) s.PHI[t] = 1.5 * LPnew[t] - LPlast[t] * half;
    do_solve();
    vertical_velocity(s, s.tW);
    // stage 2
    pressure_term(s, s.tE, s.tP, RKtime);
    breaking(s.tE);
    fs_rhs(s, s.tE, s.tP, s.tW, s.tEx, s.tPx, s.tEy, s.tPy, k2E, k2P);
    for (size_t c = 0; c < C; ++c) { s.tE[c] = s.E[c] + half * dt * k2E[c]; s.tP[c] = s.P[c] + half * dt * k2P[c]; }
    RKtime = time + half * dt;
    relax(s, s.tE, s.tP, RKtime, time);
    fs_derivs(s, s.tE, s.tP, s.tEx, s.tExx, s.tPx, s.tEy, s.tEyy, s.tPy, true);
    sigma_for(s.tE, s.tEx, s.tExx, s.tEy, s.tEyy);
    set_rhs(s.tP);
    do_solve();
    vertical_velocity(s, s.tW);
    // stage 3
    pressure_term(s, s.tE, s.tP, RKtime);
    breaking(s.tE);
    fs_rhs(s, s.tE, s.tP, s.tW, s.tEx, s.tPx, s.tEy, s.tPy, k3E, k3P);
    for (size_t c = 0; c < C; ++c) { s.tE[c] = s.E[c] + dt * k3E[c]; s.tP[c] = s.P[c] + dt * k3P[c]; }
    RKtime = time + dt;
    relax(s, s.tE, s.tP, RKtime, time);
    zero_src(true, RKtime);
    fs_derivs(s, s.tE, s.tP, s.tEx, s.tExx, s.tPx, s.tEy, s.tEyy, s.tPy, true);
    sigma_for(s.tE, s.tEx, s.tExx, s.tEy, s.tEyy);
    set_rhs(s.tP);
    if (s.p.extrapolationONOFF == 1 && tstep > 1)
        for (size_t t = 0; t < (size_t)s.N; ++t) s.PHI[t] = 2.66667 * s.PHI[t] - 2.0 * LPnew[t] + 0.333333 * LPlast[t];
    do_solve();
    vertical_velocity(s, s.tW);
    // stage 4
    pressure_term(s, s.tE, s.tP, RKtime);
    breaking(s.tE);
    fs_rhs(s, s.tE, s.tP, s.tW, s.tEx, s.tPx, s.tEy, s.tPy, k4E, k4P);
    const double six = 6.0, two = 2.0;
    for (size_t c = 0; c < C; ++c) {
        s.E[c] = s.E[c] + dt / six * (k1E[c] + two * k2E[c] + two * k3E[c] + k4E[c]);
        s.P[c] = s.P[c] + dt / six * (k1P[c] + two * k2P[c] + two * k3P[c] + k4P[c]);
    }
    if (s.smooth) {   // Runge_Kutta_4.f90:347-348
        for (size_t c = 0; c < C; ++c) s.EtatHist1[c] = 1.0 / six * (k1E[c] + two * k2E[c] + two * k3E[c] + k4E[c]);
    }
    RKtime = time + dt;
    if (s.p.filteringONOFF > 0 && (tstep % s.p.filteringONOFF) == 0) { filter(s, s.E); filter(s, s.P); }
    relax(s, s.E, s.P, RKtime, time);
    zero_src(false, RKtime);
    fs_derivs(s, s.E, s.P, s.Ex, s.Exx, s.Px, s.Ey, s.Eyy, s.Py);
    sigma_for(s.E, s.Ex, s.Exx, s.Ey, s.Eyy);
    set_rhs(s.P);
    do_solve();
    vertical_velocity(s, s.W);
    if (s.smooth) {   // Runge_Kutta_4.f90:426-427
        std::swap(s.WHist[2], s.WHist[1]); std::swap(s.WHist[1], s.WHist[0]);
        s.WHist[0] = s.W;
    }
    // OceanWave3DTakeATimeStep.f90:33-39
    local_smoothing(s);
    // rollers of the new state and the roller-angle update (OceanWave3DTakeATimeStep.f90:45-49)
    if (s.brk) detect_breaking(s, s.E, true);
    // instability check and time advance (OceanWave3DTakeATimeStep.f90:54-70)
    double me = 0, mh = 0;
    for (size_t c = 0; c < C; ++c) { me = std::max(me, std::fabs(s.E[c])); mh = std::max(mh, s.fine.h[c]); }
    if (me > 10.0 * mh) return OW3D_ERR_UNSTABLE;
    s.time = time + dt;
    return status;
}

// ------------------------------------------------------------ creation
static Sim* create(const ow3d_params* p, const double* h, const double* hx, const double* hxx, const double* hy,
                   const double* hyy, int mode) {
    std::unique_ptr<Sim> s(new Sim());
    s->p = *p; s->mode = mode;
    s->gx = (p->Nx > 1) ? p->GhostGridX : 0; s->gy = (p->Ny > 1) ? p->GhostGridY : 0; s->gz = p->GhostGridZ;
    s->Nxg = p->Nx + 2 * s->gx; s->Nyg = p->Ny + 2 * s->gy; s->Nzg = p->Nz + s->gz;
    s->C = s->Nxg * s->Nyg; s->N = s->C * s->Nzg;
    s->dimcase = (p->Ny == 1) ? 1 : (p->Nx == 1 ? 2 : 3);
    setup_fine_grid(*s);
    LevelGrid& G = s->fine;
    G.h.assign(h, h + s->C); G.hx.assign(hx, hx + s->C); G.hxx.assign(hxx, hxx + s->C);
    G.hy.assign(hy, hy + s->C); G.hyy.assign(hyy, hyy + s->C);
    s->per = (p->periodic_x != 0) ? 1 : 0;
    s->SX = s->per ? build_stencils_periodic(G.x, p->alpha) : build_stencils_xy(G.x, p->alpha);
    s->SY = build_stencils_xy(G.y, p->beta);
    s->SZ = build_stencils_z(G.z, p->Nz, s->gz, p->gamma);
    s->T = build_cross_tables(G, s->SX, s->SY, s->SZ, p->gamma, s->gx, s->gy, s->gz);
    if (p->Precond == 3) {
        if (build_hierarchy(*s) != 0) return nullptr;
        for (auto& Lv : s->lev) assemble_level(*s, Lv);
        dense_lu(s->lev[0]);
        for (size_t l = 1; l < s->lev.size(); ++l) build_ighost(s->lev[l]);
    }
    size_t C = s->C, N = s->N;
    for (auto* v : {&s->E, &s->P, &s->W, &s->Ex, &s->Exx, &s->Ey, &s->Eyy, &s->Px, &s->Py, &s->tE, &s->tP, &s->tW,
                    &s->tEx, &s->tExx, &s->tEy, &s->tEyy, &s->tPx, &s->tPy, &s->sEx, &s->sPx, &s->sEy, &s->sPy,
                    &s->tsEx, &s->tsPx})
        v->assign(C, 0.0);
    for (auto* v : {&s->PHI, &s->LASTPHI0, &s->LASTPHI1, &s->RHS}) v->assign(N, 0.0);
    update_sigma(*s, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (p->filteringONOFF > 0) filter_init(*s);
    setup_zones(*s);
    setup_pdamp(*s);
    // OceanWave3DT0Setup.f90:325-326
    if (p->current_flag) { s->Ul = p->current_Q / G.h[0]; s->Ur = p->current_Q / G.h[(size_t)s->Nxg - 2]; }
    // DetectBreaking.f90:38-70 (the first call): tan(phi) starts at tan(phi_b); Initialize.f90:7-8
    // local smoothing on for limits up to 100 g (LocalSmoothing2D.f90:37): any
    // value a deck gives, or a positive one set by a caller
    s->smooth = (p->accel_from_deck ? p->accel_tol_fact <= 100.0
                                    : (p->accel_tol_fact > 0.0 && p->accel_tol_fact <= 100.0)) ? 1 : 0;
    if (s->smooth) { for (auto& v : s->WHist) v.assign(C, 0.0); s->EtatHist1.assign(C, 0.0); }
    s->pad = p->IncWaveType == 3 ? 1 : 0;
    s->Uneu.assign((size_t)s->Nyg, 0.0);
    s->brk = (p->i_breaking > 0 && p->Ny == 1 && p->Nx > 1) ? 1 : 0;
    s->Qr_x.assign(C, 0.0);
    if (s->brk) {
        const double deg2rad = std::acos(-1.0) / 180.0;
        s->tan_b = std::tan(deg2rad * p->phi_b); s->tan_0 = std::tan(deg2rad * p->phi_0);
        s->tan_phi.assign(C, s->tan_b);
    }
    s->time = p->time0;
    return s.release();
}

}  // namespace orc

// =================================================================== C API
using namespace orc;
extern "C" {

void* orc_create(const ow3d_params* p, const double* h, const double* hx, const double* hxx, const double* hy,
                 const double* hyy, int mode) {
    return create(p, h, hx, hxx, hy, hyy, mode);
}
void orc_destroy(void* s) { delete (Sim*)s; }
void orc_set_mode(void* s, int mode) { ((Sim*)s)->mode = mode; }
int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}
int orc_dims(void* sv, int* Nxg, int* Nyg, int* Nzg, int* nlev) {
    Sim* s = (Sim*)sv; *Nxg = s->Nxg; *Nyg = s->Nyg; *Nzg = s->Nzg; *nlev = (int)s->lev.size(); return 0;
}
int orc_level_dims(void* sv, int l, int* Nx, int* Ny, int* Nz, int* ncolor) {
    Sim* s = (Sim*)sv; const Level& Lv = s->lev[l];
    *Nx = Lv.G.Nx; *Ny = Lv.G.Ny; *Nz = Lv.G.Nz; *ncolor = Lv.ncolor; return 0;
}
void orc_level_z(void* sv, int l, double* z) { Sim* s = (Sim*)sv; const Level& Lv = s->lev[l]; std::copy(Lv.G.z.begin(), Lv.G.z.end(), z); }
void orc_fine_z(void* sv, double* z) { Sim* s = (Sim*)sv; std::copy(s->fine.z.begin(), s->fine.z.end(), z); }
int orc_level_nnz(void* sv, int l) { return (int)((Sim*)sv)->lev[l].A.v.size(); }
void orc_level_csr(void* sv, int l, int* rp, int* ci, double* v) {
    const CSR& A = ((Sim*)sv)->lev[l].A;
    std::copy(A.rp.begin(), A.rp.end(), rp); std::copy(A.ci.begin(), A.ci.end(), ci); std::copy(A.v.begin(), A.v.end(), v);
}
void orc_level_matvec(void* sv, int l, const double* x, double* y) { csr_mv(((Sim*)sv)->lev[l].A, x, y); }
void orc_level_pass(void* sv, int l, int colour, double* x, const double* b) {
    Sim* s = (Sim*)sv; Level& Lv = s->lev[l];
    if (colour < 0) dm_bottoms(Lv, x, b); else dm_pass(Lv, colour, x, b);
}
void orc_level_smooth(void* sv, int l, double* x, const double* b, int nu) {
    Sim* s = (Sim*)sv; Level& Lv = s->lev[l];
    if (s->mode == 0) { gs_special(Lv, x, b); for (int i = 0; i < nu; ++i) { gs_lex(Lv.A, x, b); gs_special(Lv, x, b); } }
    else dm_smooth(Lv, x, b, nu);
}
void orc_restrict(void* sv, int lf, const double* rf, double* rc) { Sim* s = (Sim*)sv; restrict_(*s, s->lev[lf], s->lev[lf - 1], rf, rc); }
void orc_prolong(void* sv, int lf, double* pf, const double* pc) { Sim* s = (Sim*)sv; prolong_(*s, s->lev[lf], s->lev[lf - 1], pf, pc); }
void orc_coarse_solve(void* sv, double* x) { Sim* s = (Sim*)sv; dense_solve(s->lev[0], x); }
void orc_stencils(void* sv, double* SX, double* SY, double* SZ) {
    Sim* s = (Sim*)sv;
    std::copy(s->SX.w.begin(), s->SX.w.end(), SX); std::copy(s->SY.w.begin(), s->SY.w.end(), SY); std::copy(s->SZ.w.begin(), s->SZ.w.end(), SZ);
}
void orc_set_surface(void* sv, const double* E, const double* Ex, const double* Exx, const double* Ey, const double* Eyy) {
    update_sigma(*(Sim*)sv, E, Ex, Exx, Ey, Eyy);
}
void orc_matvec(void* sv, const double* phi, double* y) { matvec_ho(*(Sim*)sv, phi, y); }
void orc_precond(void* sv, const double* r, double* u) { precond(*(Sim*)sv, r, u); }
int orc_solve(void* sv, const double* rhs, double* phi, int* iters, double* resid) {
    int it = 0; double rs = 0; int st = solve(*(Sim*)sv, rhs, phi, it, rs); *iters = it; *resid = rs; return st;
}
void orc_set_state(void* sv, const double* E, const double* P, const double* W, const double* phi, double t) {
    Sim* s = (Sim*)sv;
    if (E) s->E.assign(E, E + s->C); if (P) s->P.assign(P, P + s->C); if (W) s->W.assign(W, W + s->C);
    if (phi) s->PHI.assign(phi, phi + s->N); else std::fill(s->PHI.begin(), s->PHI.end(), 0.0);
    if (s->per) { zero_images_x(*s, s->PHI.data(), s->Nzg); if (W) images_x(*s, s->W.data(), 1); }
    std::fill(s->LASTPHI0.begin(), s->LASTPHI0.end(), 0.0); std::fill(s->LASTPHI1.begin(), s->LASTPHI1.end(), 0.0);
    s->time = t; s->tstep = 0;
    std::fill(s->sPx.begin(), s->sPx.end(), 0.0);   // the set-up's sources are zero
    std::fill(s->sEx.begin(), s->sEx.end(), 0.0);
    // OceanWave3DT0Setup.f90:444,564-569: surface derivatives; linear case keeps eta = 0 coefficients.
    fs_derivs(*s, s->E, s->P, s->Ex, s->Exx, s->Px, s->Ey, s->Eyy, s->Py);
    update_sigma(*s, nullptr, nullptr, nullptr, nullptr, nullptr);
}
void orc_get_state(void* sv, double* E, double* P, double* W, double* phi, double* t) {
    Sim* s = (Sim*)sv;
    if (E) std::copy(s->E.begin(), s->E.end(), E); if (P) std::copy(s->P.begin(), s->P.end(), P);
    if (W) std::copy(s->W.begin(), s->W.end(), W);
    if (phi) {
        std::copy(s->PHI.begin(), s->PHI.end(), phi);
        if (s->per) images_x(*s, phi, s->Nzg);   // periodic: image columns filled on output
    }
    if (t) *t = s->time;
}
void orc_get_derivs(void* sv, double* Ex, double* Exx, double* Px, double* Ey, double* Eyy, double* Py) {
    Sim* s = (Sim*)sv;
    std::copy(s->Ex.begin(), s->Ex.end(), Ex); std::copy(s->Exx.begin(), s->Exx.end(), Exx); std::copy(s->Px.begin(), s->Px.end(), Px);
    std::copy(s->Ey.begin(), s->Ey.end(), Ey); std::copy(s->Eyy.begin(), s->Eyy.end(), Eyy); std::copy(s->Py.begin(), s->Py.end(), Py);
}
int orc_set_relax_target(void* sv, int zone, int mode, int nt, double dts, const double* eta, const double* phis) {
    Sim* s = (Sim*)sv; if (zone < 0 || zone >= (int)s->zones.size()) return -1;
    Zone& Z = s->zones[zone]; size_t box = (size_t)(Z.i1 - Z.i0 + 1) * (Z.j1 - Z.j0 + 1);
    Z.tmode = mode; Z.nt = nt; Z.tdt = dts; Z.eta.assign(eta, eta + box * nt); Z.phis.assign(phis, phis + box * nt);
    return 0;
}
int orc_zone_box(void* sv, int zone, int* i0, int* i1, int* j0, int* j1) {
    Sim* s = (Sim*)sv; if (zone < 0 || zone >= (int)s->zones.size()) return -1;
    const Zone& Z = s->zones[zone]; *i0 = Z.i0; *i1 = Z.i1; *j0 = Z.j0; *j1 = Z.j1; return 0;
}
void orc_zone_gamma(void* sv, int zone, double* g) { const Zone& Z = ((Sim*)sv)->zones[zone]; std::copy(Z.gam.begin(), Z.gam.end(), g); }
void orc_filter_coeffs(void* sv, double* centre, double* boundary) {
    Sim* s = (Sim*)sv; std::copy(s->fc.begin(), s->fc.end(), centre); std::copy(s->fc2.begin(), s->fc2.end(), boundary);
}
void orc_filter(void* sv, double* U) { Sim* s = (Sim*)sv; vector<double> u(U, U + s->C); filter(*s, u); std::copy(u.begin(), u.end(), U); }
int orc_step(void* sv, int nsteps) {
    Sim* s = (Sim*)sv; int st = OW3D_OK;
    for (int i = 0; i < nsteps; ++i) { int r = rk4_step(*s); if (r < 0) return r; if (r > 0) st = r; }
    return st;
}
void orc_stats(void* sv, int64_t* solves, int64_t* totit, int* minit, int* maxit, int* lastit, double* lastres, int64_t* notconv) {
    Sim* s = (Sim*)sv; *solves = s->solves; *totit = s->totit; *minit = s->minit; *maxit = s->maxit; *lastit = s->lastit;
    *lastres = s->lastres; *notconv = s->notconv;
}
// the rollers of the last completed step: count, and per roller the points
// it covers, the toe column, its position (x = (j-1) dx), the elevation at
// the toe, the thickness one column behind the toe and tan(phi) at the toe
int orc_rollers(void* sv, int cap, int* npts, int* toe, double* x, double* eta, double* thick, double* tanphi) {
    Sim* s = (Sim*)sv; const int n = (int)s->r_npts.size();
    for (int r = 0; r < n && r < cap; ++r) {
        npts[r] = s->r_npts[r]; toe[r] = s->r_toe[r]; x[r] = s->r_x[r]; eta[r] = s->r_eta[r];
        thick[r] = s->r_thick[r]; tanphi[r] = s->r_tan[r];
    }
    return n;
}
// one detect_breaking call on the surface E (update: the call after a step)
int orc_detect_breaking(void* sv, const double* E, int update) {
    Sim* s = (Sim*)sv; if (!s->brk) return -1;
    vector<double> e(E, E + s->C); detect_breaking(*s, e, update != 0); return 0;
}
// setupWavePaddle.f90:89-122: the signal (flux time-major, nt x n2) and
// eta_x = -u_t / g from the 5-point time derivative (one-sided at the ends)
int orc_set_paddle(void* sv, int nt, int n2, double dt, const double* y, const double* flux) {
    Sim* s = (Sim*)sv; if (!s->pad || nt < 5 || n2 < 1) return -1;
    s->pad_nt = nt; s->pad_n2 = n2; s->pad_dt = dt;
    s->pad_y.assign(y, y + n2); s->pad_flux.assign(flux, flux + (size_t)nt * n2);
    s->pad_etax.assign((size_t)nt * n2, 0.0);
    double ft[5], fc[5][5];
    for (int i = 0; i < 5; ++i) ft[i] = i * dt;
    for (int i = 0; i < 5; ++i) fd_weights(ft[i], ft, 4, 1, fc[i]);
    const double gfac = -1.0 / s->p.g;
    for (int j = 1; j <= n2; ++j) {
        auto F = [&](int i) { return s->pad_flux[(size_t)(i - 1) * n2 + j - 1]; };
        auto dot = [&](int row, int i0) { double a = 0; for (int q = 0; q < 5; ++q) a += fc[row - 1][q] * F(i0 + q); return a; };
        for (int i = 1; i <= 2; ++i) s->pad_etax[(size_t)(i - 1) * n2 + j - 1] = gfac * dot(i, 1);
        for (int i = 3; i <= nt - 2; ++i) s->pad_etax[(size_t)(i - 1) * n2 + j - 1] = gfac * dot(3, i - 2);
        for (int i = nt - 1; i <= nt; ++i) s->pad_etax[(size_t)(i - 1) * n2 + j - 1] = gfac * dot(5 - (nt - i), nt - 4);
    }
    return 0;
}
// the last local-smoothing call: dw/dt at the surface (C values) and the
// columns where it exceeded the limit; returns their count (-1: off)
int orc_accel_state(void* sv, double* Wt, int cap, int* cols) {
    Sim* s = (Sim*)sv; if (!s->smooth) return -1;
    if (Wt && !s->accel_Wt.empty()) std::copy(s->accel_Wt.begin(), s->accel_Wt.end(), Wt);
    const int n = (int)s->accel_pts.size();
    for (int q = 0; q < n && q < cap; ++q) cols[q] = s->accel_pts[q];
    return n;
}
void orc_breaking_state(void* sv, double* tan_phi, double* Qr_x) {
    Sim* s = (Sim*)sv;
    if (tan_phi && !s->tan_phi.empty()) std::copy(s->tan_phi.begin(), s->tan_phi.end(), tan_phi);
    if (Qr_x) std::copy(s->Qr_x.begin(), s->Qr_x.end(), Qr_x);
}
void orc_reset_stats(void* sv) { Sim* s = (Sim*)sv; s->solves = s->totit = s->notconv = 0; s->minit = 1 << 30; s->maxit = 0; }
}
