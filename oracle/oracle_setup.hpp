// ORACLE -- test infrastructure only. CPU restatement of the OceanWave3D
// reference algorithm (FP64). Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference arm of bench.py may load it; the product library
// never links or calls anything under oracle/.
//
// This header restates the set-up half of the reference: grids, Fornberg
// stencils, sigma coefficients, cross-derivative tables, the multigrid
// hierarchy and the assembled low-order preconditioning matrices.
#pragma once
#include <vector>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <string>
#include "../include/ow3d.h"

namespace orc {

using std::vector;

// Fornberg's recursion for finite-difference weights.
// Restates `weights` (src/utilities/stream_func_wave_finite.f:128-168):
// z expansion point, x[0..n] nodes, m highest derivative; c[j*(m+1)+k].
inline void fornberg(double z, const double* x, int n, int m, double* c) {
    double c1 = 1.0, c4 = x[0] - z;
    for (int k = 0; k <= m; ++k)
        for (int j = 0; j <= n; ++j) c[j * (m + 1) + k] = 0.0;
    c[0] = 1.0;
    for (int i = 1; i <= n; ++i) {
        int mn = std::min(i, m);
        double c2 = 1.0, c5 = c4;
        c4 = x[i] - z;
        for (int j = 0; j <= i - 1; ++j) {
            double c3 = x[i] - x[j];
            c2 = c2 * c3;
            if (j == i - 1) {
                for (int k = mn; k >= 1; --k)
                    c[i * (m + 1) + k] = c1 * (k * c[(i - 1) * (m + 1) + k - 1] - c5 * c[(i - 1) * (m + 1) + k]) / c2;
                c[i * (m + 1) + 0] = -c1 * c5 * c[(i - 1) * (m + 1) + 0] / c2;
            }
            for (int k = mn; k >= 1; --k)
                c[j * (m + 1) + k] = (c4 * c[j * (m + 1) + k] - k * c[j * (m + 1) + k - 1]) / c3;
            c[j * (m + 1) + 0] = c4 * c[j * (m + 1) + 0] / c3;
        }
        c1 = c2;
    }
}

// Stencil of `order` (1 or 2) on nodes xs[0..n] expanded at z -> w[0..n].
inline void fd_weights(double z, const double* xs, int n, int order, double* w) {
    vector<double> c((n + 1) * (order + 1));
    fornberg(z, xs, n, order, c.data());
    for (int j = 0; j <= n; ++j) w[j] = c[j * (order + 1) + order];
}

// Per-position stencil tables, layout S[(order-1)][pos][m], pos 0-based.
struct Stencil1D {
    int n = 0, rank = 0;
    vector<double> w;
    double at(int order, int pos, int m) const { return w[((size_t)(order - 1) * n + pos) * rank + m]; }
    double& at(int order, int pos, int m) { return w[((size_t)(order - 1) * n + pos) * rank + m]; }
};

// BuildStencilsGridX / BuildStencilsGridY (src/initialization/BuildStencilsGridX.f90:1-66,
// BuildStencilsGridY.f90:1-49): uniform-grid stencils of half width a, with
// shifted one-sided windows at the first/last a points. Nodes are given as 1-D
// coordinates x[0..n-1] (the reference uses x(:,1) resp. y(1,:)).
inline Stencil1D build_stencils_xy(const vector<double>& x, int a) {
    Stencil1D s; s.n = (int)x.size(); s.rank = 2 * a + 1;
    s.w.assign((size_t)2 * s.n * s.rank, 0.0);
    if (s.n == 1) return s;  // derivative of a one-point field is zero
    vector<double> nodes(s.rank), w(s.rank);
    for (int order = 1; order <= 2; ++order) {
        for (int i = 1; i <= s.n; ++i) {  // 1-based as in the reference
            int diff;
            if (i - 1 < a) diff = a - i + 1;
            else if (i >= s.n - a + 1) diff = (s.n - a) - i;
            else diff = 0;
            for (int m = 0; m < s.rank; ++m) nodes[m] = x[i + (m - a) + diff - 1];
            fd_weights(x[i - 1], nodes.data(), s.rank - 1, order, w.data());
            for (int m = 0; m < s.rank; ++m) s.at(order, i - 1, m) = w[m];
        }
    }
    return s;
}

// Periodic direction (no counterpart in the reference, whose lateral rows
// are walls): every position takes the centred stencil of half width a,
// formed on the nodes around the middle position of the uniform grid.
inline Stencil1D build_stencils_periodic(const vector<double>& x, int a) {
    Stencil1D s; s.n = (int)x.size(); s.rank = 2 * a + 1;
    s.w.assign((size_t)2 * s.n * s.rank, 0.0);
    vector<double> w(s.rank);
    const int mid = s.n / 2;
    for (int order = 1; order <= 2; ++order) {
        fd_weights(x[mid], &x[mid - a], s.rank - 1, order, w.data());
        for (int i = 0; i < s.n; ++i)
            for (int m = 0; m < s.rank; ++m) s.at(order, i, m) = w[m];
    }
    return s;
}

// Periodic x: the distinct columns are 2..Nxg-2 (1-based, ghosts counted);
// column Nxg-1 repeats column 2 and the ghost columns 1 and Nxg are unused.
// wrap_x maps any column index into the distinct range.
inline int wrap_x(int i, int Nxg) {
    const int M = Nxg - 3;
    while (i < 2) i += M;
    while (i > Nxg - 2) i -= M;
    return i;
}

// TaylorFDStencils1DArbitrary (src/functions/TaylorFDStencils1DArbitrary.f90:1-14):
// alp+bet+1 nodes, expansion at node alp.
inline void taylor(int alp, int bet, int order, const double* x, double* w) {
    fd_weights(x[alp], x, alp + bet, order, w);
}

// z stencils: PreProcessDiffStencils.f90:108-132 (Nzp = Nz + GhostGridZ levels).
inline Stencil1D build_stencils_z(const vector<double>& z, int Nz, int ghostz, int g) {
    Stencil1D s; int Nzp = Nz + ghostz; s.n = Nzp; s.rank = 2 * g + 1;
    s.w.assign((size_t)2 * s.n * s.rank, 0.0);
    vector<double> nodes(s.rank), w(s.rank);
    for (int order = 1; order <= 2; ++order) {
        for (int i = 1; i <= Nzp; ++i) {
            int alp, bet, diff, off;
            if (i - 1 < g) { diff = g - i + 1; alp = g - diff; bet = g + diff; off = diff; }
            else if (i >= Nz - g + 1) { diff = i - (Nzp - g); alp = g + diff; bet = g - diff; off = -diff; }
            else { alp = g; bet = g; off = 0; }
            for (int m = 0; m < s.rank; ++m) nodes[m] = z[i + (m - g) + off - 1];
            taylor(alp, bet, order, nodes.data(), w.data());
            for (int m = 0; m < s.rank; ++m) s.at(order, i - 1, m) = w[m];
        }
    }
    return s;
}

// DiffStencilsZ_modif (src/functions/DiffStencilsZ_modif.f90:1-46): the level-k
// z stencil shifted by idxg_c (corner treatment), returns order-1 weights.
inline void stencil_z_modif(int k, const vector<double>& z, int Nz, int ghostz, int g, int idxg_c,
                            double* w1) {
    int Nzp = ghostz == 0 ? Nz : Nz + 1;
    int rank = 2 * g + 1;
    vector<double> nodes(rank);
    int i = k, alp, bet, off;
    if (i - 1 < g) { int diff = g - i + 1; alp = g - diff - idxg_c; bet = g + diff + idxg_c; off = diff + idxg_c; }
    else if (i >= Nz - g + 1) { int diff = i - (Nzp - g); alp = g + diff - idxg_c; bet = g - diff + idxg_c; off = -diff + idxg_c; }
    else { alp = g - idxg_c; bet = g + idxg_c; off = idxg_c; }
    for (int m = 0; m < rank; ++m) nodes[m] = z[i + (m - g) + off - 1];
    taylor(alp, bet, 1, nodes.data(), w1);
}

// Sigma coefficients at one point: DetermineTransformationConstantsArray.f90:98-120
// (3-D branch), :60-78 (Ny==1), :79-97 (Nx==1). out[0..4] = sigma, sx, lap, sy, sz.
inline void sigma_coeffs(int dim_case, double z, double E, double Ex, double Exx, double Ey, double Eyy,
                         double h, double hx, double hxx, double hy, double hyy, double* out) {
    const double one = 1.0, two = 2.0;
    double d = E + h;
    double s1 = z;
    out[0] = s1; out[1] = 0.0; out[2] = 0.0; out[3] = 0.0; out[4] = 0.0;
    if (dim_case == 1) {  // Ny == 1
        out[1] = ((one - s1) * hx - s1 * Ex) / d;
        out[2] = -two * (one - s1) * (hx * hx) / (d * d) + two * (two * s1 - one) * (Ex * hx) / (d * d) +
                 (one - s1) * (hxx) / d + two * s1 * (Ex * Ex) / (d * d) - s1 * (Exx) / d;
        out[4] = one / d;
    } else if (dim_case == 2) {  // Nx == 1
        out[2] = -two * (one - s1) * (hy * hy) / (d * d) + two * (two * s1 - one) * (Ey * hy) / (d * d) +
                 (one - s1) * (hyy) / d + two * s1 * (Ey * Ey) / (d * d) - s1 * (Eyy) / d;
        out[3] = ((one - s1) * hy - s1 * Ey) / d;
        out[4] = one / d;
    } else {
        out[1] = ((one - s1) * hx - s1 * Ex) / d;
        out[2] = -two * (one - s1) * (hx * hx + hy * hy) / (d * d) +
                 two * (two * s1 - one) * (Ex * hx + Ey * hy) / (d * d) + (one - s1) * (hxx + hyy) / d +
                 two * s1 * (Ex * Ex + Ey * Ey) / (d * d) - s1 * (Exx + Eyy) / d;
        out[3] = ((one - s1) * hy - s1 * Ey) / d;
        out[4] = one / d;
    }
}

// Cross-derivative index/weight tables of ConstructTableCrossDerivatives
// (src/functions/ConstructTableCrossDerivatives.f90:90-264), flattened per
// point (k,i,j) 1-based -> p = (k-1) + Nzg*((i-1) + Nxg*(j-1)), entry m.
struct CrossTables {
    int Nxg = 0, Nyg = 0, Nzg = 0, rank = 0;
    vector<int> IX, IY, IZ1, IZ2;          // 1-based indices
    vector<double> SX, SY, SZ1, SZ2;
    size_t id(int k, int i, int j, int m) const {
        return ((size_t)(k - 1) + (size_t)Nzg * ((size_t)(i - 1) + (size_t)Nxg * (size_t)(j - 1))) * rank + m;
    }
};

struct LevelGrid {
    int Nx = 1, Ny = 1, Nz = 1;      // interior counts
    int Nxg = 1, Nyg = 1, Nzg = 1;   // with ghosts
    vector<double> x, y, z;          // 1-D coordinates (Nxg, Nyg, Nzg)
    vector<double> h, hx, hxx, hy, hyy;  // Nxg*Nyg, i fastest
};

inline CrossTables build_cross_tables(const LevelGrid& G, const Stencil1D& SXs, const Stencil1D& SYs,
                                      const Stencil1D& SZs, int kappa, int gx, int gy, int gz) {
    CrossTables T;
    const int Nxg = G.Nxg, Nyg = G.Nyg, Nzg = G.Nzg;
    const int rank = 2 * kappa + 1;
    T.Nxg = Nxg; T.Nyg = Nyg; T.Nzg = Nzg; T.rank = rank;
    size_t Np = (size_t)Nxg * Nyg * Nzg * rank;
    T.IX.assign(Np, 0); T.IY.assign(Np, 0); T.IZ1.assign(Np, 0); T.IZ2.assign(Np, 0);
    T.SX.assign(Np, 0.0); T.SY.assign(Np, 0.0); T.SZ1.assign(Np, 0.0); T.SZ2.assign(Np, 0.0);
    int alpha, ranka, beta, rankb;
    if (Nxg > 1) { alpha = kappa; ranka = rank; } else { alpha = 0; ranka = 1; }
    if (Nyg > 1) { beta = kappa; rankb = rank; } else { beta = 0; rankb = 1; }
    vector<int> idx(rank), idxa(rank), idxb(rank), idxg(rank);
    for (int m = 0; m < rank; ++m) idx[m] = m - kappa;
    vector<double> wz(rank);
    for (int j = 1; j <= Nyg; ++j) {
        int diffb = (j < beta + 1) ? beta + 1 - j : (j > Nyg - beta ? (Nyg - beta) - j : 0);
        for (int m = 0; m < rank; ++m) idxb[m] = j + idx[m] + diffb;
        for (int i = 1; i <= Nxg; ++i) {
            int diffa = (i < alpha + 1) ? alpha + 1 - i : (i > Nxg - alpha ? (Nxg - alpha) - i : 0);
            for (int m = 0; m < rank; ++m) idxa[m] = i + idx[m] + diffa;
            for (int k = 1; k <= Nzg; ++k) {
                int idxa_c = 0, idxb_c = 0, idxg_c = 0, idxg_c2 = 0;
                int diffg = (k < kappa + 1) ? kappa + 1 - k : (k > Nzg - kappa ? (Nzg - kappa) - k : 0);
                for (int m = 0; m < rank; ++m) idxg[m] = k + idx[m] + diffg;
                if (i == 1 || i == Nxg) { if (idxg[0] == 1) idxg_c = 1; }
                if (j == 1 || j == Nyg) { if (idxg[0] == 1) idxg_c2 = 1; }
                if (k == 1) {
                    if (idxa[0] == 1) idxa_c = 1;
                    if (idxa[ranka - 1] == Nxg) idxa_c = -1;
                    if (idxb[0] == 1) idxb_c = 1;
                    if (idxb[rankb - 1] == Nyg) idxb_c = -1;
                }
                if (i == 1 || i == Nxg) idxa_c = 0;
                if (j == 1 || j == Nyg) idxb_c = 0;
                if (k == 1 || k == Nzg) { idxg_c = 0; idxg_c2 = 0; }
                // XZ tables
                for (int m = 0; m < ranka; ++m) {
                    T.IX[T.id(k, i, j, m)] = idxa[m] + idxa_c;
                    if (Nxg > 1) T.SX[T.id(k, i, j, m)] = SXs.at(1, i - idxa_c - 1, m);
                }
                for (int m = 0; m < rank; ++m) T.IZ1[T.id(k, i, j, m)] = idxg[m] + idxg_c;
                if (idxg_c == 0) { for (int m = 0; m < rank; ++m) wz[m] = SZs.at(1, k - 1, m); }
                else stencil_z_modif(k, G.z, G.Nz, gz, kappa, idxg_c, wz.data());
                for (int m = 0; m < rank; ++m) T.SZ1[T.id(k, i, j, m)] = wz[m];
                // YZ tables
                for (int m = 0; m < rankb; ++m) {
                    T.IY[T.id(k, i, j, m)] = idxb[m] + idxb_c;
                    if (Nyg > 1) T.SY[T.id(k, i, j, m)] = SYs.at(1, j - idxb_c - 1, m);
                }
                for (int m = 0; m < rank; ++m) T.IZ2[T.id(k, i, j, m)] = idxg[m] + idxg_c2;
                if (idxg_c2 == 0) { for (int m = 0; m < rank; ++m) wz[m] = SZs.at(1, k - 1, m); }
                else stencil_z_modif(k, G.z, G.Nz, gz, kappa, idxg_c2, wz.data());
                for (int m = 0; m < rank; ++m) T.SZ2[T.id(k, i, j, m)] = wz[m];
            }
        }
    }
    (void)gx; (void)gy;
    return T;
}

// Compressed sparse row matrix with the diagonal stored first in every row
// (CSRdiaREORDER.f90:1-40); duplicates summed (CleanSparseMatrixCOO.f90:31).
struct CSR {
    int n = 0;
    vector<int> rp, ci;
    vector<double> v;
};

// Row builder: accumulates (col, val) pairs, summing duplicates in order of
// first appearance.
struct RowAcc {
    vector<int> cols; vector<double> vals;
    void clear() { cols.clear(); vals.clear(); }
    void add(int c, double v) {
        for (size_t t = 0; t < cols.size(); ++t) if (cols[t] == c) { vals[t] += v; return; }
        cols.push_back(c); vals.push_back(v);
    }
};

}  // namespace orc
