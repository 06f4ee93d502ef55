// Multigrid preconditioner on the low-order (alpha = beta = gamma = 1),
// linearised (eta = 0) operator, matrix free.
//
// The row equations are the ones BuildLinearSystemMatrix.f90:1-338 assembles
// from PrepareFullOperatorStencils.f90 and the Precond==1 part of
// ConstructTableCrossDerivatives.f90:266-351 (including that part's
// replication of the mixed-derivative stencil over the three neighbouring
// y-planes for d2/dxds and x-planes for d2/dyds). Coefficients are evaluated in
// the kernels from the level's depth fields instead of being stored as CSR.
//
// Smoother (device-matched ordering, deterministic):
//   special pass  : rows of the ghost columns (lateral Neumann / identity) and
//                   the bottom rows of the interior columns (the reference's
//                   iGhost list, MGPreProcess.f90:376-439)
//   colour sweeps : interior columns in 2 or 4 colours, Gauss-Seidel up each
//                   column (k = 2..Nzg, free surface row last)
// sequence per smoothing step as MultiGridSolver.f90:118-126,174-181:
//   special; [colours; special] x nu
#include "ow3d_internal.h"
#include <vector>

namespace ow3d {

namespace {

template <typename T>
__device__ __forceinline__ int64_t IX(const LevelDev<T>& L, int k, int i, int j) {
    return (int64_t)(k - 1) + (int64_t)L.Nzg * ((int64_t)(i - 1) + (int64_t)L.Nxg * (j - 1));
}
template <typename T>
__device__ __forceinline__ T sx(const LevelDev<T>& L, int o, int i, int m) { return L.SX[((o - 1) * L.Nxg + (i - 1)) * 3 + m]; }
template <typename T>
__device__ __forceinline__ T sy(const LevelDev<T>& L, int o, int j, int m) { return L.SY[((o - 1) * L.Nyg + (j - 1)) * 3 + m]; }
template <typename T>
__device__ __forceinline__ T sz(const LevelDev<T>& L, int o, int k, int m) { return L.SZ[((o - 1) * L.Nzg + (k - 1)) * 3 + m]; }

// Interior row (2 <= k <= Nzg-1, interior column). Returns A x at the row and
// the diagonal coefficient.
template <typename T, bool THREE>
__device__ T lo_interior(const LevelDev<T>& L, const T* x, int k, int i, int j, T& diag) {
    const int64_t c = (int64_t)(i - 1) + (int64_t)L.Nxg * (j - 1);
    const T h = L.h[c], hx = L.hx[c], hxx = L.hxx[c];
    const T hy = THREE ? L.hy[c] : T(0), hyy = THREE ? L.hyy[c] : T(0);
    const T sg = L.zs[k - 1], om = T(1) - sg;
    const T d = h;
    // DetermineTransformationConstantsArray with eta = 0
    const T s2 = (om * hx) / d;
    const T s4 = (om * hy) / d;
    const T s5 = T(1) / d;
    const T s3 = -T(2) * om * (hx * hx + hy * hy) / (d * d) + om * (hxx + hyy) / d;
    const T cz = s2 * s2 + s4 * s4 + s5 * s5;
    T acc = 0;
    // d2/dx2, d2/dy2 (centred 3-point, PrepareFullOperatorStencils.f90:213-231)
#pragma unroll
    for (int m = 0; m < 3; ++m) acc += sx(L, 2, i, m) * x[IX(L, k, i - 1 + m, j)];
    if (THREE) {
#pragma unroll
        for (int m = 0; m < 3; ++m) acc += sy(L, 2, j, m) * x[IX(L, k, i, j - 1 + m)];
    }
    T dz = 0, dzz = 0;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const T v = x[IX(L, k - 1 + m, i, j)];
        dz += sz(L, 1, k, m) * v;
        dzz += sz(L, 2, k, m) * v;
    }
    acc += s3 * dz + cz * dzz;
    diag = sx(L, 2, i, 1) + (THREE ? sy(L, 2, j, 1) : T(0)) + s3 * sz(L, 1, k, 1) + cz * sz(L, 2, k, 1);
    // mixed d2/dxds: sum over y-planes J of Dz(Dx x), the x stencil at level 1
    // shifted away from the ghost corner columns.
    if (s2 != T(0)) {
        T xz = 0;
        const int jlo = THREE ? j - 1 : j, jhi = THREE ? j + 1 : j;
        for (int jj = jlo; jj <= jhi; ++jj) {
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
                const int kz = k - 1 + kk;
                int sh = 0;
                if (kz == 1) { if (i - 1 == 1) sh = 1; if (i + 1 == L.Nxg) sh = -1; }
                T dx = 0;
#pragma unroll
                for (int m = 0; m < 3; ++m) dx += sx(L, 1, i - sh, m) * x[IX(L, kz, i - 1 + sh + m, jj)];
                xz += sz(L, 1, k, kk) * dx;
            }
        }
        acc += T(2) * s2 * xz;
        diag += T(2) * s2 * (sz(L, 1, k, 1) * sx(L, 1, i, 1));
    }
    if (THREE && s4 != T(0)) {
        T yz = 0;
        for (int ii = i - 1; ii <= i + 1; ++ii) {
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
                const int kz = k - 1 + kk;
                int sh = 0;
                if (kz == 1) { if (j - 1 == 1) sh = 1; if (j + 1 == L.Nyg) sh = -1; }
                T dy = 0;
#pragma unroll
                for (int m = 0; m < 3; ++m) dy += sy(L, 1, j - sh, m) * x[IX(L, kz, ii, j - 1 + sh + m)];
                yz += sz(L, 1, k, kk) * dy;
            }
        }
        acc += T(2) * s4 * yz;
        diag += T(2) * s4 * (sz(L, 1, k, 1) * sy(L, 1, j, 1));
    }
    return acc;
}

// Bottom row (k = 1, interior column), BuildLinearSystemMatrix.f90:50-70.
template <typename T, bool THREE>
__device__ T lo_bottom(const LevelDev<T>& L, const T* x, int i, int j, T& diag) {
    const int64_t c = (int64_t)(i - 1) + (int64_t)L.Nxg * (j - 1);
    const T h = L.h[c], hx = L.hx[c];
    const T hy = THREE ? L.hy[c] : T(0);
    const T om = T(1) - L.zs[1];
    const T s2 = (om * hx) / h, s4 = (om * hy) / h, s5 = T(1) / h;
    const T f = THREE ? (s5 + hx * s2 + hy * s4) : (s5 + hx * s2);
    T dz = 0;
#pragma unroll
    for (int m = 0; m < 3; ++m) dz += sz(L, 1, 2, m) * x[IX(L, 1 + m, i, j)];
    T dx = 0;
#pragma unroll
    for (int m = 0; m < 3; ++m) dx += sx(L, 1, i, m) * x[IX(L, 2, i - 1 + m, j)];
    T acc = f * dz + hx * dx;
    if (THREE) {
        T dy = 0;
#pragma unroll
        for (int m = 0; m < 3; ++m) dy += sy(L, 1, j, m) * x[IX(L, 2, i, j - 1 + m)];
        acc += hy * dy;
    }
    diag = f * sz(L, 1, 2, 0);
    return acc;
}

// Ghost-column row (lateral Neumann or identity).
template <typename T, bool THREE>
__device__ T lo_ghost(const LevelDev<T>& L, const T* x, int k, int i, int j, T& diag) {
    const bool gxx = (i == 1 || i == L.Nxg), gyy = THREE && (j == 1 || j == L.Nyg);
    if ((gxx && gyy) || k == 1) { diag = T(1); return x[IX(L, k, i, j)]; }
    T acc = 0;
    if (gxx) {
        const int ia = (i == 1) ? 2 : L.Nxg - 1;
#pragma unroll
        for (int m = 0; m < 3; ++m) acc += sx(L, 1, ia, m) * x[IX(L, k, ia - 1 + m, j)];
        diag = sx(L, 1, ia, (i == 1) ? 0 : 2);
    } else {
        const int ja = (j == 1) ? 2 : L.Nyg - 1;
#pragma unroll
        for (int m = 0; m < 3; ++m) acc += sy(L, 1, ja, m) * x[IX(L, k, i, ja - 1 + m)];
        diag = sy(L, 1, ja, (j == 1) ? 0 : 2);
    }
    return acc;
}

template <typename T, bool THREE>
__device__ __forceinline__ bool is_ghost_col(const LevelDev<T>& L, int i, int j) {
    return i == 1 || i == L.Nxg || (THREE && (j == 1 || j == L.Nyg));
}

template <typename T, bool THREE>
__device__ T lo_row(const LevelDev<T>& L, const T* x, int k, int i, int j, T& diag) {
    if (is_ghost_col<T, THREE>(L, i, j)) return lo_ghost<T, THREE>(L, x, k, i, j, diag);
    if (k == L.Nzg) { diag = T(1); return x[IX(L, k, i, j)]; }
    if (k == 1) return lo_bottom<T, THREE>(L, x, i, j, diag);
    return lo_interior<T, THREE>(L, x, k, i, j, diag);
}

// ------------------------------------------------------------- kernels
template <typename T, bool THREE>
__global__ void k_lo_matvec(LevelDev<T> L, const T* __restrict__ x, T* __restrict__ y) {
    const int64_t n = L.N;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(p % L.Nzg) + 1;
        const int64_t c = p / L.Nzg;
        const int i = (int)(c % L.Nxg) + 1, j = (int)(c / L.Nxg) + 1;
        T dg;
        y[p] = lo_row<T, THREE>(L, x, k, i, j, dg);
    }
}

// r = b - A x
template <typename T, bool THREE>
__global__ void k_lo_residual(LevelDev<T> L) {
    const int64_t n = L.N;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(p % L.Nzg) + 1;
        const int64_t c = p / L.Nzg;
        const int i = (int)(c % L.Nxg) + 1, j = (int)(c / L.Nxg) + 1;
        T dg;
        L.rv[p] = L.bv[p] - lo_row<T, THREE>(L, L.xv, k, i, j, dg);
    }
}

// Special pass, part 1: every row of the ghost columns (lateral Neumann rows
// and identity rows). These rows only read interior-column values, so the
// columns update independently.
template <typename T, bool THREE>
__global__ void k_lo_special_ghost(LevelDev<T> L) {
    // ghost columns enumerated along the perimeter: west/east (all j), then
    // south/north (interior i) in 3-D
    const int Nxg = L.Nxg, Nyg = L.Nyg;
    const int64_t nper = THREE ? (int64_t)2 * Nyg + 2 * (Nxg - 2) : 2;
    const int64_t total = nper * L.Nzg;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(q % L.Nzg) + 1;
        const int64_t e = q / L.Nzg;
        int i, j;
        if (!THREE) { i = (e == 0) ? 1 : Nxg; j = 1; }
        else if (e < 2 * Nyg) { i = (e % 2 == 0) ? 1 : Nxg; j = (int)(e / 2) + 1; }
        else { const int64_t f = e - 2 * Nyg; j = (f % 2 == 0) ? 1 : Nyg; i = (int)(f / 2) + 2; }
        T dg;
        const T a = lo_ghost<T, THREE>(L, L.xv, k, i, j, dg);
        const int64_t p = IX(L, k, i, j);
        L.xv[p] = L.xv[p] + (L.bv[p] - a) / dg;
    }
}

// Special pass, part 2: bottom rows of the interior columns (they read the
// ghost-column values part 1 produced, and no other bottom row).
template <typename T, bool THREE>
__global__ void k_lo_special_bottom(LevelDev<T> L) {
    const int64_t C = (int64_t)L.Nxg * L.Nyg;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % L.Nxg) + 1, j = (int)(c / L.Nxg) + 1;
        if (is_ghost_col<T, THREE>(L, i, j)) continue;
        T dg;
        const T a = lo_bottom<T, THREE>(L, L.xv, i, j, dg);
        const int64_t p = IX(L, 1, i, j);
        L.xv[p] = L.xv[p] + (L.bv[p] - a) / dg;
    }
}

// Read-only load: the neighbour columns a colour phase reads belong to other
// colours and are not written during the phase.
template <typename T>
__device__ __forceinline__ T ro(const T* p) { return __ldg(p); }

// Colour phase: Gauss-Seidel up the interior rows k = 2..Nzg-1 of every
// interior column of this colour, then the free-surface row. The column's own
// unknowns stay in registers (NZ > 0: compile-time Nzg); rows 1 and Nzg of the
// column are constant during the sweep.
template <typename T, bool THREE, int NZ>
__global__ void __launch_bounds__(128) k_lo_colour(LevelDev<T> L, int colour) {
    constexpr int ZM = NZ > 0 ? NZ : kMaxNzg;
    const int Nzg = NZ > 0 ? NZ : L.Nzg;
    const int Nxg = L.Nxg, Nyg = L.Nyg;
    const int nxi = Nxg - 2, nyi = THREE ? Nyg - 2 : 1;
    const int64_t total = (int64_t)nxi * nyi;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % nxi) + 2, j = THREE ? (int)(q / nxi) + 2 : 1;
        const int col = (L.ncolor == 4) ? ((i & 1) + 2 * (j & 1)) : ((i + j) & 1);
        if (col != colour) continue;
        const int64_t c = (int64_t)(i - 1) + (int64_t)Nxg * (j - 1);
        T* xc = L.xv + c * Nzg;
        const T* bc = L.bv + c * Nzg;
        const T h = L.h[c], hx = L.hx[c], hxx = L.hxx[c];
        const T hy = THREE ? L.hy[c] : T(0), hyy = THREE ? L.hyy[c] : T(0);
        const bool cross = (hx != T(0)) || (hy != T(0));
        T xo[ZM];
#pragma unroll
        for (int k = 0; k < ZM; ++k) if (NZ > 0 || k < Nzg) xo[k] = xc[k];
        const T* xw = L.xv + (c - 1) * Nzg;           // west column
        const T* xe = L.xv + (c + 1) * Nzg;           // east column
        const T* xs = THREE ? L.xv + (c - Nxg) * Nzg : xc;  // south
        const T* xn = THREE ? L.xv + (c + Nxg) * Nzg : xc;  // north
        const T sxx0 = sx(L, 2, i, 0), sxx1 = sx(L, 2, i, 1), sxx2 = sx(L, 2, i, 2);
        const T syy0 = THREE ? sy(L, 2, j, 0) : T(0), syy1 = THREE ? sy(L, 2, j, 1) : T(0), syy2 = THREE ? sy(L, 2, j, 2) : T(0);
        const T sx1c = sx(L, 1, i, 1), sy1c = THREE ? sy(L, 1, j, 1) : T(0);
#pragma unroll
        for (int k = 2; k < ZM; ++k) {
            if (k >= Nzg) break;
            const T sg = L.zs[k - 1], om = T(1) - sg;
            const T s2 = (om * hx) / h, s4 = (om * hy) / h, s5 = T(1) / h;
            const T s3 = -T(2) * om * (hx * hx + hy * hy) / (h * h) + om * (hxx + hyy) / h;
            const T cz = s2 * s2 + s4 * s4 + s5 * s5;
            const T z0 = sz(L, 1, k, 0), z1 = sz(L, 1, k, 1), z2 = sz(L, 1, k, 2);
            const T zz0 = sz(L, 2, k, 0), zz1 = sz(L, 2, k, 1), zz2 = sz(L, 2, k, 2);
            // off-column part of the row (constant during this phase)
            T off = sxx0 * ro(xw + k - 1) + sxx2 * ro(xe + k - 1);
            if (THREE) off += syy0 * ro(xs + k - 1) + syy2 * ro(xn + k - 1);
            T diag = sxx1 + syy1 + s3 * z1 + cz * zz1;
            T lo = s3 * z0 + cz * zz0, up = s3 * z2 + cz * zz2;
            if (cross && s2 != T(0)) {
                const int jlo = THREE ? j - 1 : j, jhi = THREE ? j + 1 : j;
                T xz = 0;
                for (int jj = jlo; jj <= jhi; ++jj) {
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk) {
                        const int kz = k - 1 + kk;
                        int sh = 0;
                        if (kz == 1) { if (i - 1 == 1) sh = 1; if (i + 1 == Nxg) sh = -1; }
                        T dx = 0;
#pragma unroll
                        for (int m = 0; m < 3; ++m) {
                            const int ii = i - 1 + sh + m;
                            const T w = sx(L, 1, i - sh, m);
                            if (ii == i && jj == j && kz >= 2 && kz <= Nzg - 1) {
                                // own-column unknown: goes into the tridiagonal part
                                const T cf = T(2) * s2 * sz(L, 1, k, kk) * w;
                                if (kk == 0) lo += cf; else if (kk == 1) diag += cf; else up += cf;
                            } else {
                                const T* src = L.xv + ((int64_t)(ii - 1) + (int64_t)Nxg * (jj - 1)) * Nzg + (kz - 1);
                                dx += w * ((ii == i && jj == j) ? *src : ro(src));
                            }
                        }
                        xz += sz(L, 1, k, kk) * dx;
                    }
                }
                off += T(2) * s2 * xz;
            }
            if (THREE && cross && s4 != T(0)) {
                T yz = 0;
                for (int ii = i - 1; ii <= i + 1; ++ii) {
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk) {
                        const int kz = k - 1 + kk;
                        int sh = 0;
                        if (kz == 1) { if (j - 1 == 1) sh = 1; if (j + 1 == Nyg) sh = -1; }
                        T dy = 0;
#pragma unroll
                        for (int m = 0; m < 3; ++m) {
                            const int jj = j - 1 + sh + m;
                            const T w = sy(L, 1, j - sh, m);
                            if (ii == i && jj == j && kz >= 2 && kz <= Nzg - 1) {
                                const T cf = T(2) * s4 * sz(L, 1, k, kk) * w;
                                if (kk == 0) lo += cf; else if (kk == 1) diag += cf; else up += cf;
                            } else {
                                const T* src = L.xv + ((int64_t)(ii - 1) + (int64_t)Nxg * (jj - 1)) * Nzg + (kz - 1);
                                dy += w * ((ii == i && jj == j) ? *src : ro(src));
                            }
                        }
                        yz += sz(L, 1, k, kk) * dy;
                    }
                }
                off += T(2) * s4 * yz;
            }
            (void)sx1c; (void)sy1c;
            // row residual with the current iterate: lower neighbour already updated
            const T xm = xo[k - 2], x0 = xo[k - 1], xp = xo[k];
            const T a = lo * xm + diag * x0 + up * xp + off;
            xo[k - 1] = x0 + (bc[k - 1] - a) / diag;
        }
        xo[Nzg - 1] = bc[Nzg - 1];
#pragma unroll
        for (int k = 1; k < ZM; ++k) if (k < Nzg) xc[k] = xo[k];
    }
}

// MGRestriction3DExplicit.f90:19-128 as a gather per coarse point.
template <typename T>
__global__ void k_restrict(LevelDev<T> F, LevelDev<T> Cc, const T* __restrict__ rf, T* __restrict__ rc, T* __restrict__ xc) {
    const int64_t n = Cc.N;
    const int gy = (F.Nyg > 1) ? 1 : 0;
    const int Nzf = F.Nzg - 1, Nyf = F.Nyg - 2 * gy;
    const int xcz = Cc.xc, ycz = Cc.yc, zcz = Cc.zc;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const int kc = (int)(p % Cc.Nzg) + 1;
        const int64_t cc = p / Cc.Nzg;
        const int ic = (int)(cc % Cc.Nxg) + 1, jc = (int)(cc / Cc.Nxg) + 1;
        xc[p] = T(0);
        const bool ghost = kc == 1 || ic == 1 || ic == Cc.Nxg || (gy && (jc == 1 || jc == Cc.Nyg));
        if (ghost) { rc[p] = T(0); continue; }
        const int kf = 2 + (kc - 2) * (1 + zcz), ifn = 2 + (ic - 2) * (1 + xcz), jf = gy ? 2 + (jc - 2) * (1 + ycz) : 1;
        auto R = [&](int k, int i, int j) -> T { return rf[IX(F, k, i, j)]; };
        if (kf == F.Nzg) { rc[p] = R(kf, ifn, jf); continue; }
        // x-weighted value at (k, ifn, j) (raw on ghost rows and outside 2..Nzf)
        auto Sx = [&](int k, int j) -> T {
            if (!xcz || k < 2 || k > Nzf || (gy && (j < 2 || j > Nyf + 1))) return R(k, ifn, j);
            const double dW = F.x[ifn - 1] - F.x[ifn - 2], dE = F.x[ifn] - F.x[ifn - 1];
            const T dxc = T(1.0 / (dW + dE));
            return (T(0.5) * dxc) * (T(dW) * R(k, ifn - 1, j) + T(dW + dE) * R(k, ifn, j) + T(dE) * R(k, ifn + 1, j));
        };
        auto Sxy = [&](int k) -> T {
            if (!ycz || k < 2 || k > Nzf) return Sx(k, jf);
            const double dS = F.y[jf - 1] - F.y[jf - 2], dN = F.y[jf] - F.y[jf - 1];
            const T dyc = T(1.0 / (dS + dN));
            return (T(0.5) * dyc) * (T(dS) * Sx(k, jf - 1) + T(dN + dS) * Sx(k, jf) + T(dN) * Sx(k, jf + 1));
        };
        T v;
        if (zcz) {
            const double dU = F.z[kf] - F.z[kf - 1], dD = F.z[kf - 1] - F.z[kf - 2];
            const T dzc = T(1.0 / (dD + dU));
            v = (T(0.5) * dzc) * (T(dD) * Sxy(kf - 1) + T(dU) * Sxy(kf + 1)) + T(0.5) * Sxy(kf);
        } else {
            v = Sxy(kf);
        }
        rc[p] = v;
    }
}

// MGProlongation3DExplicit.f90:19-110 as a gather per fine point, added to xf.
template <typename T>
__global__ void k_prolong_add(LevelDev<T> F, LevelDev<T> Cc, const T* __restrict__ xc, T* __restrict__ xf) {
    const int64_t n = F.N;
    const int gy = (F.Nyg > 1) ? 1 : 0;
    const int XF = Cc.xc ? 2 : 1, YF = Cc.yc ? 2 : 1, ZF = Cc.zc ? 2 : 1;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const int kf = (int)(p % F.Nzg) + 1;
        const int64_t cf = p / F.Nzg;
        const int ifn = (int)(cf % F.Nxg) + 1, jf = (int)(cf / F.Nxg) + 1;
        if (kf == 1 || kf == F.Nzg || ifn == 1 || ifn == F.Nxg || (gy && (jf == 1 || jf == F.Nyg))) continue;
        // coarse value at coincident fine indices
        auto Cv = [&](int k, int i, int j) -> T {
            if (k == F.Nzg) return T(0);  // free-surface layer is not injected
            const int kc = 2 + (k - 2) / ZF, ic = 2 + (i - 2) / XF, jc = gy ? 2 + (j - 2) / YF : 1;
            return xc[IX(Cc, kc, ic, jc)];
        };
        auto Px = [&](int k, int j) -> T {
            if (k == F.Nzg) return T(0);
            if (XF == 1 || ((ifn - 2) % 2) == 0) return Cv(k, ifn, j);
            const double dW = F.x[ifn - 1] - F.x[ifn - 2], dE = F.x[ifn] - F.x[ifn - 1];
            const T dxf = T(1.0 / (dW + dE));
            return (T(dE) * Cv(k, ifn - 1, j) + T(dW) * Cv(k, ifn + 1, j)) * dxf;
        };
        auto Py = [&](int k) -> T {
            if (k == F.Nzg) return T(0);
            if (!gy || YF == 1 || ((jf - 2) % 2) == 0) return Px(k, jf);
            const double dS = F.y[jf - 1] - F.y[jf - 2], dN = F.y[jf] - F.y[jf - 1];
            const T dyf = T(1.0 / (dS + dN));
            return (T(dN) * Px(k, jf - 1) + T(dS) * Px(k, jf + 1)) * dyf;
        };
        T v;
        if (ZF == 1 || ((kf - 2) % 2) == 0) v = Py(kf);
        else {
            const double dD = F.z[kf - 1] - F.z[kf - 2], dU = F.z[kf] - F.z[kf - 1];
            const T dzf = T(1.0 / (dD + dU));
            v = (T(dU) * Py(kf - 1) + T(dD) * Py(kf + 1)) * dzf;
        }
        xf[p] += v;
    }
}

// Coarsest level: x = A^{-1} b with the explicit inverse (the reference factors
// this matrix with HSL MA41 once, LUfactor.f90:20-66, and solves with it).
template <typename T>
__global__ void k_coarse(int n, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        T acc = 0;
        for (int c = 0; c < n; ++c) acc += inv[(int64_t)r * n + c] * b[c];
        x[r] = acc;
    }
}

template <typename T>
__global__ void k_scale_copy(const double* __restrict__ src, double s, T* __restrict__ dst, int64_t n) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        dst[p] = T(s * src[p]);
}
template <typename T>
__global__ void k_scale_copy_dev(const double* __restrict__ src, const double* __restrict__ ds, T* __restrict__ dst, int64_t n) {
    const double s = ds ? *ds : 1.0;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        dst[p] = T(s * src[p]);
}
__global__ void k_convert(const float* __restrict__ src, double* __restrict__ dst, int64_t n) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        dst[p] = (double)src[p];
}
template <typename T>
__global__ void k_fill(T* __restrict__ dst, T v, int64_t n) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) dst[p] = v;
}

inline int nblk(int64_t n, int t = 256) {
    int64_t b = (n + t - 1) / t;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

template <typename T>
void launch_lo_matvec(const LevelDev<T>& L, const T* x, T* y, cudaStream_t st) {
    if (L.Nyg > 1) k_lo_matvec<T, true><<<nblk(L.N), 256, 0, st>>>(L, x, y);
    else k_lo_matvec<T, false><<<nblk(L.N), 256, 0, st>>>(L, x, y);
}

template <typename T>
static void special(const LevelDev<T>& L, cudaStream_t st) {
    const int64_t C = (int64_t)L.Nxg * L.Nyg;
    const int64_t G = (L.Nyg > 1) ? ((int64_t)2 * L.Nyg + 2 * (L.Nxg - 2)) * L.Nzg : 2 * L.Nzg;
    if (L.Nyg > 1) {
        k_lo_special_ghost<T, true><<<nblk(G, 128), 128, 0, st>>>(L);
        k_lo_special_bottom<T, true><<<nblk(C, 128), 128, 0, st>>>(L);
    } else {
        k_lo_special_ghost<T, false><<<nblk(G, 128), 128, 0, st>>>(L);
        k_lo_special_bottom<T, false><<<nblk(C, 128), 128, 0, st>>>(L);
    }
}
template <typename T, bool THREE, int NZ>
static void colour_launch(const LevelDev<T>& L, int c, cudaStream_t st) {
    const int64_t C = (int64_t)(L.Nxg - 2) * (THREE ? L.Nyg - 2 : 1);
    k_lo_colour<T, THREE, NZ><<<nblk(C, 128), 128, 0, st>>>(L, c);
}
template <typename T, bool THREE>
static void colour_dispatch(const LevelDev<T>& L, int c, cudaStream_t st) {
    switch (L.Nzg) {
        case 4: colour_launch<T, THREE, 4>(L, c, st); break;
        case 6: colour_launch<T, THREE, 6>(L, c, st); break;
        case 8: colour_launch<T, THREE, 8>(L, c, st); break;
        case 10: colour_launch<T, THREE, 10>(L, c, st); break;
        case 14: colour_launch<T, THREE, 14>(L, c, st); break;
        case 18: colour_launch<T, THREE, 18>(L, c, st); break;
        default: colour_launch<T, THREE, 0>(L, c, st); break;
    }
}
template <typename T>
static void colours(const LevelDev<T>& L, cudaStream_t st) {
    for (int c = 0; c < L.ncolor; ++c) {
        if (L.Nyg > 1) colour_dispatch<T, true>(L, c, st);
        else colour_dispatch<T, false>(L, c, st);
    }
}

template <typename T>
void launch_lo_smooth(const LevelDev<T>& L, int nu, cudaStream_t st) {
    special(L, st);
    for (int s = 0; s < nu; ++s) { colours(L, st); special(L, st); }
}

template <typename T>
void launch_restrict(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* rf, T* rc, cudaStream_t st) {
    k_restrict<T><<<nblk(Cc.N), 256, 0, st>>>(F, Cc, rf, rc, Cc.xv);
}
template <typename T>
void launch_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* xc, T* xf, cudaStream_t st) {
    k_prolong_add<T><<<nblk(F.N), 256, 0, st>>>(F, Cc, xc, xf);
}
template <typename T>
void launch_coarse_solve(const LevelDev<T>& Lc, const T* inv, cudaStream_t st) {
    int n = (int)Lc.N;
    k_coarse<T><<<(n + 127) / 128, 128, 0, st>>>(n, inv, Lc.bv, Lc.xv);
}
template <typename T>
void launch_scale_copy(const double* src, double s, T* dst, int64_t n, cudaStream_t st) {
    k_scale_copy<T><<<nblk(n), 256, 0, st>>>(src, s, dst, n);
}
template <typename T>
void launch_fill(T* dst, T v, int64_t n, cudaStream_t st) {
    k_fill<T><<<nblk(n), 256, 0, st>>>(dst, v, n);
}
template <typename T>
void launch_scale_copy_dev(const double* src, const double* ds, T* dst, int64_t n, cudaStream_t st) {
    k_scale_copy_dev<T><<<nblk(n), 256, 0, st>>>(src, ds, dst, n);
}
void launch_convert(const float* src, double* dst, int64_t n, cudaStream_t st) {
    k_convert<<<nblk(n), 256, 0, st>>>(src, dst, n);
}

// MultiGridSolver.f90:5-192 (V cycle, gam = 1), levels lev[0] coarsest.
template <typename T>
static void vcycle(LevelDev<T>* lev, int l, const T* inv, int nu1, int nu2, cudaStream_t st) {
    if (l == 0) { launch_coarse_solve(lev[0], inv, st); return; }
    const LevelDev<T>& F = lev[l];
    LevelDev<T>& Cc = lev[l - 1];
    launch_lo_smooth(F, nu1, st);
    if (F.Nyg > 1) k_lo_residual<T, true><<<nblk(F.N), 256, 0, st>>>(F);
    else k_lo_residual<T, false><<<nblk(F.N), 256, 0, st>>>(F);
    launch_restrict(F, Cc, (const T*)F.rv, Cc.bv, st);   // also zeroes Cc.xv
    vcycle(lev, l - 1, inv, nu1, nu2, st);
    launch_prolong_add(F, Cc, (const T*)Cc.xv, F.xv, st);
    launch_lo_smooth(F, nu2, st);
}

// MultiGridSolveLinearSystem.f90:26-91: u = 0, then maxit cycles.
template <typename T>
void launch_mg_vcycle(LevelDev<T>* lev, int nlev, const T* coarse_inv, int nu1, int nu2, int maxit, cudaStream_t st) {
    LevelDev<T>& F = lev[nlev - 1];
    launch_fill<T>(F.xv, T(0), F.N, st);
    for (int it = 1; it <= maxit; ++it) {
        if (nlev == 1 && it > 1) break;
        vcycle(lev, nlev - 1, coarse_inv, nu1, nu2, st);
    }
}

#define OW3D_INST(T)                                                                                         \
    template void launch_mg_vcycle<T>(LevelDev<T>*, int, const T*, int, int, int, cudaStream_t);           \
    template void launch_lo_matvec<T>(const LevelDev<T>&, const T*, T*, cudaStream_t);                      \
    template void launch_lo_smooth<T>(const LevelDev<T>&, int, cudaStream_t);                               \
    template void launch_restrict<T>(const LevelDev<T>&, const LevelDev<T>&, const T*, T*, cudaStream_t);   \
    template void launch_prolong_add<T>(const LevelDev<T>&, const LevelDev<T>&, const T*, T*, cudaStream_t); \
    template void launch_coarse_solve<T>(const LevelDev<T>&, const T*, cudaStream_t);                       \
    template void launch_scale_copy<T>(const double*, double, T*, int64_t, cudaStream_t);                   \
    template void launch_fill<T>(T*, T, int64_t, cudaStream_t);                                             \
    template void launch_scale_copy_dev<T>(const double*, const double*, T*, int64_t, cudaStream_t);
OW3D_INST(double)
OW3D_INST(float)
#undef OW3D_INST

}  // namespace ow3d
