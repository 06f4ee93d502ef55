// Device-side pieces of the multigrid preconditioner shared by the per-phase
// kernels and the fused coarse-level kernel (mg.cu): row evaluation of the
// low-order operator, the Gauss-Seidel colour pass and the grid transfers,
// each as a function of one work item.
#pragma once
#include "ow3d_internal.h"

namespace ow3d {
namespace mgdev {

// Linear point index p (k fastest) -> 1-based (k, i, j) and column c.
// Every level has fewer than 2^31 points (the set-up rejects larger grids),
// so the decomposition runs in 32 bits.
template <typename T>
__device__ __forceinline__ void decomp(const LevelDev<T>& L, int64_t p, int& k, int64_t& c, int& i, int& j) {
    const uint32_t pp = (uint32_t)p;
    const uint32_t cc = div32(pp, L.mz32, L.sz32);
    k = (int)(pp - cc * (uint32_t)L.Nzg) + 1;
    const uint32_t jj = div32(cc, L.mx32, L.sx32);
    i = (int)(cc - jj * (uint32_t)L.Nxg) + 1;
    j = (int)jj + 1;
    c = (int64_t)cc;
}

// Column coefficients (1/h, h_x/h, h_y/h, c3), one 32- or 16-byte read.
__device__ __forceinline__ void load_cf(const double* cf, int64_t c, double& ih, double& a, double& b, double& c3) {
    const double2 u = __ldg(reinterpret_cast<const double2*>(cf) + 2 * c);
    const double2 v = __ldg(reinterpret_cast<const double2*>(cf) + 2 * c + 1);
    ih = u.x; a = u.y; b = v.x; c3 = v.y;
}
__device__ __forceinline__ void load_cf(const float* cf, int64_t c, float& ih, float& a, float& b, float& c3) {
    const float4 u = __ldg(reinterpret_cast<const float4*>(cf) + c);
    ih = u.x; a = u.y; b = u.z; c3 = u.w;
}

// Bottom-row coefficients of a column (see LevelDev::bt).
__device__ __forceinline__ void load_bt(const double* bt, int64_t c, double* o) {
    const double2* p = reinterpret_cast<const double2*>(bt) + 4 * c;
    const double2 a = __ldg(p), b = __ldg(p + 1), d = __ldg(p + 2), e = __ldg(p + 3);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = d.x; o[5] = d.y; o[6] = e.x;
}
__device__ __forceinline__ void load_bt(const float* bt, int64_t c, float* o) {
    const float4* p = reinterpret_cast<const float4*>(bt) + 2 * c;
    const float4 a = __ldg(p), b = __ldg(p + 1);
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = b.x; o[5] = b.y; o[6] = b.z;
}

// All eight bottom-row coefficients of a column.
__device__ __forceinline__ void load_bt8(const double* bt, int64_t c, double* o) {
    const double2* p = reinterpret_cast<const double2*>(bt) + 4 * c;
    const double2 a = __ldg(p), b = __ldg(p + 1), d = __ldg(p + 2), e = __ldg(p + 3);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = d.x; o[5] = d.y; o[6] = e.x; o[7] = e.y;
}
__device__ __forceinline__ void load_bt8(const float* bt, int64_t c, float* o) {
    const float4* p = reinterpret_cast<const float4*>(bt) + 2 * c;
    const float4 a = __ldg(p), b = __ldg(p + 1);
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}

template <typename T>
__device__ __forceinline__ int64_t IX(const LevelDev<T>& L, int k, int i, int j) {
    return (int64_t)(k - 1) + (int64_t)L.Nzg * ((int64_t)(i - 1) + (int64_t)L.Nxg * (j - 1));
}
// stencil tables are read-only for the whole solve
template <typename T>
__device__ __forceinline__ T sx(const LevelDev<T>& L, int o, int i, int m) { return __ldg(L.SX + ((o - 1) * L.Nxg + (i - 1)) * 3 + m); }
template <typename T>
__device__ __forceinline__ T sy(const LevelDev<T>& L, int o, int j, int m) { return __ldg(L.SY + ((o - 1) * L.Nyg + (j - 1)) * 3 + m); }
template <typename T>
__device__ __forceinline__ T sz(const LevelDev<T>& L, int o, int k, int m) { return __ldg(L.SZ + ((o - 1) * L.Nzg + (k - 1)) * 3 + m); }

// x-neighbour column index: cyclic on a periodic level.
template <typename T>
__device__ __forceinline__ int xcol(const LevelDev<T>& L, int i) { return L.per ? wrap_x(i, L.Nxg) : i; }
// Column offsets (in elements) of the left and right x-neighbours of column
// i, for addressing relative to the column: +-Nzg, or across the period on
// a periodic level.
template <typename T>
__device__ __forceinline__ int xoff_l(const LevelDev<T>& L, int i) {
    return (L.per && i == 2) ? (L.Nxg - 4) * L.Nzg : -L.Nzg;
}
template <typename T>
__device__ __forceinline__ int xoff_r(const LevelDev<T>& L, int i) {
    return (L.per && i == L.Nxg - 2) ? -(L.Nxg - 4) * L.Nzg : L.Nzg;
}

// Interior row (2 <= k <= Nzg-1, interior column). Returns A x at the row and
// the diagonal coefficient.
template <typename T, bool THREE, bool CROSS = true>
__device__ T lo_interior(const LevelDev<T>& L, const T* x, int k, int i, int j, T& diag) {
    const int64_t c = (int64_t)(i - 1) + (int64_t)L.Nxg * (j - 1);
    T s5, ca, cb, c3;
    load_cf(L.cf, c, s5, ca, cb, c3);
    const T sg = __ldg(L.zs + k - 1), om = T(1) - sg;
    // DetermineTransformationConstantsArray with eta = 0
    const T s2 = om * ca;
    const T s4 = THREE ? om * cb : T(0);
    const T s3 = om * c3;
    const T cz = s2 * s2 + s4 * s4 + s5 * s5;
    T acc = 0;
    // d2/dx2, d2/dy2 (centred 3-point, PrepareFullOperatorStencils.f90:213-231)
#pragma unroll
    for (int m = 0; m < 3; ++m) acc += sx(L, 2, i, m) * x[IX(L, k, xcol(L, i - 1 + m), j)];
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
    if (CROSS && s2 != T(0)) {
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
    if (THREE && CROSS && s4 != T(0)) {
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
    const T hx = L.hx[c];
    const T hy = THREE ? L.hy[c] : T(0);
    const T om = T(1) - L.zs[1];
    T s5, ca, cb, c3;
    load_cf(L.cf, c, s5, ca, cb, c3);
    const T s2 = om * ca, s4 = THREE ? om * cb : T(0);
    const T f = THREE ? (s5 + hx * s2 + hy * s4) : (s5 + hx * s2);
    T dz = 0;
#pragma unroll
    for (int m = 0; m < 3; ++m) dz += sz(L, 1, 2, m) * x[IX(L, 1 + m, i, j)];
    T dx = 0;
#pragma unroll
    for (int m = 0; m < 3; ++m) dx += sx(L, 1, i, m) * x[IX(L, 2, xcol(L, i - 1 + m), j)];
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
    // periodic x: the ghost and repeated columns are identity rows
    const bool pid = L.per && (gxx || i == L.Nxg - 1);
    if ((gxx && gyy) || k == 1 || pid) { diag = T(1); return x[IX(L, k, i, j)]; }
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
    return i == 1 || i == L.Nxg || (L.per && i == L.Nxg - 1) || (THREE && (j == 1 || j == L.Nyg));
}

template <typename T, bool THREE, bool CROSS = true>
__device__ T lo_row(const LevelDev<T>& L, const T* x, int k, int i, int j, T& diag) {
    if (is_ghost_col<T, THREE>(L, i, j)) return lo_ghost<T, THREE>(L, x, k, i, j, diag);
    if (k == L.Nzg) { diag = T(1); return x[IX(L, k, i, j)]; }
    if (k == 1) return lo_bottom<T, THREE>(L, x, i, j, diag);
    return lo_interior<T, THREE, CROSS>(L, x, k, i, j, diag);
}


// Iterates, right-hand sides and residuals are written by earlier phases of
// the same fused coarse-level kernel, so they are read with ordinary
// (coherent) loads, never through the read-only data path: the item functions
// below take them through pointers without __restrict__ (the per-level
// kernels, where they are read-only, put the qualifier on their own
// parameters). Only the stencil and coefficient tables, constant for the
// whole solve, use __ldg.
template <typename T>
__device__ __forceinline__ T ro(const T* p) { return *p; }

template <typename T, bool THREE, bool CROSS>
__device__ __forceinline__ void residual_item(const LevelDev<T>& L, int64_t p) {
    int k, i, j;
    int64_t c;
    decomp(L, p, k, c, i, j);
    T dg;
    L.rv[p] = L.bv[p] - lo_row<T, THREE, CROSS>(L, L.xv, k, i, j, dg);
}

// Residual r = b - A x at point p (k fastest, so a warp covers about two
// columns). On levels without mixed-derivative terms the rows of an interior
// column -- interior rows, the bottom row (BuildLinearSystemMatrix.f90:50-70)
// and the free-surface row -- are all a 7-term combination of the same seven
// values: the column at levels kk-1, kk, kk+1 and the four neighbour columns
// at level kk (kk = 2 for the bottom row, the row itself otherwise), so the
// lanes of a warp share one branch-free form and only select their
// coefficients. Ghost columns and levels with mixed-derivative terms take
// lo_row.
template <typename T, bool THREE, bool CROSS>
__device__ __forceinline__ void residual_point(const LevelDev<T>& L, int64_t p) {
    int k, i, j;
    int64_t c;
    decomp(L, p, k, c, i, j);
    const int Nzg = L.Nzg, Nxg = L.Nxg;
    T v;
    if (CROSS || is_ghost_col<T, THREE>(L, i, j)) {
        T dg;
        v = lo_row<T, THREE, CROSS>(L, L.xv, k, i, j, dg);
    } else {
        const bool bot = (k == 1), top = (k == Nzg);
        const int kk = bot ? 2 : (top ? Nzg - 1 : k);
        const T* xp = L.xv + c * Nzg + (kk - 1);
        const int oy = Nzg * Nxg;
        // interior-row coefficients of row kk
        T ih, ca, cb, c3;
        load_cf(L.cf, c, ih, ca, cb, c3);
        const T* sxp = L.SX + (Nxg + i - 1) * 3;       // order 2, position i
        const T* zp1 = L.SZ + (kk - 1) * 3;            // order 1, row kk
        const T* zp2 = L.SZ + (Nzg + kk - 1) * 3;      // order 2, row kk
        const T om = T(1) - __ldg(L.zs + kk - 1);
        const T s2 = om * ca, s4 = THREE ? om * cb : T(0);
        const T s3 = om * c3;
        const T cz = s2 * s2 + s4 * s4 + ih * ih;
        const T wx0 = __ldg(sxp), wx1 = __ldg(sxp + 1), wx2 = __ldg(sxp + 2);
        T wy0 = 0, wy1 = 0, wy2 = 0;
        if (THREE) {
            const T* syp = L.SY + (L.Nyg + j - 1) * 3;
            wy0 = __ldg(syp); wy1 = __ldg(syp + 1); wy2 = __ldg(syp + 2);
        }
        T cm = s3 * __ldg(zp1) + cz * __ldg(zp2);
        T c0 = wx1 + wy1 + s3 * __ldg(zp1 + 1) + cz * __ldg(zp2 + 1);
        T cq = s3 * __ldg(zp1 + 2) + cz * __ldg(zp2 + 2);
        T cl = wx0, cr = wx2, cd = wy0, cu = wy2;
        T bt[8];
        load_bt8(L.bt, c, bt);
        if (bot) { cm = bt[7]; c0 = bt[0]; cq = bt[1]; cl = bt[2]; cr = bt[3]; cd = bt[4]; cu = bt[5]; }
        if (top) { cm = 0; c0 = 0; cq = 1; cl = 0; cr = 0; cd = 0; cu = 0; }
        v = cm * xp[-1] + c0 * xp[0] + cq * xp[1] + cl * xp[xoff_l(L, i)] + cr * xp[xoff_r(L, i)];
        if (THREE) v += cd * xp[-oy] + cu * xp[oy];
    }
    L.rv[p] = L.bv[p] - v;
}

// Gauss-Seidel value of the bottom row (k = 1) of interior column c = (i, j)
// (BuildLinearSystemMatrix.f90:50-70), given rows 2 and 3 of the column; the
// neighbours' row-2 values are read from X.
template <typename T, bool THREE>
__device__ __forceinline__ T bottom_value(const LevelDev<T>& L, const T* X, const T* B, int64_t c, int i, int j, T x2,
                                          T x3) {
    const int Nzg = L.Nzg, Nxg = L.Nxg;
    const T hx = L.hx[c];
    const T hy = THREE ? L.hy[c] : T(0);
    T ih, ca, cb, c3;
    load_cf(L.cf, c, ih, ca, cb, c3);
    const T omb = T(1) - __ldg(L.zs + 1);
    const T s2 = omb * ca, s4 = THREE ? omb * cb : T(0);
    const T f = THREE ? (ih + hx * s2 + hy * s4) : (ih + hx * s2);
    const T dz = sz(L, 1, 2, 1) * x2 + sz(L, 1, 2, 2) * x3;
    T dx = sx(L, 1, i, 0) * X[(c - 1) * Nzg + 1] + sx(L, 1, i, 1) * x2;
    dx += sx(L, 1, i, 2) * X[(c + 1) * Nzg + 1];
    T off = f * dz + hx * dx;
    if (THREE) {
        T dy = sy(L, 1, j, 0) * X[(c - Nxg) * Nzg + 1] + sy(L, 1, j, 1) * x2;
        dy += sy(L, 1, j, 2) * X[(c + Nxg) * Nzg + 1];
        off += hy * dy;
    }
    return (B[c * Nzg] - off) / (f * sz(L, 1, 2, 0));
}

// Level-1 pass item q (levels with mixed-derivative terms relax their level-1
// rows in a pass of their own): the bottom rows of the interior columns, then
// the identity level-1 rows of the lateral ghost columns (corners excluded).
template <typename T, bool THREE>
__device__ __forceinline__ int64_t bottom_count(const LevelDev<T>& L) {
    const int64_t nyi = THREE ? L.Nyg - 2 : 1;
    return (int64_t)(L.Nxg - 2) * nyi + 2 * nyi + (THREE ? 2 * (int64_t)(L.Nxg - 2) : 0);
}
template <typename T, bool THREE>
__device__ __forceinline__ void bottom_item(const LevelDev<T>& L, int64_t q) {
    const int nxi = L.Nxg - 2, nyi = THREE ? L.Nyg - 2 : 1;
    const int64_t nint = (int64_t)nxi * nyi;
    T* X = L.xv;
    if (q < nint) {
        const int64_t tj = q / nxi;
        const int i = 2 + (int)(q - tj * nxi), j = THREE ? 2 + (int)tj : 1;
        const int64_t c = (int64_t)(i - 1) + (int64_t)L.Nxg * (j - 1);
        X[c * L.Nzg] = bottom_value<T, THREE>(L, X, L.bv, c, i, j, X[c * L.Nzg + 1], X[c * L.Nzg + 2]);
        return;
    }
    q -= nint;
    int i, j;
    if (q < 2 * nyi) { j = THREE ? 2 + (int)(q >> 1) : 1; i = (q & 1) ? L.Nxg : 1; }
    else { q -= 2 * nyi; i = 2 + (int)(q >> 1); j = (q & 1) ? L.Nyg : 1; }
    const int64_t c = (int64_t)(i - 1) + (int64_t)L.Nxg * (j - 1);
    X[c * L.Nzg] = L.bv[c * L.Nzg];
}

// Colour pass, warp-cooperative form. A segment of S lanes (S a power of two
// >= Nzg-2) owns one interior column (i, j) of the colour; lane r holds row
// k = r+2. The column's task, in the order the oracle's device mode uses:
//   1. identity corner columns diagonal to it (3-D): x = b,
//   2. the lateral ghost columns it reads (i = 2 / Nxg-1, j = 2 / Nyg-1),
//      relaxed from the current values,
//   3. its bottom row (k = 1, kinematic bottom condition), lane 0,
//   4. rows k = 2..Nzg-1 bottom to top: each lane forms its row's
//      Gauss-Seidel update as an affine map of the new value below it,
//      x_k = q_k - g_k x_{k-1}, and the chain is evaluated with a shuffle scan
//      of the composed maps; the free-surface row (identity) last,
//   5. its bottom row again, from the new column,
//   6. the lateral ghost columns whose Neumann stencil contains the column
//      (i = 2 or 3 / Nxg-1 or Nxg-2, likewise in j), from the new values.
// A ghost column so ends every smoothing step consistent with both interior
// columns of its stencil. Columns of one colour never read what another
// column of that colour writes, so all tasks of a pass run concurrently.
// Loads are coalesced along the column. CROSS: the level has mixed-derivative
// terms (sloping bottom). All 32 lanes of the warp call this with the same
// `base` (the first column index of the warp).
template <typename T, bool THREE>
__device__ __forceinline__ int64_t colour_count(const LevelDev<T>& L) {
    const int nxi = L.Nxg - 2 - L.per, nyi = THREE ? L.Nyg - 2 : 1;   // periodic: the distinct columns
    const int ni = (nxi + 1) / 2, nj = (L.ncolor == 4) ? (nyi + 1) / 2 : nyi;
    return (int64_t)ni * nj;
}

// Per-lane constants of row k = r+2 (the same for every column of a level).
template <typename T>
struct RowConst { T om, z0, z1, z2, zz0, zz1, zz2; };

template <typename T, int S>
__device__ __forceinline__ RowConst<T> row_const(const LevelDev<T>& L) {
    const int r = (threadIdx.x & 31) & (S - 1);
    const int k = min(r + 2, L.Nzg - 1);
    RowConst<T> c;
    c.om = T(1) - __ldg(L.zs + k - 1);
    c.z0 = sz(L, 1, k, 0); c.z1 = sz(L, 1, k, 1); c.z2 = sz(L, 1, k, 2);
    c.zz0 = sz(L, 2, k, 0); c.zz1 = sz(L, 2, k, 1); c.zz2 = sz(L, 2, k, 2);
    return c;
}

template <typename T, bool THREE, int S, bool CROSS>
__device__ void colour_warp(const LevelDev<T>& L, int colour, int base, const RowConst<T>& rk) {
    const int Nxg = L.Nxg, Nyg = L.Nyg, Nzg = L.Nzg, R = Nzg - 2;
    const int lane = threadIdx.x & 31, r = lane & (S - 1);
    const int nxi = Nxg - 2 - L.per, nyi = THREE ? Nyg - 2 : 1;
    // columns of this colour: every other i (and every other j with 4 colours)
    const bool four = (L.ncolor == 4);
    const int ni = (nxi + 1) / 2;
    const int nj = four ? (nyi + 1) / 2 : nyi;
    const int total = ni * nj;                // columns of one colour (< 2^31)
    const unsigned segmask = 0xffffffffu;   // the whole warp runs the scan together
    T* const X = L.xv;
    const T* const B = L.bv;

    const int q = base + (lane / S);
    bool act = q < total;
    int i = 2, j = THREE ? 2 : 1;
    if (act) {
        const int tj = q / ni, ti = q - tj * ni;   // 32-bit division
        if (four) {
            j = THREE ? 2 + 2 * tj + (colour >> 1) : 1;
            i = 2 + 2 * ti + (colour & 1);
        } else {
            j = THREE ? 2 + tj : 1;
            i = 2 + 2 * ti + ((colour + j) & 1);    // (i + j) & 1 == colour
        }
        act = (i <= Nxg - 1 - L.per) && (!THREE || j <= Nyg - 1);
    }
    const bool rowact = act && (r < R);
    const int k = r + 2;
    // the column's base; neighbours and rows are 32-bit offsets from it
    // (every level has fewer than 2^31 points)
    const int c = (i - 1) + Nxg * (j - 1);
    T* const xc = X + (int64_t)c * Nzg;
    const T* const bc = B + (int64_t)c * Nzg;
    const int ox = Nzg, oy = Nzg * Nxg;
    // the column borders a ghost column (ghost relaxation before or after it,
    // and the corner columns)
    const bool edge = act && (i <= 3 || i >= Nxg - 2 || (THREE && (j <= 3 || j >= Nyg - 2)));

    auto colidx = [&](int ii, int jj) -> int64_t { return (int64_t)(ii - 1) + (int64_t)Nxg * (jj - 1); };
    // Relax ghost column cg: Neumann rows k = 2..Nzg with the 3-point stencil
    // wa x(ca) + wb x(cb) + wg x(cg) = b, identity row k = 1. With post set,
    // the value of this column (ca if own == 1, cb if own == 2) is the lane's
    // new one (xnew for rows 2..Nzg-1, xfsn for the free-surface row).
    auto relax_ghost = [&](int64_t cg, int64_t ca, T wa, int64_t cb, T wb, T wg, int own, bool post, T xnew, T xfsn) {
        auto row = [&](int kk, T xo) {
            const T va = (post && own == 1) ? xo : X[ca * Nzg + kk - 1];
            const T vb = (post && own == 2) ? xo : X[cb * Nzg + kk - 1];
            X[cg * Nzg + kk - 1] = (B[cg * Nzg + kk - 1] - (wa * va + wb * vb)) / wg;
        };
        if (r < R) row(k, xnew);
        if (r == R - 1) row(Nzg, xfsn);
        if (!CROSS && r == 0) X[cg * Nzg] = B[cg * Nzg];   // identity level-1 row
    };
    // the four ghost columns that can touch column (i, j); `pre` selects the
    // ones this column reads, otherwise the ones whose stencil contains it
    auto ghosts = [&](bool post, T xnew, T xfsn) {
        // periodic x has no x ghost columns to relax
        if (!L.per && (i == 2 || (post && i == 3)))
            relax_ghost(colidx(1, j), colidx(2, j), sx(L, 1, 2, 1), colidx(3, j), sx(L, 1, 2, 2), sx(L, 1, 2, 0),
                        i == 2 ? 1 : 2, post, xnew, xfsn);
        if (!L.per && (i == Nxg - 1 || (post && i == Nxg - 2)))
            relax_ghost(colidx(Nxg, j), colidx(Nxg - 2, j), sx(L, 1, Nxg - 1, 0), colidx(Nxg - 1, j),
                        sx(L, 1, Nxg - 1, 1), sx(L, 1, Nxg - 1, 2), i == Nxg - 1 ? 2 : 1, post, xnew, xfsn);
        if (THREE) {
            if (j == 2 || (post && j == 3))
                relax_ghost(colidx(i, 1), colidx(i, 2), sy(L, 1, 2, 1), colidx(i, 3), sy(L, 1, 2, 2), sy(L, 1, 2, 0),
                            j == 2 ? 1 : 2, post, xnew, xfsn);
            if (j == Nyg - 1 || (post && j == Nyg - 2))
                relax_ghost(colidx(i, Nyg), colidx(i, Nyg - 2), sy(L, 1, Nyg - 1, 0), colidx(i, Nyg - 1),
                            sy(L, 1, Nyg - 1, 1), sy(L, 1, Nyg - 1, 2), j == Nyg - 1 ? 2 : 1, post, xnew, xfsn);
        }
    };
    if (edge) {
        // 1. identity corner column diagonal to (i, j) (3-D; at most one)
        if (THREE && !L.per && (i == 2 || i == Nxg - 1) && (j == 2 || j == Nyg - 1)) {
            const int64_t cc = colidx(i == 2 ? 1 : Nxg, j == 2 ? 1 : Nyg);
            for (int kk = r; kk < Nzg; kk += S) X[cc * Nzg + kk] = B[cc * Nzg + kk];
        }
        // 2. ghost columns this column reads, from the current values
        ghosts(false, T(0), T(0));
    }
    __syncwarp();

    // 3.-5. the column. Every lane of an active segment evaluates its row
    // (lanes past the last interior row evaluate row Nzg-1 and discard it)
    // and the pieces of the bottom row, loads first and without lane-dependent
    // branches, so that one round trip to memory serves the whole task.
    const int kr = (r < R) ? k : R + 1;
    const int o = kr - 1;
    T qv = 0, gv = 0, x1 = 0;
    T bb1 = 0, bl = 0, br = 0, bd = 0, bu = 0;
    T t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0;   // bottom-row coefficients
    if (act) {
        T ih, ca, cb, c3;
        load_cf(L.cf, (int64_t)c, ih, ca, cb, c3);
        const int oxl = xoff_l(L, i), oxr = xoff_r(L, i);
        const T xl = xc[o + oxl], xr = xc[o + oxr];
        const T xd = THREE ? xc[o - oy] : T(0), xu = THREE ? xc[o + oy] : T(0);
        const T x0 = xc[o];
        const T xp = xc[o + 1];                // old value of the row above (row Nzg: free surface)
        const T bk = bc[o];
        T x2o = 0, x3o = 0;
        if (!CROSS) {
            T btv[7];
            load_bt(L.bt, (int64_t)c, btv);
            t0 = btv[0]; t1 = btv[1]; t2 = btv[2]; t3 = btv[3]; t4 = btv[4]; t5 = btv[5]; t6 = btv[6];
            x2o = xc[1]; x3o = xc[2]; bb1 = bc[0];
            bl = xc[1 + oxl]; br = xc[1 + oxr];
            if (THREE) { bd = xc[1 - oy]; bu = xc[1 + oy]; }
        } else {
            x1 = xc[0];                        // bottom rows are fixed during this pass
        }
        const T* sxp = L.SX + (Nxg + i - 1) * 3;          // order 2, position i
        const T om = rk.om;
        const T s2 = om * ca, s4 = THREE ? om * cb : T(0);
        const T s3 = om * c3;
        const T cz = s2 * s2 + s4 * s4 + ih * ih;
        T off = __ldg(sxp) * xl + __ldg(sxp + 2) * xr;
        T diag = __ldg(sxp + 1) + s3 * rk.z1 + cz * rk.zz1;
        if (THREE) {
            const T* syp = L.SY + (Nyg + j - 1) * 3;
            off += __ldg(syp) * xd + __ldg(syp + 2) * xu;
            diag += __ldg(syp + 1);
        }
        T lo = s3 * rk.z0 + cz * rk.zz0, up = s3 * rk.z2 + cz * rk.zz2;
        if (CROSS && s2 != T(0)) {
            const int jlo = THREE ? j - 1 : j, jhi = THREE ? j + 1 : j;
            T xz = 0;
            for (int jj = jlo; jj <= jhi; ++jj) {
#pragma unroll
                for (int kk = 0; kk < 3; ++kk) {
                    const int kz = kr - 1 + kk;
                    int sh = 0;
                    if (kz == 1) { if (i - 1 == 1) sh = 1; if (i + 1 == Nxg) sh = -1; }
                    T dx = 0;
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        const int ii = i - 1 + sh + m;
                        const T w = sx(L, 1, i - sh, m);
                        if (ii == i && jj == j && kz <= Nzg - 1) {
                            // own column: the term joins the scan (below / diagonal / above)
                            const T cf2 = T(2) * s2 * sz(L, 1, kr, kk) * w;
                            if (kk == 0) lo += cf2; else if (kk == 1) diag += cf2; else up += cf2;
                        } else {
                            dx += w * xc[(ii - i) * ox + (jj - j) * oy + (kz - 1)];
                        }
                    }
                    xz += sz(L, 1, kr, kk) * dx;
                }
            }
            off += T(2) * s2 * xz;
        }
        if (THREE && CROSS && s4 != T(0)) {
            T yz = 0;
            for (int ii = i - 1; ii <= i + 1; ++ii) {
#pragma unroll
                for (int kk = 0; kk < 3; ++kk) {
                    const int kz = kr - 1 + kk;
                    int sh = 0;
                    if (kz == 1) { if (j - 1 == 1) sh = 1; if (j + 1 == Nyg) sh = -1; }
                    T dy = 0;
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        const int jj = j - 1 + sh + m;
                        const T w = sy(L, 1, j - sh, m);
                        if (ii == i && jj == j && kz <= Nzg - 1) {
                            const T cf2 = T(2) * s4 * sz(L, 1, kr, kk) * w;
                            if (kk == 0) lo += cf2; else if (kk == 1) diag += cf2; else up += cf2;
                        } else {
                            dy += w * xc[(ii - i) * ox + (jj - j) * oy + (kz - 1)];
                        }
                    }
                    yz += sz(L, 1, kr, kk) * dy;
                }
            }
            off += T(2) * s4 * yz;
        }
        // row update x0 + (b - (lo x_{k-1} + diag x0 + up xp + off)) / diag
        const T id = T(1) / diag;
        if (r < R) {
            qv = x0 + (bk - diag * x0 - up * xp - off) * id;
            gv = lo * id;
        }
        // bottom row from the current column
        if (!CROSS) {
            T boff = t0 * x2o + t1 * x3o + t2 * bl + t3 * br;
            if (THREE) boff += t4 * bd + t5 * bu;
            x1 = (bb1 - boff) * t6;
        }
    }
    // inclusive scan of the affine maps x -> a x + b, a = -g, b = q (in row order)
    T a = -gv, bb = qv;
#pragma unroll
    for (int d = 1; d < S; d <<= 1) {
        const T ap = __shfl_up_sync(segmask, a, d, S);
        const T bp = __shfl_up_sync(segmask, bb, d, S);
        if (r >= d) { bb = a * bp + bb; a = a * ap; }
    }
    const T xn = a * x1 + bb;                  // new value of row k
    const T x2n = __shfl_sync(segmask, xn, 0, S);
    const T x3n = __shfl_sync(segmask, xn, 1, S);
    if (rowact) xc[k - 1] = xn;
    const T xfs = act ? bc[Nzg - 1] : T(0);
    if (act && r == R - 1) xc[Nzg - 1] = xfs;  // free-surface row
    // 5. bottom row again, from the new column (the neighbours are unchanged)
    if (!CROSS && act && r == 0) {
        T boff = t0 * x2n + t1 * x3n + t2 * bl + t3 * br;
        if (THREE) boff += t4 * bd + t5 * bu;
        xc[0] = (bb1 - boff) * t6;
    }
    // 6. ghost columns whose stencil contains this column, from the new values
    if (edge) ghosts(true, xn, xfs);
}

// Row constants of row k (clamped to the interior rows 2..Nzg-1).
template <typename T>
__device__ __forceinline__ RowConst<T> row_const_k(const LevelDev<T>& L, int k) {
    k = min(max(k, 2), L.Nzg - 1);
    RowConst<T> c;
    c.om = T(1) - __ldg(L.zs + k - 1);
    c.z0 = sz(L, 1, k, 0); c.z1 = sz(L, 1, k, 1); c.z2 = sz(L, 1, k, 2);
    c.zz0 = sz(L, 2, k, 0); c.zz1 = sz(L, 2, k, 1); c.zz2 = sz(L, 2, k, 2);
    return c;
}

// Colour pass with two rows per lane: a segment of S lanes (S a power of two
// >= (Nzg-2)/2) owns one column, lane r its rows ka = 2+2r and kb = ka+1. The
// column's task and its order are colour_warp's; a lane composes its two
// rows' affine maps before the segment's shuffle scan, so a warp solves 32/S
// columns and the per-column work (column decode, coefficient and bottom-row
// loads, the bottom row itself) is shared by twice as many rows.
//
// colour_col2 is the task of column (i, j) for its segment (act false: the
// segment joins the warp's shuffles and touches no memory). x is read through
// xr, the column's first row, with neighbour columns at +-Nzg (x) and +-oy (y);
// b through br; x is written in global memory. With TILE the reads come from
// a shared-memory tile (cfs, bts: the column's coefficients and bottom-row
// table there) and the column is not next to a wall; otherwise they come from
// global memory and the ghost-column and corner work of the wall columns runs
// here.
template <typename T, bool THREE, int S, bool CROSS, bool TILE>
__device__ __forceinline__ void colour_col2(const LevelDev<T>& L, int i, int j, bool act, const RowConst<T>& rka,
                                            const RowConst<T>& rkb, const T* xr, int oy, const T* br, const T* cfs,
                                            const T* bts) {
    const int Nxg = L.Nxg, Nyg = L.Nyg, Nzg = L.Nzg, R = Nzg - 2;
    const int lane = threadIdx.x & 31, r = lane & (S - 1);
    const unsigned segmask = 0xffffffffu;   // the whole warp runs the scan together
    T* const X = L.xv;
    const T* const B = L.bv;

    const int ka = 2 + 2 * r, kb = ka + 1;
    const bool va = act && ka <= Nzg - 1, vb = act && kb <= Nzg - 1;
    const int last = (R - 1) / 2;           // lane holding row Nzg-1 (the free surface follows it)
    const int c = (i - 1) + Nxg * (j - 1);
    T* const xc = X + (int64_t)c * Nzg;
    const T* const bc = br;
    const int ox = Nzg;
    const bool edge = !TILE && act && (i <= 3 || i >= Nxg - 2 || (THREE && (j <= 3 || j >= Nyg - 2)));

    auto colidx = [&](int ii, int jj) -> int64_t { return (int64_t)(ii - 1) + (int64_t)Nxg * (jj - 1); };
    // ghost column cg: Neumann rows of this lane's levels, wa x(ca) + wb x(cb) + wg x(cg) = b;
    // with post set, the value of this column (ca if own == 1, cb if own == 2)
    // is the lane's new one
    auto relax_ghost = [&](int64_t cg, int64_t ca, T wa, int64_t cb, T wb, T wg, int own, bool post, T xna, T xnb,
                           T xfsn) {
        auto row = [&](int kk, T xo) {
            const T v1 = (post && own == 1) ? xo : X[ca * Nzg + kk - 1];
            const T v2 = (post && own == 2) ? xo : X[cb * Nzg + kk - 1];
            X[cg * Nzg + kk - 1] = (B[cg * Nzg + kk - 1] - (wa * v1 + wb * v2)) / wg;
        };
        if (ka <= Nzg - 1) row(ka, xna);
        if (kb <= Nzg - 1) row(kb, xnb);
        if (r == last) row(Nzg, xfsn);
        if (!CROSS && r == 0) X[cg * Nzg] = B[cg * Nzg];   // identity level-1 row
    };
    auto ghosts = [&](bool post, T xna, T xnb, T xfsn) {
        // periodic x has no x ghost columns to relax
        if (!L.per && (i == 2 || (post && i == 3)))
            relax_ghost(colidx(1, j), colidx(2, j), sx(L, 1, 2, 1), colidx(3, j), sx(L, 1, 2, 2), sx(L, 1, 2, 0),
                        i == 2 ? 1 : 2, post, xna, xnb, xfsn);
        if (!L.per && (i == Nxg - 1 || (post && i == Nxg - 2)))
            relax_ghost(colidx(Nxg, j), colidx(Nxg - 2, j), sx(L, 1, Nxg - 1, 0), colidx(Nxg - 1, j),
                        sx(L, 1, Nxg - 1, 1), sx(L, 1, Nxg - 1, 2), i == Nxg - 1 ? 2 : 1, post, xna, xnb, xfsn);
        if (THREE) {
            if (j == 2 || (post && j == 3))
                relax_ghost(colidx(i, 1), colidx(i, 2), sy(L, 1, 2, 1), colidx(i, 3), sy(L, 1, 2, 2), sy(L, 1, 2, 0),
                            j == 2 ? 1 : 2, post, xna, xnb, xfsn);
            if (j == Nyg - 1 || (post && j == Nyg - 2))
                relax_ghost(colidx(i, Nyg), colidx(i, Nyg - 2), sy(L, 1, Nyg - 1, 0), colidx(i, Nyg - 1),
                            sy(L, 1, Nyg - 1, 1), sy(L, 1, Nyg - 1, 2), j == Nyg - 1 ? 2 : 1, post, xna, xnb, xfsn);
        }
    };
    if (!TILE) {
        if (edge) {
            if (THREE && !L.per && (i == 2 || i == Nxg - 1) && (j == 2 || j == Nyg - 1)) {
                const int64_t cc = colidx(i == 2 ? 1 : Nxg, j == 2 ? 1 : Nyg);
                for (int kk = r; kk < Nzg; kk += S) X[cc * Nzg + kk] = B[cc * Nzg + kk];
            }
            ghosts(false, T(0), T(0), T(0));
        }
        __syncwarp();
    }

    // rows ka and kb (clamped for loads; lanes past the last row discard theirs)
    const int kra = min(ka, Nzg - 1), krb = min(kb, Nzg - 1);
    T qa = 0, ga = 0, qb = 0, gb = 0, x1 = 0;
    T bb1 = 0, bl = 0, br1 = 0, bd = 0, bu = 0;
    T t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0;
    if (act) {
        T ih, ca, cb, c3;
        if (TILE) { ih = cfs[0]; ca = cfs[1]; cb = cfs[2]; c3 = cfs[3]; }
        else load_cf(L.cf, (int64_t)c, ih, ca, cb, c3);
        const T* sxp = L.SX + (Nxg + i - 1) * 3;
        const T wxl = __ldg(sxp), wxc = __ldg(sxp + 1), wxr = __ldg(sxp + 2);
        T wyd = 0, wyc = 0, wyu = 0;
        if (THREE) {
            const T* syp = L.SY + (Nyg + j - 1) * 3;
            wyd = __ldg(syp); wyc = __ldg(syp + 1); wyu = __ldg(syp + 2);
        }
        // q, g of row kr (x_kr = q - g x_{kr-1})
        const int oxl = xoff_l(L, i), oxr = xoff_r(L, i);
        auto rowq = [&](int kr, const RowConst<T>& rk, T x0, T xp, T& qo, T& go) {
            const int o = kr - 1;
            const T xl = xr[o + oxl], xrr = xr[o + oxr];
            const T xd = THREE ? xr[o - oy] : T(0), xu = THREE ? xr[o + oy] : T(0);
            const T bk = bc[o];
            const T om = rk.om;
            const T s2 = om * ca, s4 = THREE ? om * cb : T(0);
            const T s3 = om * c3;
            const T cz = s2 * s2 + s4 * s4 + ih * ih;
            T off = wxl * xl + wxr * xrr;
            T diag = wxc + s3 * rk.z1 + cz * rk.zz1;
            if (THREE) { off += wyd * xd + wyu * xu; diag += wyc; }
            T lo = s3 * rk.z0 + cz * rk.zz0, up = s3 * rk.z2 + cz * rk.zz2;
            if (CROSS && s2 != T(0)) {
                const int jlo = THREE ? j - 1 : j, jhi = THREE ? j + 1 : j;
                T xz = 0;
                for (int jj = jlo; jj <= jhi; ++jj) {
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk) {
                        const int kz = kr - 1 + kk;
                        int sh = 0;
                        if (kz == 1) { if (i - 1 == 1) sh = 1; if (i + 1 == Nxg) sh = -1; }
                        T dx = 0;
#pragma unroll
                        for (int m = 0; m < 3; ++m) {
                            const int ii = i - 1 + sh + m;
                            const T w = sx(L, 1, i - sh, m);
                            if (ii == i && jj == j && kz <= Nzg - 1) {
                                const T cf2 = T(2) * s2 * sz(L, 1, kr, kk) * w;
                                if (kk == 0) lo += cf2; else if (kk == 1) diag += cf2; else up += cf2;
                            } else {
                                dx += w * xr[(ii - i) * ox + (jj - j) * oy + (kz - 1)];
                            }
                        }
                        xz += sz(L, 1, kr, kk) * dx;
                    }
                }
                off += T(2) * s2 * xz;
            }
            if (THREE && CROSS && s4 != T(0)) {
                T yz = 0;
                for (int ii = i - 1; ii <= i + 1; ++ii) {
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk) {
                        const int kz = kr - 1 + kk;
                        int sh = 0;
                        if (kz == 1) { if (j - 1 == 1) sh = 1; if (j + 1 == Nyg) sh = -1; }
                        T dy = 0;
#pragma unroll
                        for (int m = 0; m < 3; ++m) {
                            const int jj = j - 1 + sh + m;
                            const T w = sy(L, 1, j - sh, m);
                            if (ii == i && jj == j && kz <= Nzg - 1) {
                                const T cf2 = T(2) * s4 * sz(L, 1, kr, kk) * w;
                                if (kk == 0) lo += cf2; else if (kk == 1) diag += cf2; else up += cf2;
                            } else {
                                dy += w * xr[(ii - i) * ox + (jj - j) * oy + (kz - 1)];
                            }
                        }
                        yz += sz(L, 1, kr, kk) * dy;
                    }
                }
                off += T(2) * s4 * yz;
            }
            const T id = T(1) / diag;
            qo = x0 + (bk - diag * x0 - up * xp - off) * id;
            go = lo * id;
        };
        const T x0a = xr[kra - 1], xpa = xr[kra], xpb = xr[krb];
        rowq(kra, rka, x0a, xpa, qa, ga);
        rowq(krb, rkb, xpa, xpb, qb, gb);            // row kb's old value is row ka's "above"
        if (!va) { qa = 0; ga = 0; }
        if (!vb) { qb = 0; gb = 0; }
        if (!CROSS) {
            if (TILE) {
                t0 = bts[0]; t1 = bts[1]; t2 = bts[2]; t3 = bts[3]; t4 = bts[4]; t5 = bts[5]; t6 = bts[6];
            } else {
                T btv[7];
                load_bt(L.bt, (int64_t)c, btv);
                t0 = btv[0]; t1 = btv[1]; t2 = btv[2]; t3 = btv[3]; t4 = btv[4]; t5 = btv[5]; t6 = btv[6];
            }
            bb1 = bc[0];
            bl = xr[1 + oxl]; br1 = xr[1 + oxr];
            if (THREE) { bd = xr[1 - oy]; bu = xr[1 + oy]; }
            T boff = t0 * xr[1] + t1 * xr[2] + t2 * bl + t3 * br1;
            if (THREE) boff += t4 * bd + t5 * bu;
            x1 = (bb1 - boff) * t6;
        } else {
            x1 = xr[0];
        }
    }
    // this lane's two rows as one map x_{ka-1} -> x_kb, then the segment scan
    T a = 1, bb = 0;
    if (va) { bb = qa; a = -ga; }
    if (vb) { bb = qb - gb * bb; a = -gb * a; }
#pragma unroll
    for (int d = 1; d < S; d <<= 1) {
        const T ap = __shfl_up_sync(segmask, a, d, S);
        const T bp = __shfl_up_sync(segmask, bb, d, S);
        if (r >= d) { bb = a * bp + bb; a = a * ap; }
    }
    const T ae = __shfl_up_sync(segmask, a, 1, S), be = __shfl_up_sync(segmask, bb, 1, S);
    const T xin = (r == 0) ? x1 : ae * x1 + be;   // new value of row ka-1
    const T xna = qa - ga * xin;
    const T xnb = qb - gb * xna;
    const T x2n = __shfl_sync(segmask, xna, 0, S);
    const T x3n = __shfl_sync(segmask, xnb, 0, S);
    if (va) xc[ka - 1] = xna;
    if (vb) xc[kb - 1] = xnb;
    const T xfs = act ? bc[Nzg - 1] : T(0);
    if (act && r == last) xc[Nzg - 1] = xfs;  // free-surface row
    if (!CROSS && act && r == 0) {
        T boff = t0 * x2n + t1 * x3n + t2 * bl + t3 * br1;
        if (THREE) boff += t4 * bd + t5 * bu;
        xc[0] = (bb1 - boff) * t6;
    }
    if (!TILE && edge) ghosts(true, xna, xnb, xfs);
}

// Ask for the column data of the group a warp solves from `base` on to be
// brought into L1 (the rows of x this lane reads in the column and its four
// neighbours, and of b): one prefetch per 32-byte sector the lane touches.
template <typename T, bool THREE, int S>
__device__ __forceinline__ void colour_prefetch(const LevelDev<T>& L, int colour, int base) {
    const int Nxg = L.Nxg, Nyg = L.Nyg, Nzg = L.Nzg;
    const int lane = threadIdx.x & 31, r = lane & (S - 1);
    const int nxi = Nxg - 2 - L.per, nyi = THREE ? Nyg - 2 : 1;
    const bool four = (L.ncolor == 4);
    const int ni = (nxi + 1) / 2, nj = four ? (nyi + 1) / 2 : nyi;
    const int q = base + (lane / S);
    if (q >= ni * nj) return;
    const int tj = q / ni, ti = q - tj * ni;
    int i, j;
    if (four) { j = THREE ? 2 + 2 * tj + (colour >> 1) : 1; i = 2 + 2 * ti + (colour & 1); }
    else { j = THREE ? 2 + tj : 1; i = 2 + 2 * ti + ((colour + j) & 1); }
    if (i > Nxg - 1 - L.per || (THREE && j > Nyg - 1)) return;
    const int64_t c = (int64_t)(i - 1) + (int64_t)Nxg * (j - 1);
    const int k = min(2 + 2 * r, Nzg - 1) - 1;
    const T* x = L.xv + c * Nzg + k;
    auto pf = [](const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); };
    pf(x);
    pf(x + xoff_l(L, i));
    pf(x + xoff_r(L, i));
    if (THREE) { pf(x - (int64_t)Nzg * Nxg); pf(x + (int64_t)Nzg * Nxg); }
    pf(L.bv + c * Nzg + k);
}

// The colour's columns in order (rows of constant j, i fastest), 32/S per
// warp from column `base` on.
template <typename T, bool THREE, int S, bool CROSS>
__device__ void colour_warp2(const LevelDev<T>& L, int colour, int base, const RowConst<T>& rka,
                             const RowConst<T>& rkb) {
    const int Nxg = L.Nxg, Nyg = L.Nyg, Nzg = L.Nzg;
    const int lane = threadIdx.x & 31;
    const int nxi = Nxg - 2 - L.per, nyi = THREE ? Nyg - 2 : 1;   // periodic: the distinct columns
    const bool four = (L.ncolor == 4);
    const int ni = (nxi + 1) / 2;
    const int nj = four ? (nyi + 1) / 2 : nyi;
    const int total = ni * nj;
    const int q = base + (lane / S);
    bool act = q < total;
    int i = 2, j = THREE ? 2 : 1;
    if (act) {
        const int tj = q / ni, ti = q - tj * ni;
        if (four) {
            j = THREE ? 2 + 2 * tj + (colour >> 1) : 1;
            i = 2 + 2 * ti + (colour & 1);
        } else {
            j = THREE ? 2 + tj : 1;
            i = 2 + 2 * ti + ((colour + j) & 1);
        }
        act = (i <= Nxg - 1 - L.per) && (!THREE || j <= Nyg - 1);
    }
    const int64_t c = (int64_t)(i - 1) + (int64_t)Nxg * (j - 1);
    colour_col2<T, THREE, S, CROSS, false>(L, i, j, act, rka, rkb, L.xv + c * Nzg, Nzg * Nxg, L.bv + c * Nzg,
                                           nullptr, nullptr);
}

// Number of columns of one colour (two colours, 3-D) within two columns of a
// wall: rows j = 2, 3, Nyg-2, Nyg-1 whole, and on the rows between them the
// columns i = 2, 3, Nxg-2, Nxg-1. The tiled pass covers the rest.
template <typename T>
__device__ __host__ __forceinline__ int wall_band_count(const LevelDev<T>& L) {
    const int ni = (L.Nxg - 1) / 2;
    return 4 * ni + 2 * (L.Nyg - 6);
}

// The wall-band columns of `colour` (wall_band_count of them), 32/S per warp
// from band column `base` on.
template <typename T, int S>
__device__ void colour_band2(const LevelDev<T>& L, int colour, int base, const RowConst<T>& rka,
                             const RowConst<T>& rkb) {
    const int Nxg = L.Nxg, Nyg = L.Nyg, Nzg = L.Nzg;
    const int ni = (Nxg - 1) / 2;
    const int q = base + ((threadIdx.x & 31) / S);
    bool act = q < wall_band_count(L);
    int i = 2, j = 2;
    if (act) {
        if (q < 4 * ni) {
            const int rr = q / ni, ti = q - rr * ni;
            j = rr < 2 ? 2 + rr : Nyg - 4 + rr;
            i = 2 + 2 * ti + ((colour + j) & 1);
            act = i <= Nxg - 1;
        } else {
            const int q2 = q - 4 * ni;
            j = 4 + (q2 >> 1);
            i = (q2 & 1) ? Nxg - 2 + ((colour + j - (Nxg - 2)) & 1) : 2 + ((colour + j) & 1);
        }
    }
    const int64_t c = (int64_t)(i - 1) + (int64_t)Nxg * (j - 1);
    colour_col2<T, true, S, false, false>(L, i, j, act, rka, rkb, L.xv + c * Nzg, Nzg * Nxg, L.bv + c * Nzg,
                                          nullptr, nullptr);
}

// MGRestriction3DExplicit.f90:19-128 as a gather for coarse point p (also zeroes the coarse iterate).
template <typename T>
__device__ void restrict_item(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* rf, T* rc, T* xc, int64_t p) {

    const int gy = (F.Nyg > 1) ? 1 : 0;
    const int Nzf = F.Nzg - 1, Nyf = F.Nyg - 2 * gy;
    const int xcz = Cc.xc, ycz = Cc.yc, zcz = Cc.zc;

        int kc, ic, jc;
        int64_t cc;
        decomp(Cc, p, kc, cc, ic, jc);
        xc[p] = T(0);
        const bool ghost = kc == 1 || ic == 1 || ic == Cc.Nxg || (Cc.per && ic == Cc.Nxg - 1) ||
                           (gy && (jc == 1 || jc == Cc.Nyg));
        if (ghost) { rc[p] = T(0); return; }
        const int kf = 2 + (kc - 2) * (1 + zcz), ifn = 2 + (ic - 2) * (1 + xcz), jf = gy ? 2 + (jc - 2) * (1 + ycz) : 1;
        // fine values by 32-bit offsets from (kf, ifn, jf) (levels have < 2^31 points)
        const T* rb = rf + IX(F, kf, ifn, jf);
        const int fox = F.Nzg, foy = F.Nzg * F.Nxg;
        auto R = [&](int k, int i, int j) -> T { return rb[(k - kf) + (i - ifn) * fox + (j - jf) * foy]; };
        if (kf == F.Nzg) { rc[p] = R(kf, ifn, jf); return; }
        // x-weighted value at (k, ifn, j) (raw on ghost rows and outside 2..Nzf)
        auto Sx = [&](int k, int j) -> T {
            if (!xcz || k < 2 || k > Nzf || (gy && (j < 2 || j > Nyf + 1))) return R(k, ifn, j);
            const double dW = F.x[ifn - 1] - F.x[ifn - 2], dE = F.x[ifn] - F.x[ifn - 1];
            const T dxc = T(F.ix[ifn - 1]);
            // periodic x: the west neighbour of the first column is the last distinct one
            const int iw = F.per ? wrap_x(ifn - 1, F.Nxg) : ifn - 1;
            return (T(0.5) * dxc) * (T(dW) * R(k, iw, j) + T(dW + dE) * R(k, ifn, j) + T(dE) * R(k, ifn + 1, j));
        };
        auto Sxy = [&](int k) -> T {
            if (!ycz || k < 2 || k > Nzf) return Sx(k, jf);
            const double dS = F.y[jf - 1] - F.y[jf - 2], dN = F.y[jf] - F.y[jf - 1];
            const T dyc = T(F.iy[jf - 1]);
            return (T(0.5) * dyc) * (T(dS) * Sx(k, jf - 1) + T(dN + dS) * Sx(k, jf) + T(dN) * Sx(k, jf + 1));
        };
        T v;
        if (zcz) {
            const double dU = F.z[kf] - F.z[kf - 1], dD = F.z[kf - 1] - F.z[kf - 2];
            const T dzc = T(F.iz[kf - 1]);
            v = (T(0.5) * dzc) * (T(dD) * Sxy(kf - 1) + T(dU) * Sxy(kf + 1)) + T(0.5) * Sxy(kf);
        } else {
            v = Sxy(kf);
        }
        rc[p] = v;
    }

// MGProlongation3DExplicit.f90:19-110 as a gather for fine point p, added to
// xf: the sequential x, y, z interpolation sweeps are a tensor product, so the
// value is the weighted sum over (at most) 2 x 2 x 2 coarse points with the
// fine level's per-direction tables. The free-surface row, the bottom ghost
// row and the ghost columns are not touched.
template <typename T>
__device__ void prolong_item(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* xc, T* xf, int64_t p) {
    const int gy = (F.Nyg > 1) ? 1 : 0;
    int kf, ifn, jf;
    int64_t cfl;
    decomp(F, p, kf, cfl, ifn, jf);
    if (kf == 1 || kf == F.Nzg || ifn == 1 || ifn == F.Nxg || (gy && (jf == 1 || jf == F.Nyg))) return;
    if (F.per && ifn == F.Nxg - 1) return;   // periodic x: the repeated column stays zero
    const int2 zi = __ldg(reinterpret_cast<const int2*>(F.piz) + (kf - 1));
    const int2 xi = __ldg(reinterpret_cast<const int2*>(F.pix) + (ifn - 1));
    const int2 yi = __ldg(reinterpret_cast<const int2*>(F.piy) + (gy ? jf - 1 : 0));
    const T wz0 = __ldg(F.pwz + 2 * (kf - 1)), wz1 = __ldg(F.pwz + 2 * (kf - 1) + 1);
    const T wx0 = __ldg(F.pwx + 2 * (ifn - 1)), wx1 = __ldg(F.pwx + 2 * (ifn - 1) + 1);
    const T wy0 = __ldg(F.pwy + 2 * (gy ? jf - 1 : 0)), wy1 = __ldg(F.pwy + 2 * (gy ? jf - 1 : 0) + 1);
    const int Ncz = Cc.Nzg, Ncx = Cc.Nxg;
    auto C = [&](int kc, int ic, int jc) -> T {   // 32-bit: levels have < 2^31 points
        return xc[(kc - 1) + Ncz * ((ic - 1) + Ncx * (jc - 1))];
    };
    auto Px = [&](int kc, int jc) -> T {
        T v = wx0 * C(kc, xi.x, jc);
        if (wx1 != T(0)) v += wx1 * C(kc, xi.y, jc);
        return v;
    };
    auto Py = [&](int kc) -> T {
        T v = wy0 * Px(kc, yi.x);
        if (wy1 != T(0)) v += wy1 * Px(kc, yi.y);
        return v;
    };
    T v = wz0 * Py(zi.x);
    if (wz1 != T(0)) v += wz1 * Py(zi.y);
    xf[p] += v;
}

// Coarsest level, row r of x = A^{-1} b.
template <typename T>
__device__ __forceinline__ void coarse_item(int n, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x, int r) {
    T acc = 0;
    for (int c = 0; c < n; ++c) acc += inv[(int64_t)r * n + c] * b[c];
    x[r] = acc;
}

}  // namespace mgdev
}  // namespace ow3d
