// Device-side pieces of the multigrid preconditioner shared by the per-phase
// kernels (mg.cu) and the fused coarse-level kernel (mg_coarse.cu): row
// evaluation of the low-order operator, the Gauss-Seidel phases and the grid
// transfers, each as a function of one work item.
#pragma once
#include "ow3d_internal.h"

namespace ow3d {
namespace mgdev {

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

// Interior row (2 <= k <= Nzg-1, interior column). Returns A x at the row and
// the diagonal coefficient.
template <typename T, bool THREE>
__device__ T lo_interior(const LevelDev<T>& L, const T* x, int k, int i, int j, T& diag) {
    const int64_t c = (int64_t)(i - 1) + (int64_t)L.Nxg * (j - 1);
    const T h = L.h[c], hx = L.hx[c], hxx = L.hxx[c];
    const T hy = THREE ? L.hy[c] : T(0), hyy = THREE ? L.hyy[c] : T(0);
    const T sg = __ldg(L.zs + k - 1), om = T(1) - sg;
    // DetermineTransformationConstantsArray with eta = 0
    const T s5 = T(1) / h;
    const T s2 = om * hx * s5;
    const T s4 = om * hy * s5;
    const T s3 = om * ((hxx + hyy) * s5 - T(2) * (hx * hx + hy * hy) * s5 * s5);
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
    const T s5 = T(1) / h, s2 = om * hx * s5, s4 = om * hy * s5;
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

// Gauss-Seidel value of a ghost-column row, (b - off-diagonal part) / diagonal.
// It does not read the row's own current value, so a thread that needs the
// updated ghost value can recompute it while another thread writes it.
template <typename T, bool THREE>
__device__ T ghost_gs(const LevelDev<T>& L, int k, int i, int j) {
    const int64_t p = IX(L, k, i, j);
    const bool gxx = (i == 1 || i == L.Nxg), gyy = THREE && (j == 1 || j == L.Nyg);
    if ((gxx && gyy) || k == 1) return L.bv[p];
    T off = 0, dg;
    if (gxx) {
        const int ia = (i == 1) ? 2 : L.Nxg - 1;
        const int self = (i == 1) ? 0 : 2;
#pragma unroll
        for (int m = 0; m < 3; ++m) if (m != self) off += sx(L, 1, ia, m) * L.xv[IX(L, k, ia - 1 + m, j)];
        dg = sx(L, 1, ia, self);
    } else {
        const int ja = (j == 1) ? 2 : L.Nyg - 1;
        const int self = (j == 1) ? 0 : 2;
#pragma unroll
        for (int m = 0; m < 3; ++m) if (m != self) off += sy(L, 1, ja, m) * L.xv[IX(L, k, i, ja - 1 + m)];
        dg = sy(L, 1, ja, self);
    }
    return (L.bv[p] - off) / dg;
}

template <typename T, bool THREE>
__device__ T lo_row(const LevelDev<T>& L, const T* x, int k, int i, int j, T& diag) {
    if (is_ghost_col<T, THREE>(L, i, j)) return lo_ghost<T, THREE>(L, x, k, i, j, diag);
    if (k == L.Nzg) { diag = T(1); return x[IX(L, k, i, j)]; }
    if (k == 1) return lo_bottom<T, THREE>(L, x, i, j, diag);
    return lo_interior<T, THREE>(L, x, k, i, j, diag);
}


template <typename T>
__device__ __forceinline__ T ro(const T* p) { return __ldg(p); }

template <typename T, bool THREE>
__device__ __forceinline__ void residual_item(const LevelDev<T>& L, int64_t p) {
    const int k = (int)(p % L.Nzg) + 1;
    const int64_t c = p / L.Nzg;
    const int i = (int)(c % L.Nxg) + 1, j = (int)(c / L.Nxg) + 1;
    T dg;
    L.rv[p] = L.bv[p] - lo_row<T, THREE>(L, L.xv, k, i, j, dg);
}

// Special pass item q in [0, special_count): ghost-column rows first, then
// the bottom rows of the interior columns (the reference's iGhost rows,
// MGPreProcess.f90:376-439). A bottom row next to a ghost column uses the ghost
// value of this pass, recomputed with ghost_gs (the ghost thread's arithmetic).
template <typename T, bool THREE>
__device__ __forceinline__ int64_t special_count(const LevelDev<T>& L) {
    const int64_t nper = THREE ? (int64_t)2 * L.Nyg + 2 * (L.Nxg - 2) : 2;
    return nper * L.Nzg + (int64_t)L.Nxg * L.Nyg;
}
template <typename T, bool THREE>
__device__ void special_item(const LevelDev<T>& L, int64_t q) {
    const int Nxg = L.Nxg, Nyg = L.Nyg, Nzg = L.Nzg;
    const int64_t nper = THREE ? (int64_t)2 * Nyg + 2 * (Nxg - 2) : 2;
    const int64_t nghost = nper * Nzg;

        if (q < nghost) {
            const int k = (int)(q % Nzg) + 1;
            const int64_t e = q / Nzg;
            int i, j;
            if (!THREE) { i = (e == 0) ? 1 : Nxg; j = 1; }
            else if (e < 2 * Nyg) { i = (e % 2 == 0) ? 1 : Nxg; j = (int)(e / 2) + 1; }
            else { const int64_t f = e - 2 * Nyg; j = (f % 2 == 0) ? 1 : Nyg; i = (int)(f / 2) + 2; }
            L.xv[IX(L, k, i, j)] = ghost_gs<T, THREE>(L, k, i, j);
            return;
        }
        const int64_t c = q - nghost;
        const int i = (int)(c % Nxg) + 1, j = (int)(c / Nxg) + 1;
        if (is_ghost_col<T, THREE>(L, i, j)) return;
        const T h = L.h[c], hx = L.hx[c];
        const T hy = THREE ? L.hy[c] : T(0);
        const T om = T(1) - L.zs[1], ih = T(1) / h;
        const T s2 = om * hx * ih, s4 = om * hy * ih;
        const T f = THREE ? (ih + hx * s2 + hy * s4) : (ih + hx * s2);
        const T* xc = L.xv + c * Nzg;
        const T dz = sz(L, 1, 2, 1) * xc[1] + sz(L, 1, 2, 2) * xc[2];
        T dx = 0;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const int ii = i - 1 + m;
            dx += sx(L, 1, i, m) * (is_ghost_col<T, THREE>(L, ii, j) ? ghost_gs<T, THREE>(L, 2, ii, j) : L.xv[IX(L, 2, ii, j)]);
        }
        T off = f * dz + hx * dx;
        if (THREE) {
            T dy = 0;
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                const int jj = j - 1 + m;
                dy += sy(L, 1, j, m) * (is_ghost_col<T, THREE>(L, i, jj) ? ghost_gs<T, THREE>(L, 2, i, jj) : L.xv[IX(L, 2, i, jj)]);
            }
            off += hy * dy;
        }
        L.xv[c * Nzg] = (L.bv[c * Nzg] - off) / (f * sz(L, 1, 2, 0));
    }

// Colour phase, warp-cooperative form. A segment of S lanes (S a power of two
// >= Nzg-2) owns one interior column of the colour; lane r holds row k = r+2.
// Each lane forms its row's Gauss-Seidel update as an affine map of the new
// value below it, x_k = q_k - g_k x_{k-1}; the chain over the column (the
// bottom-to-top Gauss-Seidel order) is evaluated with a shuffle scan of the
// composed maps. Loads are coalesced along the column. CROSS: the level has
// mixed-derivative terms (sloping bottom). All 32 lanes of the warp call this
// with the same `base` (the first column index of the warp).
template <typename T, bool THREE>
__device__ __forceinline__ int64_t colour_count(const LevelDev<T>& L) {
    const int nxi = L.Nxg - 2, nyi = THREE ? L.Nyg - 2 : 1;
    const int ni = (nxi + 1) / 2, nj = (L.ncolor == 4) ? (nyi + 1) / 2 : nyi;
    return (int64_t)ni * nj;
}
template <typename T, bool THREE, int S, bool CROSS>
__device__ void colour_warp(const LevelDev<T>& L, int colour, int64_t base) {
    const int Nxg = L.Nxg, Nyg = L.Nyg, Nzg = L.Nzg, R = Nzg - 2;
    const int lane = threadIdx.x & 31, r = lane & (S - 1);
    const int seg_per_warp = 32 / S;
    const int nxi = Nxg - 2, nyi = THREE ? Nyg - 2 : 1;
    // columns of this colour: every other i (and every other j with 4 colours)
    const bool four = (L.ncolor == 4);
    const int ni = (nxi + 1) / 2;
    const int nj = four ? (nyi + 1) / 2 : nyi;
    const int64_t total = (int64_t)ni * nj;
    const unsigned segmask = 0xffffffffu;   // the whole warp runs the scan together

        const int64_t q = base + (lane / S);
        bool act = q < total;
        int i = 0, j = 1;
        if (act) {
            const int ti = (int)(q % ni), tj = (int)(q / ni);
            if (four) {
                j = THREE ? 2 + 2 * tj + (((colour >> 1) - 2) & 1) : 1;
                i = 2 + 2 * ti + (((colour & 1) - 2) & 1);
            } else {
                j = THREE ? 2 + tj : 1;
                i = 2 + 2 * ti + ((colour + j) & 1);    // (i + j) & 1 == colour
            }
            act = (i <= Nxg - 1) && (!THREE || j <= Nyg - 1);
        }
        const bool rowact = act && (r < R);
        const int k = r + 2;
        T qv = 0, gv = 0, x1 = 0;
        const int64_t c = (int64_t)(i - 1) + (int64_t)Nxg * (j - 1);
        if (rowact) {
            const T* xc = L.xv + c * Nzg;
            const T h = L.h[c], hx = L.hx[c], hxx = L.hxx[c];
            const T hy = THREE ? L.hy[c] : T(0), hyy = THREE ? L.hyy[c] : T(0);
                const T ih = T(1) / h;
            const T sg = __ldg(L.zs + k - 1), om = T(1) - sg;
            const T s2 = om * hx * ih, s4 = om * hy * ih;
            const T s3 = om * ((hxx + hyy) * ih - T(2) * (hx * hx + hy * hy) * ih * ih);
            const T cz = s2 * s2 + s4 * s4 + ih * ih;
            const T z0 = sz(L, 1, k, 0), z1 = sz(L, 1, k, 1), z2 = sz(L, 1, k, 2);
            const T zz0 = sz(L, 2, k, 0), zz1 = sz(L, 2, k, 1), zz2 = sz(L, 2, k, 2);
            T off = sx(L, 2, i, 0) * ro(L.xv + (c - 1) * Nzg + k - 1) + sx(L, 2, i, 2) * ro(L.xv + (c + 1) * Nzg + k - 1);
            T diag = sx(L, 2, i, 1) + s3 * z1 + cz * zz1;
            if (THREE) {
                off += sy(L, 2, j, 0) * ro(L.xv + (c - Nxg) * Nzg + k - 1) + sy(L, 2, j, 2) * ro(L.xv + (c + Nxg) * Nzg + k - 1);
                diag += sy(L, 2, j, 1);
            }
            T lo = s3 * z0 + cz * zz0, up = s3 * z2 + cz * zz2;
            if (CROSS && s2 != T(0)) {
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
            if (THREE && CROSS && s4 != T(0)) {
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
            const T x0 = xc[k - 1];
            const T xp = xc[k];                    // old value of the row above (row Nzg: free surface)
            const T bk = L.bv[c * Nzg + k - 1];
            // row update x0 + (b - (lo x_{k-1} + diag x0 + up xp + off)) / diag
            const T id = T(1) / diag;
            qv = x0 + (bk - diag * x0 - up * xp - off) * id;
            gv = lo * id;
            if (r == 0) x1 = xc[0];                // bottom row: constant during the phase
        }
        // inclusive scan of the affine maps x -> a x + b, a = -g, b = q (in row order)
        T a = -gv, bb = qv;
#pragma unroll
        for (int d = 1; d < S; d <<= 1) {
            const T ap = __shfl_up_sync(segmask, a, d, S);
            const T bp = __shfl_up_sync(segmask, bb, d, S);
            if (r >= d) { bb = a * bp + bb; a = a * ap; }
        }
        x1 = __shfl_sync(segmask, x1, 0, S);
        if (rowact) {
            T* xc = L.xv + c * Nzg;
            xc[k - 1] = a * x1 + bb;
            if (r == R - 1) xc[Nzg - 1] = L.bv[c * Nzg + Nzg - 1];   // free-surface row
        }
    }

// MGRestriction3DExplicit.f90:19-128 as a gather for coarse point p (also zeroes the coarse iterate).
template <typename T>
__device__ void restrict_item(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* __restrict__ rf, T* __restrict__ rc, T* __restrict__ xc, int64_t p) {

    const int gy = (F.Nyg > 1) ? 1 : 0;
    const int Nzf = F.Nzg - 1, Nyf = F.Nyg - 2 * gy;
    const int xcz = Cc.xc, ycz = Cc.yc, zcz = Cc.zc;

        const int kc = (int)(p % Cc.Nzg) + 1;
        const int64_t cc = p / Cc.Nzg;
        const int ic = (int)(cc % Cc.Nxg) + 1, jc = (int)(cc / Cc.Nxg) + 1;
        xc[p] = T(0);
        const bool ghost = kc == 1 || ic == 1 || ic == Cc.Nxg || (gy && (jc == 1 || jc == Cc.Nyg));
        if (ghost) { rc[p] = T(0); return; }
        const int kf = 2 + (kc - 2) * (1 + zcz), ifn = 2 + (ic - 2) * (1 + xcz), jf = gy ? 2 + (jc - 2) * (1 + ycz) : 1;
        auto R = [&](int k, int i, int j) -> T { return rf[IX(F, k, i, j)]; };
        if (kf == F.Nzg) { rc[p] = R(kf, ifn, jf); return; }
        // x-weighted value at (k, ifn, j) (raw on ghost rows and outside 2..Nzf)
        auto Sx = [&](int k, int j) -> T {
            if (!xcz || k < 2 || k > Nzf || (gy && (j < 2 || j > Nyf + 1))) return R(k, ifn, j);
            const double dW = F.x[ifn - 1] - F.x[ifn - 2], dE = F.x[ifn] - F.x[ifn - 1];
            const T dxc = T(F.ix[ifn - 1]);
            return (T(0.5) * dxc) * (T(dW) * R(k, ifn - 1, j) + T(dW + dE) * R(k, ifn, j) + T(dE) * R(k, ifn + 1, j));
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

// MGProlongation3DExplicit.f90:19-110 as a gather for fine point p, added to xf.
template <typename T>
__device__ void prolong_item(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* __restrict__ xc, T* __restrict__ xf, int64_t p) {

    const int gy = (F.Nyg > 1) ? 1 : 0;
    const int XF = Cc.xc ? 2 : 1, YF = Cc.yc ? 2 : 1, ZF = Cc.zc ? 2 : 1;

        const int kf = (int)(p % F.Nzg) + 1;
        const int64_t cf = p / F.Nzg;
        const int ifn = (int)(cf % F.Nxg) + 1, jf = (int)(cf / F.Nxg) + 1;
        if (kf == 1 || kf == F.Nzg || ifn == 1 || ifn == F.Nxg || (gy && (jf == 1 || jf == F.Nyg))) return;
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
            const T dxf = T(F.ix[ifn - 1]);
            return (T(dE) * Cv(k, ifn - 1, j) + T(dW) * Cv(k, ifn + 1, j)) * dxf;
        };
        auto Py = [&](int k) -> T {
            if (k == F.Nzg) return T(0);
            if (!gy || YF == 1 || ((jf - 2) % 2) == 0) return Px(k, jf);
            const double dS = F.y[jf - 1] - F.y[jf - 2], dN = F.y[jf] - F.y[jf - 1];
            const T dyf = T(F.iy[jf - 1]);
            return (T(dN) * Px(k, jf - 1) + T(dS) * Px(k, jf + 1)) * dyf;
        };
        T v;
        if (ZF == 1 || ((kf - 2) % 2) == 0) v = Py(kf);
        else {
            const double dD = F.z[kf - 1] - F.z[kf - 2], dU = F.z[kf] - F.z[kf - 1];
            const T dzf = T(F.iz[kf - 1]);
            v = (T(dU) * Py(kf - 1) + T(dD) * Py(kf + 1)) * dzf;
        }
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
