// High-order sigma-transformed Laplace operator, y = A(eta) phi.
//
// Restates BuildLinearSystem (src/functions/BuildLinearSystem.f90:1-290) with
// the derivative routines DiffXEven/DiffYEven/DiffZArbitrary and the
// corner-corrected mixed derivatives DiffXEven_CD/DiffZArbitrary_CD whose
// index tables ConstructTableCrossDerivatives.f90:90-264 builds. Instead of
// the reference's per-point index/weight tables and its five 3-D sigma
// coefficient arrays (DetermineTransformationConstantsArray.f90), the kernel
// applies the table rules in closed form and recomputes the sigma
// coefficients per column from eta, h and their horizontal derivatives.
//
// Work decomposition (one launch):
//  * interior tiles: the columns at least kBand points from every wall, in
//    tiles of BX x BY columns, one thread per column. A tile stages phi of
//    its columns plus a halo of 3 in shared memory (odd column pitch: the
//    column-per-thread accesses are free of bank conflicts). Inside the
//    bands every x/y stencil is the centred one, which is a kernel parameter
//    (constant bank), as are the sigma stencils. A thread walks its column
//    bottom to top, forms d/dx, d/dy and the horizontal Laplacian of each
//    level once, and emits each row of y as soon as the last level of its
//    sigma stencil has been read, so only a window of levels is live;
//  * wall bands: the ghost columns and the columns within kBand points of a
//    wall (one-sided windows, shifted windows below the bottom), one thread
//    per column reading phi from global memory, per-position stencils from
//    the tables. These blocks come first in the grid so that they start
//    early and overlap the tiles.
#include "ow3d_internal.h"
#include <cstring>

namespace ow3d {

namespace {

constexpr int kZMax = 34;   // largest Nzg the library accepts (Nz <= 33)
constexpr int kBand = 5;    // columns from each wall handled by the band path

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
// Levels of a tile's first staging group: the rows these complete are
// computed while the remaining levels are still arriving.
__host__ __device__ constexpr int stage_split(int nzg) { return nzg > 0 ? (nzg + 2) / 2 : 0; }

__device__ __forceinline__ int win_start(int i, int n) {  // 1-based DiffXEven window start, half width 3
    return i <= 3 ? 1 : (i <= n - 3 ? i - 3 : n - 6);
}
// first level of the sigma stencil of row k (DiffZArbitrary, PreProcessDiffStencils.f90:108-132)
__host__ __device__ constexpr int zwin(int k, int nzg) { return k <= 3 ? 1 : (k <= nzg - 3 ? k - 3 : nzg - 6); }
// last level that row k of y depends on
__host__ __device__ constexpr int zlast(int k, int nzg) {
    return k == nzg ? nzg : (k == 1 ? zwin(2, nzg) + 6 : zwin(k, nzg) + 6);
}

template <int NZ>
struct ZTab {
    double s1[NZ][kHoRank];   // d/dsigma stencil of row k
    double s2[NZ][kHoRank];   // d2/dsigma2 stencil of row k
    double zs[NZ];            // sigma levels, zs[0] = 0
    double cx[2][kHoRank];    // the centred x stencil (orders 1, 2) of every interior position
    double cy[2][kHoRank];    // the centred y stencil
};

template <bool THREE>
struct Tile {
    static constexpr int BX = THREE ? 32 : 256;
    static constexpr int BY = THREE ? 8 : 1;
    static constexpr int HX = BX + 6;                 // staged columns in x (halo 3)
    static constexpr int HY = THREE ? BY + 6 : 1;     // staged rows in y
};

// Sigma-transformation coefficients of column col (linear in sigma).
struct ColCoef {
    double id, a2, b2, a4, b4, a3, b3, hx, hy;
};
template <bool THREE>
__device__ __forceinline__ ColCoef col_coef(const HoGrid& g, const Surface& s, int64_t col) {
    double E = 0, Ex = 0, Exx = 0, Ey = 0, Eyy = 0;
    if (g.nonlinear) {
        if (s.E) E = s.E[col];
        if (s.Ex) Ex = s.Ex[col];
        if (s.Exx) Exx = s.Exx[col];
        if (THREE) { if (s.Ey) Ey = s.Ey[col]; if (s.Eyy) Eyy = s.Eyy[col]; }
    }
    ColCoef c;
    c.hx = g.hx[col];
    const double hxx = g.hxx[col];
    c.hy = THREE ? g.hy[col] : 0.0;
    const double hyy = THREE ? g.hyy[col] : 0.0;
    const double d = E + g.h[col];
    c.id = 1.0 / d;
    const double id2 = c.id * c.id;
    c.a2 = c.hx * c.id; c.b2 = -(c.hx + Ex) * c.id;
    c.a4 = c.hy * c.id; c.b4 = -(c.hy + Ey) * c.id;
    const double P1 = -2.0 * (c.hx * c.hx + c.hy * c.hy) * id2 + (hxx + hyy) * c.id;
    const double P2 = 2.0 * (Ex * c.hx + Ey * c.hy) * id2;
    const double P3 = 2.0 * (Ex * Ex + Ey * Ey) * id2 - (Exx + Eyy) * c.id;
    c.a3 = P1 - P2; c.b3 = P3 + 2.0 * P2 - P1;
    return c;
}

// ---------------------------------------------------------------- wall bands
// Band column q -> (i, j); with `all`, every column of the grid.
__device__ __forceinline__ void band_col(int64_t q, int Nxg, int Nyg, bool all, int& i, int& j) {
    if (all) {
        j = (int)(q / Nxg) + 1;
        i = (int)(q - (int64_t)(j - 1) * Nxg) + 1;
        return;
    }
    const int64_t nx = 2 * kBand;
    if (q < nx * Nyg) {
        j = (int)(q / nx) + 1;
        const int r = (int)(q - (int64_t)(j - 1) * nx);
        i = r < kBand ? r + 1 : Nxg - (int)nx + 1 + r;
        return;
    }
    q -= nx * Nyg;   // y bands (3-D only), interior x positions
    const int w = Nxg - 2 * kBand;
    const int t = (int)(q / w);
    i = kBand + 1 + (int)(q - (int64_t)t * w);
    j = t < kBand ? t + 1 : Nyg - 2 * kBand + 1 + t;
}

// One column (i, j) of any kind, phi read from global memory, per-position
// stencils from the tables: the general path.
template <bool THREE, typename TIN, typename ZT>
__device__ void ho_column_general(const HoGrid& g, const Surface& s, const TIN* __restrict__ phi, double scale,
                                  const double* __restrict__ b, double* __restrict__ y, int mode, const ZT& zt,
                                  int i, int j) {
    const int Nxg = g.Nxg, Nyg = g.Nyg, Nzg = g.Nzg;
    auto P = [&](int k, int ii, int jj) -> double {   // 1-based
        return (double)__ldg(phi + (int64_t)(k - 1) + (int64_t)Nzg * ((int64_t)(ii - 1) + (int64_t)Nxg * (jj - 1)));
    };
    const double* SX1 = g.SX;
    const double* SX2 = g.SX + (int64_t)Nxg * kHoRank;
    const double* SY1 = g.SY;
    const double* SY2 = g.SY + (int64_t)Nyg * kHoRank;
    const int64_t col = (int64_t)(i - 1) + (int64_t)Nxg * (j - 1);
    const int64_t gb = col * Nzg;
    auto emit = [&](int k, double v) {
        if (mode == 0) y[gb + k - 1] = scale * v;
        else y[gb + k - 1] = b[gb + k - 1] - v;
    };
    const bool ghost_x = (i == 1 || i == Nxg);
    const bool ghost_y = THREE && (j == 1 || j == Nyg);
    if (g.per && (ghost_x || i == Nxg - 1)) {
        // periodic x: ghost and repeated columns are identity rows
        for (int k = 1; k <= Nzg; ++k) emit(k, P(k, i, j));
        return;
    }
    if (ghost_x || ghost_y) {
        // Lateral Neumann rows and identity corners (BuildLinearSystem.f90:150-284)
        const bool corner = ghost_x && ghost_y;
        for (int k = 1; k <= Nzg; ++k) {
            double v;
            if (corner || k == 1) v = P(k, i, j);
            else if (ghost_x) {
                const int ia = (i == 1) ? 2 : Nxg - 1, ws = win_start(ia, Nxg);
                v = 0.0;
                for (int m = 0; m < kHoRank; ++m) v += SX1[(ia - 1) * kHoRank + m] * P(k, ws + m, j);
            } else {
                const int ja = (j == 1) ? 2 : Nyg - 1, ws = win_start(ja, Nyg);
                v = 0.0;
                for (int m = 0; m < kHoRank; ++m) v += SY1[(ja - 1) * kHoRank + m] * P(k, i, ws + m);
            }
            emit(k, v);
        }
        return;
    }
    // pass 1: horizontal derivatives at every level (periodic x: the centred
    // window, its columns taken cyclically)
    double tx[kZMax], ty[kZMax], lap[kZMax], pc[kZMax];
    const int wsx = g.per ? i - 3 : win_start(i, Nxg);
    const int wsy = THREE ? win_start(j, Nyg) : 1;
    for (int k = 1; k <= Nzg; ++k) {
        double dx = 0, dxx = 0;
        for (int m = 0; m < kHoRank; ++m) {
            const double v = P(k, g.per ? wrap_x(wsx + m, Nxg) : wsx + m, j);
            dx += SX1[(i - 1) * kHoRank + m] * v;
            dxx += SX2[(i - 1) * kHoRank + m] * v;
        }
        double dy = 0, dyy = 0;
        if (THREE) {
            for (int m = 0; m < kHoRank; ++m) {
                const double v = P(k, i, wsy + m);
                dy += SY1[(j - 1) * kHoRank + m] * v;
                dyy += SY2[(j - 1) * kHoRank + m] * v;
            }
        }
        tx[k - 1] = dx; ty[k - 1] = dy; lap[k - 1] = dxx + dyy;
        pc[k - 1] = P(k, i, j);
    }
    // Level k = 1 (below the bottom): the x/y derivative entering the mixed
    // derivative avoids the ghost corner columns (ConstructTableCrossDerivatives.f90:173-186,231-235).
    {
        int sh = 0;
        if (!g.per && wsx == 1) sh = 1;
        if (!g.per && wsx + 6 == Nxg) sh = -1;
        if (sh != 0) {
            double dx = 0;
            for (int m = 0; m < kHoRank; ++m) dx += SX1[(i - sh - 1) * kHoRank + m] * P(1, wsx + sh + m, j);
            tx[0] = dx;
        }
        if (THREE) {
            int shy = 0;
            if (wsy == 1) shy = 1;
            if (wsy + 6 == Nyg) shy = -1;
            if (shy != 0) {
                double dy = 0;
                for (int m = 0; m < kHoRank; ++m) dy += SY1[(j - shy - 1) * kHoRank + m] * P(1, i, wsy + shy + m);
                ty[0] = dy;
            }
        }
    }
    const ColCoef c = col_coef<THREE>(g, s, col);
    // pass 2: rows of this column
    for (int k = 1; k <= Nzg; ++k) {
        double v;
        if (k == Nzg) {
            v = pc[k - 1];  // free surface, Dirichlet
        } else if (k == 1) {
            // kinematic bottom condition evaluated at k = 2 (BuildLinearSystem.f90:121-126)
            const double z2 = zt.zs[1];
            const double s2 = fma(z2, c.b2, c.a2), s4 = fma(z2, c.b4, c.a4);
            double dz = 0;
            for (int m = 0; m < kHoRank; ++m) dz += zt.s1[1][m] * pc[m];
            v = (c.id + c.hx * s2 + c.hy * s4) * dz + c.hx * tx[1] + c.hy * ty[1];
        } else {
            const int wz = zwin(k, Nzg);
            const double sg = zt.zs[k - 1];
            const double s2 = fma(sg, c.b2, c.a2), s4 = fma(sg, c.b4, c.a4), s3 = fma(sg, c.b3, c.a3);
            double dz = 0, dzz = 0, dzx = 0, dzy = 0;
            for (int m = 0; m < kHoRank; ++m) {
                const double w1 = zt.s1[k - 1][m], w2 = zt.s2[k - 1][m];
                const int kk = wz + m - 1;
                dz += w1 * pc[kk];
                dzz += w2 * pc[kk];
                dzx += w1 * tx[kk];
                if (THREE) dzy += w1 * ty[kk];
            }
            const double cz = s2 * s2 + s4 * s4 + c.id * c.id;
            v = lap[k - 1] + s3 * dz + 2.0 * (s2 * dzx + s4 * dzy) + cz * dzz;
        }
        emit(k, v);
    }
}

// ------------------------------------------------------------ interior tiles
// Interior column (i, j) of a tile; P(k, di, dj) reads the staged phi at
// (i + di, j + dj). NZG > 0: levels unrolled, rows emitted as their windows
// complete; NZG == 0: any Nzg, two passes.
template <int NZG, bool THREE, typename ZT, typename PF>
__device__ __forceinline__ void ho_column_tile(const HoGrid& g, const Surface& s, double scale,
                                               const double* __restrict__ b, double* __restrict__ y, int mode,
                                               const ZT& zt, int i, int j, bool active, const PF& P) {
    constexpr int ZA = NZG > 0 ? NZG : kZMax;
    const int Nzg = NZG > 0 ? NZG : g.Nzg;
    const int64_t col = (int64_t)(i - 1) + (int64_t)g.Nxg * (j - 1);
    const int64_t gb = col * Nzg;
    auto emit = [&](int k, double v) {
        if (!active) return;
        if (mode == 0) y[gb + k - 1] = scale * v;
        else y[gb + k - 1] = b[gb + k - 1] - v;
    };
    const ColCoef c = col_coef<THREE>(g, s, col);
    double pw[ZA], tx[ZA], ty[ZA], lap[ZA];
    auto level = [&](int kk) {
        double dx = 0, dxx = 0, dy = 0, dyy = 0;
#pragma unroll
        for (int m = 0; m < kHoRank; ++m) {
            const double v = P(kk, m - 3, 0);
            dx = fma(zt.cx[0][m], v, dx);
            dxx = fma(zt.cx[1][m], v, dxx);
            if (m == 3) pw[kk - 1] = v;
        }
        if (THREE) {
#pragma unroll
            for (int m = 0; m < kHoRank; ++m) {
                const double v = (m == 3) ? pw[kk - 1] : P(kk, 0, m - 3);
                dy = fma(zt.cy[0][m], v, dy);
                dyy = fma(zt.cy[1][m], v, dyy);
            }
        }
        tx[kk - 1] = dx;
        ty[kk - 1] = dy;
        lap[kk - 1] = dxx + dyy;
    };
    auto row = [&](int k) -> double {
        if (k == Nzg) return pw[k - 1];   // free surface, Dirichlet
        if (k == 1) {
            // kinematic bottom condition evaluated at k = 2 (BuildLinearSystem.f90:121-126)
            const double z2 = zt.zs[1];
            const double s2 = fma(z2, c.b2, c.a2), s4 = fma(z2, c.b4, c.a4);
            double dz = 0;
#pragma unroll
            for (int m = 0; m < kHoRank; ++m) dz += zt.s1[1][m] * pw[m];
            return (c.id + c.hx * s2 + c.hy * s4) * dz + c.hx * tx[1] + c.hy * ty[1];
        }
        const int wz = zwin(k, Nzg);
        const double sg = zt.zs[k - 1];
        const double s2 = fma(sg, c.b2, c.a2), s4 = fma(sg, c.b4, c.a4), s3 = fma(sg, c.b3, c.a3);
        double dz = 0, dzz = 0, dzx = 0, dzy = 0;
#pragma unroll
        for (int m = 0; m < kHoRank; ++m) {
            const double w1 = zt.s1[k - 1][m], w2 = zt.s2[k - 1][m];
            const int q = wz + m - 1;
            dz += w1 * pw[q];
            dzz += w2 * pw[q];
            dzx += w1 * tx[q];
            if (THREE) dzy += w1 * ty[q];
        }
        const double cz = s2 * s2 + s4 * s4 + c.id * c.id;
        return lap[k - 1] + s3 * dz + 2.0 * (s2 * dzx + s4 * dzy) + cz * dzz;
    };
    if constexpr (NZG > 0) {
#pragma unroll
        for (int kk = 1; kk <= NZG; ++kk) {
            if (kk == stage_split(NZG) + 1) {   // the upper levels of the tile
                cp_wait<0>();
                __syncthreads();
            }
            level(kk);
#pragma unroll
            for (int k = 1; k <= NZG; ++k)
                if (zlast(k, NZG) == kk) emit(k, row(k));
        }
    } else {
        for (int kk = 1; kk <= Nzg; ++kk) level(kk);
        for (int k = 1; k <= Nzg; ++k) emit(k, row(k));
    }
}

template <int NZG, bool THREE, typename TIN>
__global__ void __launch_bounds__(THREE ? 256 : 256, 2)
    k_ho_matvec(HoGrid g, Surface s, const TIN* __restrict__ phi, const double* __restrict__ dscale,
                const double* __restrict__ b, double* __restrict__ y, int mode,
                const __grid_constant__ ZTab<(NZG > 0 ? NZG : kZMax)> zt, int band_blocks, int64_t nband, int all,
                int tiles_x) {
    pdl_entry();
    constexpr int BX = Tile<THREE>::BX, BY = Tile<THREE>::BY, HX = Tile<THREE>::HX, HY = Tile<THREE>::HY;
    const int Nxg = g.Nxg, Nyg = g.Nyg, Nzg = NZG > 0 ? NZG : g.Nzg;
    const double scale = dscale ? *dscale : 1.0;
    const int tid = threadIdx.x;
    if ((int)blockIdx.x < band_blocks) {
        const int64_t q = (int64_t)blockIdx.x * blockDim.x + tid;
        if (q >= nband) return;
        int i, j;
        band_col(q, Nxg, Nyg, all != 0, i, j);
        ho_column_general<THREE, TIN>(g, s, phi, scale, b, y, mode, zt, i, j);
        return;
    }
    // interior tile: columns i0..i0+BX-1 (x), j0..j0+BY-1 (y) inside [kBand+1, N-kBand]
    extern __shared__ __align__(16) unsigned char smraw[];
    TIN* const sm = reinterpret_cast<TIN*>(smraw);
    const int NZP = Nzg | 1;   // odd column pitch
    const int t = (int)blockIdx.x - band_blocks;
    const int ty_ = t / tiles_x, tx_ = t - ty_ * tiles_x;
    const int i0 = kBand + 1 + tx_ * BX;
    const int j0 = THREE ? kBand + 1 + ty_ * BY : 1;
    const int ilo = i0 - 3, jlo = THREE ? j0 - 3 : 1;
    // stage with cp.async in two groups, levels [0, KA) then [KA, Nzg); each
    // staged y row's column range is contiguous in global memory
    constexpr int KA0 = stage_split(NZG);
    const int KA = NZG > 0 ? KA0 : Nzg;
    const int ncolx = min(HX, Nxg - ilo + 1);
    auto stage = [&](int k0, int k1) {
        const int nk = k1 - k0;
        if (nk <= 0) return;
        for (int r = 0; r < HY; ++r) {
            const int jj = jlo + r;
            if (jj > Nyg) break;
            const TIN* src = phi + ((int64_t)(jj - 1) * Nxg + (ilo - 1)) * Nzg;
            TIN* dst = sm + (int64_t)r * HX * NZP;
            const int cnt = ncolx * nk;
            for (int e = tid; e < cnt; e += blockDim.x) {
                const int cc = e / nk, k = k0 + (e - cc * nk);
                cp_async<sizeof(TIN)>(dst + cc * NZP + k, src + (int64_t)cc * Nzg + k);
            }
        }
    };
    stage(0, KA);
    cp_commit();
    stage(KA, Nzg);
    cp_commit();
    if (NZG > 0) cp_wait<1>();
    else cp_wait<0>();
    __syncthreads();
    // every thread stays to the end (the tile's second barrier); threads past
    // the interior work on the nearest interior column and store nothing
    const int lx = tid % BX, ly = tid / BX;
    const int i = i0 + lx, j = j0 + ly;
    const bool active = i <= Nxg - kBand && (!THREE || j <= Nyg - kBand);
    const int ic = min(i, Nxg - kBand), jc = THREE ? min(j, Nyg - kBand) : 1;
    const TIN* base = sm + ((int64_t)(jc - j0 + (THREE ? 3 : 0)) * HX + (ic - i0 + 3)) * NZP;
    auto P = [&](int k, int di, int dj) -> double { return (double)base[((int64_t)dj * HX + di) * NZP + (k - 1)]; };
    ho_column_tile<NZG, THREE>(g, s, scale, b, y, mode, zt, ic, jc, active, P);
}

template <int NZG, bool THREE, typename TIN>
void launch_impl(const HoGrid& g, const Surface& s, const TIN* phi, const double* scale, const double* b, double* y,
                 int mode, cudaStream_t st) {
    constexpr int ZA = NZG > 0 ? NZG : kZMax;
    constexpr int BX = Tile<THREE>::BX, BY = Tile<THREE>::BY, HX = Tile<THREE>::HX, HY = Tile<THREE>::HY;
    ZTab<ZA> zt;
    std::memset(&zt, 0, sizeof(zt));
    for (int k = 0; k < g.Nzg && k < ZA; ++k) {
        for (int m = 0; m < kHoRank; ++m) {
            zt.s1[k][m] = g.hSZ[k * kHoRank + m];
            zt.s2[k][m] = g.hSZ[((int64_t)g.Nzg + k) * kHoRank + m];
        }
        zt.zs[k] = g.hzs[k];
    }
    // centred x / y stencils, and whether every position outside the wall
    // bands carries exactly them (then the tiles may use them)
    bool uniform = true;
    auto centred = [&](const double* tab, int n, double (*c)[kHoRank]) {
        const int r = n / 2;   // 0-based representative interior position
        for (int o = 0; o < 2; ++o)
            for (int m = 0; m < kHoRank; ++m) c[o][m] = tab[((int64_t)o * n + r) * kHoRank + m];
        for (int o = 0; o < 2; ++o)
            for (int q = kBand; q < n - kBand; ++q)
                for (int m = 0; m < kHoRank; ++m)
                    if (tab[((int64_t)o * n + q) * kHoRank + m] != c[o][m]) uniform = false;
    };
    centred(g.hSX, g.Nxg, zt.cx);
    if (THREE) centred(g.hSY, g.Nyg, zt.cy);
    const bool split = uniform && g.Nxg > 2 * kBand && (!THREE || g.Nyg > 2 * kBand);
    int64_t nband;
    int tiles_x = 1, tiles = 0;
    if (split) {
        nband = (int64_t)2 * kBand * g.Nyg + (THREE ? (int64_t)2 * kBand * (g.Nxg - 2 * kBand) : 0);
        tiles_x = (g.Nxg - 2 * kBand + BX - 1) / BX;
        const int tiles_y = THREE ? (g.Nyg - 2 * kBand + BY - 1) / BY : 1;
        tiles = tiles_x * tiles_y;
    } else {
        nband = (int64_t)g.Nxg * g.Nyg;
    }
    const int threads = BX * BY;
    const int band_blocks = (int)((nband + threads - 1) / threads);
    const int NZP = g.Nzg | 1;
    const size_t smem = (size_t)HX * HY * NZP * sizeof(TIN);
    // the shared-memory opt-in is per device; setting it twice is harmless,
    // so concurrent first launches from several host threads need no lock
    static std::atomic<unsigned long long> attr_set{0ull};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_set.load(std::memory_order_relaxed) & bit)) {
        cudaFuncSetAttribute(k_ho_matvec<NZG, THREE, TIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set.fetch_or(bit, std::memory_order_relaxed);
    }
    launch_k(k_ho_matvec<NZG, THREE, TIN>, dim3(band_blocks + tiles), dim3(threads), smem, st, 
        g, s, phi, scale, b, y, mode, zt, band_blocks, nband, split ? 0 : 1, tiles_x);
}

template <bool THREE, typename TIN>
void dispatch_nz(const HoGrid& g, const Surface& s, const TIN* phi, const double* scale, const double* b, double* y,
                 int mode, cudaStream_t st) {
    switch (g.Nzg) {
        case 8: launch_impl<8, THREE, TIN>(g, s, phi, scale, b, y, mode, st); break;
        case 10: launch_impl<10, THREE, TIN>(g, s, phi, scale, b, y, mode, st); break;
        case 14: launch_impl<14, THREE, TIN>(g, s, phi, scale, b, y, mode, st); break;
        case 18: launch_impl<18, THREE, TIN>(g, s, phi, scale, b, y, mode, st); break;
        default: launch_impl<0, THREE, TIN>(g, s, phi, scale, b, y, mode, st); break;
    }
}

}  // namespace

template <typename TIN>
void launch_ho_matvec(const HoGrid& g, const Surface& s, const TIN* phi, const double* scale, const double* b,
                      double* y, int mode, cudaStream_t st) {
    if (g.three) dispatch_nz<true, TIN>(g, s, phi, scale, b, y, mode, st);
    else dispatch_nz<false, TIN>(g, s, phi, scale, b, y, mode, st);
}

template void launch_ho_matvec<double>(const HoGrid&, const Surface&, const double*, const double*, const double*,
                                       double*, int, cudaStream_t);
template void launch_ho_matvec<float>(const HoGrid&, const Surface&, const float*, const double*, const double*,
                                      double*, int, cudaStream_t);

}  // namespace ow3d
