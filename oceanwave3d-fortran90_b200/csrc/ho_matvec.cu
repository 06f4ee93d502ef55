// High-order sigma-transformed Laplace operator, y = A(eta) phi.
//
// Restates BuildLinearSystem (src/functions/BuildLinearSystem.f90:1-290) with
// the derivative routines DiffXEven/DiffYEven/DiffZArbitrary and the
// corner-corrected mixed derivatives DiffXEven_CD/DiffZArbitrary_CD whose
// index tables ConstructTableCrossDerivatives.f90:90-264 builds. Instead of
// the reference's per-point index/weight tables and its five 3-D sigma
// coefficient arrays (DetermineTransformationConstantsArray.f90), the kernel
// derives the table rules in closed form and recomputes the sigma
// coefficients per column from eta, h and their horizontal derivatives.
//
// Work decomposition: one thread per water column (i,j) holding the whole
// sigma column in registers; a CTA covers BX x BY columns and stages the
// planes j-3..j+3 (x-halo 3) of phi in shared memory with a padded column
// stride (odd number of doubles: bank-conflict free for the column-per-thread
// access pattern).
#include "ow3d_internal.h"
#include <cstdio>

namespace ow3d {

namespace {

__device__ __forceinline__ int win_start(int i, int n) {  // 1-based DiffXEven window start, half width 3
    return i <= 3 ? 1 : (i <= n - 3 ? i - 3 : n - 6);
}

template <int NZG>
struct NzgT { static constexpr int v = NZG; };

template <int NZG, bool THREE, typename TIN>
__global__ void __launch_bounds__(128) k_ho_matvec(HoGrid g, Surface s, const TIN* __restrict__ phi, const double* __restrict__ dscale,
                                                   const double* __restrict__ b, double* __restrict__ y, int mode,
                                                   int BX, int BY) {
    extern __shared__ double sm[];
    constexpr int ZMAX = NZG > 0 ? NZG : kMaxNzg;
    const int Nxg = g.Nxg, Nyg = g.Nyg, Nzg = NZG > 0 ? NZG : g.Nzg;
    const int NZP = Nzg | 1;  // padded column stride (odd)
    const int i0 = blockIdx.x * BX + 1, j0 = blockIdx.y * BY + 1;
    const int ilast = min(i0 + BX - 1, Nxg), jlast = min(j0 + BY - 1, Nyg);
    // staged ranges (1-based, inclusive)
    const int ilo = max(1, win_start(i0, Nxg) - 1), ihi = min(Nxg, win_start(ilast, Nxg) + 7);
    int jlo = 1, jhi = 1;
    if (THREE) { jlo = max(1, win_start(j0, Nyg) - 1); jhi = min(Nyg, win_start(jlast, Nyg) + 7); }
    const int ncol = ihi - ilo + 1, npl = jhi - jlo + 1;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y, nth = blockDim.x * blockDim.y;
    // cooperative staging: each plane's column range is contiguous in global memory
    for (int p = 0; p < npl; ++p) {
        const int64_t gbase = ((int64_t)(jlo + p - 1) * Nxg + (ilo - 1)) * Nzg;
        const int cnt = ncol * Nzg;
        double* dst = sm + (int64_t)p * ncol * NZP;
        for (int e = tid; e < cnt; e += nth) {
            int c = e / Nzg, k = e - c * Nzg;
            dst[c * NZP + k] = (double)phi[gbase + e];
        }
    }
    __syncthreads();
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    if (i > Nxg || j > Nyg) return;
    auto P = [&](int k, int ii, int jj) -> double {  // 1-based
        return sm[((int64_t)(jj - jlo) * ncol + (ii - ilo)) * NZP + (k - 1)];
    };
    const double* SX1 = g.SX;
    const double* SX2 = g.SX + (int64_t)Nxg * kHoRank;
    const double* SY1 = g.SY;
    const double* SY2 = g.SY + (int64_t)Nyg * kHoRank;
    const double* SZ1 = g.SZ;
    const double* SZ2 = g.SZ + (int64_t)Nzg * kHoRank;
    const int64_t col = (int64_t)(i - 1) + (int64_t)Nxg * (j - 1);
    const int64_t gb = col * Nzg;
    const bool ghost_x = (i == 1 || i == Nxg);
    const bool ghost_y = THREE && (j == 1 || j == Nyg);
    const double scale = dscale ? *dscale : 1.0;
    auto emit = [&](int k, double v) {
        if (mode == 0) y[gb + k - 1] = scale * v;
        else y[gb + k - 1] = b[gb + k - 1] - v;
    };
    if (ghost_x || ghost_y) {
        // Lateral Neumann rows and identity corners (BuildLinearSystem.f90:150-284)
        const bool corner = ghost_x && ghost_y;
        for (int k = 1; k <= Nzg; ++k) {
            double v;
            if (corner || k == 1) v = P(k, i, j);
            else if (ghost_x) {
                int ia = (i == 1) ? 2 : Nxg - 1, ws = win_start(ia, Nxg);
                v = 0.0;
#pragma unroll
                for (int m = 0; m < kHoRank; ++m) v += SX1[(ia - 1) * kHoRank + m] * P(k, ws + m, j);
            } else {
                int ja = (j == 1) ? 2 : Nyg - 1, ws = win_start(ja, Nyg);
                v = 0.0;
#pragma unroll
                for (int m = 0; m < kHoRank; ++m) v += SY1[(ja - 1) * kHoRank + m] * P(k, i, ws + m);
            }
            emit(k, v);
        }
        return;
    }
    // ---- interior column: pass 1, horizontal derivatives at every level
    double tx[ZMAX], ty[ZMAX], lap[ZMAX], pc[ZMAX];
    const int wsx = win_start(i, Nxg);
    const int wsy = THREE ? win_start(j, Nyg) : 1;
    double sx1[kHoRank], sx2[kHoRank], sy1[kHoRank], sy2[kHoRank];
#pragma unroll
    for (int m = 0; m < kHoRank; ++m) {
        sx1[m] = SX1[(i - 1) * kHoRank + m];
        sx2[m] = SX2[(i - 1) * kHoRank + m];
        if (THREE) { sy1[m] = SY1[(j - 1) * kHoRank + m]; sy2[m] = SY2[(j - 1) * kHoRank + m]; }
    }
#pragma unroll
    for (int k = 1; k <= ZMAX; ++k) {
        if (NZG == 0 && k > Nzg) break;
        double dx = 0, dxx = 0;
#pragma unroll
        for (int m = 0; m < kHoRank; ++m) {
            double v = P(k, wsx + m, j);
            dx += sx1[m] * v;
            dxx += sx2[m] * v;
        }
        double dy = 0, dyy = 0;
        if (THREE) {
#pragma unroll
            for (int m = 0; m < kHoRank; ++m) {
                double v = P(k, i, wsy + m);
                dy += sy1[m] * v;
                dyy += sy2[m] * v;
            }
        }
        tx[k - 1] = dx; ty[k - 1] = dy; lap[k - 1] = dxx + dyy;
        pc[k - 1] = P(k, i, j);
    }
    // Level k = 1 (below the bottom): the x/y derivative entering the mixed
    // derivative avoids the ghost corner columns (ConstructTableCrossDerivatives.f90:173-186,231-235).
    {
        int sh = 0;
        if (wsx == 1) sh = 1;
        if (wsx + 6 == Nxg) sh = -1;
        if (sh != 0) {
            double dx = 0;
#pragma unroll
            for (int m = 0; m < kHoRank; ++m) dx += SX1[(i - sh - 1) * kHoRank + m] * P(1, wsx + sh + m, j);
            tx[0] = dx;
        }
        if (THREE) {
            int shy = 0;
            if (wsy == 1) shy = 1;
            if (wsy + 6 == Nyg) shy = -1;
            if (shy != 0) {
                double dy = 0;
#pragma unroll
                for (int m = 0; m < kHoRank; ++m) dy += SY1[(j - shy - 1) * kHoRank + m] * P(1, i, wsy + shy + m);
                ty[0] = dy;
            }
        }
    }
    // ---- sigma coefficients of this column (linear in sigma)
    double E = 0, Ex = 0, Exx = 0, Ey = 0, Eyy = 0;
    if (g.nonlinear) {
        if (s.E) E = s.E[col];
        if (s.Ex) Ex = s.Ex[col];
        if (s.Exx) Exx = s.Exx[col];
        if (THREE) { if (s.Ey) Ey = s.Ey[col]; if (s.Eyy) Eyy = s.Eyy[col]; }
    }
    const double hx = g.hx[col], hxx = g.hxx[col];
    const double hy = THREE ? g.hy[col] : 0.0, hyy = THREE ? g.hyy[col] : 0.0;
    const double d = E + g.h[col], id = 1.0 / d, id2 = id * id;
    const double a2 = hx * id, b2 = -(hx + Ex) * id;
    const double a4 = hy * id, b4 = -(hy + Ey) * id;
    const double P1 = -2.0 * (hx * hx + hy * hy) * id2 + (hxx + hyy) * id;
    const double P2 = 2.0 * (Ex * hx + Ey * hy) * id2;
    const double P3 = 2.0 * (Ex * Ex + Ey * Ey) * id2 - (Exx + Eyy) * id;
    const double a3 = P1 - P2, b3 = P3 + 2.0 * P2 - P1;
    // ---- pass 2: rows of this column
#pragma unroll
    for (int k = 1; k <= ZMAX; ++k) {
        if (NZG == 0 && k > Nzg) break;
        double v;
        if (k == Nzg) {
            v = pc[k - 1];  // free surface, Dirichlet
        } else if (k == 1) {
            // kinematic bottom condition evaluated at k = 2 (BuildLinearSystem.f90:121-126)
            const double z2 = g.zs[1];
            const double s2 = fma(z2, b2, a2), s4 = fma(z2, b4, a4);
            double dz = 0;
#pragma unroll
            for (int m = 0; m < kHoRank; ++m) dz += SZ1[1 * kHoRank + m] * pc[m];
            v = (id + hx * s2 + hy * s4) * dz + hx * tx[1] + hy * ty[1];
        } else {
            const int wz = k <= 3 ? 1 : (k <= Nzg - 3 ? k - 3 : Nzg - 6);
            const double sg = g.zs[k - 1];
            const double s2 = fma(sg, b2, a2), s4 = fma(sg, b4, a4), s3 = fma(sg, b3, a3);
            double dz = 0, dzz = 0, dzx = 0, dzy = 0;
#pragma unroll
            for (int m = 0; m < kHoRank; ++m) {
                const double w1 = SZ1[(k - 1) * kHoRank + m], w2 = SZ2[(k - 1) * kHoRank + m];
                const int kk = wz + m - 1;
                dz += w1 * pc[kk];
                dzz += w2 * pc[kk];
                dzx += w1 * tx[kk];
                if (THREE) dzy += w1 * ty[kk];
            }
            const double cz = s2 * s2 + s4 * s4 + id * id;
            v = lap[k - 1] + s3 * dz + 2.0 * (s2 * dzx + s4 * dzy) + cz * dzz;
        }
        emit(k, v);
    }
}

template <int NZG, bool THREE, typename TIN>
void launch_impl(const HoGrid& g, const Surface& s, const TIN* phi, const double* scale, const double* b, double* y, int mode,
                 cudaStream_t st) {
    const int BX = THREE ? 32 : 128, BY = THREE ? 4 : 1;
    dim3 blk(BX, BY), grd((g.Nxg + BX - 1) / BX, (g.Nyg + BY - 1) / BY);
    const int NZP = g.Nzg | 1;
    size_t smem = (size_t)(THREE ? BY + 9 : 1) * (BX + 9) * NZP * sizeof(double);
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
    note_launch(), k_ho_matvec<NZG, THREE, TIN><<<grd, blk, smem, st>>>(g, s, phi, scale, b, y, mode, BX, BY);
}

template <bool THREE, typename TIN>
void dispatch_nz(const HoGrid& g, const Surface& s, const TIN* phi, const double* scale, const double* b, double* y, int mode,
                 cudaStream_t st) {
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
