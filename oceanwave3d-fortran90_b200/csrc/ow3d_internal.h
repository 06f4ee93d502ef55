// Internal declarations of the B200 OceanWave3D hot path.
//
// Device layout (all simulations): the reference's Fortran layout is kept as
// is, so host arrays are copied without transposition:
//   3-D fields  PHI(k,i,j): k (sigma) fastest, then x, then y,
//               index (k-1) + Nzg*((i-1) + Nxg*(j-1))  (1-based k,i,j)
//   2-D fields  E(i,j):     i fastest, index (i-1) + Nxg*(j-1)
// Ghost points are included (one layer in x, y and below the bottom).
#pragma once
#include <atomic>
#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>
#include "../../include/ow3d.h"

namespace ow3d {

// Kernels launched by this library since load (all handles, all threads).
extern std::atomic<unsigned long long> g_kernel_launches;
inline void note_launch() { g_kernel_launches.fetch_add(1ull, std::memory_order_relaxed); }

constexpr int kMaxLevels = 16;
constexpr int kMaxKrylov = 64;     // maximum GMRESmaxiterations
constexpr int kHoRank = 7;         // 6th-order operator, half width 3
constexpr int kMaxNzg = 64;

// ------------------------------------------------------------------ grids
// High-order (fine) operator description, BuildLinearSystem.f90:1-290.
struct HoGrid {
    int Nxg, Nyg, Nzg;      // with ghosts
    int gx, gy;             // ghost layers present in x / y (0 in a 2-D direction)
    int three;              // 1: 3-D (Nx>1 and Ny>1); 0: 2-D in x (Ny == 1)
    int nonlinear;          // sigma coefficients from eta (LinearONOFF == 1)
    // per-position stencils, [order-1][pos][7], order 1 and 2 (BuildStencilsGridX.f90)
    const double* SX;       // 2*Nxg*7
    const double* SY;       // 2*Nyg*7 (unused in 2-D)
    const double* SZ;       // 2*Nzg*7 (PreProcessDiffStencils.f90:108-132)
    const double* zs;       // sigma levels with zs[0] = 0 (DetermineTransformationConstantsArray.f90:59)
    const double *h, *hx, *hxx, *hy, *hyy;   // bathymetry, Nxg*Nyg
};

// Surface state that defines the sigma coefficients of one solve.
struct Surface {
    const double *E, *Ex, *Exx, *Ey, *Eyy;   // Nxg*Nyg each; may be null (= 0)
};

// One multigrid level (low-order operator, alpha = beta = gamma = 1).
template <typename T>
struct LevelDev {
    int Nx, Ny, Nz;         // interior counts
    int Nxg, Nyg, Nzg;
    int64_t N;
    int ncolor;             // 2 or 4 (multicolour column Gauss-Seidel)
    int cross;              // mixed-derivative terms present (h_x or h_y nonzero on the level)
    int xc, yc, zc;         // this level is coarsened w.r.t. the next finer one
    const T* SX;            // [2][Nxg][3]
    const T* SY;            // [2][Nyg][3]
    const T* SZ;            // [2][Nzg][3]
    const T* zs;            // sigma with zs[0] = 0
    const T *h, *hx, *hxx, *hy, *hyy;  // Nxg*Nyg (ghost values as MGPreProcess sets them)
    const double *x, *y, *z;           // coordinates for transfer weights (FP64)
    const double *ix, *iy, *iz;        // 1/(x[i+1]-x[i-1]) etc. (computed as (dW+dE)) per index
    T* xv;                  // iterate
    T* bv;                  // right-hand side
    T* rv;                  // residual
};

// ------------------------------------------------ Krylov device scalars
struct KrylovState {
    double H[kMaxKrylov + 1][kMaxKrylov + 1];   // H[col][row]
    double cs[kMaxKrylov + 1], sn[kMaxKrylov + 1], g[kMaxKrylov + 2];
    double scale[kMaxKrylov + 2];               // v_i = scale[i] * V_i (stored unnormalised)
    double y[kMaxKrylov + 1];
    double dots[kMaxKrylov + 2];                // result of the last multi-dot
    double w0, w1;                              // |w|^2 before / after projection
    double beta, tol, resid;
    int k;                                      // Arnoldi steps done
    int reorth;                                 // re-orthogonalise this step
    int done;                                   // converged / stopped
    int converged;
    int iters;                                  // matvec count
    int status;
};

// --------------------------------------------------------- kernel entry
// High-order operator: y = s * A(phi) (mode 0) or y = b - A(phi) (mode 1).
// dscale: device pointer to a scalar multiplying phi (null = 1).
template <typename TIN>
void launch_ho_matvec(const HoGrid& g, const Surface& s, const TIN* phi, const double* dscale, const double* b,
                      double* y, int mode, cudaStream_t st);

// Multigrid (T = double or float)
template <typename T>
void launch_mg_vcycle(LevelDev<T>* lev, int nlev, const T* coarse_inv, int nu1, int nu2, int maxit,
                      cudaStream_t st);
template <typename T>
void launch_lo_matvec(const LevelDev<T>& L, const T* x, T* y, cudaStream_t st);
template <typename T>
void launch_lo_smooth(const LevelDev<T>& L, int nu, cudaStream_t st);
template <typename T>
void launch_restrict(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* rf, T* rc, cudaStream_t st);
template <typename T>
void launch_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* xc, T* xf, cudaStream_t st);
template <typename T>
void launch_coarse_solve(const LevelDev<T>& Lc, const T* inv, cudaStream_t st);
template <typename T>
void launch_scale_copy(const double* src, double s, T* dst, int64_t n, cudaStream_t st);
template <typename T>
void launch_fill(T* dst, T v, int64_t n, cudaStream_t st);
// dst = (*dscale) * src (dscale device pointer, null = 1), converted to T
template <typename T>
void launch_scale_copy_dev(const double* src, const double* dscale, T* dst, int64_t n, cudaStream_t st);
void launch_convert(const float* src, double* dst, int64_t n, cudaStream_t st);

// Krylov
struct DotScratch {
    double* partial;        // [kMaxKrylov+2][nblocks]
    unsigned int* counter;
    int nblocks;
};
void launch_multidot(const double* V, int64_t ldv, int k, const double* w, int64_t n, const DotScratch& sc,
                     KrylovState* ks, int cond, cudaStream_t st);
// Projection pass; the last block finishes the Arnoldi step (Givens rotation,
// stopping test) when no re-orthogonalisation pass follows.
void launch_project(const double* V, int64_t ldv, int k, double* w, int64_t n, const DotScratch& sc, KrylovState* ks,
                    int cond, int maxmv, int m, cudaStream_t st);
void launch_arnoldi_finish(KrylovState* ks, int maxmv, int m, cudaStream_t st);
void launch_norm_init(const double* v, int64_t n, const DotScratch& sc, KrylovState* ks, double rtol, double atol,
                      cudaStream_t st);
void launch_backsolve(KrylovState* ks, cudaStream_t st);
template <typename TZ>
void launch_solution_update(double* x, const TZ* Z, int64_t ldz, int64_t n, const KrylovState* ks, int use_scale,
                            cudaStream_t st);
void launch_krylov_reset(KrylovState* ks, cudaStream_t st);
void launch_krylov_restart(KrylovState* ks, cudaStream_t st);

}  // namespace ow3d
