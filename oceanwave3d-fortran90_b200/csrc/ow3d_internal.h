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
#include <utility>
#include <cstdint>
#include <cstddef>
#include <cstdio>
#include <string>
#include <cuda_runtime.h>
#include "../../include/ow3d.h"

namespace ow3d {

// Kernels launched by this library since load (all handles, all threads).
extern std::atomic<unsigned long long> g_kernel_launches;
// Block count cap of the fused coarse-level kernel (0: one block per SM).
extern std::atomic<int> g_coarse_blocks;
extern std::atomic<int64_t> g_coop_max_points;
extern std::atomic<int64_t> g_tail_max_points;
extern std::atomic<int> g_tail_cluster;
extern std::atomic<int> g_colour_tiles;
extern std::atomic<int> g_colour_prefetch;

// Set (on the capturing thread) when a launch sequence under stream capture
// issued a host-to-device copy whose source the host later overwrites.
extern thread_local bool g_capture_unsafe;
inline void note_launch() { g_kernel_launches.fetch_add(1ull, std::memory_order_relaxed); }

// Programmatic dependent launch on the solver path: a kernel launched by
// launch_k may start (its blocks resident, its launch latency spent) while
// the kernel before it on the stream finishes; it waits at pdl_entry for
// that kernel to complete and its writes to be visible, before touching any
// memory, and lets its own successor start as soon as all its blocks run.
// g_pdl = 0 launches plainly (the wait is then a no-op).
extern std::atomic<int> g_pdl;
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    note_launch();
    if (g_pdl.load(std::memory_order_relaxed)) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
    } else {
        kernel<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
    }
}
#endif  // __CUDACC__

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
    int per;                // periodic in x: distinct columns 2..Nxg-2, the
                            // others identity rows (see wrap_x)
    // per-position stencils, [order-1][pos][7], order 1 and 2 (BuildStencilsGridX.f90)
    const double* SX;       // 2*Nxg*7
    const double* SY;       // 2*Nyg*7 (unused in 2-D)
    const double* SZ;       // 2*Nzg*7 (PreProcessDiffStencils.f90:108-132)
    const double* zs;       // sigma levels with zs[0] = 0 (DetermineTransformationConstantsArray.f90:59)
    const double *h, *hx, *hxx, *hy, *hyy;   // bathymetry, Nxg*Nyg
    // host copies of the stencil tables and levels (owned by the handle), for
    // kernel parameters
    const double *hSX, *hSY, *hSZ, *hzs;
};

// Inputs of the kinematics passes (kinematics.cu, StoreKinematicData.f90).
struct KinArgs {
    int Nxg, Nyg, Nzg;
    int dox, doy;          // x / y derivatives present (Nx > 1, Ny > 1)
    int chain;             // LinearONOFF != 0: the s_x, s_y terms
    int64_t N;
    const double *SX, *SY, *SZ;   // order-1 blocks of the per-position stencils, [pos][7]
    const double* z;              // sigma levels, ghost level included
    const double *h, *hx, *hy, *E, *Ex, *Ey;
};
// One Fortran unformatted record of n parts (io.cpp).
bool write_record(std::FILE* f, const void* const* parts, const size_t* bytes, int n);

// out: 13 fields of N doubles: u, v, phi_s, w, then the 9 gradient fields.
void launch_kinematics(const KinArgs& a, const double* phi, double* out, cudaStream_t st);

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
    int per;                // periodic in x (never together with cross)
    int xc, yc, zc;         // this level is coarsened w.r.t. the next finer one
    const T* SX;            // [2][Nxg][3]
    const T* SY;            // [2][Nyg][3]
    const T* SZ;            // [2][Nzg][3]
    const T* zs;            // sigma with zs[0] = 0
    const T *h, *hx, *hxx, *hy, *hyy;  // Nxg*Nyg (ghost values as MGPreProcess sets them)
    const double *x, *y, *z;           // coordinates for transfer weights (FP64)
    const double *ix, *iy, *iz;        // 1/(x[i+1]-x[i-1]) etc. (computed as (dW+dE)) per index
    // per column: 1/h, h_x/h, h_y/h, (h_xx+h_yy)/h - 2(h_x^2+h_y^2)/h^2 -- the
    // eta = 0 sigma coefficients divided by (1 - sigma)
    const T* cf;            // [Nxg*Nyg][4]
    // per column, the bottom row's Gauss-Seidel coefficients (levels without
    // mixed-derivative terms): x2, x3 of the column, row 2 of the left, right,
    // lower and upper neighbours, 1/diagonal, and the diagonal (coefficient
    // of x1)
    const T* bt;            // [Nxg*Nyg][8]
    uint64_t mz, mx;        // division magics for Nzg and Nxg (see qdiv)
    uint32_t mz32, mx32;    // 32-bit magics for Nzg and Nxg (see div32) and their shifts
    int sz32, sx32;
    // prolongation from the next coarser level onto this one
    // (MGProlongation3DExplicit.f90:19-110) as per-direction tables over this
    // level's indices: coarse indices (1-based) and weights of the two coarse
    // points that interpolate fine index n; weight 0 marks an unused point
    const int *pix, *piy, *piz;        // [2*Nxg], [2*Nyg], [2*Nzg]
    const T *pwx, *pwy, *pwz;          // same layout
    T* xv;                  // iterate
    T* bv;                  // right-hand side
    T* rv;                  // residual
};

// Periodic x: the Nx points of a row span one period with both ends, so
// column Nxg-1 repeats column 2; the distinct columns are 2..Nxg-2 and a
// column index outside that range is taken cyclically. Ghost column 1,
// the repeated column Nxg-1 and ghost column Nxg carry identity rows with a
// zero right-hand side inside every solve.
__host__ __device__ __forceinline__ int wrap_x(int i, int Nxg) {
    const int M = Nxg - 3;
    return i < 2 ? i + M : (i > Nxg - 2 ? i - M : i);
}

// n / d as a 64-bit multiply-high with m = floor((2^64-1)/d) + 1: exact for
// every n < 2^48 and 2 <= d < 2^16 (the error term n*(m*d - 2^64) / 2^64 stays
// below 1/d), and a few instructions instead of a 64-bit division.
inline uint64_t div_magic(uint64_t d) { return ~0ull / d + 1ull; }
#ifdef __CUDACC__
__device__ __forceinline__ uint64_t qdiv(uint64_t n, uint64_t m) { return __umul64hi(n, m); }
#endif
// n / d for every n < 2^31 and d >= 2 as umulhi(n, m) >> sh with
// m = ceil(2^(31+l) / d), l = ceil(log2 d), sh = l - 1 (Granlund and
// Montgomery's round-up method; m < 2^32).
inline void div_magic32(uint32_t d, uint32_t& m, int& sh) {
    int l = 0;
    while ((1ull << l) < d) ++l;
    m = (uint32_t)(((1ull << (31 + l)) + d - 1) / d);
    sh = l - 1;
}
#ifdef __CUDACC__
__device__ __forceinline__ uint32_t div32(uint32_t n, uint32_t m, int sh) { return __umulhi(n, m) >> sh; }
#endif

// The incident wave of a generation zone on the device (incwave.cu): the
// components set up on the host (incident_wave_setup), device copies.
struct IncidentWaveDev {
    int bx, by, nt, ny_eval, N, kmax, heading, mono;
    double cosb, sinb, g, domega;
    double amp, nu, omega, phifact, t0, dt;   // mono-chromatic wave
    const double *dx, *dy, *dy_rows;          // [bx], [ny_eval], [by]
    const double *nus, *kcos, *ksin;          // [kmax]; kcos, ksin null unless spread
    const double2 *c, *W;                     // amplitudes [kmax], twiddles [N]
    double2 *A, *B;                           // per point and mode [ny_eval*bx][kmax]
};
// eta, phis: nt x (bx*by) samples (i fastest, then j), the zone's target layout.
int launch_incident_wave(const IncidentWaveDev& w, double* eta, double* phis, cudaStream_t st);

// sqrt(sum y^2) of a device vector using only fixed file-scope device scratch
// (noalloc.cu); result written to host memory, stream synchronised.
int noalloc_norm2(int dev, const double* d_y, int64_t n, double* host_norm2, cudaStream_t st, std::string& err);

// ------------------------------------------------ Krylov device scalars
struct KrylovState {
    double H[kMaxKrylov + 1][kMaxKrylov + 1];   // H[col][row] (FGMRES: unrotated columns)
    double R[kMaxKrylov + 1][kMaxKrylov + 2];   // FGMRES: rotated columns (upper triangle)
    double gsave[kMaxKrylov + 2];               // FGMRES: g[col] before rotation col
    double coefA[kMaxKrylov + 2];               // FGMRES update: V_j -= coefA_i V_i
    double coefB[kMaxKrylov + 2];               // FGMRES update: W -= coefB_i V_i (i <= j)
    double cs[kMaxKrylov + 1], sn[kMaxKrylov + 1], g[kMaxKrylov + 2];
    double scale[kMaxKrylov + 2];               // v_i = scale[i] * V_i (stored unnormalised)
    // left preconditioning: T[j][i], i <= j, expresses the vector step j
    // multiplied (V_j after one Gram-Schmidt pass, times its provisional
    // scale) in the final basis v_0..v_j
    double T[kMaxKrylov + 1][kMaxKrylov + 1];
    double y[kMaxKrylov + 1];
    // the scalars from here on are what the host reads after each Arnoldi step
    double w0, w1;                              // spare
    double beta, tol, resid;
    int k;                                      // Arnoldi steps done
    int reorth;                                 // spare
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
// Device copy of the level table for the fused coarse-level kernel, with the
// host image of what was last uploaded.
template <typename T>
struct LevelTable {
    LevelDev<T>* dev = nullptr;
    LevelDev<T> host[kMaxLevels];
    // the whole fused coarse cycle in one thread-block cluster instead of a
    // cooperative grid over every SM (ow3d_set_coarse_cluster)
    bool cluster = false;
    // Gauss-Seidel in the reference's lexicographic order on every level
    // (ow3d_set_smoother_order): no fused coarse cycle, no dense sub-cycle
    // operator (the V cycle descends to the coarsest level's inverse)
    bool lex = false;
};

// M: dense operator of level ld (the coarsest level's inverse when ld = 0).
template <typename T>
void launch_mg_vcycle(LevelDev<T>* lev, int nlev, const T* M, int ld, int nu1, int nu2, int maxit,
                      LevelTable<T>& pack, cudaStream_t st);
template <typename T>
void launch_mg_subcycle(LevelDev<T>* lev, int nlev, int l, int ld, const T* M, int nu1, int nu2,
                        LevelTable<T>& pack, cudaStream_t st);
template <typename T>
void launch_dense_apply(const LevelDev<T>& L, const T* M, cudaStream_t st);
template <typename T>
void launch_lo_matvec(const LevelDev<T>& L, const T* x, T* y, cudaStream_t st);
template <typename T>
void launch_lo_smooth(const LevelDev<T>& L, int nu, cudaStream_t st);
// the same smoothing steps in the reference's lexicographic order (mg_lex.cu)
template <typename T>
void launch_lo_smooth_lex(const LevelDev<T>& L, int nu, cudaStream_t st);
// One smoother phase: colour pass `colour`, or the bottom-row pass (colour < 0).
template <typename T>
void launch_lo_pass(const LevelDev<T>& L, int colour, cudaStream_t st);
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
// Arnoldi step j with delayed classical Gram-Schmidt (DCGS2): the one
// reduction pass and the one update pass; the new vector W (A z_j, or
// M^{-1} A v_j with left preconditioning) sits in V_{j+1}.
void launch_dcgs_reduce(const double* V, int64_t ldv, int j, const double* W, int64_t n, const DotScratch& sc,
                        KrylovState* ks, cudaStream_t st);
// hnext: inside a captured step graph, the condition of the node that runs
// Arnoldi step j+1 (set to "not done" by the step's stopping test); 0 otherwise.
void launch_dcgs_update(double* V, int64_t ldv, int j, double* W, int64_t n, const DotScratch& sc, KrylovState* ks,
                        int maxmv, int m, cudaStream_t st, cudaGraphConditionalHandle hnext = 0);
void launch_norm_init(const double* v, int64_t n, const DotScratch& sc, KrylovState* ks, double rtol, double atol,
                      cudaStream_t st, cudaGraphConditionalHandle hnext = 0);
// The outcome of one solve, copied from the Krylov state when it ends (the
// step graph's record of its four solves).
struct SolveLog {
    int iters, converged;
    double resid, beta, tol;
};
void launch_solve_log(const KrylovState* ks, SolveLog* out, cudaStream_t st);
void launch_backsolve(KrylovState* ks, cudaStream_t st, int rotated_R = 0, int in_basis = 0);
template <typename TZ>
void launch_solution_update(double* x, const TZ* Z, int64_t ldz, int64_t n, const KrylovState* ks, int use_scale,
                            cudaStream_t st);
void launch_krylov_reset(KrylovState* ks, cudaStream_t st);
void launch_krylov_restart(KrylovState* ks, cudaStream_t st);

}  // namespace ow3d
