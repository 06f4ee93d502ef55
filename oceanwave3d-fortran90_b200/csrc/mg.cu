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
//
// Levels with few points run inside one cooperative kernel (k_mg_coarse_cycle)
// that executes the phases of every coarse level back to back with grid-wide
// barriers, instead of one launch per phase.
#include "ow3d_internal.h"
#include "mg_device.cuh"
#include <cooperative_groups.h>
#include <vector>

namespace ow3d {

namespace {
using namespace mgdev;
namespace cg = cooperative_groups;

#define OW3D_GRID_STRIDE(var, n) \
    for (int64_t var = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; var < (n); var += (int64_t)gridDim.x * blockDim.x)

// Points per level below which the level runs in the fused coarse kernel.
constexpr int64_t kCoopMaxPoints = 160000;

template <typename T, bool THREE>
__global__ void k_lo_matvec(LevelDev<T> L, const T* __restrict__ x, T* __restrict__ y) {
    OW3D_GRID_STRIDE(p, L.N) {
        const int k = (int)(p % L.Nzg) + 1;
        const int64_t c = p / L.Nzg;
        const int i = (int)(c % L.Nxg) + 1, j = (int)(c / L.Nxg) + 1;
        T dg;
        y[p] = lo_row<T, THREE>(L, x, k, i, j, dg);
    }
}

template <typename T, bool THREE>
__global__ void k_lo_residual(LevelDev<T> L) {
    OW3D_GRID_STRIDE(p, L.N) residual_item<T, THREE>(L, p);
}

template <typename T, bool THREE>
__global__ void k_lo_special(LevelDev<T> L) {
    OW3D_GRID_STRIDE(q, (special_count<T, THREE>(L))) special_item<T, THREE>(L, q);
}

template <typename T, bool THREE, int S, bool CROSS>
__global__ void __launch_bounds__(128) k_lo_colour(LevelDev<T> L, int colour) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t total = colour_count<T, THREE>(L);
    for (int64_t base = warp * (32 / S); base < total; base += nwarps * (32 / S))
        colour_warp<T, THREE, S, CROSS>(L, colour, base);
}

template <typename T>
__global__ void k_restrict(LevelDev<T> F, LevelDev<T> Cc, const T* __restrict__ rf, T* __restrict__ rc, T* __restrict__ xc) {
    OW3D_GRID_STRIDE(p, Cc.N) restrict_item<T>(F, Cc, rf, rc, xc, p);
}

template <typename T>
__global__ void k_prolong_add(LevelDev<T> F, LevelDev<T> Cc, const T* __restrict__ xc, T* __restrict__ xf) {
    OW3D_GRID_STRIDE(p, F.N) prolong_item<T>(F, Cc, xc, xf, p);
}

// Coarsest level: x = A^{-1} b with the explicit inverse (the reference factors
// this matrix with HSL MA41 once, LUfactor.f90:20-66, and solves with it).
template <typename T>
__global__ void k_coarse(int n, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x) {
    OW3D_GRID_STRIDE(r, n) coarse_item<T>(n, inv, b, x, (int)r);
}

template <typename T>
__global__ void k_scale_copy(const double* __restrict__ src, double s, T* __restrict__ dst, int64_t n) {
    OW3D_GRID_STRIDE(p, n) dst[p] = T(s * src[p]);
}
template <typename T>
__global__ void k_scale_copy_dev(const double* __restrict__ src, const double* __restrict__ ds, T* __restrict__ dst, int64_t n) {
    const double s = ds ? *ds : 1.0;
    OW3D_GRID_STRIDE(p, n) dst[p] = T(s * src[p]);
}
__global__ void k_convert(const float* __restrict__ src, double* __restrict__ dst, int64_t n) {
    OW3D_GRID_STRIDE(p, n) dst[p] = (double)src[p];
}
template <typename T>
__global__ void k_fill(T* __restrict__ dst, T v, int64_t n) {
    OW3D_GRID_STRIDE(p, n) dst[p] = v;
}

// ------------------------------------------------- fused coarse levels
template <typename T>
struct LevelPack { LevelDev<T> l[kMaxLevels]; };

inline int seg_width(int Nzg) {
    const int R = Nzg - 2;
    return R <= 2 ? 2 : (R <= 4 ? 4 : (R <= 8 ? 8 : (R <= 16 ? 16 : 32)));
}

template <typename T, bool THREE, int S, bool CROSS>
__device__ void coop_colour_loop(const LevelDev<T>& L, int colour) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t total = colour_count<T, THREE>(L);
    for (int64_t base = warp * (32 / S); base < total; base += nwarps * (32 / S))
        colour_warp<T, THREE, S, CROSS>(L, colour, base);
}

template <typename T, bool THREE>
__device__ void coop_colour(const LevelDev<T>& L, int colour) {
    const int R = L.Nzg - 2;
    const bool cr = L.cross != 0;
#define OW3D_CC(SW) { if (cr) coop_colour_loop<T, THREE, SW, true>(L, colour); else coop_colour_loop<T, THREE, SW, false>(L, colour); }
    if (R <= 2) OW3D_CC(2) else if (R <= 4) OW3D_CC(4) else if (R <= 8) OW3D_CC(8) else if (R <= 16) OW3D_CC(16) else OW3D_CC(32)
#undef OW3D_CC
}

template <typename T, bool THREE>
__device__ void coop_smooth(const LevelDev<T>& L, int nu, cg::grid_group& grid) {
    OW3D_GRID_STRIDE(q, (special_count<T, THREE>(L))) special_item<T, THREE>(L, q);
    grid.sync();
    for (int s = 0; s < nu; ++s) {
        for (int c = 0; c < L.ncolor; ++c) { coop_colour<T, THREE>(L, c); grid.sync(); }
        OW3D_GRID_STRIDE(q, (special_count<T, THREE>(L))) special_item<T, THREE>(L, q);
        grid.sync();
    }
}

// V cycle over levels lc..0 (MultiGridSolver.f90:5-192) in one cooperative
// launch. Level lc's right-hand side is set and its iterate zeroed on entry.
template <typename T, bool THREE>
__global__ void __launch_bounds__(256) k_mg_coarse_cycle(LevelPack<T> P, int lc, const T* __restrict__ inv, int nu1,
                                                         int nu2) {
    cg::grid_group grid = cg::this_grid();
    for (int l = lc; l >= 1; --l) {
        const LevelDev<T>& L = P.l[l];
        const LevelDev<T>& Cc = P.l[l - 1];
        coop_smooth<T, THREE>(L, nu1, grid);
        OW3D_GRID_STRIDE(p, L.N) residual_item<T, THREE>(L, p);
        grid.sync();
        OW3D_GRID_STRIDE(p, Cc.N) restrict_item<T>(L, Cc, L.rv, Cc.bv, Cc.xv, p);
        grid.sync();
    }
    {
        const LevelDev<T>& L0 = P.l[0];
        OW3D_GRID_STRIDE(r, L0.N) coarse_item<T>((int)L0.N, inv, L0.bv, L0.xv, (int)r);
        grid.sync();
    }
    for (int l = 1; l <= lc; ++l) {
        const LevelDev<T>& L = P.l[l];
        const LevelDev<T>& Cc = P.l[l - 1];
        OW3D_GRID_STRIDE(p, L.N) prolong_item<T>(L, Cc, Cc.xv, L.xv, p);
        grid.sync();
        coop_smooth<T, THREE>(L, nu2, grid);
    }
}

inline int nblk(int64_t n, int t = 256) {
    int64_t b = (n + t - 1) / t;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

template <typename T>
void launch_lo_matvec(const LevelDev<T>& L, const T* x, T* y, cudaStream_t st) {
    if (L.Nyg > 1) note_launch(), k_lo_matvec<T, true><<<nblk(L.N), 256, 0, st>>>(L, x, y);
    else note_launch(), k_lo_matvec<T, false><<<nblk(L.N), 256, 0, st>>>(L, x, y);
}

template <typename T>
static void special(const LevelDev<T>& L, cudaStream_t st) {
    const int64_t n = (int64_t)L.Nxg * L.Nyg + ((L.Nyg > 1) ? ((int64_t)2 * L.Nyg + 2 * (L.Nxg - 2)) : 2) * L.Nzg;
    if (L.Nyg > 1) note_launch(), k_lo_special<T, true><<<nblk(n, 128), 128, 0, st>>>(L);
    else note_launch(), k_lo_special<T, false><<<nblk(n, 128), 128, 0, st>>>(L);
}

template <typename T, bool THREE, int S>
static void colour_launch(const LevelDev<T>& L, int c, cudaStream_t st) {
    const int64_t cols = (int64_t)((L.Nxg - 1) / 2) * (THREE ? L.Nyg - 2 : 1);
    const int64_t warps = (cols + (32 / S) - 1) / (32 / S);
    int64_t blocks = (warps * 32 + 127) / 128;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks < 1) blocks = 1;
    if (L.cross) note_launch(), k_lo_colour<T, THREE, S, true><<<(int)blocks, 128, 0, st>>>(L, c);
    else note_launch(), k_lo_colour<T, THREE, S, false><<<(int)blocks, 128, 0, st>>>(L, c);
}
template <typename T, bool THREE>
static void colour_dispatch(const LevelDev<T>& L, int c, cudaStream_t st) {
    switch (seg_width(L.Nzg)) {
        case 2: colour_launch<T, THREE, 2>(L, c, st); break;
        case 4: colour_launch<T, THREE, 4>(L, c, st); break;
        case 8: colour_launch<T, THREE, 8>(L, c, st); break;
        case 16: colour_launch<T, THREE, 16>(L, c, st); break;
        default: colour_launch<T, THREE, 32>(L, c, st); break;
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
    note_launch(), k_restrict<T><<<nblk(Cc.N), 256, 0, st>>>(F, Cc, rf, rc, Cc.xv);
}
template <typename T>
void launch_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* xc, T* xf, cudaStream_t st) {
    note_launch(), k_prolong_add<T><<<nblk(F.N), 256, 0, st>>>(F, Cc, xc, xf);
}
template <typename T>
void launch_coarse_solve(const LevelDev<T>& Lc, const T* inv, cudaStream_t st) {
    int n = (int)Lc.N;
    note_launch(), k_coarse<T><<<(n + 127) / 128, 128, 0, st>>>(n, inv, Lc.bv, Lc.xv);
}
template <typename T>
void launch_scale_copy(const double* src, double s, T* dst, int64_t n, cudaStream_t st) {
    note_launch(), k_scale_copy<T><<<nblk(n), 256, 0, st>>>(src, s, dst, n);
}
template <typename T>
void launch_fill(T* dst, T v, int64_t n, cudaStream_t st) {
    note_launch(), k_fill<T><<<nblk(n), 256, 0, st>>>(dst, v, n);
}
template <typename T>
void launch_scale_copy_dev(const double* src, const double* ds, T* dst, int64_t n, cudaStream_t st) {
    note_launch(), k_scale_copy_dev<T><<<nblk(n), 256, 0, st>>>(src, ds, dst, n);
}
void launch_convert(const float* src, double* dst, int64_t n, cudaStream_t st) {
    note_launch(), k_convert<<<nblk(n), 256, 0, st>>>(src, dst, n);
}

// Launch the fused coarse cycle over levels lc..0 with a fully co-resident grid.
template <typename T, bool THREE>
static void coarse_cycle(const LevelDev<T>* lev, int lc, const T* inv, int nu1, int nu2, cudaStream_t st) {
    static int grid = 0;
    if (grid == 0) {
        int dev = 0, nsm = 148, per = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_mg_coarse_cycle<T, THREE>, 256, 0);
        grid = nsm * (per < 2 ? (per < 1 ? 1 : per) : 2);
    }
    LevelPack<T> P;
    for (int l = 0; l <= lc; ++l) P.l[l] = lev[l];
    void* args[] = {(void*)&P, (void*)&lc, (void*)&inv, (void*)&nu1, (void*)&nu2};
    note_launch();
    cudaLaunchCooperativeKernel((const void*)k_mg_coarse_cycle<T, THREE>, dim3(grid), dim3(256), args, 0, st);
}

template <typename T>
static int coop_level(const LevelDev<T>* lev, int nlev) {
    int lc = -1;
    for (int l = 0; l < nlev; ++l) if (lev[l].N <= kCoopMaxPoints) lc = l;
    return lc;
}

// MultiGridSolver.f90:5-192 (V cycle, gam = 1), levels lev[0] coarsest.
template <typename T>
static void vcycle(LevelDev<T>* lev, int l, int lc, const T* inv, int nu1, int nu2, cudaStream_t st) {
    if (l <= lc) {
        if (lev[0].Nyg > 1) coarse_cycle<T, true>(lev, l, inv, nu1, nu2, st);
        else coarse_cycle<T, false>(lev, l, inv, nu1, nu2, st);
        return;
    }
    if (l == 0) { launch_coarse_solve(lev[0], inv, st); return; }
    const LevelDev<T>& F = lev[l];
    LevelDev<T>& Cc = lev[l - 1];
    launch_lo_smooth(F, nu1, st);
    if (F.Nyg > 1) note_launch(), k_lo_residual<T, true><<<nblk(F.N), 256, 0, st>>>(F);
    else note_launch(), k_lo_residual<T, false><<<nblk(F.N), 256, 0, st>>>(F);
    launch_restrict(F, Cc, (const T*)F.rv, Cc.bv, st);   // also zeroes Cc.xv
    vcycle(lev, l - 1, lc, inv, nu1, nu2, st);
    launch_prolong_add(F, Cc, (const T*)Cc.xv, F.xv, st);
    launch_lo_smooth(F, nu2, st);
}

// MultiGridSolveLinearSystem.f90:26-91: u = 0, then maxit cycles.
template <typename T>
void launch_mg_vcycle(LevelDev<T>* lev, int nlev, const T* coarse_inv, int nu1, int nu2, int maxit, cudaStream_t st) {
    LevelDev<T>& F = lev[nlev - 1];
    launch_fill<T>(F.xv, T(0), F.N, st);
    const int lc = (nlev > 1) ? coop_level(lev, nlev) : -1;
    for (int it = 1; it <= maxit; ++it) {
        if (nlev == 1 && it > 1) break;
        vcycle(lev, nlev - 1, lc, coarse_inv, nu1, nu2, st);
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
