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
// Smoother (device-matched ordering, deterministic): one smoothing step is one
// pass per colour of the interior columns (2 colours, or 4 when the level has
// mixed-derivative terms). A column's task relaxes its bottom row, then its
// rows k = 2..Nzg bottom to top, then the rows of the lateral ghost columns it
// borders -- so the reference's special rows (iGhost, MGPreProcess.f90:376-439,
// relaxed by GaussSeidelSpecialPoints around each sweep in
// MultiGridSolver.f90:118-126,174-181) are relaxed inside the colour passes
// instead of in separate strided passes. A handle may ask for the reference's
// own lexicographic order instead (mg_lex.cu, ow3d_set_smoother_order).
//
// Levels with few points run inside one cooperative kernel (k_mg_coarse_cycle)
// that executes the phases of every coarse level back to back with grid-wide
// barriers, instead of one launch per phase.
#include "ow3d_internal.h"
#include "mg_device.cuh"
#include <cooperative_groups.h>
#include <cstring>
#include <vector>

namespace ow3d {

namespace {
using namespace mgdev;
namespace cg = cooperative_groups;

#define OW3D_GRID_STRIDE(var, n) \
    for (int64_t var = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; var < (n); var += (int64_t)gridDim.x * blockDim.x)

// Points per level below which the level runs in the fused coarse kernel.
// Threads per block of the fused coarse kernel (one block per SM: fewer
// blocks make the grid-wide barrier cheaper).
constexpr int kCoopThreads = 512;

template <typename T, bool THREE>
__global__ void k_lo_matvec(LevelDev<T> L, const T* __restrict__ x, T* __restrict__ y) {
    pdl_entry();
    OW3D_GRID_STRIDE(p, L.N) {
        int k, i, j;
        int64_t c;
        decomp(L, p, k, c, i, j);
        T dg;
        y[p] = lo_row<T, THREE>(L, x, k, i, j, dg);
    }
}

template <typename T, bool THREE, bool CROSS>
__global__ void k_lo_residual(LevelDev<T> L) {
    pdl_entry();
    OW3D_GRID_STRIDE(p, L.N) residual_point<T, THREE, CROSS>(L, p);
}

template <typename T, bool THREE>
__global__ void k_lo_bottom(LevelDev<T> L) {
    pdl_entry();
    OW3D_GRID_STRIDE(q, (bottom_count<T, THREE>(L))) bottom_item<T, THREE>(L, q);
}

// Per-level colour pass: two rows per lane (colour_warp2), S lanes per column.
// With prefetch set, each warp asks for the next group's column data (its
// rows of x in the column and the four neighbour columns, and of b) to be
// brought into L1 before it solves the current group.
// Resident blocks per SM. Without mixed-derivative terms: FP64 5 (at most
// 96 registers, a few spilled: measured on a B200 at 1025x257x17, the finest
// pass 51.8 against 57.6 us and the FP64 step 78.8 against 79.6 ms; 6 blocks
// spill more and are slower), FP32 7 (72 registers, none spilled: the mixed
// step 62.9 against 63.4 ms; 8 blocks spill and gain less). With them 4
// (their larger rows would spill far more under the same caps).
constexpr int colour_blocks_per_sm(bool cross, bool fp32) { return cross ? 4 : (fp32 ? 7 : 5); }

template <typename T, bool THREE, int S, bool CROSS>
__global__ void __launch_bounds__(128, colour_blocks_per_sm(CROSS, sizeof(T) == 4))
    k_lo_colour(LevelDev<T> L, int colour, int prefetch) {
    pdl_entry();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t total = colour_count<T, THREE>(L);
    const int r = (threadIdx.x & 31) & (S - 1);
    const RowConst<T> rka = row_const_k<T>(L, 2 + 2 * r), rkb = row_const_k<T>(L, 3 + 2 * r);
    const int step = (int)nwarps * (32 / S);
    for (int base = (int)warp * (32 / S); base < (int)total; base += step) {
        if (prefetch && base + step < (int)total) colour_prefetch<T, THREE, S>(L, colour, base + step);
        colour_warp2<T, THREE, S, CROSS>(L, colour, base, rka, rkb);
    }
}

// ------------------------------------------------- tiled colour pass
//
// Levels without mixed-derivative terms (two colours, 3-D): every column of
// the inner part (i in 4..Nxg-3, j in 4..Nyg-3) is solved from a tile staged
// in shared memory by cp.async: kCTX x kCTY columns of x with one ring of
// neighbour columns, and the colour's b, coefficients and bottom-row tables.
// The tile arrives in two groups (tile rows 0-3 with their neighbour rows,
// then the rest), and the first half is solved while the second arrives. The
// columns within two columns of a wall (their ghost and corner work included)
// run in the leading blocks of the same launch from global memory. Within one
// colour no column reads another column that the pass writes, so both parts
// read the values the per-column pass reads, and the arithmetic per column is
// the same code (colour_col2).
constexpr int kCTX = 32, kCTY = 8, kCTThreads = 256;
constexpr int kCTSlots = kCTX * kCTY / 2;      // columns of one colour in a tile

// Shared-memory layout of a tile, in elements: x rows RS apart (row rj holds
// the columns i0-1.. of row j0-1+rj), b in slots BS apart, then 4 coefficients
// and 8 bottom-row values per slot. Rows are copied in 16-byte chunks from the
// 16-byte boundary at or below their first element; RS has the residue of a
// global row (Nxg*Nzg) modulo a chunk, so the chunks of every row land on
// 16-byte boundaries and neighbouring rows stay RS apart.
template <typename T>
struct TileShape {
    int RS, BS, oB, oCF, oBT, bytes;
};
template <typename T>
inline TileShape<T> tile_shape(int Nxg, int Nzg) {
    constexpr int V = 16 / (int)sizeof(T);
    TileShape<T> sh;
    const int rmin = (kCTX + 2) * Nzg + 2 * V;
    const int want = (int)(((int64_t)Nxg * Nzg) % V);
    sh.RS = rmin + ((want - rmin % V) % V + V) % V;
    sh.BS = (Nzg + 3 * V - 1) / V * V;
    sh.oB = ((kCTY + 2) * sh.RS + V - 1) / V * V;
    sh.oCF = sh.oB + kCTSlots * sh.BS;
    sh.oBT = sh.oCF + kCTSlots * 4;
    sh.bytes = (sh.oBT + kCTSlots * 8) * (int)sizeof(T);
    return sh;
}

__device__ __forceinline__ void cp16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename T>
__device__ __forceinline__ int chunk_pad(const T* p) {
    return (int)(((uintptr_t)p & 15u) / sizeof(T));
}

template <typename T, int S>
__global__ void __launch_bounds__(kCTThreads, 2) k_lo_colour_tile(LevelDev<T> L, int colour, int nband, int ntx,
                                                                  TileShape<T> sh) {
    pdl_entry();
    extern __shared__ __align__(16) unsigned char ct_smem[];
    constexpr int V = 16 / (int)sizeof(T);
    constexpr int CPW = 32 / S;                       // columns per warp
    constexpr int NW = kCTThreads / 32;
    const int warp = threadIdx.x >> 5, r = (threadIdx.x & 31) & (S - 1);
    const RowConst<T> rka = row_const_k<T>(L, 2 + 2 * r), rkb = row_const_k<T>(L, 3 + 2 * r);
    if ((int)blockIdx.x < nband) {
        colour_band2<T, S>(L, colour, ((int)blockIdx.x * NW + warp) * CPW, rka, rkb);
        return;
    }
    const int t = (int)blockIdx.x - nband;
    const int ty = t / ntx, tx = t - ty * ntx;
    const int i0 = 4 + tx * kCTX, j0 = 4 + ty * kCTY;
    const int Nxg = L.Nxg, Nyg = L.Nyg, Nzg = L.Nzg;
    T* const xs = reinterpret_cast<T*>(ct_smem);
    T* const bs = xs + sh.oB;
    T* const cfs = xs + sh.oCF;
    T* const bts = xs + sh.oBT;
    const T* const X = L.xv;
    const T* const B = L.bv;
    const int tid = threadIdx.x;
    const int ncols = min(kCTX + 2, Nxg - i0);       // x columns i0-1 .. at most Nxg-2
    const int P = chunk_pad(X + ((int64_t)(i0 - 2) + (int64_t)Nxg * (j0 - 2)) * Nzg);
    // x rows rj in [rlo, rhi) (level rows j0-1+rj up to Nyg-2)
    auto stage_rows = [&](int rlo, int rhi) {
        for (int rj = rlo; rj < rhi; ++rj) {
            const int jj = j0 - 1 + rj;
            if (jj > Nyg - 2) break;
            const T* g = X + ((int64_t)(i0 - 2) + (int64_t)Nxg * (jj - 1)) * Nzg;
            const int pad = chunk_pad(g);
            const int n16 = (pad + ncols * Nzg + V - 1) / V;
            T* d = xs + rj * sh.RS + P - pad;
            const T* ga = g - pad;
            for (int e = tid; e < n16; e += kCTThreads) cp16(d + e * V, ga + e * V);
        }
    };
    // b, coefficients and bottom-row table of the colour's columns in slots [slo, shi)
    auto stage_slots = [&](int slo, int shi) {
        constexpr int CFC = 4 / V, BTC = 8 / V;
        const int nb = sh.BS / V, per = nb + CFC + BTC;
        for (int e = tid; e < (shi - slo) * per; e += kCTThreads) {
            const int q = e / per, w = e - q * per, s = slo + q;
            const int rr = s / (kCTX / 2), m = s - rr * (kCTX / 2);
            const int j = j0 + rr, i = i0 + 2 * m + ((colour + j - i0) & 1);
            if (i > Nxg - 3 || j > Nyg - 3) continue;
            const int64_t c = (int64_t)(i - 1) + (int64_t)Nxg * (j - 1);
            if (w < nb) {
                const T* gb = B + c * Nzg;
                cp16(bs + s * sh.BS + w * V, gb - chunk_pad(gb) + w * V);
            } else if (w < nb + CFC) {
                cp16(cfs + s * 4 + (w - nb) * V, L.cf + c * 4 + (w - nb) * V);
            } else {
                cp16(bts + s * 8 + (w - nb - CFC) * V, L.bt + c * 8 + (w - nb - CFC) * V);
            }
        }
    };
    stage_rows(0, kCTY / 2 + 2);
    stage_slots(0, kCTSlots / 2);
    cp_commit();
    stage_rows(kCTY / 2 + 2, kCTY + 2);
    stage_slots(kCTSlots / 2, kCTSlots);
    cp_commit();
    constexpr int GPR = (kCTX / 2) / CPW;            // warp groups per tile row
    constexpr int G = kCTSlots / CPW;                // warp groups per tile
    auto group = [&](int g) {
        const int rr = g / GPR, m = (g - rr * GPR) * CPW + ((threadIdx.x & 31) / S);
        const int s = rr * (kCTX / 2) + m;
        const int j = j0 + rr, i = i0 + 2 * m + ((colour + j - i0) & 1);
        const bool act = i <= Nxg - 3 && j <= Nyg - 3;
        const int64_t c = (int64_t)(i - 1) + (int64_t)Nxg * (j - 1);
        const T* xr = xs + (rr + 1) * sh.RS + P + (i - i0 + 1) * Nzg;
        const T* br = bs + s * sh.BS + chunk_pad(B + c * Nzg);
        colour_col2<T, true, S, false, true>(L, i, j, act, rka, rkb, xr, sh.RS, br, cfs + s * 4, bts + s * 8);
    };
    cp_wait<1>();
    __syncthreads();
    for (int g = warp; g < G / 2; g += NW) group(g);
    cp_wait<0>();
    __syncthreads();
    for (int g = G / 2 + warp; g < G; g += NW) group(g);
}

template <typename T>
__global__ void k_restrict(LevelDev<T> F, LevelDev<T> Cc, const T* __restrict__ rf, T* __restrict__ rc, T* __restrict__ xc) {
    pdl_entry();
    OW3D_GRID_STRIDE(p, Cc.N) restrict_item<T>(F, Cc, rf, rc, xc, p);
}

template <typename T>
__global__ void k_prolong_add(LevelDev<T> F, LevelDev<T> Cc, const T* __restrict__ xc, T* __restrict__ xf) {
    pdl_entry();
    OW3D_GRID_STRIDE(p, F.N) prolong_item<T>(F, Cc, xc, xf, p);
}

// Coarsest level: x = A^{-1} b with the explicit inverse (the reference factors
// this matrix with HSL MA41 once, LUfactor.f90:20-66, and solves with it).
template <typename T>
__global__ void k_coarse(int n, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x) {
    pdl_entry();
    OW3D_GRID_STRIDE(r, n) coarse_item<T>(n, inv, b, x, (int)r);
}

// x = M b for a dense row-major n x n operator: one warp per row, lanes
// stride along the row (coalesced), shuffle reduction.
template <typename T>
__device__ __forceinline__ void dense_rows(int n, const T* __restrict__ M, const T* b, T* x) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < n; r += nwarps) {
        const T* row = M + r * n;
        T acc = 0;
        for (int c = lane; c < n; c += 32) acc += row[c] * b[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) x[r] = acc;
    }
}

template <typename T>
__global__ void k_dense_apply(int n, const T* __restrict__ M, const T* __restrict__ b, T* __restrict__ x) {
    pdl_entry();
    dense_rows<T>(n, M, b, x);
}

template <typename T>
__global__ void k_scale_copy(const double* __restrict__ src, double s, T* __restrict__ dst, int64_t n) {
    pdl_entry();
    OW3D_GRID_STRIDE(p, n) dst[p] = T(s * src[p]);
}
template <typename T>
__global__ void k_scale_copy_dev(const double* __restrict__ src, const double* __restrict__ ds, T* __restrict__ dst, int64_t n) {
    pdl_entry();
    const double s = ds ? *ds : 1.0;
    OW3D_GRID_STRIDE(p, n) dst[p] = T(s * src[p]);
}
__global__ void k_convert(const float* __restrict__ src, double* __restrict__ dst, int64_t n) {
    pdl_entry();
    OW3D_GRID_STRIDE(p, n) dst[p] = (double)src[p];
}
template <typename T>
__global__ void k_fill(T* __restrict__ dst, T v, int64_t n) {
    pdl_entry();
    OW3D_GRID_STRIDE(p, n) dst[p] = v;
}

// ------------------------------------------------- fused coarse levels

inline int seg_width(int Nzg) {
    const int R = Nzg - 2;
    return R <= 2 ? 2 : (R <= 4 ? 4 : (R <= 8 ? 8 : (R <= 16 ? 16 : 32)));
}

template <typename T, bool THREE, int S, bool CROSS>
__device__ void coop_colour_loop(const LevelDev<T>& L, int colour) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t total = colour_count<T, THREE>(L);
    const RowConst<T> rk = row_const<T, S>(L);
    for (int base = (int)warp * (32 / S); base < (int)total; base += (int)nwarps * (32 / S))
        colour_warp<T, THREE, S, CROSS>(L, colour, base, rk);
}

template <typename T, bool THREE>
__device__ void coop_colour(const LevelDev<T>& L, int colour) {
    const int R = L.Nzg - 2;
    const bool cr = L.cross != 0;
#define OW3D_CC(SW) { if (cr) coop_colour_loop<T, THREE, SW, true>(L, colour); else coop_colour_loop<T, THREE, SW, false>(L, colour); }
    if (R <= 2) OW3D_CC(2) else if (R <= 4) OW3D_CC(4) else if (R <= 8) OW3D_CC(8) else if (R <= 16) OW3D_CC(16) else OW3D_CC(32)
#undef OW3D_CC
}

// Barriers of the fused coarse kernels: the whole cooperative grid, or the
// one thread-block cluster of the tail kernel (a hardware barrier among the
// cluster's SMs, with release / acquire ordering of their global-memory
// accesses at cluster scope).
struct GridSync {
    cg::grid_group g;
    __device__ void sync() { g.sync(); }
};
struct ClusterSync {
    __device__ void sync() { cg::this_cluster().sync(); }
};

template <typename T, bool THREE, typename SY>
__device__ void coop_bottoms(const LevelDev<T>& L, SY& sy) {
    OW3D_GRID_STRIDE(q, (bottom_count<T, THREE>(L))) bottom_item<T, THREE>(L, q);
    sy.sync();
}

template <typename T, bool THREE, typename SY>
__device__ void coop_smooth(const LevelDev<T>& L, int nu, SY& sy) {
    if (L.cross) coop_bottoms<T, THREE>(L, sy);
    for (int s = 0; s < nu; ++s) {
        for (int c = 0; c < L.ncolor; ++c) { coop_colour<T, THREE>(L, c); sy.sync(); }
        if (L.cross) coop_bottoms<T, THREE>(L, sy);
    }
}

// Parts of the V cycle over levels lc..ld that one launch of a fused kernel
// runs: all of it, the descent from lc to level lo (ending with lo's
// right-hand side restricted and its iterate zeroed), or the ascent from lo.
enum CoarsePart : int { kWhole = 0, kDown = 1, kUp = 2 };

// V cycle over levels lc..ld (MultiGridSolver.f90:5-192) in one launch whose
// phases are separated by the barrier SY; level ld is solved with the dense
// operator M (the coarsest level's inverse when ld = 0, otherwise the V cycle
// below ld as one precomputed map). Level lc's right-hand side is set and its
// iterate zeroed on entry. Level lc is read from `top` (the table's entry with
// the iterate and right-hand side of this launch), the others from the table.
// part / lo select the piece of the cycle (CoarsePart); lo = ld for kWhole.
template <typename T, bool THREE, typename SY>
__device__ void coarse_body(const LevelDev<T>* __restrict__ P, const LevelDev<T>& top, int lc, int ld, int lo,
                            int part, const T* __restrict__ M, int nu1, int nu2, SY& sy) {
    auto lv = [&](int l) -> const LevelDev<T>& { return l == lc ? top : P[l]; };
    if (part != kUp) {
        for (int l = lc; l > lo; --l) {
            const LevelDev<T>& L = lv(l);
            const LevelDev<T>& Cc = P[l - 1];
            coop_smooth<T, THREE>(L, nu1, sy);
            if (L.cross) { OW3D_GRID_STRIDE(p, L.N) residual_point<T, THREE, true>(L, p); }
            else { OW3D_GRID_STRIDE(p, L.N) residual_point<T, THREE, false>(L, p); }
            sy.sync();
            OW3D_GRID_STRIDE(p, Cc.N) restrict_item<T>(L, Cc, L.rv, Cc.bv, Cc.xv, p);
            sy.sync();
        }
    }
    if (part == kWhole) {
        const LevelDev<T>& Ld = P[ld];
        dense_rows<T>((int)Ld.N, M, Ld.bv, Ld.xv);
        sy.sync();
    }
    if (part != kDown) {
        for (int l = lo + 1; l <= lc; ++l) {
            const LevelDev<T>& L = lv(l);
            const LevelDev<T>& Cc = P[l - 1];
            OW3D_GRID_STRIDE(p, L.N) prolong_item<T>(L, Cc, Cc.xv, L.xv, p);
            sy.sync();
            coop_smooth<T, THREE>(L, nu2, sy);
        }
    }
}

template <typename T, bool THREE>
__global__ void __launch_bounds__(kCoopThreads) k_mg_coarse_cycle(const LevelDev<T>* __restrict__ P, int lc, int ld,
                                                                  int lo, int part, const T* __restrict__ M, int nu1,
                                                                  int nu2, T* xtop, T* btop) {
    __shared__ LevelDev<T> top;
    if (threadIdx.x == 0) {
        top = P[lc];
        top.xv = xtop;
        top.bv = btop;
    }
    __syncthreads();
    GridSync sy{cg::this_grid()};
    coarse_body<T, THREE>(P, top, lc, ld, lo, part, M, nu1, nu2, sy);
}

// The small coarse levels (the tail of the cycle) in one thread-block
// cluster: a cluster barrier costs a fraction of a grid-wide one, and these
// levels have fewer points than the cluster has threads.
template <typename T, bool THREE>
__global__ void __launch_bounds__(kCoopThreads) k_mg_tail_cycle(const LevelDev<T>* __restrict__ P, int lc, int ld,
                                                                const T* __restrict__ M, int nu1, int nu2, T* xtop,
                                                                T* btop) {
    __shared__ LevelDev<T> top;
    if (threadIdx.x == 0) {
        top = P[lc];
        top.xv = xtop;
        top.bv = btop;
    }
    __syncthreads();
    ClusterSync sy;
    coarse_body<T, THREE>(P, top, lc, ld, ld, kWhole, M, nu1, nu2, sy);
}

inline int nblk(int64_t n, int t = 256) {
    int64_t b = (n + t - 1) / t;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

template <typename T>
void launch_lo_matvec(const LevelDev<T>& L, const T* x, T* y, cudaStream_t st) {
    if (L.Nyg > 1) launch_k(k_lo_matvec<T, true>, dim3(nblk(L.N)), dim3(256), 0, st, L, x, y);
    else launch_k(k_lo_matvec<T, false>, dim3(nblk(L.N)), dim3(256), 0, st, L, x, y);
}

// Tiled colour pass for the levels it covers (see k_lo_colour_tile); false
// when the level takes the per-column pass. Measured on one B200 (1025 x 257
// x 17): alone after an L2 flush the tiled pass is faster on the two finest
// levels (49 against 55 us, 19 against 24 us, FP64), but inside the solve,
// where the previous kernel leaves x and b in L2, the per-column pass is as
// fast in FP64 and 2-3 ms per step faster in mixed precision; on 2049 x 513
// x 9 (4 lanes per column) the tiled pass is slower alone too (111 against
// 94 us). It is therefore off by default (g_colour_tiles).
template <typename T, int S>
static bool colour_tile_launch(const LevelDev<T>& L, int c, cudaStream_t st) {
    const int min_tiles = g_colour_tiles.load(std::memory_order_relaxed);
    if (S < 4 || L.cross || L.per || L.ncolor != 2 || L.Nxg < 12 || L.Nyg < 12 || min_tiles <= 0) return false;
    const int ntx = (L.Nxg - 6 + kCTX - 1) / kCTX, nty = (L.Nyg - 6 + kCTY - 1) / kCTY;
    if (ntx * nty < min_tiles) return false;
    const TileShape<T> sh = tile_shape<T>(L.Nxg, L.Nzg);
    if (sh.bytes > 200 * 1024) return false;
    static std::atomic<unsigned long long> attr_set{0ull};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_set.load(std::memory_order_relaxed) & bit)) {
        cudaFuncSetAttribute(k_lo_colour_tile<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set.fetch_or(bit, std::memory_order_relaxed);
    }
    const int per_block = (kCTThreads / 32) * (32 / S);
    const int nband = (mgdev::wall_band_count(L) + per_block - 1) / per_block;
    launch_k(k_lo_colour_tile<T, S>, dim3(nband + ntx * nty), dim3(kCTThreads), sh.bytes, st, L, c, nband, ntx, sh);
    return true;
}

template <typename T, bool THREE, int S>
static void colour_launch(const LevelDev<T>& L, int c, cudaStream_t st) {
    if (THREE && colour_tile_launch<T, S>(L, c, st)) return;
    const int64_t cols = (int64_t)((L.Nxg - 1) / 2) * (THREE ? L.Nyg - 2 : 1);
    const int64_t warps = (cols + (32 / S) - 1) / (32 / S);
    int64_t blocks = (warps * 32 + 127) / 128;
    // g_colour_prefetch: 0 = one pass over the columns with up to 32 blocks
    // per SM; 1 = the grid capped at the resident blocks per SM, each warp
    // prefetching its next group into L1; 2 = the capped grid alone; -1 (the
    // default) = 2 for FP64 levels, 0 for FP32 ones, the faster of each
    // measured on a B200 (1025x257x17: FP64 step 80.7 against 82.4 ms, mixed
    // 65.7 against 68.1 ms)
    int pf = g_colour_prefetch.load(std::memory_order_relaxed);
    if (pf < 0) pf = sizeof(T) == 8 ? 2 : 0;
    const int64_t cap = pf ? 148 * colour_blocks_per_sm(L.cross != 0, sizeof(T) == 4) : 148 * 32;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    const int pre = pf == 1 ? 1 : 0;
    if (L.cross) launch_k(k_lo_colour<T, THREE, S, true>, dim3((int)blocks), dim3(128), 0, st, L, c, pre);
    else launch_k(k_lo_colour<T, THREE, S, false>, dim3((int)blocks), dim3(128), 0, st, L, c, pre);
}
// Lanes per column of the two-rows-per-lane pass.
inline int seg_width2(int Nzg) {
    const int R2 = (Nzg - 2 + 1) / 2;
    return R2 <= 2 ? 2 : (R2 <= 4 ? 4 : (R2 <= 8 ? 8 : (R2 <= 16 ? 16 : 32)));
}
template <typename T, bool THREE>
static void colour_dispatch(const LevelDev<T>& L, int c, cudaStream_t st) {
    switch (seg_width2(L.Nzg)) {
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
static void bottoms(const LevelDev<T>& L, cudaStream_t st) {
    const int64_t nyi = L.Nyg > 1 ? L.Nyg - 2 : 1;
    const int64_t n = (int64_t)(L.Nxg - 2) * nyi + 2 * nyi + (L.Nyg > 1 ? 2 * (int64_t)(L.Nxg - 2) : 0);
    if (L.Nyg > 1) launch_k(k_lo_bottom<T, true>, dim3(nblk(n)), dim3(256), 0, st, L);
    else launch_k(k_lo_bottom<T, false>, dim3(nblk(n)), dim3(256), 0, st, L);
}

template <typename T>
void launch_lo_pass(const LevelDev<T>& L, int colour, cudaStream_t st) {
    if (colour < 0) { bottoms(L, st); return; }
    if (L.Nyg > 1) colour_dispatch<T, true>(L, colour, st);
    else colour_dispatch<T, false>(L, colour, st);
}

template <typename T>
void launch_lo_smooth(const LevelDev<T>& L, int nu, cudaStream_t st) {
    if (L.cross) bottoms(L, st);
    for (int s = 0; s < nu; ++s) {
        colours(L, st);
        if (L.cross) bottoms(L, st);
    }
}

template <typename T>
void launch_restrict(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* rf, T* rc, cudaStream_t st) {
    launch_k(k_restrict<T>, dim3(nblk(Cc.N)), dim3(256), 0, st, F, Cc, rf, rc, Cc.xv);
}
template <typename T>
void launch_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* xc, T* xf, cudaStream_t st) {
    launch_k(k_prolong_add<T>, dim3(nblk(F.N)), dim3(256), 0, st, F, Cc, xc, xf);
}
template <typename T>
void launch_coarse_solve(const LevelDev<T>& Lc, const T* inv, cudaStream_t st) {
    int n = (int)Lc.N;
    launch_k(k_coarse<T>, dim3((n + 127) / 128), dim3(128), 0, st, n, inv, Lc.bv, Lc.xv);
}
template <typename T>
void launch_scale_copy(const double* src, double s, T* dst, int64_t n, cudaStream_t st) {
    launch_k(k_scale_copy<T>, dim3(nblk(n)), dim3(256), 0, st, src, s, dst, n);
}
template <typename T>
void launch_fill(T* dst, T v, int64_t n, cudaStream_t st) {
    launch_k(k_fill<T>, dim3(nblk(n)), dim3(256), 0, st, dst, v, n);
}
template <typename T>
void launch_scale_copy_dev(const double* src, const double* ds, T* dst, int64_t n, cudaStream_t st) {
    launch_k(k_scale_copy_dev<T>, dim3(nblk(n)), dim3(256), 0, st, src, ds, dst, n);
}
void launch_convert(const float* src, double* dst, int64_t n, cudaStream_t st) {
    launch_k(k_convert, dim3(nblk(n)), dim3(256), 0, st, src, dst, n);
}

template <typename T>
void launch_dense_apply(const LevelDev<T>& L, const T* M, cudaStream_t st) {
    const int n = (int)L.N;
    const int warps_per_block = 8;
    int blocks = (n + warps_per_block - 1) / warps_per_block;
    if (blocks > 148 * 8) blocks = 148 * 8;
    launch_k(k_dense_apply<T>, dim3(blocks), dim3(32 * warps_per_block), 0, st, n, M, L.bv, L.xv);
}

// Block count of the fused coarse kernel: 0 = one block per SM, else at most
// this many (a tuning knob for measurements, set through the test API).
std::atomic<int> g_coarse_blocks{0};
// Levels with at most this many points run in the fused coarse kernel.
std::atomic<int64_t> g_coop_max_points{160000};
// Levels with at most this many points run in the cluster (tail) kernel (0: none).
std::atomic<int64_t> g_tail_max_points{0};
// Blocks of the tail kernel's cluster (16 needs the non-portable cluster
// size; the launcher falls back to 8 where 16 cannot be resident).
std::atomic<int> g_tail_cluster{16};
// Levels of at least this many tiles take the tiled colour pass (0: none, the
// default: inside the solve the per-column pass measured faster, see the
// launcher).
std::atomic<int> g_colour_tiles{0};
std::atomic<int> g_colour_prefetch{-1};
// Programmatic dependent launch between the solver-path kernels (launch_k).
std::atomic<int> g_pdl{1};

thread_local bool g_capture_unsafe = false;

// Cluster size the tail kernel can run with on this device (0: none):
// the requested size if a cluster of it can be resident, else 8, else 0.
template <typename T, bool THREE>
static int tail_cluster_size(int want) {
    static std::atomic<int> cached[64][17];
    int dev = 0;
    cudaGetDevice(&dev);
    if (want < 1 || want > 16) return 0;
    std::atomic<int>& c = cached[dev & 63][want];
    int v = c.load(std::memory_order_relaxed);
    if (v != 0) return v > 0 ? v : 0;
    auto fits = [&](int cl) {
        if (cl > 8 && cudaFuncSetAttribute((const void*)k_mg_tail_cycle<T, THREE>,
                                           cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            (void)cudaGetLastError();
            return false;
        }
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)cl;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)cl);
        cfg.blockDim = dim3(kCoopThreads);
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (const void*)k_mg_tail_cycle<T, THREE>, &cfg) != cudaSuccess) {
            (void)cudaGetLastError();
            return false;
        }
        return n >= 1;
    };
    v = fits(want) ? want : (want > 8 && fits(8) ? 8 : -1);
    c.store(v, std::memory_order_relaxed);
    return v > 0 ? v : 0;
}

// Launch the fused coarse cycle over levels lc..ld: the levels of at most
// g_tail_max_points points in one thread-block cluster, the larger ones with
// a fully co-resident grid (its descent, then the tail, then its ascent).
template <typename T, bool THREE>
static void coarse_cycle(const LevelDev<T>* lev, int lc, int ld, const T* M, int nu1, int nu2, LevelTable<T>& pack,
                         cudaStream_t st) {
    // one block per SM; a grid that cannot be co-resident makes the launch
    // fail (cudaErrorCooperativeLaunchTooLarge), which the caller's error
    // check reports
    static std::atomic<int> sm_count[64];
    int dev = 0;
    cudaGetDevice(&dev);
    int grid = sm_count[dev & 63].load(std::memory_order_relaxed);
    if (grid == 0) {
        cudaDeviceGetAttribute(&grid, cudaDevAttrMultiProcessorCount, dev);
        sm_count[dev & 63].store(grid, std::memory_order_relaxed);
    }
    const int cap = g_coarse_blocks.load(std::memory_order_relaxed);
    if (cap > 0 && cap < grid) grid = cap;
    // the level table lives in device memory (a by-value parameter indexed
    // by a run-time level would be copied to every thread's stack); upload it
    // only when a level's pointers or sizes changed since the last launch.
    // The top level's iterate and right-hand side are launch arguments (they
    // change between Arnoldi steps when the top level is the finest), so the
    // table holds them as null and stays the same.
    LevelDev<T> cur[kMaxLevels];
    std::memcpy(cur, lev, sizeof(LevelDev<T>) * (size_t)(lc + 1));
    cur[lc].xv = nullptr;
    cur[lc].bv = nullptr;
    if (std::memcmp(pack.host, cur, sizeof(LevelDev<T>) * (size_t)(lc + 1)) != 0) {
        // Inside a stream capture this copy would replay from a host buffer
        // that later calls overwrite: mark the capture unusable and leave the
        // host image as it was, so that the direct launches that replace the
        // capture upload the table themselves.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(st, &cs);
        if (cs != cudaStreamCaptureStatusNone) {
            g_capture_unsafe = true;
        } else {
            std::memcpy(pack.host, cur, sizeof(LevelDev<T>) * (size_t)(lc + 1));
            cudaMemcpyAsync(pack.dev, pack.host, sizeof(LevelDev<T>) * (size_t)(lc + 1), cudaMemcpyHostToDevice, st);
        }
    }
    const LevelDev<T>* P = pack.dev;
    // the tail: levels ld+1..lt of at most g_tail_max_points points
    const int64_t tmax = pack.cluster ? INT64_MAX : g_tail_max_points.load(std::memory_order_relaxed);
    const int cl = tmax > 0 ? tail_cluster_size<T, THREE>(g_tail_cluster.load(std::memory_order_relaxed)) : 0;
    int lt = ld;
    if (cl > 0)
        for (int l = ld + 1; l <= lc && lev[l].N <= tmax; ++l) lt = l;
    auto coop = [&](int lo, int part) {
        T* xtop = lev[lc].xv;
        T* btop = lev[lc].bv;
        void* args[] = {(void*)&P, (void*)&lc, (void*)&ld, (void*)&lo, (void*)&part, (void*)&M,
                        (void*)&nu1, (void*)&nu2, (void*)&xtop, (void*)&btop};
        note_launch();
        cudaLaunchCooperativeKernel((const void*)k_mg_coarse_cycle<T, THREE>, dim3(grid), dim3(kCoopThreads), args, 0,
                                    st);
    };
    if (lt == ld) {
        coop(ld, kWhole);
        return;
    }
    if (lt < lc) coop(lt, kDown);
    {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)cl;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)cl);
        cfg.blockDim = dim3(kCoopThreads);
        cfg.stream = st;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        note_launch();
        cudaLaunchKernelEx(&cfg, k_mg_tail_cycle<T, THREE>, P, lt, ld, M, nu1, nu2, lev[lt].xv, lev[lt].bv);
    }
    if (lt < lc) coop(lt, kUp);
}

template <typename T>
static int coop_level(const LevelDev<T>* lev, int nlev) {
    int lc = -1;
    const int64_t cap = g_coop_max_points.load(std::memory_order_relaxed);
    for (int l = 0; l < nlev; ++l) if (lev[l].N <= cap) lc = l;
    return lc;
}

// MultiGridSolver.f90:5-192 (V cycle, gam = 1), levels lev[0] coarsest;
// level ld is solved by the dense operator M.
template <typename T>
static void vcycle(LevelDev<T>* lev, int l, int lc, int ld, const T* M, int nu1, int nu2, LevelTable<T>& pack,
                   cudaStream_t st) {
    if (l == ld) { launch_dense_apply(lev[l], M, st); return; }
    if (l <= lc) {
        if (lev[0].Nyg > 1) coarse_cycle<T, true>(lev, l, ld, M, nu1, nu2, pack, st);
        else coarse_cycle<T, false>(lev, l, ld, M, nu1, nu2, pack, st);
        return;
    }
    const LevelDev<T>& F = lev[l];
    LevelDev<T>& Cc = lev[l - 1];
    if (pack.lex) launch_lo_smooth_lex(F, nu1, st);
    else launch_lo_smooth(F, nu1, st);
    if (F.Nyg > 1) {
        if (F.cross) launch_k(k_lo_residual<T, true, true>, dim3(nblk(F.N)), dim3(256), 0, st, F);
        else launch_k(k_lo_residual<T, true, false>, dim3(nblk(F.N)), dim3(256), 0, st, F);
    } else {
        if (F.cross) launch_k(k_lo_residual<T, false, true>, dim3(nblk(F.N)), dim3(256), 0, st, F);
        else launch_k(k_lo_residual<T, false, false>, dim3(nblk(F.N)), dim3(256), 0, st, F);
    }
    launch_restrict(F, Cc, (const T*)F.rv, Cc.bv, st);   // also zeroes Cc.xv
    vcycle(lev, l - 1, lc, ld, M, nu1, nu2, pack, st);
    launch_prolong_add(F, Cc, (const T*)Cc.xv, F.xv, st);
    if (pack.lex) launch_lo_smooth_lex(F, nu2, st);
    else launch_lo_smooth(F, nu2, st);
}

// One V cycle from level l (its b set, its x zeroed by the caller) down to the
// dense level ld; used to build the dense operator of a coarse level.
template <typename T>
void launch_mg_subcycle(LevelDev<T>* lev, int nlev, int l, int ld, const T* M, int nu1, int nu2, LevelTable<T>& pack,
                        cudaStream_t st) {
    const int lc = (nlev > 1 && !pack.lex) ? coop_level(lev, nlev) : -1;
    vcycle(lev, l, lc, ld, M, nu1, nu2, pack, st);
}

// MultiGridSolveLinearSystem.f90:26-91: u = 0, then maxit cycles.
template <typename T>
void launch_mg_vcycle(LevelDev<T>* lev, int nlev, const T* M, int ld, int nu1, int nu2, int maxit, LevelTable<T>& pack,
                      cudaStream_t st) {
    LevelDev<T>& F = lev[nlev - 1];
    launch_fill<T>(F.xv, T(0), F.N, st);
    const int lc = (nlev > 1 && !pack.lex) ? coop_level(lev, nlev) : -1;
    for (int it = 1; it <= maxit; ++it) {
        if (nlev == 1 && it > 1) break;
        vcycle(lev, nlev - 1, lc, ld, M, nu1, nu2, pack, st);
    }
}

#define OW3D_INST(T)                                                                                         \
    template void launch_mg_vcycle<T>(LevelDev<T>*, int, const T*, int, int, int, int, LevelTable<T>&, cudaStream_t); \
    template void launch_mg_subcycle<T>(LevelDev<T>*, int, int, int, const T*, int, int, LevelTable<T>&, cudaStream_t); \
    template void launch_dense_apply<T>(const LevelDev<T>&, const T*, cudaStream_t);                        \
    template void launch_lo_matvec<T>(const LevelDev<T>&, const T*, T*, cudaStream_t);                      \
    template void launch_lo_smooth<T>(const LevelDev<T>&, int, cudaStream_t);                               \
    template void launch_lo_pass<T>(const LevelDev<T>&, int, cudaStream_t);                                 \
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
