// Gauss-Seidel smoother in the reference's own (lexicographic) order, for the
// multigrid preconditioner when a handle asks for it (ow3d_set_smoother_order).
//
// The reference relaxes the rows of a level one after another in index order
// (k fastest, then i, then j; GaussSeidel.f90:15-26) and relaxes its "special"
// rows -- the bottom row of every column and every row of a lateral ghost
// column (iGhost, MGPreProcess.f90:376-439) -- once more, in index order,
// before the first and after every sweep (GaussSeidelSpecialPoints.f90:43-53,
// MultiGridSolver.f90:118-126,174-181). This file gives both the same results
// on the device, without their sequence:
//
// * The sweep runs as wavefronts. Row (k, i, j) goes in wave
//   (k-1) + 2 (i-1) + B (j-1). For every row r and every point c its equation
//   reads, the wave of c is below the wave of r exactly when the index of c is
//   below the index of r, so each row sees the new values of the points it
//   reads that precede it and the old values of those that follow it, as in
//   the sequential sweep, and no two rows of one wave read each other. The
//   reach of a row (mg_device.cuh): points one step away in k, i and j; the
//   bottom row also k+2; the ghost rows i +-2 or j +-2 at their own k; on
//   levels with mixed-derivative terms the row k = 2 next to a ghost column
//   reads the level-1 points two columns along, one plane to the side
//   (offset (-1, +-2, +-1)), which sets B = 6 there (B = 2 without mixed terms;
//   periodic levels never have them, and their cyclic x-neighbours lie on the
//   same j). One block runs every wave of a level, with a block barrier
//   between waves; levels small enough run entirely in shared memory.
// * The special pass needs no order beyond three phases: a ghost row reads
//   only its own point and interior points of rows k >= 2, which the pass
//   does not change, and a bottom row reads, besides interior points, the k = 2
//   rows of the ghost columns on its sides. The ghost columns at i = 1 / j = 1
//   precede their neighbours in index order and those at i = Nxg / j = Nyg
//   follow them, so the phases are: the low ghost columns, then the bottom
//   rows, then the high ghost columns, each fully parallel.
#include "ow3d_internal.h"
#include "mg_device.cuh"
#include <atomic>

namespace ow3d {

namespace {
using namespace mgdev;

constexpr int kLexThreads = 512;
// levels whose iterate fits in this much shared memory are swept there
constexpr size_t kLexStageBytes = 200 * 1024;

inline unsigned lex_blocks(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (unsigned)(b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

// x_r += (b_r - (A x)_r) / a_rr for row (k, i, j).
template <typename T, bool THREE>
__device__ __forceinline__ void relax_row(const LevelDev<T>& L, T* x, const T* b, int k, int i, int j) {
    T dg;
    const T ax = lo_row<T, THREE>(L, x, k, i, j, dg);
    const int64_t p = IX(L, k, i, j);
    x[p] += (b[p] - ax) / dg;
}

template <typename T, bool THREE>
__global__ void __launch_bounds__(kLexThreads) k_lex_sweep(LevelDev<T> L, int B, int staged) {
    pdl_entry();
    extern __shared__ __align__(16) unsigned char lex_smem[];
    T* const xg = L.xv;
    const T* const b = L.bv;
    T* const x = staged ? reinterpret_cast<T*>(lex_smem) : xg;
    if (staged) {
        for (int64_t p = threadIdx.x; p < L.N; p += blockDim.x) x[p] = xg[p];
        __syncthreads();
    }
    // rows of one wave share the parity of k - 1 (B is even), so a wave has
    // at most ceil(Nzg/2) rows per line j
    const int nk = (L.Nzg + 1) / 2;
    const int cand = L.Nyg * nk;
    const int waves = (L.Nzg - 1) + 2 * (L.Nxg - 1) + B * (L.Nyg - 1) + 1;
    for (int w = 0; w < waves; ++w) {
        const int par = w & 1;
        for (int t = threadIdx.x; t < cand; t += blockDim.x) {
            const int jj = t / nk;
            const int k = 2 * (t - jj * nk) + par + 1;
            const int r2 = w - (k - 1) - B * jj;
            if (k > L.Nzg || r2 < 0) continue;
            const int i = (r2 >> 1) + 1;
            if (i > L.Nxg) continue;
            relax_row<T, THREE>(L, x, b, k, i, jj + 1);
        }
        __syncthreads();
    }
    if (staged)
        for (int64_t p = threadIdx.x; p < L.N; p += blockDim.x) xg[p] = x[p];
}

// One phase of the special pass: 0 the ghost columns at i = 1 or j = 1 (all
// their rows), 1 the bottom rows of the other columns, 2 the remaining ghost
// columns (i = Nxg or j = Nyg).
template <typename T, bool THREE>
__global__ void k_lex_special(LevelDev<T> L, int phase) {
    pdl_entry();
    const int64_t C = (int64_t)L.Nxg * L.Nyg;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(c / L.Nxg) + 1;
        const int i = (int)(c - (int64_t)(j - 1) * L.Nxg) + 1;
        const bool lo = i == 1 || (THREE && j == 1);
        const bool hi = i == L.Nxg || (THREE && j == L.Nyg);
        int k1;
        if (phase == 0) { if (!lo) continue; k1 = L.Nzg; }
        else if (phase == 2) { if (!hi || lo) continue; k1 = L.Nzg; }
        else { if (lo || hi) continue; k1 = 1; }
        for (int k = 1; k <= k1; ++k) relax_row<T, THREE>(L, L.xv, L.bv, k, i, j);
    }
}

template <typename T, bool THREE>
void lex_special(const LevelDev<T>& L, cudaStream_t st) {
    const int64_t C = (int64_t)L.Nxg * L.Nyg;
    for (int ph = 0; ph < 3; ++ph)
        launch_k(k_lex_special<T, THREE>, dim3(lex_blocks(C)), dim3(256), 0, st, L, ph);
}

template <typename T, bool THREE>
void lex_sweep(const LevelDev<T>& L, cudaStream_t st) {
    const int B = THREE ? (L.cross ? 6 : 2) : 0;
    const size_t bytes = (size_t)L.N * sizeof(T);
    const int staged = bytes <= kLexStageBytes ? 1 : 0;
    if (staged) {
        // the shared-memory opt-in is per device; setting it twice is harmless
        static std::atomic<unsigned long long> attr_set{0ull};
        int dev = 0;
        cudaGetDevice(&dev);
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(attr_set.load(std::memory_order_relaxed) & bit)) {
            cudaFuncSetAttribute(k_lex_sweep<T, THREE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLexStageBytes);
            attr_set.fetch_or(bit, std::memory_order_relaxed);
        }
    }
    launch_k(k_lex_sweep<T, THREE>, dim3(1), dim3(kLexThreads), staged ? bytes : 0, st, L, B, staged);
}

template <typename T, bool THREE>
void lex_smooth(const LevelDev<T>& L, int nu, cudaStream_t st) {
    lex_special<T, THREE>(L, st);
    for (int s = 0; s < nu; ++s) {
        lex_sweep<T, THREE>(L, st);
        lex_special<T, THREE>(L, st);
    }
}
}  // namespace

// Special pass, then nu times (lexicographic sweep, special pass):
// MultiGridSolver.f90:118-126 (pre-smoothing) and 174-181 (post-smoothing).
template <typename T>
void launch_lo_smooth_lex(const LevelDev<T>& L, int nu, cudaStream_t st) {
    if (L.Nyg > 1) lex_smooth<T, true>(L, nu, st);
    else lex_smooth<T, false>(L, nu, st);
}

template void launch_lo_smooth_lex<double>(const LevelDev<double>&, int, cudaStream_t);
template void launch_lo_smooth_lex<float>(const LevelDev<float>&, int, cudaStream_t);

}  // namespace ow3d
