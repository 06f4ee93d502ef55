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
//   between waves, entirely in shared memory where the level fits there. A
//   larger 3-D level runs in a thread-block cluster instead: each block owns
//   a band of lines j and keeps the band and two lines on either side in its
//   shared memory; a new value goes to the owner's copy and, through
//   distributed shared memory, to the copies in the neighbouring blocks, and
//   a cluster barrier separates the waves.
// * The special pass needs no order beyond three phases: a ghost row reads
//   only its own point and interior points of rows k >= 2, which the pass
//   does not change, and a bottom row reads, besides interior points, the k = 2
//   rows of the ghost columns on its sides. The ghost columns at i = 1 / j = 1
//   precede their neighbours in index order and those at i = Nxg / j = Nyg
//   follow them, so the phases are: the low ghost columns, then the bottom
//   rows, then the high ghost columns, each fully parallel.
#include "ow3d_internal.h"
#include "mg_device.cuh"
#include <cooperative_groups.h>
#include <algorithm>
#include <atomic>

namespace ow3d {

namespace {
using namespace mgdev;
namespace cg = cooperative_groups;

constexpr int kLexThreads = 512;
// levels whose iterate fits in this much shared memory are swept there
constexpr size_t kLexStageBytes = 200 * 1024;

inline unsigned lex_blocks(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (unsigned)(b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

// x_r += (b_r - (A x)_r) / a_rr for row (k, i, j); returns the new value.
template <typename T, bool THREE>
__device__ __forceinline__ T relax_row(const LevelDev<T>& L, T* x, T b, int k, int i, int j) {
    T dg;
    const T ax = lo_row<T, THREE>(L, x, k, i, j, dg);
    const int64_t p = IX(L, k, i, j);
    const T v = x[p] + (b - ax) / dg;
    x[p] = v;
    return v;
}

// Candidate t of wave w among the lines j0..j1-1: its row (k, i, j), or
// false. Rows of one wave share the parity of k - 1 (B is even), so a wave
// has at most ceil(Nzg/2) rows per line.
template <typename T>
__device__ __forceinline__ bool wave_row(const LevelDev<T>& L, int B, int w, int t, int j0, int nk, int& k, int& i,
                                         int& j) {
    const int jj = t / nk;
    k = 2 * (t - jj * nk) + (w & 1) + 1;
    j = j0 + jj + 1;
    const int r2 = w - (k - 1) - B * (j - 1);
    if (k > L.Nzg || r2 < 0) return false;
    i = (r2 >> 1) + 1;
    return i <= L.Nxg;
}

template <typename T>
__device__ __forceinline__ int wave_count(const LevelDev<T>& L, int B) {
    return (L.Nzg - 1) + 2 * (L.Nxg - 1) + B * (L.Nyg - 1) + 1;
}

// One block, all lines. Each thread's right-hand side for the next wave is
// read while the current wave runs (b does not change during the sweep).
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
    const int nk = (L.Nzg + 1) / 2;
    const int cand = L.Nyg * nk;
    const int waves = wave_count(L, B);
    const int t0 = threadIdx.x;
    int k, i, j;
    bool have = t0 < cand && wave_row(L, B, 0, t0, 0, nk, k, i, j);
    T bn = have ? b[IX(L, k, i, j)] : T(0);
    for (int w = 0; w < waves; ++w) {
        const bool cur = have;
        const int kc = k, ic = i, jc = j;
        const T bc = bn;
        have = w + 1 < waves && t0 < cand && wave_row(L, B, w + 1, t0, 0, nk, k, i, j);
        if (have) bn = b[IX(L, k, i, j)];
        if (cur) relax_row<T, THREE>(L, x, bc, kc, ic, jc);
        for (int t = t0 + blockDim.x; t < cand; t += blockDim.x) {
            int k2, i2, j2;
            if (wave_row(L, B, w, t, 0, nk, k2, i2, j2)) relax_row<T, THREE>(L, x, b[IX(L, k2, i2, j2)], k2, i2, j2);
        }
        __syncthreads();
    }
    if (staged)
        for (int64_t p = threadIdx.x; p < L.N; p += blockDim.x) xg[p] = x[p];
}

// Lines of the band of block r of n: [band_start(r), band_start(r + 1)).
__device__ __forceinline__ int band_start(int r, int n, int Nyg) { return (int)((int64_t)r * Nyg / n); }

// A thread-block cluster over a 3-D level. Block c owns the lines of its band
// and holds them, with up to two lines on either side (the reach of a row in
// j), in its shared memory; every line belongs to one band, so one block
// writes it and the blocks whose window holds it receive each new value.
// Every band has at least one line (the cluster has at most Nyg blocks), so
// the windows that hold a line of band c are those of blocks c-2..c+2.
template <typename T, bool THREE>
__global__ void __launch_bounds__(kLexThreads) k_lex_sweep_cluster(LevelDev<T> L, int B) {
    pdl_entry();
    cg::cluster_group cl = cg::this_cluster();
    const int nc = (int)cl.num_blocks();
    const int c = (int)cl.block_rank();
    extern __shared__ __align__(16) unsigned char lex_smem[];
    T* const win = reinterpret_cast<T*>(lex_smem);
    const int Nyg = L.Nyg;
    const int64_t line = (int64_t)L.Nxg * L.Nzg;
    const int j0 = band_start(c, nc, Nyg), j1 = band_start(c + 1, nc, Nyg);
    const int w0 = max(0, j0 - 2), w1 = min(Nyg, j1 + 2);
    T* const xs = win - (int64_t)w0 * line;   // addressed by the level's linear index
    for (int64_t q = threadIdx.x; q < (int64_t)(w1 - w0) * line; q += blockDim.x) win[q] = L.xv[(int64_t)w0 * line + q];
    T* peer[4];
    int pw0[4], pw1[4], np = 0;
    for (int d = -2; d <= 2; ++d) {
        const int r = c + d;
        if (d == 0 || r < 0 || r >= nc) continue;
        const int a = max(0, band_start(r, nc, Nyg) - 2), e = min(Nyg, band_start(r + 1, nc, Nyg) + 2);
        if (a >= j1 || e <= j0) continue;
        peer[np] = cl.map_shared_rank(win, r) - (int64_t)a * line;
        pw0[np] = a;
        pw1[np] = e;
        ++np;
    }
    cl.sync();   // every window loaded before any block writes
    const T* const b = L.bv;
    const int nk = (L.Nzg + 1) / 2;
    const int cand = (j1 - j0) * nk;
    const int waves = wave_count(L, B);
    const int t0 = threadIdx.x;
    int k, i, j;
    bool have = t0 < cand && wave_row(L, B, 0, t0, j0, nk, k, i, j);
    T bn = have ? b[IX(L, k, i, j)] : T(0);
    auto publish = [&](int64_t p, int jr, T v) {
        for (int q = 0; q < np; ++q)
            if (jr - 1 >= pw0[q] && jr - 1 < pw1[q]) peer[q][p] = v;
    };
    for (int w = 0; w < waves; ++w) {
        const bool cur = have;
        const int kc = k, ic = i, jc = j;
        const T bc = bn;
        have = w + 1 < waves && t0 < cand && wave_row(L, B, w + 1, t0, j0, nk, k, i, j);
        if (have) bn = b[IX(L, k, i, j)];
        if (cur) publish(IX(L, kc, ic, jc), jc, relax_row<T, THREE>(L, xs, bc, kc, ic, jc));
        for (int t = t0 + blockDim.x; t < cand; t += blockDim.x) {
            int k2, i2, j2;
            if (wave_row(L, B, w, t, j0, nk, k2, i2, j2))
                publish(IX(L, k2, i2, j2), j2, relax_row<T, THREE>(L, xs, b[IX(L, k2, i2, j2)], k2, i2, j2));
        }
        cl.sync();
    }
    for (int64_t q = (int64_t)j0 * line + threadIdx.x; q < (int64_t)j1 * line; q += blockDim.x) L.xv[q] = xs[q];
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
        for (int k = 1; k <= k1; ++k) relax_row<T, THREE>(L, L.xv, L.bv[IX(L, k, i, j)], k, i, j);
    }
}

template <typename T, bool THREE>
void lex_special(const LevelDev<T>& L, cudaStream_t st) {
    const int64_t C = (int64_t)L.Nxg * L.Nyg;
    for (int ph = 0; ph < 3; ++ph)
        launch_k(k_lex_special<T, THREE>, dim3(lex_blocks(C)), dim3(256), 0, st, L, ph);
}

// Blocks of the cluster the sweep of a 3-D level can run with on this device
// (16, else 8, else 0), for a window of kLexStageBytes.
template <typename T>
int lex_cluster_size() {
    static std::atomic<int> cached[64];
    int dev = 0;
    cudaGetDevice(&dev);
    std::atomic<int>& c = cached[dev & 63];
    int v = c.load(std::memory_order_relaxed);
    if (v != 0) return v > 0 ? v : 0;
    auto fits = [&](int n) {
        const void* f = (const void*)k_lex_sweep_cluster<T, true>;
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLexStageBytes) != cudaSuccess ||
            (n > 8 && cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
            (void)cudaGetLastError();
            return false;
        }
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)n;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)n);
        cfg.blockDim = dim3(kLexThreads);
        cfg.dynamicSmemBytes = kLexStageBytes;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int m = 0;
        if (cudaOccupancyMaxActiveClusters(&m, f, &cfg) != cudaSuccess) {
            (void)cudaGetLastError();
            return false;
        }
        return m >= 1;
    };
    v = fits(16) ? 16 : (fits(8) ? 8 : -1);
    c.store(v, std::memory_order_relaxed);
    return v > 0 ? v : 0;
}

// Shared memory a block of an n-block cluster needs for its window.
template <typename T>
size_t lex_window_bytes(const LevelDev<T>& L, int n) {
    const int band = (L.Nyg + n - 1) / n;
    const int lines = std::min(L.Nyg, band + 4);
    return (size_t)lines * L.Nxg * L.Nzg * sizeof(T);
}

template <typename T, bool THREE>
void lex_sweep(const LevelDev<T>& L, cudaStream_t st) {
    const int B = THREE ? (L.cross ? 6 : 2) : 0;
    const size_t bytes = (size_t)L.N * sizeof(T);
    if (THREE && bytes > kLexStageBytes) {
        int n = lex_cluster_size<T>();
        if (n > L.Nyg) n = L.Nyg >= 8 ? 8 : 0;
        if (n > 0 && lex_window_bytes(L, n) <= kLexStageBytes) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = (unsigned)n;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3((unsigned)n);
            cfg.blockDim = dim3(kLexThreads);
            cfg.dynamicSmemBytes = lex_window_bytes(L, n);
            cfg.stream = st;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            note_launch();
            cudaLaunchKernelEx(&cfg, k_lex_sweep_cluster<T, THREE>, L, B);
            return;
        }
    }
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
