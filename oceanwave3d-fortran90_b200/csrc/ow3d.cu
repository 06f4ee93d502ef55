// C ABI and drivers of the B200 OceanWave3D hot path (include/ow3d.h).
//
// One ow3d_handle owns one simulation on one device: grid and stencils, the
// multigrid hierarchy, the Krylov workspace and the free-surface state, all
// resident in device memory for the handle's lifetime. Host pointers passed
// to the API are only read or written during the call.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ow3d_fs.h"
#include "ow3d_internal.h"
#include "../../include/ow3d_test.h"
#include "setup.h"

using namespace ow3d;

std::atomic<unsigned long long> ow3d::g_kernel_launches{0ull};

namespace {

thread_local std::string g_last_error;

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);             \
            return (e_ == cudaErrorMemoryAllocation) ? OW3D_ERR_OOM : OW3D_ERR_CUDA;       \
        }                                                                                  \
    } while (0)

template <typename T>
struct MgSet {
    std::vector<LevelDev<T>> lev;
    T* coarse_inv = nullptr;
    T* dense_op = nullptr;  // dense operator of level dense_level (coarse_inv when 0)
    int dense_level = 0;
    LevelTable<T> table;    // level table of the fused coarse-level kernel
    T* fine_b = nullptr;    // right-hand side of the finest level
    T* fine_x = nullptr;    // iterate of the finest level when not written in place
};

}  // namespace

struct ow3d_handle {
    ow3d_params p;
    GridHost G;
    std::vector<ZoneHost> zones_h;
    int dev = 0;
    cudaStream_t st = nullptr;
    size_t bytes = 0;
    std::vector<void*> allocs;
    bool mixed = false;
    // geometry
    double *SX = nullptr, *SY = nullptr, *SZ = nullptr, *zs = nullptr;
    double *h = nullptr, *hx = nullptr, *hxx = nullptr, *hy = nullptr, *hyy = nullptr;
    HoGrid hg;
    FsArgs fa;
    // multigrid
    MgSet<double> mg64;
    MgSet<float> mg32;
    int nlev = 0;
    // Krylov
    int m = 0;
    int64_t ldv = 0;
    double* V = nullptr;      // (m+1) vectors, stride ldv
    void* Z = nullptr;        // m vectors (FGMRES), element type of the preconditioner
    double* w = nullptr;      // scratch vector
    KrylovState* ks = nullptr;
    KrylovState* ks_host = nullptr;   // pinned
    DotScratch dsc;
    // state
    double *E, *P, *W, *Ex, *Exx, *Ey, *Eyy, *Px, *Py;
    double *tE, *tP, *tW, *tEx, *tExx, *tEy, *tEyy, *tPx, *tPy;
    double *kE[4], *kP[4], *ftmp;
    double *PHI, *LP[2], *RHS;
    double* zerosC = nullptr;
    // host-API staging (allocated on first use)
    double *s_rhs = nullptr, *s_phi = nullptr, *s_E[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // relaxation and filtering
    std::vector<RelaxZoneDev> zones;
    double *fc = nullptr, *F2 = nullptr;
    // pressure damping (2-D decks)
    PDampHost pd_h;
    PDampDev pd{};
    bool pd_on = false;
    // roller breaking model (x flumes with i_breaking > 0)
    BreakDev brk{};
    bool brk_on = false;
    // local smoothing by the vertical acceleration (accel_tol_fact <= 100)
    SmoothDev sm{};
    bool sm_on = false;
    // the flux wavemaker (IncWaveType 3): its signal tables, installed by
    // ow3d_set_paddle_signal before the first step
    PaddleDev pad{};
    bool pad_on = false, pad_set = false;
    int* flag = nullptr;
    int* flag_host = nullptr;
    double hmax = 0;
    // bookkeeping
    double time = 0;
    int64_t tstep = 0;
    ow3d_stats stats{};
    // CUDA graphs of the FGMRES Arnoldi step (preconditioner, operator,
    // DCGS2 passes), one per step index j and sigma-surface arrays
    struct IterGraph {
        const double* surf[5];
        int j;
        cudaGraphExec_t exec;
        unsigned long long kernels;   // kernel nodes, counted per replay
    };
    std::vector<IterGraph> iter_graphs;
    int graphs = 1;
    bool graphs_failed = false;
    // One CUDA graph per RK4 step (from the second step on), by the parity of
    // the step number (the extrapolation history alternates between two
    // buffers). Each of the step's four solves is its initial residual, one
    // conditional node per Arnoldi step whose condition the previous step's
    // stopping test sets on the device, and the solution update; no host
    // round trip happens inside a step.
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        unsigned long long base = 0;       // kernels outside the Arnoldi steps
        unsigned long long per_step = 0;   // kernels of one Arnoldi step
        bool failed = false;
    };
    StepGraph step_graph[2];
    cudaStream_t st2 = nullptr;            // captures the conditional bodies
    StepDev* sd = nullptr;                 // device time level
    SolveLog* slog = nullptr;              // the four solves of the last graph step
    SolveLog* slog_host = nullptr;         // pinned copy
};

namespace {

template <typename T>
int dalloc(ow3d_handle* H, T** p, size_t n) {
    void* q = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) {
        g_last_error = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return OW3D_ERR_OOM;
    }
    H->allocs.push_back(q);
    H->bytes += n * sizeof(T);
    *p = (T*)q;
    return OW3D_OK;
}

template <typename T>
int upload(ow3d_handle* H, T** p, const std::vector<double>& v) {
    int r = dalloc(H, p, v.size());
    if (r) return r;
    std::vector<T> t(v.begin(), v.end());
    CK(cudaMemcpy(*p, t.data(), t.size() * sizeof(T), cudaMemcpyHostToDevice));
    return OW3D_OK;
}

#define TRY(x) do { int r_ = (x); if (r_) return r_; } while (0)

template <typename T>
int build_levels(ow3d_handle* H, MgSet<T>& S, bool alloc_fine_x) {
    const int L = (int)H->G.levels.size();
    S.lev.resize(L);
    for (int l = 0; l < L; ++l) {
        const LevelHost& h = H->G.levels[l];
        LevelDev<T>& d = S.lev[l];
        d.Nx = h.Nx; d.Ny = h.Ny; d.Nz = h.Nz; d.Nxg = h.Nxg; d.Nyg = h.Nyg; d.Nzg = h.Nzg;
        d.N = (int64_t)h.Nxg * h.Nyg * h.Nzg;
        d.ncolor = h.ncolor; d.xc = h.xc; d.yc = h.yc; d.zc = h.zc;
        d.per = H->G.per;
        d.cross = 0;
        for (size_t q = 0; q < h.hx.size(); ++q) if (h.hx[q] != 0.0 || h.hy[q] != 0.0) { d.cross = 1; break; }
        T *sx, *sy, *sz, *zs, *hh, *hx, *hxx, *hy, *hyy;
        TRY(upload(H, &sx, h.SX.w)); TRY(upload(H, &sy, h.SY.w.empty() ? std::vector<double>(1, 0.0) : h.SY.w));
        TRY(upload(H, &sz, h.SZ.w)); TRY(upload(H, &zs, h.zs));
        TRY(upload(H, &hh, h.h)); TRY(upload(H, &hx, h.hx)); TRY(upload(H, &hxx, h.hxx));
        TRY(upload(H, &hy, h.hy)); TRY(upload(H, &hyy, h.hyy));
        d.SX = sx; d.SY = sy; d.SZ = sz; d.zs = zs; d.h = hh; d.hx = hx; d.hxx = hxx; d.hy = hy; d.hyy = hyy;
        double *x, *y, *z, *ix, *iy, *iz;
        TRY(upload(H, &x, h.x)); TRY(upload(H, &y, h.y)); TRY(upload(H, &z, h.z));
        d.x = x; d.y = y; d.z = z;
        // reciprocal of the two-sided spacing, 1/((c[i]-c[i-1]) + (c[i+1]-c[i])), the
        // weight normaliser of MGRestriction3DExplicit.f90:55 / MGProlongation3DExplicit.f90:69
        auto recip = [](const std::vector<double>& c) {
            std::vector<double> r(c.size(), 0.0);
            for (size_t q = 1; q + 1 < c.size(); ++q) r[q] = 1.0 / ((c[q] - c[q - 1]) + (c[q + 1] - c[q]));
            return r;
        };
        TRY(upload(H, &ix, recip(h.x))); TRY(upload(H, &iy, recip(h.y))); TRY(upload(H, &iz, recip(h.z)));
        d.ix = ix; d.iy = iy; d.iz = iz;
        {
            std::vector<double> cf(4 * h.h.size());
            for (size_t q = 0; q < h.h.size(); ++q) {
                const double ih = 1.0 / h.h[q];
                const bool three = h.Nyg > 1;   // 2-D levels ignore any y-derivatives of h
                const double hyq = three ? h.hy[q] : 0.0, hyyq = three ? h.hyy[q] : 0.0;
                cf[4 * q + 0] = ih;
                cf[4 * q + 1] = h.hx[q] * ih;
                cf[4 * q + 2] = hyq * ih;
                cf[4 * q + 3] = (h.hxx[q] + hyyq) * ih - 2.0 * (h.hx[q] * h.hx[q] + hyq * hyq) * ih * ih;
            }
            T* c;
            TRY(upload(H, &c, cf));
            d.cf = c;
        }
        {
            // bottom row (k = 1) of column (i, j): f Dz(x)|_2 + h_x Dx(x)|_2 + h_y Dy(x)|_2
            // with f = 1/h + h_x s2 + h_y s4 at sigma_2 (BuildLinearSystemMatrix.f90:50-70)
            const bool three = h.Nyg > 1;
            const double omb = 1.0 - h.zs[1];
            const double z0 = h.SZ.w[3 + 0], z1 = h.SZ.w[3 + 1], z2 = h.SZ.w[3 + 2];   // order 1, row 2
            std::vector<double> bt(8 * h.h.size(), 0.0);
            for (int jj = 1; jj <= h.Nyg; ++jj)
                for (int ii = 1; ii <= h.Nxg; ++ii) {
                    const size_t q = (size_t)(ii - 1) + (size_t)h.Nxg * (jj - 1);
                    const double ih = 1.0 / h.h[q];
                    const double hxq = h.hx[q], hyq = three ? h.hy[q] : 0.0;
                    const double s2 = omb * (hxq * ih), s4 = omb * (hyq * ih);
                    const double f = three ? (ih + hxq * s2 + hyq * s4) : (ih + hxq * s2);
                    const double* wx = &h.SX.w[(size_t)(ii - 1) * 3];
                    double* o = &bt[8 * q];
                    o[0] = f * z1 + hxq * wx[1];
                    o[1] = f * z2;
                    o[2] = hxq * wx[0];
                    o[3] = hxq * wx[2];
                    if (three) {
                        const double* wy = &h.SY.w[(size_t)(jj - 1) * 3];
                        o[0] += hyq * wy[1];
                        o[4] = hyq * wy[0];
                        o[5] = hyq * wy[2];
                    }
                    o[6] = 1.0 / (f * z0);
                    o[7] = f * z0;
                }
            T* btd;
            TRY(upload(H, &btd, bt));
            d.bt = btd;
        }
        d.mz = div_magic((uint64_t)d.Nzg);
        d.mx = div_magic((uint64_t)d.Nxg);
        div_magic32((uint32_t)d.Nzg, d.mz32, d.sz32);
        div_magic32((uint32_t)d.Nxg, d.mx32, d.sx32);
        d.pix = d.piy = d.piz = nullptr;
        d.pwx = d.pwy = d.pwz = nullptr;
        if (l > 0) {
            // interpolation along one direction of MGProlongation3DExplicit.f90:62-110:
            // coincident fine index n -> coarse 2 + (n-2)/F; in between ->
            // (dE c(n-1) + dW c(n+1)) / (dW + dE). The free-surface row of the
            // coarse grid is not injected (its contribution is zero).
            const LevelHost& hc = H->G.levels[l - 1];
            auto table = [&](const std::vector<double>& cf, int ng, int coarsened, bool zdir,
                             std::vector<int>& idx, std::vector<double>& w) {
                idx.assign(2 * (size_t)ng, 1); w.assign(2 * (size_t)ng, 0.0);
                const int ff = coarsened ? 2 : 1;
                for (int n = 2; n <= ng - 1; ++n) {
                    auto cidx = [&](int m) { return 2 + (m - 2) / ff; };
                    if (!coarsened || ((n - 2) % 2) == 0) {
                        idx[2 * (n - 1)] = cidx(n); w[2 * (n - 1)] = 1.0;
                        idx[2 * (n - 1) + 1] = cidx(n); w[2 * (n - 1) + 1] = 0.0;
                    } else {
                        const double dW = cf[n - 1] - cf[n - 2], dE = cf[n] - cf[n - 1];
                        const double inv = 1.0 / (dW + dE);
                        idx[2 * (n - 1)] = cidx(n - 1); w[2 * (n - 1)] = dE * inv;
                        idx[2 * (n - 1) + 1] = cidx(n + 1); w[2 * (n - 1) + 1] = dW * inv;
                        if (zdir && n + 1 == ng) w[2 * (n - 1) + 1] = 0.0;
                    }
                }
            };
            std::vector<int> ix_, iy_, iz_;
            std::vector<double> wx_, wy_, wz_;
            table(h.x, h.Nxg, hc.xc, false, ix_, wx_);
            if (H->G.per) {
                // periodic x: the coarse repeated column holds zero, so the
                // last distinct fine column interpolates towards coarse
                // column 2; the fine repeated column takes nothing
                for (size_t q = 0; q < ix_.size(); ++q)
                    if (ix_[q] == hc.Nxg - 1) ix_[q] = 2;
                wx_[2 * (size_t)(h.Nxg - 2)] = 0.0; wx_[2 * (size_t)(h.Nxg - 2) + 1] = 0.0;
            }
            if (h.Nyg > 1) table(h.y, h.Nyg, hc.yc, false, iy_, wy_);
            else { iy_.assign(2, 1); wy_.assign(2, 0.0); wy_[0] = 1.0; }
            table(h.z, h.Nzg, hc.zc, true, iz_, wz_);
            auto upi = [&](const int** dst, const std::vector<int>& v) -> int {
                int* q;
                int rr = dalloc(H, &q, v.size());
                if (rr) return rr;
                CK(cudaMemcpy(q, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice));
                *dst = q;
                return OW3D_OK;
            };
            TRY(upi(&d.pix, ix_)); TRY(upi(&d.piy, iy_)); TRY(upi(&d.piz, iz_));
            T *a1, *a2, *a3;
            TRY(upload(H, &a1, wx_)); TRY(upload(H, &a2, wy_)); TRY(upload(H, &a3, wz_));
            d.pwx = a1; d.pwy = a2; d.pwz = a3;
        }
        T* r;
        TRY(dalloc(H, &r, d.N)); d.rv = r;
        if (l < L - 1) {
            T *xv, *bv;
            TRY(dalloc(H, &xv, d.N)); TRY(dalloc(H, &bv, d.N));
            d.xv = xv; d.bv = bv;
        }
    }
    TRY(dalloc(H, &S.table.dev, (size_t)kMaxLevels));
    std::memset((void*)S.table.host, 0, sizeof(S.table.host));
    LevelDev<T>& F = S.lev[L - 1];
    TRY(dalloc(H, &S.fine_b, F.N));
    F.bv = S.fine_b;
    if (alloc_fine_x) TRY(dalloc(H, &S.fine_x, F.N));
    F.xv = S.fine_x;
    return OW3D_OK;
}

// Dense inverse of the coarsest-level operator, probing the matrix-free
// operator with unit vectors (FP64), Gauss-Jordan with partial pivoting.
template <typename T>
int coarse_inverse(ow3d_handle* H, MgSet<T>& S) {
    // FP64 probe on a temporary FP64 copy of the coarsest level
    MgSet<double> tmp;
    ow3d_handle& h = *H;
    const LevelHost& Lh = h.G.levels[0];
    const int n = Lh.Nxg * Lh.Nyg * Lh.Nzg;
    if (n > 4096) { g_last_error = "coarsest multigrid level too large for the dense solve (raise MGmaxgrids)"; return OW3D_ERR_UNSUPPORTED; }
    std::vector<LevelHost> keep = h.G.levels;
    h.G.levels.assign(1, Lh);
    int r = build_levels<double>(H, tmp, false);
    h.G.levels = keep;
    if (r) return r;
    LevelDev<double> L0 = tmp.lev[0];
    double *X, *Y;
    TRY(dalloc(H, &X, (size_t)n * n)); TRY(dalloc(H, &Y, (size_t)n * n));
    std::vector<double> I((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c) I[(size_t)c * n + c] = 1.0;
    CK(cudaMemcpy(X, I.data(), I.size() * sizeof(double), cudaMemcpyHostToDevice));
    for (int c = 0; c < n; ++c) launch_lo_matvec<double>(L0, X + (size_t)c * n, Y + (size_t)c * n, h.st);
    CK(cudaStreamSynchronize(h.st));
    std::vector<double> A((size_t)n * n), colmaj((size_t)n * n);
    CK(cudaMemcpy(colmaj.data(), Y, colmaj.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int c = 0; c < n; ++c) for (int rr = 0; rr < n; ++rr) A[(size_t)rr * n + c] = colmaj[(size_t)c * n + rr];
    std::vector<double> inv((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
    for (int k = 0; k < n; ++k) {
        int pr = k;
        for (int rr = k + 1; rr < n; ++rr) if (std::fabs(A[(size_t)rr * n + k]) > std::fabs(A[(size_t)pr * n + k])) pr = rr;
        if (A[(size_t)pr * n + k] == 0.0) { g_last_error = "singular coarsest-level operator"; return OW3D_ERR_BAD_INPUT; }
        if (pr != k)
            for (int c = 0; c < n; ++c) { std::swap(A[(size_t)k * n + c], A[(size_t)pr * n + c]); std::swap(inv[(size_t)k * n + c], inv[(size_t)pr * n + c]); }
        const double d = A[(size_t)k * n + k];
        for (int c = 0; c < n; ++c) { A[(size_t)k * n + c] /= d; inv[(size_t)k * n + c] /= d; }
        for (int rr = 0; rr < n; ++rr) {
            if (rr == k) continue;
            const double f = A[(size_t)rr * n + k];
            if (f == 0.0) continue;
            for (int c = 0; c < n; ++c) { A[(size_t)rr * n + c] -= f * A[(size_t)k * n + c]; inv[(size_t)rr * n + c] -= f * inv[(size_t)k * n + c]; }
        }
    }
    TRY(upload(H, &S.coarse_inv, inv));
    return OW3D_OK;
}

// Levels with at most this many points, below the finest, may be replaced by
// one dense operator (row-major, n^2 values).
constexpr int64_t kDenseMaxPoints = 2500;

// The preconditioner is independent of the free surface (the low-order
// operator linearises about eta = 0), so the V cycle from a coarse level ld
// down to the coarsest level -- pre-smoothing, residual, restriction, the
// recursion, prolongation and post-smoothing, started from x = 0 -- is a fixed
// linear map b_ld -> x_ld. Build it once by applying that sub-cycle to every
// unit vector, and apply it as one dense product: this replaces ~10 dependent
// phases per level below ld with one.
template <typename T>
int dense_subcycle(ow3d_handle* H, MgSet<T>& S) {
    S.dense_op = S.coarse_inv;
    S.dense_level = 0;
    const int L = (int)S.lev.size();
    int ld = 0;
    for (int l = 1; l <= L - 2; ++l) if (S.lev[l].N <= kDenseMaxPoints) ld = l;
    if (ld == 0) return OW3D_OK;
    LevelDev<T>* lev = S.lev.data();
    const int64_t n = lev[ld].N;
    T* Mcol;
    TRY(dalloc(H, &Mcol, (size_t)(n * n)));
    const T one = T(1);
    for (int64_t c = 0; c < n; ++c) {
        launch_fill<T>(lev[ld].bv, T(0), n, H->st);
        launch_fill<T>(lev[ld].xv, T(0), n, H->st);
        CK(cudaMemcpyAsync(lev[ld].bv + c, &one, sizeof(T), cudaMemcpyHostToDevice, H->st));
        launch_mg_subcycle<T>(lev, L, ld, 0, S.coarse_inv, H->p.nu1, H->p.nu2, S.table, H->st);
        CK(cudaMemcpyAsync(Mcol + c * n, lev[ld].xv, n * sizeof(T), cudaMemcpyDeviceToDevice, H->st));
    }
    CK(cudaStreamSynchronize(H->st));
    CK(cudaGetLastError());
    std::vector<T> col((size_t)(n * n));
    CK(cudaMemcpy(col.data(), Mcol, col.size() * sizeof(T), cudaMemcpyDeviceToHost));
    std::vector<T> row((size_t)(n * n));
    for (int64_t c = 0; c < n; ++c)
        for (int64_t r = 0; r < n; ++r) row[(size_t)(r * n + c)] = col[(size_t)(c * n + r)];
    CK(cudaMemcpy(Mcol, row.data(), row.size() * sizeof(T), cudaMemcpyHostToDevice));
    S.dense_op = Mcol;
    S.dense_level = ld;
    return OW3D_OK;
}

int alloc_state(ow3d_handle* H) {
    const size_t C = (size_t)H->G.C, N = (size_t)H->G.N;
    double** cs[] = {&H->E, &H->P, &H->W, &H->Ex, &H->Exx, &H->Ey, &H->Eyy, &H->Px, &H->Py,
                     &H->tE, &H->tP, &H->tW, &H->tEx, &H->tExx, &H->tEy, &H->tEyy, &H->tPx, &H->tPy,
                     &H->kE[0], &H->kE[1], &H->kE[2], &H->kE[3], &H->kP[0], &H->kP[1], &H->kP[2], &H->kP[3],
                     &H->ftmp, &H->zerosC};
    for (double** q : cs) { TRY(dalloc(H, q, C)); CK(cudaMemset(*q, 0, C * sizeof(double))); }
    double** ns[] = {&H->PHI, &H->LP[0], &H->LP[1], &H->RHS};
    for (double** q : ns) { TRY(dalloc(H, q, N)); CK(cudaMemset(*q, 0, N * sizeof(double))); }
    return OW3D_OK;
}

Surface surface_of(const ow3d_handle* H, const double* E, const double* Ex, const double* Exx, const double* Ey,
                   const double* Eyy) {
    Surface s{E, Ex, Exx, Ey, Eyy};
    return s;
}

template <typename T>
void run_precond(ow3d_handle* H, MgSet<T>& S, const double* src, const double* dscale, T* out) {
    LevelDev<T>* lev = S.lev.data();
    const int L = (int)S.lev.size();
    LevelDev<T>& F = lev[L - 1];
    launch_scale_copy_dev<T>(src, dscale, S.fine_b, F.N, H->st);
    F.xv = out;
    if (S.table.lex)  // the recursion to the coarsest level, as the reference runs it
        launch_mg_vcycle<T>(lev, L, S.coarse_inv, 0, H->p.nu1, H->p.nu2, H->p.maxit, S.table, H->st);
    else
        launch_mg_vcycle<T>(lev, L, S.dense_op, S.dense_level, H->p.nu1, H->p.nu2, H->p.maxit, S.table, H->st);
}

// Apply M^{-1} to src (times *dscale) into the FP64 vector dst.
void precond_into(ow3d_handle* H, const double* src, const double* dscale, double* dst) {
    if (H->nlev == 0) {  // no preconditioner
        launch_scale_copy_dev<double>(src, dscale, dst, H->G.N, H->st);
        return;
    }
    if (!H->mixed) run_precond<double>(H, H->mg64, src, dscale, dst);
    else {
        run_precond<float>(H, H->mg32, src, dscale, H->mg32.fine_x);
        launch_convert(H->mg32.fine_x, dst, H->G.N, H->st);
    }
}

int sync_ks(ow3d_handle* H) {
    CK(cudaMemcpyAsync(H->ks_host, H->ks, sizeof(KrylovState), cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    return OW3D_OK;
}

int sync_ks_small(ow3d_handle* H) {
    // the scalars after the Hessenberg/rotation arrays
    const size_t off = offsetof(KrylovState, w0);
    CK(cudaMemcpyAsync((char*)H->ks_host + off, (char*)H->ks + off, sizeof(KrylovState) - off,
                       cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    return OW3D_OK;
}

// The kernels of Arnoldi step j with the multigrid preconditioner, then the
// DCGS2 reduction and update of the new vector V_{j+1}:
//   FGMRES (right):  z_j = M^{-1} v_j, V_{j+1} = A z_j;
//   left GMRES:      w = A v_j, V_{j+1} = M^{-1} w.
void arnoldi_step_launches(ow3d_handle* H, const Surface& s, int j, int maxmv, int m,
                           cudaGraphConditionalHandle hnext = 0) {
    const int64_t N = H->G.N;
    double* Vj = H->V + (int64_t)j * H->ldv;
    double* Vn = H->V + (int64_t)(j + 1) * H->ldv;
    const double* sj = &H->ks->scale[j];
    if (H->p.krylov == OW3D_KRYLOV_LGMRES) {
        launch_ho_matvec<double>(H->hg, s, Vj, sj, nullptr, H->w, 0, H->st);
        precond_into(H, H->w, nullptr, Vn);
    } else if (!H->mixed) {
        double* Zj = (double*)H->Z + (int64_t)j * H->ldv;
        run_precond<double>(H, H->mg64, Vj, sj, Zj);
        launch_ho_matvec<double>(H->hg, s, Zj, nullptr, nullptr, Vn, 0, H->st);
    } else {
        float* Zj = (float*)H->Z + (int64_t)j * H->ldv;
        run_precond<float>(H, H->mg32, Vj, sj, Zj);
        launch_ho_matvec<float>(H->hg, s, Zj, nullptr, nullptr, Vn, 0, H->st);
    }
    launch_dcgs_reduce(H->V, H->ldv, j, Vn, N, H->dsc, H->ks, H->st);
    launch_dcgs_update(H->V, H->ldv, j, Vn, N, H->dsc, H->ks, maxmv, m, H->st, hnext);
}

// The initial residual of a solve into V_0 (FGMRES: b - A phi; left GMRES:
// M^{-1}(b - A phi)).
void initial_residual_launches(ow3d_handle* H, const Surface& s, const double* rhs, const double* phi) {
    if (H->p.krylov == OW3D_KRYLOV_LGMRES) {
        launch_ho_matvec<double>(H->hg, s, phi, nullptr, rhs, H->w, 1, H->st);
        precond_into(H, H->w, nullptr, H->V);
    } else {
        launch_ho_matvec<double>(H->hg, s, phi, nullptr, rhs, H->V, 1, H->st);
    }
}

// phi += the solve's combination: of Z (FGMRES) or of the final basis V (left
// GMRES, after the back-substitution took the coefficients there).
void solution_update_launches(ow3d_handle* H, double* phi) {
    const int64_t N = H->G.N;
    if (H->p.krylov == OW3D_KRYLOV_LGMRES) {
        launch_backsolve(H->ks, H->st, 1, 1);
        launch_solution_update<double>(phi, H->V, H->ldv, N, H->ks, 1, H->st);
    } else {
        launch_backsolve(H->ks, H->st, 1, 0);
        if (!H->mixed) launch_solution_update<double>(phi, (const double*)H->Z, H->ldv, N, H->ks, 0, H->st);
        else launch_solution_update<float>(phi, (const float*)H->Z, H->ldv, N, H->ks, 0, H->st);
    }
}

// Arnoldi step j as a CUDA graph: captured on its first use (the handle has finished
// a solve by then, so every one-time set-up of the launches is done),
// replayed afterwards. The launch sequence depends on j and on the surface
// arrays only; everything else it touches is fixed for the handle's
// lifetime. A capture that fails switches the handle to direct launches.
int arnoldi_step_graph(ow3d_handle* H, const Surface& s, int j, int maxmv, int m) {
    const double* key[5] = {s.E, s.Ex, s.Exx, s.Ey, s.Eyy};
    ow3d_handle::IterGraph* g = nullptr;
    for (auto& q : H->iter_graphs)
        if (q.j == j && std::memcmp(q.surf, key, sizeof key) == 0) { g = &q; break; }
    if (!g) {
        const unsigned long long k0 = g_kernel_launches.load(std::memory_order_relaxed);
        cudaGraph_t graph = nullptr;
        g_capture_unsafe = false;
        cudaError_t e = cudaStreamBeginCapture(H->st, cudaStreamCaptureModeThreadLocal);
        unsigned long long nk = 0;
        if (e == cudaSuccess) {
            arnoldi_step_launches(H, s, j, maxmv, m);
            e = cudaStreamEndCapture(H->st, &graph);
            if (e == cudaSuccess && g_capture_unsafe) e = cudaErrorStreamCaptureUnsupported;
        }
        // the captured launches did not run: count them per replay instead
        nk = g_kernel_launches.load(std::memory_order_relaxed) - k0;
        g_kernel_launches.fetch_sub(nk, std::memory_order_relaxed);
        cudaGraphExec_t ex = nullptr;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            cudaGetLastError();
            H->graphs_failed = true;
            arnoldi_step_launches(H, s, j, maxmv, m);
            CK(cudaGetLastError());
            return OW3D_OK;
        }
        ow3d_handle::IterGraph ng;
        std::memcpy(ng.surf, key, sizeof key);
        ng.j = j; ng.exec = ex; ng.kernels = nk;
        H->iter_graphs.push_back(ng);
        g = &H->iter_graphs.back();
    }
    CK(cudaGraphLaunch(g->exec, H->st));
    g_kernel_launches.fetch_add(g->kernels, std::memory_order_relaxed);
    return OW3D_OK;
}

// The counters of OceanWave3DTakeATimeStep.f90:76-122 for one solve.
void record_solve(ow3d_handle* H, int it, double resid, double r0, double tol, bool not_converged) {
    ow3d_stats& S = H->stats;
    S.solves++;
    S.total_iterations += it;
    S.min_iterations = (S.solves == 1) ? it : std::min(S.min_iterations, it);
    S.max_iterations = std::max(S.max_iterations, it);
    S.last_iterations = it;
    S.last_residual = resid;
    S.last_initial_residual = r0;
    S.last_tolerance = tol;
    if (not_converged) S.not_converged++;
}

// One Laplace solve on the device: phi <- A^{-1} rhs, initial guess in phi.
int solve_device(ow3d_handle* H, const double* rhs, double* phi, const Surface& s, int* iters_out) {
    const int64_t N = H->G.N;
    const int m = H->m, maxmv = H->p.GMRESmaxiterations;
    launch_krylov_reset(H->ks, H->st);
    int status = OW3D_OK;
    double r0 = 0, tol = 0;
    for (int cycle = 0; cycle < 1000; ++cycle) {
        initial_residual_launches(H, s, rhs, phi);
        launch_norm_init(H->V, N, H->dsc, H->ks, H->p.reltol, H->p.abstol, H->st);
        TRY(sync_ks_small(H));
        if (cycle == 0) { r0 = H->ks_host->beta; tol = H->ks_host->tol; }
        int j = 0;
        while (!H->ks_host->done) {
            if (H->nlev > 0 && H->graphs && !H->graphs_failed && H->stats.solves > 0) {
                // Arnoldi step j as one graph launch
                TRY(arnoldi_step_graph(H, s, j, maxmv, m));
            } else if (H->nlev == 0 && H->p.krylov != OW3D_KRYLOV_LGMRES) {
                // FGMRES without a preconditioner: z_j = v_j
                double* Vj = H->V + (int64_t)j * H->ldv;
                double* Vn = H->V + (int64_t)(j + 1) * H->ldv;
                double* Zj = (double*)H->Z + (int64_t)j * H->ldv;
                launch_scale_copy_dev<double>(Vj, &H->ks->scale[j], Zj, N, H->st);
                launch_ho_matvec<double>(H->hg, s, Zj, nullptr, nullptr, Vn, 0, H->st);
                launch_dcgs_reduce(H->V, H->ldv, j, Vn, N, H->dsc, H->ks, H->st);
                launch_dcgs_update(H->V, H->ldv, j, Vn, N, H->dsc, H->ks, maxmv, m, H->st);
            } else {
                arnoldi_step_launches(H, s, j, maxmv, m);
            }
            TRY(sync_ks_small(H));
            ++j;
        }
        if (H->ks_host->k > 0) solution_update_launches(H, phi);
        TRY(sync_ks_small(H));
        if (H->ks_host->converged) break;
        if (H->ks_host->iters >= maxmv) { status = OW3D_NOT_CONVERGED; break; }
        // restart: the subspace filled before the matvec limit
        launch_krylov_restart(H->ks, H->st);
    }
    const int it = H->ks_host->iters;
    if (iters_out) *iters_out = it;
    record_solve(H, it, H->ks_host->resid, r0, tol, status == OW3D_NOT_CONVERGED);
    CK(cudaGetLastError());
    return status;
}

int check_dims(const ow3d_params* p) {
    if (!p) return OW3D_ERR_BAD_INPUT;
    if (p->solver != 1) { g_last_error = "only GMRES (solver = 1) is supported"; return OW3D_ERR_UNSUPPORTED; }
    if (p->Precond != 3 && p->Precond != 0) { g_last_error = "Precond must be 3 (multigrid) or 0"; return OW3D_ERR_UNSUPPORTED; }
    if (p->cyclet != 'V' && p->cyclet != 'v') { g_last_error = "only V cycles are supported"; return OW3D_ERR_UNSUPPORTED; }
    if (p->GMRESmaxiterations < 2 || p->GMRESmaxiterations > kMaxKrylov) { g_last_error = "GMRESmaxiterations out of range"; return OW3D_ERR_BAD_INPUT; }
    if (p->timemethod != 1) { g_last_error = "only RK4 (timemethod = 1) is supported"; return OW3D_ERR_UNSUPPORTED; }
    if (p->PressureTermOnOff != 0) { g_last_error = "applied surface pressure is not supported"; return OW3D_ERR_UNSUPPORTED; }
    return OW3D_OK;
}

int create_impl(const ow3d_params* p, const double* h, const double* hx, const double* hxx, const double* hy,
                const double* hyy, ow3d_handle** out) {
    TRY(check_dims(p));
    std::string err;
    if (check_supported(*p, &err) != 0) { g_last_error = err; return OW3D_ERR_UNSUPPORTED; }
    std::unique_ptr<ow3d_handle> H(new ow3d_handle());
    H->p = *p;
    H->mixed = (p->precision == OW3D_PREC_MIXED);
    int r = build_grid(*p, h, hx, hxx, hy, hyy, H->G, &err);
    if (r) { g_last_error = err; return r; }
    // the inputs are checked before any device work, so a bad deck is
    // reported as such on a machine without a GPU too
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { g_last_error = "no CUDA device"; return OW3D_ERR_NO_DEVICE; }
    H->dev = p->device;
    CK(cudaSetDevice(H->dev));
    CK(cudaStreamCreateWithFlags(&H->st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&H->st2, cudaStreamNonBlocking));
    GridHost& G = H->G;
    TRY(upload(H.get(), &H->SX, G.SX.w));
    TRY(upload(H.get(), &H->SY, G.SY.w.empty() ? std::vector<double>(1, 0.0) : G.SY.w));
    TRY(upload(H.get(), &H->SZ, G.SZ.w));
    TRY(upload(H.get(), &H->zs, G.zs));
    TRY(upload(H.get(), &H->h, G.h)); TRY(upload(H.get(), &H->hx, G.hx)); TRY(upload(H.get(), &H->hxx, G.hxx));
    TRY(upload(H.get(), &H->hy, G.hy)); TRY(upload(H.get(), &H->hyy, G.hyy));
    HoGrid& hg = H->hg;
    hg.Nxg = G.Nxg; hg.Nyg = G.Nyg; hg.Nzg = G.Nzg; hg.gx = G.gx; hg.gy = G.gy; hg.three = G.three;
    hg.nonlinear = (p->LinearONOFF == 1); hg.per = G.per; hg.SX = H->SX; hg.SY = H->SY; hg.SZ = H->SZ; hg.zs = H->zs;
    hg.h = H->h; hg.hx = H->hx; hg.hxx = H->hxx; hg.hy = H->hy; hg.hyy = H->hyy;
    hg.hSX = G.SX.w.data(); hg.hSY = G.SY.w.data(); hg.hSZ = G.SZ.w.data(); hg.hzs = G.zs.data();
    FsArgs& fa = H->fa;
    fa.Nxg = G.Nxg; fa.Nyg = G.Nyg; fa.Nzg = G.Nzg; fa.three = G.three; fa.nonlinear = hg.nonlinear; fa.g = p->g;
    fa.per = G.per;
    fa.SX = H->SX; fa.SY = H->SY; fa.SZ = H->SZ; fa.h = H->h;
    // OceanWave3DT0Setup.f90:325-326: Ul = Q / h(1,1), Ur = Q / h(Nx+GhostGridX,1)
    fa.Ul = p->current_flag ? p->current_Q / G.h[0] : 0.0;
    fa.Ur = p->current_flag ? p->current_Q / G.h[(size_t)G.Nxg - 2] : 0.0;
    H->hmax = *std::max_element(G.h.begin(), G.h.end());
    // multigrid
    H->nlev = (int)G.levels.size();
    if (H->nlev > 0) {
        if (!H->mixed) {
            TRY(build_levels<double>(H.get(), H->mg64, true));
            TRY(coarse_inverse<double>(H.get(), H->mg64));
            TRY(dense_subcycle<double>(H.get(), H->mg64));
        } else {
            TRY(build_levels<float>(H.get(), H->mg32, true));
            TRY(coarse_inverse<float>(H.get(), H->mg32));
            TRY(dense_subcycle<float>(H.get(), H->mg32));
        }
    }
    // Krylov workspace
    H->m = p->GMRESmaxiterations;
    H->ldv = (G.N + 31) / 32 * 32;
    TRY(dalloc(H.get(), &H->V, (size_t)(H->m + 1) * H->ldv));
    if (p->krylov == OW3D_KRYLOV_FGMRES) {
        if (H->mixed) { float* z; TRY(dalloc(H.get(), &z, (size_t)H->m * H->ldv)); H->Z = z; }
        else { double* z; TRY(dalloc(H.get(), &z, (size_t)H->m * H->ldv)); H->Z = z; }
    }
    TRY(dalloc(H.get(), &H->w, (size_t)H->ldv));
    // the Krylov kernels read element pairs up to n rounded up: padding stays zero
    CK(cudaMemset(H->V, 0, sizeof(double) * (size_t)(H->m + 1) * H->ldv));
    CK(cudaMemset(H->w, 0, sizeof(double) * (size_t)H->ldv));
    if (H->Z) CK(cudaMemset(H->Z, 0, (H->mixed ? sizeof(float) : sizeof(double)) * (size_t)H->m * H->ldv));
    TRY(dalloc(H.get(), &H->ks, 1));
    CK(cudaMallocHost(&H->ks_host, sizeof(KrylovState)));
    std::memset(H->ks_host, 0, sizeof(KrylovState));
    H->dsc.nblocks = 148 * 4;
    TRY(dalloc(H.get(), &H->dsc.partial, (size_t)(kMaxKrylov + 2) * H->dsc.nblocks));
    TRY(dalloc(H.get(), &H->dsc.counter, 1));
    CK(cudaMemset(H->dsc.counter, 0, sizeof(unsigned int)));
    TRY(alloc_state(H.get()));
    // relaxation zones and filter
    H->zones_h = build_zones(*p, G);
    for (const ZoneHost& z : H->zones_h) {
        RelaxZoneDev d{};
        d.i0 = z.i0; d.i1 = z.i1; d.j0 = z.j0; d.j1 = z.j1; d.xdir = z.xdir; d.wavegen = z.wavegen; d.phion = z.phion;
        double* g;
        TRY(upload(H.get(), &g, z.gam));
        d.gam = g; d.tmode = 0; d.nt = 0; d.tdt = 1.0; d.eta = nullptr; d.phis = nullptr;
        H->zones.push_back(d);
    }
    if (p->PDampingONOFF != 0) {
        std::string e;
        if (int r = build_pdamp(*p, G, H->pd_h, &e)) { g_last_error = "ow3d_create: " + e; return r; }
        PDampDev& d = H->pd;
        const PDampHost& ph = H->pd_h;
        d.type = ph.type; d.i1 = ph.i1; d.nd = ph.nd; d.rank = ph.rank;
        d.Ur = p->current_flag ? p->current_Q / G.h[(size_t)G.Nxg - 2] : 0.0;
        double *gp, *ge;
        TRY(upload(H.get(), &gp, ph.gamPhi)); TRY(upload(H.get(), &ge, ph.gamEta));
        d.gamPhi = gp; d.gamEta = ge;
        if (d.type == 0) {
            double *w, *li;
            TRY(upload(H.get(), &w, ph.D1)); TRY(upload(H.get(), &li, ph.Linv));
            d.D1 = w; d.Linv = li;
            TRY(dalloc(H.get(), &d.f, (size_t)ph.nd)); TRY(dalloc(H.get(), &d.r, (size_t)ph.nd));
            TRY(dalloc(H.get(), &d.x, (size_t)ph.nd));
        }
        TRY(dalloc(H.get(), &d.NuD, (size_t)G.C)); TRY(dalloc(H.get(), &d.Pd, (size_t)G.C));
        CK(cudaMemset(d.NuD, 0, sizeof(double) * (size_t)G.C));
        CK(cudaMemset(d.Pd, 0, sizeof(double) * (size_t)G.C));
        H->pd_h.L.clear(); H->pd_h.L.shrink_to_fit(); H->pd_h.Linv.clear(); H->pd_h.Linv.shrink_to_fit();
        H->pd_on = true;
    }
    if (p->IncWaveType == 3) {
        PaddleDev& d = H->pad;
        d.Nyg = G.Nyg; d.j0 = 1 + G.gy; d.j1 = G.Ny + G.gy; d.ramp = p->flux_ramp;
        TRY(dalloc(H.get(), &d.Uw, (size_t)G.Nyg)); TRY(dalloc(H.get(), &d.Es, (size_t)G.Nyg));
        CK(cudaMemset(d.Uw, 0, sizeof(double) * (size_t)G.Nyg));
        CK(cudaMemset(d.Es, 0, sizeof(double) * (size_t)G.Nyg));
        H->fa.Uw = d.Uw; H->fa.Es = d.Es;
        H->pad_on = true;
    }
    if (smoothing_on(*p)) {
        SmoothDev& m = H->sm;
        m.tol = p->accel_tol_fact * p->g;
        m.dt_inv = 1.0 / p->dt;
        m.z = H->zs; m.hx = H->hx; m.hy = H->hy;
        for (int q = 0; q < 3; ++q) {
            TRY(dalloc(H.get(), &m.WH[q], (size_t)G.C));
            CK(cudaMemset(m.WH[q], 0, sizeof(double) * (size_t)G.C));
        }
        TRY(dalloc(H.get(), &m.Wt, (size_t)G.C)); TRY(dalloc(H.get(), &m.flag, (size_t)G.C));
        TRY(dalloc(H.get(), &m.any, 1)); TRY(dalloc(H.get(), &m.sE, (size_t)G.C)); TRY(dalloc(H.get(), &m.sP, (size_t)G.C));
        CK(cudaMemset(m.Wt, 0, sizeof(double) * (size_t)G.C));
        CK(cudaMemset(m.flag, 0, sizeof(int) * (size_t)G.C));
        H->sm_on = true;
    }
    if (breaking_on(*p)) {
        // DetectBreaking.f90:38-70 (its first call): tan(phi) starts at tan(phi_b)
        BreakDev& b = H->brk;
        const int nfx = G.Nxg;
        b.nfx = nfx; b.cap = nfx; b.dynamics = p->i_breaking == 1 ? 1 : 0;
        b.dx = p->Lx / ((double)p->Nx - 1.0); b.dx_inv = 1.0 / b.dx;
        b.g = p->g; b.del_fac = p->del_fac; b.dt = p->dt; b.T_half = p->T_half;
        const double deg2rad = std::acos(-1.0) / 180.0;   // Initialize.f90:7-8
        b.tan_b = std::tan(deg2rad * p->phi_b); b.tan_0 = std::tan(deg2rad * p->phi_0);
        TRY(upload(H.get(), &b.tan_phi, std::vector<double>((size_t)nfx, b.tan_b)));
        TRY(dalloc(H.get(), &b.tan_old, (size_t)nfx)); TRY(dalloc(H.get(), &b.eta_x, (size_t)nfx + 1));
        TRY(dalloc(H.get(), &b.thick, (size_t)nfx + 1)); TRY(dalloc(H.get(), &b.Qr_x, (size_t)nfx));
        TRY(dalloc(H.get(), &b.n_rollers, 1));
        TRY(dalloc(H.get(), &b.npts, (size_t)nfx)); TRY(dalloc(H.get(), &b.toe, (size_t)nfx));
        TRY(dalloc(H.get(), &b.xr, (size_t)nfx)); TRY(dalloc(H.get(), &b.sr, (size_t)nfx));
        TRY(dalloc(H.get(), &b.r_thick, (size_t)nfx)); TRY(dalloc(H.get(), &b.r_tan, (size_t)nfx));
        CK(cudaMemset(b.Qr_x, 0, sizeof(double) * (size_t)nfx));
        CK(cudaMemset(b.n_rollers, 0, sizeof(int)));
        H->brk_on = true;
    }
    if (p->filteringONOFF > 0) {
        std::vector<double> fc, F2;
        filter_coeffs(*p, fc, F2);
        TRY(upload(H.get(), &H->fc, fc)); TRY(upload(H.get(), &H->F2, F2));
    }
    TRY(dalloc(H.get(), &H->flag, 1));
    CK(cudaMemset(H->flag, 0, sizeof(int)));
    CK(cudaMallocHost(&H->flag_host, sizeof(int)));
    TRY(dalloc(H.get(), &H->slog, 4));
    CK(cudaMallocHost(&H->slog_host, 4 * sizeof(SolveLog)));
    TRY(dalloc(H.get(), &H->sd, 1));
    {
        const StepDev s0{p->time0, 0};
        CK(cudaMemcpy(H->sd, &s0, sizeof(StepDev), cudaMemcpyHostToDevice));
    }
    H->time = p->time0;
    H->stats.time = H->time;
    CK(cudaStreamSynchronize(H->st));
    CK(cudaGetLastError());
    *out = H.release();
    return OW3D_OK;
}

int ensure_staging(ow3d_handle* H) {
    if (H->s_rhs) return OW3D_OK;
    TRY(dalloc(H, &H->s_rhs, (size_t)H->G.N));
    TRY(dalloc(H, &H->s_phi, (size_t)H->G.N));
    for (int q = 0; q < 5; ++q) TRY(dalloc(H, &H->s_E[q], (size_t)H->G.C));
    return OW3D_OK;
}

int stage_surface(ow3d_handle* H, const double* E, const double* Ex, const double* Exx, const double* Ey,
                  const double* Eyy, Surface& s) {
    const double* src[5] = {E, Ex, Exx, Ey, Eyy};
    const double* dst[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int q = 0; q < 5; ++q) {
        if (!src[q]) continue;
        CK(cudaMemcpyAsync(H->s_E[q], src[q], sizeof(double) * H->G.C, cudaMemcpyHostToDevice, H->st));
        dst[q] = H->s_E[q];
    }
    s = Surface{dst[0], dst[1], dst[2], dst[3], dst[4]};
    return OW3D_OK;
}

// ------------------------------------------------------------- RK4 step
// The kernels of RK4 step number `tstep` (Runge_Kutta_4.f90:1-429, the
// reference's stage sequence) on the handle's stream. solve(surface, k)
// performs or enqueues the k-th Laplace solve of the step (k = 0..3). With
// `graph` set the step is being captured: the records the host reads after
// the step (instability flag, the solves' outcomes) are copied to pinned
// memory at its end.
template <typename SolveF>
int enqueue_step(ow3d_handle* H, int64_t tstep, bool graph, SolveF&& solve) {
    if (H->pad_on && !H->pad_set) {
        g_last_error = "IncWaveType 3: install the paddle signal (ow3d_set_paddle_signal) before stepping";
        return OW3D_ERR_BAD_INPUT;
    }
    cudaStream_t st = H->st;
    const double dt = H->p.dt, half = 0.5, time = H->time;
    const int64_t N = H->G.N;
    double* LPnew = H->LP[(tstep - 1) % 2];
    double* LPlast = H->LP[tstep % 2];
    fs_step_begin(H->sd, st);
    CK(cudaMemcpyAsync(LPnew, H->PHI, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    const FsArgs& fa = H->fa;
    auto relax = [&](double* E, double* P, double off) {
        if (H->p.relaxONOFF == 1)
            fs_relax(fa, H->zones.data(), (int)H->zones.size(), E, P, H->sd, off, H->p.relaxTransientTime, st);
    };
    auto derivs = [&](double* E, double* P, double* Ex, double* Exx, double* Px, double* Ey, double* Eyy, double* Py,
                      int src) { fs_derivs(fa, E, P, Ex, Exx, Px, Ey, Eyy, Py, src, st); };
    // waveGenerationFromPaddleSignal at RK time (step start) + off: stages 1
    // and 3 (Runge_Kutta_4.f90:83-85,264-266); the last stage's call, at the
    // same time as stage 3's, gives the same values
    auto paddle = [&](double off) {
        if (H->pad_on) fs_paddle(H->pad, H->sd, off, st);
    };
    const bool nl = H->p.LinearONOFF == 1;
    auto surf = [&](const double* E, const double* Ex, const double* Exx, const double* Ey, const double* Eyy) {
        return nl ? Surface{E, Ex, Exx, Ey, Eyy} : Surface{nullptr, nullptr, nullptr, nullptr, nullptr};
    };
    // funPressureTerm at each stage (Runge_Kutta_4.f90:50,159,239,334): the
    // damping terms of the stage's state when its time is positive; at
    // t <= 0 they keep their last values (steps with pressure damping are
    // never captured, so the host time is the step's)
    const double* NuD = H->pd_on ? H->pd.NuD : nullptr;
    const double* Pd = H->pd_on ? H->pd.Pd : nullptr;
    auto pdamp = [&](const double* E, const double* P, double t) {
        if (H->pd_on && t > 0) fs_pdamp(fa, H->pd, E, P, st);
    };
    // detect_breaking at each stage (Runge_Kutta_4.f90:55-57,164-166,241-243,
    // 336-338): the stage's rollers give the Qr_x its fs_stage subtracts; it
    // only changes the dynamics with i_breaking == 1
    const bool brk_dyn = H->brk_on && H->brk.dynamics;
    const double* Qr = brk_dyn ? H->brk.Qr_x : nullptr;
    auto breaking = [&](const double* E) {
        if (brk_dyn) fs_breaking(H->brk, E, 0, st);
    };
    // stage 1
    pdamp(H->E, H->P, time);
    breaking(H->E);
    fs_stage(fa, H->E, H->P, H->W, H->Ex, H->Px, H->Ey, H->Py, H->E, H->P, half * dt, H->kE[0], H->kP[0], H->tE, H->tP,
             NuD, Pd, Qr, st);
    relax(H->tE, H->tP, half * dt);
    paddle(half * dt);
    derivs(H->tE, H->tP, H->tEx, H->tExx, H->tPx, H->tEy, H->tEyy, H->tPy, 1);
    fs_set_rhs(fa, H->tP, H->RHS, st);
    if (H->p.extrapolationONOFF == 1) fs_extrap(H->PHI, LPnew, LPlast, N, 0, H->sd, st);
    TRY(solve(surf(H->tE, H->tEx, H->tExx, H->tEy, H->tEyy), 0));
    fs_wvel(fa, H->PHI, H->tE, H->tW, st);
    // stage 2
    pdamp(H->tE, H->tP, time + half * dt);
    breaking(H->tE);
    fs_stage(fa, H->tE, H->tP, H->tW, H->tEx, H->tPx, H->tEy, H->tPy, H->E, H->P, half * dt, H->kE[1], H->kP[1], H->tE,
             H->tP, NuD, Pd, Qr, st);
    relax(H->tE, H->tP, half * dt);
    derivs(H->tE, H->tP, H->tEx, H->tExx, H->tPx, H->tEy, H->tEyy, H->tPy, 1);
    fs_set_rhs(fa, H->tP, H->RHS, st);
    TRY(solve(surf(H->tE, H->tEx, H->tExx, H->tEy, H->tEyy), 1));
    fs_wvel(fa, H->PHI, H->tE, H->tW, st);
    // stage 3
    pdamp(H->tE, H->tP, time + half * dt);
    breaking(H->tE);
    fs_stage(fa, H->tE, H->tP, H->tW, H->tEx, H->tPx, H->tEy, H->tPy, H->E, H->P, dt, H->kE[2], H->kP[2], H->tE, H->tP,
             NuD, Pd, Qr, st);
    relax(H->tE, H->tP, dt);
    paddle(dt);
    derivs(H->tE, H->tP, H->tEx, H->tExx, H->tPx, H->tEy, H->tEyy, H->tPy, 1);
    fs_set_rhs(fa, H->tP, H->RHS, st);
    // Runge_Kutta_4.f90:294-303, from the second step on (checked on the device)
    if (H->p.extrapolationONOFF == 1) fs_extrap(H->PHI, LPnew, LPlast, N, 1, H->sd, st);
    TRY(solve(surf(H->tE, H->tEx, H->tExx, H->tEy, H->tEyy), 2));
    fs_wvel(fa, H->PHI, H->tE, H->tW, st);
    // stage 4 and the new time level
    pdamp(H->tE, H->tP, time + dt);
    breaking(H->tE);
    fs_stage(fa, H->tE, H->tP, H->tW, H->tEx, H->tPx, H->tEy, H->tPy, nullptr, nullptr, 0.0, H->kE[3], H->kP[3], nullptr,
             nullptr, NuD, Pd, Qr, st);
    fs_rk_final(fa, H->E, H->P, H->kE, H->kP, dt, st);
    if (H->p.filteringONOFF > 0) {
        // every filteringONOFF steps (Runge_Kutta_4.f90:355-362; the step number is checked on the device)
        FilterDev f{H->p.filterALPHA, H->fc, H->F2};
        fs_filter(fa, f, H->E, H->ftmp, H->sd, H->p.filteringONOFF, st);
        fs_filter(fa, f, H->P, H->ftmp, H->sd, H->p.filteringONOFF, st);
    }
    relax(H->E, H->P, dt);
    derivs(H->E, H->P, H->Ex, H->Exx, H->Px, H->Ey, H->Eyy, H->Py, 2);
    fs_set_rhs(fa, H->P, H->RHS, st);
    TRY(solve(surf(H->E, H->Ex, H->Exx, H->Ey, H->Eyy), 3));
    fs_wvel(fa, H->PHI, H->E, H->W, st);
    // OceanWave3DTakeATimeStep.f90:33-39: local smoothing (from the third
    // step on; the step number is read on the device)
    if (H->sm_on) TRY(fs_local_smoothing(fa, H->sm, H->PHI, H->E, H->P, H->Ex, H->Ey, H->W, H->kE, H->sd, st));
    // the rollers of the new state and the roller-angle update
    // (OceanWave3DTakeATimeStep.f90:45-49)
    if (H->brk_on) fs_breaking(H->brk, H->E, 1, st);
    fs_step_end(H->sd, dt, st);
    // OceanWave3DTakeATimeStep.f90:54-70
    fs_unstable(fa, H->E, 10.0 * H->hmax, H->flag, st);
    CK(cudaMemcpyAsync(H->flag_host, H->flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (graph) CK(cudaMemcpyAsync(H->slog_host, H->slog, 4 * sizeof(SolveLog), cudaMemcpyDeviceToHost, st));
    return OW3D_OK;
}

// Host bookkeeping after step number tstep completed on the device.
int finish_step(ow3d_handle* H, int64_t tstep) {
    if (*H->flag_host) { g_last_error = "max|eta| > 10 max h: the solution went unstable"; return OW3D_ERR_UNSTABLE; }
    H->tstep = tstep;
    H->time = H->time + H->p.dt;
    H->stats.time = H->time;
    H->stats.tstep = H->tstep;
    return OW3D_OK;
}

// One RK4 step with host-driven solves (per Arnoldi step graphs where they apply).
int rk4_step(ow3d_handle* H) {
    const int64_t tstep = H->tstep + 1;
    int status = OW3D_OK;
    auto solve = [&](const Surface& s, int) -> int {
        int it = 0;
        int r = solve_device(H, H->RHS, H->PHI, s, &it);
        if (r < 0) return r;
        if (r == OW3D_NOT_CONVERGED) status = OW3D_NOT_CONVERGED;
        return OW3D_OK;
    };
    TRY(enqueue_step(H, tstep, false, solve));
    CK(cudaStreamSynchronize(H->st));
    TRY(finish_step(H, tstep));
    CK(cudaGetLastError());
    return status;
}

// One solve of a captured step: the initial residual, then one conditional
// node per Arnoldi step (FGMRES with the multigrid preconditioner): node j
// runs step j when its condition, set by the stopping test of step j-1 (or
// of the initial residual), says the solve is not done. The subspace holds
// m = GMRESmaxiterations vectors and the matvec limit is the same m, so a
// solve never restarts. kin / bodies count the kernels and the nodes of the
// Arnoldi steps.
int enqueue_solve_graph(ow3d_handle* H, const Surface& s, int slot, unsigned long long& kin, int& bodies) {
    cudaStream_t st = H->st;
    const int m = H->m, maxmv = H->p.GMRESmaxiterations;
    launch_krylov_reset(H->ks, st);
    initial_residual_launches(H, s, H->RHS, H->PHI);
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    std::vector<cudaGraphConditionalHandle> hc((size_t)m, 0);
    for (int j = 0; j < m; ++j) CK(cudaGraphConditionalHandleCreate(&hc[(size_t)j], g, 0, cudaGraphCondAssignDefault));
    launch_norm_init(H->V, H->G.N, H->dsc, H->ks, H->p.reltol, H->p.abstol, st, hc[0]);
    for (int j = 0; j < m; ++j) {
        CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
        // the parameter block has no default constructor (its union holds
        // kernel parameters with dim3 members): zeroed raw storage instead
        alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)] = {};
        cudaGraphNodeParams& np = *reinterpret_cast<cudaGraphNodeParams*>(raw);
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = hc[(size_t)j];
        np.conditional.type = cudaGraphCondTypeIf;
        np.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        CK(cudaGraphAddNode(&node, g, deps, nd, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
        CK(cudaStreamBeginCaptureToGraph(H->st2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        const unsigned long long k0 = g_kernel_launches.load(std::memory_order_relaxed);
        H->st = H->st2;   // the step's launches go to the body's capture
        arnoldi_step_launches(H, s, j, maxmv, m, j + 1 < m ? hc[(size_t)j + 1] : 0);
        H->st = st;
        kin += g_kernel_launches.load(std::memory_order_relaxed) - k0;
        ++bodies;
        cudaGraph_t bout = nullptr;
        CK(cudaStreamEndCapture(H->st2, &bout));
    }
    solution_update_launches(H, H->PHI);
    launch_solve_log(H->ks, H->slog + slot, st);
    return OW3D_OK;
}

// Whether the next step may run as a captured graph: GMRES (either side)
// with the multigrid preconditioner, no pressure damping (its terms are
// gated on the host time), graphs on, and the first step done directly (it
// performs the one-time set-ups of the launches and uploads the level
// tables).
bool step_graph_eligible(const ow3d_handle* H) {
    return H->graphs && H->nlev > 0 && !H->pd_on && H->tstep >= 1 && !H->step_graph[(H->tstep + 1) & 1].failed;
}

// Capture the graph of steps with the parity of `tstep`.
int capture_step_graph(ow3d_handle* H, int64_t tstep) {
    ow3d_handle::StepGraph& G = H->step_graph[tstep & 1];
    cudaStream_t st = H->st;
    g_capture_unsafe = false;
    const unsigned long long k0 = g_kernel_launches.load(std::memory_order_relaxed);
    unsigned long long kin = 0;
    int bodies = 0;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    int err = OW3D_OK;
    if (e == cudaSuccess) {
        auto solve = [&](const Surface& s, int slot) -> int { return enqueue_solve_graph(H, s, slot, kin, bodies); };
        err = enqueue_step(H, tstep, true, solve);
        H->st = st;
        e = cudaStreamEndCapture(st, &graph);
        if (e == cudaSuccess && (err != OW3D_OK || g_capture_unsafe)) e = cudaErrorStreamCaptureUnsupported;
    }
    // the captured launches did not run: they are counted per replay instead
    const unsigned long long nk = g_kernel_launches.load(std::memory_order_relaxed) - k0;
    g_kernel_launches.fetch_sub(nk, std::memory_order_relaxed);
    cudaGraphExec_t ex = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        G.failed = true;
        return OW3D_ERR_UNSUPPORTED;   // the caller steps directly
    }
    G.exec = ex;
    G.per_step = bodies > 0 ? kin / (unsigned long long)bodies : 0;
    G.base = nk - kin;
    return OW3D_OK;
}

// Launch the next step as a graph (capturing it first if needed); the host
// work after it is finish_graph_step. Returns OW3D_ERR_UNSUPPORTED when the
// step has to run directly.
int launch_graph_step(ow3d_handle* H) {
    if (!step_graph_eligible(H)) return OW3D_ERR_UNSUPPORTED;
    const int64_t tstep = H->tstep + 1;
    ow3d_handle::StepGraph& G = H->step_graph[tstep & 1];
    if (!G.exec) TRY(capture_step_graph(H, tstep));
    CK(cudaGraphLaunch(G.exec, H->st));
    return OW3D_OK;
}

int finish_graph_step(ow3d_handle* H) {
    const int64_t tstep = H->tstep + 1;
    const ow3d_handle::StepGraph& G = H->step_graph[tstep & 1];
    CK(cudaStreamSynchronize(H->st));
    int status = OW3D_OK;
    unsigned long long kernels = G.base;
    const int maxmv = H->p.GMRESmaxiterations;
    for (int q = 0; q < 4; ++q) {
        const SolveLog& l = H->slog_host[q];
        // iterative_solution.f90:117-134: the limit reached without convergence
        const bool nc = !l.converged && l.iters >= maxmv;
        record_solve(H, l.iters, l.resid, l.beta, l.tol, nc);
        if (nc) status = OW3D_NOT_CONVERGED;
        kernels += (unsigned long long)(l.iters > 1 ? l.iters - 1 : 0) * G.per_step;
    }
    g_kernel_launches.fetch_add(kernels, std::memory_order_relaxed);
    TRY(finish_step(H, tstep));
    CK(cudaGetLastError());
    return status;
}

// The next step, as a graph where it applies, directly otherwise.
int next_step(ow3d_handle* H) {
    int r = launch_graph_step(H);
    if (r == OW3D_ERR_UNSUPPORTED) return rk4_step(H);
    if (r < 0) return r;
    return finish_graph_step(H);
}

void drop_step_graphs(ow3d_handle* H) {
    for (auto& g : H->step_graph) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = ow3d_handle::StepGraph{};
    }
}

}  // namespace

namespace {
template <typename T>
int level_op_t(ow3d_handle* H, MgSet<T>& S, int l, int op, int nu, const double* in1, const double* in2, double* out) {
    const int L = (int)S.lev.size();
    LevelDev<T> Lv = S.lev[l];
    const size_t n = (size_t)Lv.N;
    T *a, *b, *c;
    // temporary device buffers for the probe (freed at the end of the call)
    size_t nmax = n;
    if (l > 0) nmax = std::max(nmax, (size_t)S.lev[l - 1].N);
    CK(cudaMalloc(&a, nmax * sizeof(T))); CK(cudaMalloc(&b, nmax * sizeof(T))); CK(cudaMalloc(&c, nmax * sizeof(T)));
    auto put = [&](T* d, const double* h, size_t k) -> int {
        std::vector<T> t(h, h + k);
        CK(cudaMemcpy(d, t.data(), k * sizeof(T), cudaMemcpyHostToDevice));
        return OW3D_OK;
    };
    auto get = [&](double* h, const T* d, size_t k) -> int {
        std::vector<T> t(k);
        CK(cudaMemcpy(t.data(), d, k * sizeof(T), cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < k; ++q) h[q] = (double)t[q];
        return OW3D_OK;
    };
    int r = OW3D_OK;
    if (op == 0) {  // y = A_l x
        r = put(a, in1, n);
        if (!r) { launch_lo_matvec<T>(Lv, a, b, H->st); cudaStreamSynchronize(H->st); r = get(out, b, n); }
    } else if (op == 1) {  // smoothing: x <- S(x, b), nu steps
        r = put(a, in1, n); if (!r) r = put(b, in2, n);
        if (!r) {
            Lv.xv = a; Lv.bv = b;
            if (S.table.lex) launch_lo_smooth_lex<T>(Lv, nu, H->st);
            else launch_lo_smooth<T>(Lv, nu, H->st);
            cudaStreamSynchronize(H->st); r = get(out, a, n);
        }
    } else if (op == 2 && l > 0) {  // restriction of a fine residual to level l-1
        LevelDev<T> Cc = S.lev[l - 1];
        r = put(a, in1, n);
        if (!r) { Cc.xv = c; launch_restrict<T>(Lv, Cc, a, b, H->st); cudaStreamSynchronize(H->st); r = get(out, b, (size_t)Cc.N); }
    } else if (op == 3 && l > 0) {  // prolongation of a level l-1 vector, added to zero
        LevelDev<T> Cc = S.lev[l - 1];
        r = put(a, in1, (size_t)Cc.N);
        if (!r) {
            cudaMemsetAsync(b, 0, n * sizeof(T), H->st);
            launch_prolong_add<T>(Lv, Cc, a, b, H->st); cudaStreamSynchronize(H->st); r = get(out, b, n);
        }
    } else if (op == 5) {  // one smoother phase: colour pass nu, or the bottom-row pass (nu < 0)
        r = put(a, in1, n); if (!r) r = put(b, in2, n);
        if (!r) { Lv.xv = a; Lv.bv = b; launch_lo_pass<T>(Lv, nu, H->st); cudaStreamSynchronize(H->st); r = get(out, a, n); }
    } else if (op == 4 && l == 0) {  // coarse solve
        r = put(b, in1, n);
        if (!r) { Lv.bv = b; Lv.xv = a; launch_coarse_solve<T>(Lv, S.coarse_inv, H->st); cudaStreamSynchronize(H->st); r = get(out, a, n); }
    } else r = OW3D_ERR_BAD_INPUT;
    cudaFree(a); cudaFree(b); cudaFree(c);
    (void)L;
    CK(cudaGetLastError());
    return r;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

unsigned long long ow3d_launch_count(void) { return g_kernel_launches.load(std::memory_order_relaxed); }

int ow3d_test_set_coarse_blocks(int blocks) { return g_coarse_blocks.exchange(blocks < 0 ? 0 : blocks); }
int ow3d_test_set_colour_tiles(int min_tiles) { return g_colour_tiles.exchange(min_tiles < 0 ? 0 : min_tiles); }
int ow3d_test_set_colour_prefetch(int mode) { return g_colour_prefetch.exchange(mode < 0 ? -1 : mode); }
long long ow3d_test_set_tail_max_points(long long points) {
    return g_tail_max_points.exchange(points < 0 ? 0 : (int64_t)points);
}
int ow3d_test_set_pdl(int on) { return g_pdl.exchange(on ? 1 : 0); }
int ow3d_test_set_tail_cluster(int blocks) { return g_tail_cluster.exchange(blocks < 0 ? 0 : blocks); }
long long ow3d_test_set_coop_max_points(long long points) {
    return g_coop_max_points.exchange(points < 0 ? 0 : (int64_t)points);
}

int ow3d_test_graph_count(const ow3d_handle* H) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    return H->graphs_failed ? -1 : (int)H->iter_graphs.size();
}

int ow3d_test_step_graph_count(const ow3d_handle* H) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    int n = 0;
    for (const auto& g : H->step_graph) {
        if (g.failed) return -1;
        if (g.exec) ++n;
    }
    return n;
}

int ow3d_default_params(ow3d_params* p) { return default_params(p); }

int ow3d_read_deck(const char* path, ow3d_params* p) {
    if (!path || !p) return OW3D_ERR_BAD_INPUT;
    std::string err;
    int r = read_deck(path, p, &err);
    if (r) g_last_error = err;
    return r;
}

int ow3d_initial_condition(const ow3d_params* p, double* h, double* hx, double* hxx, double* hy, double* hyy,
                           double* E, double* P) {
    if (!p) return OW3D_ERR_BAD_INPUT;
    std::string err;
    const int r = initial_condition(*p, h, hx, hxx, hy, hyy, E, P, &err);
    if (r) g_last_error = err;
    return r;
}

int ow3d_read_bathymetry(const ow3d_params* p, const char* path, double* h, double* hx, double* hxx, double* hy,
                         double* hyy, int* flag) {
    if (!p) return OW3D_ERR_BAD_INPUT;
    std::string err;
    const int r = read_bathymetry(*p, path, h, hx, hxx, hy, hyy, flag, &err);
    if (r) g_last_error = err;
    return r;
}

int ow3d_stream_function_wave(const ow3d_params* p, int n, const double* x, double t, double* eta, double* phis,
                              double* info) {
    if (!p || n < 0 || (n > 0 && !x)) return OW3D_ERR_BAD_INPUT;
    SFWave w;
    std::string err;
    const int r = stream_function_solve(*p, w, &err);
    if (r) { g_last_error = err; return r; }
    stream_function_eval(w, n, x, t, eta, phis);
    if (info) { info[0] = w.k; info[1] = w.L; info[2] = w.T; info[3] = w.c; }
    return OW3D_OK;
}

int ow3d_incident_wave(const ow3d_params* p, int zone, int nt, double* eta, double* phis, int* box) {
    if (!p) return OW3D_ERR_BAD_INPUT;
    std::string err;
    const int r = incident_wave(*p, zone, nt, eta, phis, box, &err);
    if (r) g_last_error = err;
    return r;
}

int ow3d_create(const ow3d_params* p, const double* h, const double* hx, const double* hxx, const double* hy,
                const double* hyy, ow3d_handle** out) {
    if (!out) return OW3D_ERR_BAD_INPUT;
    *out = nullptr;
    return create_impl(p, h, hx, hxx, hy, hyy, out);
}

int ow3d_destroy(ow3d_handle* H) {
    if (!H) return OW3D_OK;
    cudaSetDevice(H->dev);
    if (H->st) cudaStreamSynchronize(H->st);
    for (auto& g : H->iter_graphs) cudaGraphExecDestroy(g.exec);
    for (auto& g : H->step_graph) if (g.exec) cudaGraphExecDestroy(g.exec);
    for (void* q : H->allocs) cudaFree(q);
    if (H->ks_host) cudaFreeHost(H->ks_host);
    if (H->flag_host) cudaFreeHost(H->flag_host);
    if (H->slog_host) cudaFreeHost(H->slog_host);
    if (H->st) cudaStreamDestroy(H->st);
    if (H->st2) cudaStreamDestroy(H->st2);
    delete H;
    return OW3D_OK;
}

int ow3d_dims(const ow3d_handle* H, int* Nxg, int* Nyg, int* Nzg, size_t* bytes) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    if (Nxg) *Nxg = H->G.Nxg;
    if (Nyg) *Nyg = H->G.Nyg;
    if (Nzg) *Nzg = H->G.Nzg;
    if (bytes) *bytes = H->bytes;
    return OW3D_OK;
}

int ow3d_estimate_bytes(const ow3d_params* p, size_t* bytes) {
    if (!p || !bytes) return OW3D_ERR_BAD_INPUT;
    {
        std::string err;
        if (check_params(*p, &err) != 0) { g_last_error = err; return OW3D_ERR_BAD_INPUT; }
        if (check_supported(*p, &err) != 0) { g_last_error = err; return OW3D_ERR_UNSUPPORTED; }
        if (p->GMRESmaxiterations < 2 || p->GMRESmaxiterations > kMaxKrylov) { g_last_error = "GMRESmaxiterations out of range"; return OW3D_ERR_BAD_INPUT; }
    }
    const int gx = p->Nx > 1 ? 1 : 0, gy = p->Ny > 1 ? 1 : 0;
    const double C = (double)(p->Nx + 2 * gx) * (p->Ny + 2 * gy);
    const double N = C * (p->Nz + 1);
    const double s = (p->precision == OW3D_PREC_MIXED) ? 4.0 : 8.0;
    const int m = p->GMRESmaxiterations;
    double b = 8.0 * N * (m + 1) + s * N * m + 8.0 * N * 5 + 3.0 * s * N * 1.6 + 8.0 * C * 60 +
               s * (double)kDenseMaxPoints * (double)kDenseMaxPoints * 2.0;
    // the inverse of a type-0 pressure-damping zone matrix: at most a row squared
    if (p->PDampingONOFF != 0 && p->pd_type == 0) b += 8.0 * (double)(p->Nx + 2) * (double)(p->Nx + 2);
    // local smoothing: the W history, dw/dt, flags and two scratch fields;
    // the breaking model: its per-column state and roller records
    if (smoothing_on(*p)) b += 8.0 * C * 7;
    if (breaking_on(*p)) b += 8.0 * C * 12;
    *bytes = (size_t)(b * 1.05) + ((size_t)64 << 20);
    return OW3D_OK;
}

int ow3d_solve_device(ow3d_handle* H, const double* rhs, double* phi, const double* E, const double* Ex,
                      const double* Exx, const double* Ey, const double* Eyy, int* iterations) {
    if (!H || !rhs || !phi) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    const bool nl = H->p.LinearONOFF == 1;
    Surface s = nl ? Surface{E, Ex, Exx, Ey, Eyy} : Surface{nullptr, nullptr, nullptr, nullptr, nullptr};
    return solve_device(H, rhs, phi, s, iterations);
}

int ow3d_solve(ow3d_handle* H, const double* rhs, double* phi, const double* E, const double* Ex, const double* Exx,
               const double* Ey, const double* Eyy, int* iterations) {
    if (!H || !rhs || !phi) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    TRY(ensure_staging(H));
    const size_t nb = sizeof(double) * (size_t)H->G.N;
    CK(cudaMemcpyAsync(H->s_rhs, rhs, nb, cudaMemcpyHostToDevice, H->st));
    CK(cudaMemcpyAsync(H->s_phi, phi, nb, cudaMemcpyHostToDevice, H->st));
    Surface s;
    TRY(stage_surface(H, E, Ex, Exx, Ey, Eyy, s));
    if (H->p.LinearONOFF != 1) s = Surface{nullptr, nullptr, nullptr, nullptr, nullptr};
    int r = solve_device(H, H->s_rhs, H->s_phi, s, iterations);
    if (r < 0) return r;
    CK(cudaMemcpyAsync(phi, H->s_phi, nb, cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    return r;
}

int ow3d_matvec(ow3d_handle* H, const double* phi, double* y, const double* E, const double* Ex, const double* Exx,
                const double* Ey, const double* Eyy) {
    if (!H || !phi || !y) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    TRY(ensure_staging(H));
    const size_t nb = sizeof(double) * (size_t)H->G.N;
    CK(cudaMemcpyAsync(H->s_phi, phi, nb, cudaMemcpyHostToDevice, H->st));
    Surface s;
    TRY(stage_surface(H, E, Ex, Exx, Ey, Eyy, s));
    if (H->p.LinearONOFF != 1) s = Surface{nullptr, nullptr, nullptr, nullptr, nullptr};
    launch_ho_matvec<double>(H->hg, s, H->s_phi, nullptr, nullptr, H->s_rhs, 0, H->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(y, H->s_rhs, nb, cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    return OW3D_OK;
}

int ow3d_residual_device_noalloc(ow3d_handle* H, const double* d_rhs, const double* d_phi, const double* d_E,
                                 const double* d_Ex, const double* d_Exx, const double* d_Ey, const double* d_Eyy,
                                 double* d_res, double* norm2) {
    if (!H || !d_rhs || !d_phi || !d_res || !norm2) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    const bool nl = H->p.LinearONOFF == 1;
    if (nl && (!d_E || !d_Ex || !d_Exx || (H->G.three && (!d_Ey || !d_Eyy)))) {
        g_last_error = "ow3d_residual_device_noalloc: the nonlinear operator needs E, Ex, Exx (and Ey, Eyy in 3-D)";
        return OW3D_ERR_BAD_INPUT;
    }
    const Surface s = nl ? Surface{d_E, d_Ex, d_Exx, d_Ey, d_Eyy} : Surface{nullptr, nullptr, nullptr, nullptr, nullptr};
    launch_ho_matvec<double>(H->hg, s, d_phi, nullptr, d_rhs, d_res, 1, H->st);
    CK(cudaGetLastError());
    std::string err;
    const int r = noalloc_norm2(H->dev, d_res, H->G.N, norm2, H->st, err);
    if (r) g_last_error = err;
    return r;
}

int ow3d_precondition(ow3d_handle* H, const double* r, double* u) {
    if (!H || !r || !u) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    TRY(ensure_staging(H));
    const size_t nb = sizeof(double) * (size_t)H->G.N;
    CK(cudaMemcpyAsync(H->s_rhs, r, nb, cudaMemcpyHostToDevice, H->st));
    precond_into(H, H->s_rhs, nullptr, H->s_phi);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(u, H->s_phi, nb, cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    return OW3D_OK;
}

int ow3d_set_state(ow3d_handle* H, const double* E, const double* P, const double* W, const double* phi, double t) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    const size_t cb = sizeof(double) * (size_t)H->G.C, nb = sizeof(double) * (size_t)H->G.N;
    if (E) CK(cudaMemcpyAsync(H->E, E, cb, cudaMemcpyHostToDevice, H->st)); else CK(cudaMemsetAsync(H->E, 0, cb, H->st));
    if (P) CK(cudaMemcpyAsync(H->P, P, cb, cudaMemcpyHostToDevice, H->st)); else CK(cudaMemsetAsync(H->P, 0, cb, H->st));
    if (W) CK(cudaMemcpyAsync(H->W, W, cb, cudaMemcpyHostToDevice, H->st)); else CK(cudaMemsetAsync(H->W, 0, cb, H->st));
    if (phi) CK(cudaMemcpyAsync(H->PHI, phi, nb, cudaMemcpyHostToDevice, H->st)); else CK(cudaMemsetAsync(H->PHI, 0, nb, H->st));
    if (H->G.per) {
        // periodic x: the image columns of phi stay zero inside the solves
        // (identity rows), those of W hold the distinct columns' values
        fs_images(H->fa, H->PHI, H->G.Nzg, 1, H->st);
        fs_images(H->fa, H->W, 1, 0, H->st);
    }
    CK(cudaMemsetAsync(H->LP[0], 0, nb, H->st));
    CK(cudaMemsetAsync(H->LP[1], 0, nb, H->st));
    CK(cudaMemsetAsync(H->RHS, 0, nb, H->st));
    // OceanWave3DT0Setup.f90:444 -- surface derivatives of the initial state
    // (the current's ghost source is still zero there)
    fs_derivs(H->fa, H->E, H->P, H->Ex, H->Exx, H->Px, H->Ey, H->Eyy, H->Py, 0, H->st);
    {
        const StepDev s0{t, 0};
        CK(cudaMemcpyAsync(H->sd, &s0, sizeof(StepDev), cudaMemcpyHostToDevice, H->st));
        CK(cudaStreamSynchronize(H->st));   // s0 lives on this stack frame
    }
    H->time = t;
    H->tstep = 0;
    H->stats.time = t;
    H->stats.tstep = 0;
    CK(cudaStreamSynchronize(H->st));
    return OW3D_OK;
}

int ow3d_put_surface(ow3d_handle* H, const double* E, const double* P) {
    if (!H || !E || !P) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    const size_t cb = sizeof(double) * (size_t)H->G.C;
    CK(cudaMemcpyAsync(H->E, E, cb, cudaMemcpyHostToDevice, H->st));
    CK(cudaMemcpyAsync(H->P, P, cb, cudaMemcpyHostToDevice, H->st));
    // after a step the ghost sources hold the current's flux and the
    // wavemaker's values of the step's end
    fs_derivs(H->fa, H->E, H->P, H->Ex, H->Exx, H->Px, H->Ey, H->Eyy, H->Py, H->tstep > 0 ? 2 : 0, H->st);
    CK(cudaGetLastError());
    return OW3D_OK;
}

int ow3d_get_state(ow3d_handle* H, double* E, double* P, double* W, double* phi, double* t) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    const size_t cb = sizeof(double) * (size_t)H->G.C, nb = sizeof(double) * (size_t)H->G.N;
    if (E) CK(cudaMemcpyAsync(E, H->E, cb, cudaMemcpyDeviceToHost, H->st));
    if (P) CK(cudaMemcpyAsync(P, H->P, cb, cudaMemcpyDeviceToHost, H->st));
    if (W) CK(cudaMemcpyAsync(W, H->W, cb, cudaMemcpyDeviceToHost, H->st));
    if (phi) CK(cudaMemcpyAsync(phi, H->PHI, nb, cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    if (phi && H->G.per) {
        // periodic x: phi's image columns are filled on output (column 1 <-
        // Nxg-2, Nxg-1 <- 2, Nxg <- 3); on the device they stay zero
        const int Nx = H->G.Nxg, Nz = H->G.Nzg;
        for (int j = 0; j < H->G.Nyg; ++j) {
            double* r = phi + (size_t)Nz * Nx * j;
            std::memcpy(r, r + (size_t)Nz * (Nx - 3), sizeof(double) * Nz);
            std::memcpy(r + (size_t)Nz * (Nx - 2), r + (size_t)Nz * 1, sizeof(double) * Nz);
            std::memcpy(r + (size_t)Nz * (Nx - 1), r + (size_t)Nz * 2, sizeof(double) * Nz);
        }
    }
    if (t) *t = H->time;
    return OW3D_OK;
}

int ow3d_set_relax_target(ow3d_handle* H, int zone, int mode, int nt, double dts, const double* eta, const double* phis) {
    if (!H || zone < 0 || zone >= (int)H->zones.size() || nt <= 0 || !eta || !phis || dts <= 0) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    RelaxZoneDev& z = H->zones[zone];
    const size_t box = (size_t)(z.i1 - z.i0 + 1) * (z.j1 - z.j0 + 1);
    double *de, *dp;
    TRY(dalloc(H, &de, box * nt)); TRY(dalloc(H, &dp, box * nt));
    CK(cudaMemcpy(de, eta, box * nt * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dp, phis, box * nt * sizeof(double), cudaMemcpyHostToDevice));
    z.eta = de; z.phis = dp; z.nt = nt; z.tdt = dts; z.tmode = mode;
    drop_step_graphs(H);   // the captured relaxation launches hold the old table
    return OW3D_OK;
}

int ow3d_incident_wave_device(ow3d_handle* H, int zone, int nt) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    if (zone < 0 || zone >= (int)H->zones.size()) { g_last_error = "ow3d_incident_wave_device: no such zone"; return OW3D_ERR_BAD_INPUT; }
    CK(cudaSetDevice(H->dev));
    IncidentWave w;
    std::string err;
    if (int r = incident_wave_setup(H->p, zone, nt, w, nullptr, nullptr, &err)) { g_last_error = err; return r; }
    RelaxZoneDev& z = H->zones[(size_t)zone];
    const size_t box = (size_t)(z.i1 - z.i0 + 1) * (z.j1 - z.j0 + 1);
    if (box != (size_t)w.bx * w.by) { g_last_error = "ow3d_incident_wave_device: zone box mismatch"; return OW3D_ERR_BAD_INPUT; }
    // the series, kept as the zone's target for the handle's lifetime
    double *de, *dp;
    TRY(dalloc(H, &de, box * (size_t)nt)); TRY(dalloc(H, &dp, box * (size_t)nt));
    // the components and work arrays, freed at the end of the call
    std::vector<void*> tmp;
    // src = nullptr: an uninitialised work array
    auto put = [&](const void* src, size_t bytes) -> void* {
        void* d = nullptr;
        if (cudaMalloc(&d, bytes ? bytes : 16) != cudaSuccess) { tmp.push_back(nullptr); return nullptr; }
        tmp.push_back(d);
        if (src && bytes && cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            tmp.push_back(nullptr);
            return nullptr;
        }
        return d;
    };
    auto release = [&]() { for (void* q : tmp) cudaFree(q); };
    const double pi = std::acos(-1.0);
    std::vector<double> dy_rows((size_t)w.by, 0.0);
    if (w.heading) dy_rows = w.dy;
    IncidentWaveDev d{};
    d.bx = w.bx; d.by = w.by; d.nt = nt; d.ny_eval = w.ny_eval; d.N = w.N; d.kmax = w.kmax;
    d.heading = w.heading ? 1 : 0; d.mono = w.mono ? 1 : 0;
    d.cosb = w.cosb; d.sinb = w.sinb; d.g = w.g; d.domega = w.domega;
    d.amp = w.amp; d.nu = w.nu; d.omega = w.omega; d.phifact = w.phifact; d.t0 = w.t0; d.dt = w.dt;
    d.dx = (const double*)put(w.dx.data(), w.dx.size() * sizeof(double));
    d.dy = (const double*)put(w.dy.data(), w.dy.size() * sizeof(double));
    d.dy_rows = (const double*)put(dy_rows.data(), dy_rows.size() * sizeof(double));
    if (!w.mono) {
        std::vector<double2> c((size_t)w.kmax), W((size_t)w.N);
        for (int k = 0; k < w.kmax; ++k) c[(size_t)k] = make_double2(w.c[(size_t)k].real(), w.c[(size_t)k].imag());
        for (int m = 0; m < w.N; ++m) {
            const double a = -2.0 * pi * (double)m / (double)w.N;
            W[(size_t)m] = make_double2(std::cos(a), std::sin(a));
        }
        d.c = (const double2*)put(c.data(), c.size() * sizeof(double2));
        d.W = (const double2*)put(W.data(), W.size() * sizeof(double2));
        d.nus = (const double*)put(w.nus.data(), w.nus.size() * sizeof(double));
        if (!w.kcos.empty()) {
            d.kcos = (const double*)put(w.kcos.data(), w.kcos.size() * sizeof(double));
            d.ksin = (const double*)put(w.ksin.data(), w.ksin.size() * sizeof(double));
        }
        const size_t modes = (size_t)w.bx * w.ny_eval * (size_t)w.kmax;
        d.A = (double2*)put(nullptr, modes * sizeof(double2));
        d.B = (double2*)put(nullptr, modes * sizeof(double2));
    }
    for (void* q : tmp)
        if (!q) {
            release();
            (void)cudaGetLastError();
            g_last_error = "ow3d_incident_wave_device: device allocation or upload failed";
            return OW3D_ERR_OOM;
        }
    int r = launch_incident_wave(d, de, dp, H->st);
    if (r == OW3D_OK && cudaStreamSynchronize(H->st) != cudaSuccess) r = OW3D_ERR_CUDA;
    release();
    if (r) {
        g_last_error = "ow3d_incident_wave_device: kernel launch or execution failed";
        return r;
    }
    z.eta = de; z.phis = dp; z.nt = nt; z.tdt = H->p.dt; z.tmode = 0;
    drop_step_graphs(H);   // the captured relaxation launches hold the old table
    return OW3D_OK;
}

int ow3d_rollers(ow3d_handle* H, int cap, int* n_rollers, int* npts, int* toe, double* x, double* eta,
                 double* thickness, double* tan_phi) {
    if (!H || !n_rollers) { g_last_error = "ow3d_rollers: null argument"; return OW3D_ERR_BAD_INPUT; }
    if (!H->brk_on) { *n_rollers = 0; return OW3D_OK; }
    int n = 0;
    CK(cudaSetDevice(H->dev));
    CK(cudaMemcpyAsync(&n, H->brk.n_rollers, sizeof(int), cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    *n_rollers = n;
    const int k = n < cap ? n : (cap > 0 ? cap : 0);
    if (k > 0) {
        const BreakDev& b = H->brk;
        auto get = [&](void* dst, const void* src, size_t sz) -> int {
            if (dst) CK(cudaMemcpyAsync(dst, src, sz * (size_t)k, cudaMemcpyDeviceToHost, H->st));
            return OW3D_OK;
        };
        TRY(get(npts, b.npts, sizeof(int))); TRY(get(toe, b.toe, sizeof(int)));
        TRY(get(x, b.xr, sizeof(double))); TRY(get(eta, b.sr, sizeof(double)));
        TRY(get(thickness, b.r_thick, sizeof(double))); TRY(get(tan_phi, b.r_tan, sizeof(double)));
        CK(cudaStreamSynchronize(H->st));
    }
    return OW3D_OK;
}

int ow3d_test_detect_breaking(ow3d_handle* H, const double* E, int update) {
    if (!H || !H->brk_on || !E) {
        g_last_error = "ow3d_test_detect_breaking: no breaking model on this handle";
        return OW3D_ERR_BAD_INPUT;
    }
    CK(cudaSetDevice(H->dev));
    CK(cudaMemcpyAsync(H->tE, E, sizeof(double) * (size_t)H->G.C, cudaMemcpyHostToDevice, H->st));
    fs_breaking(H->brk, H->tE, update, H->st);
    CK(cudaStreamSynchronize(H->st));
    CK(cudaGetLastError());
    return OW3D_OK;
}

int ow3d_test_accel_state(ow3d_handle* H, double* Wt, int* flags) {
    if (!H || !H->sm_on) {
        g_last_error = "ow3d_test_accel_state: no local smoothing on this handle";
        return OW3D_ERR_BAD_INPUT;
    }
    CK(cudaSetDevice(H->dev));
    const size_t n = (size_t)H->G.C;
    if (Wt) CK(cudaMemcpyAsync(Wt, H->sm.Wt, sizeof(double) * n, cudaMemcpyDeviceToHost, H->st));
    if (flags) CK(cudaMemcpyAsync(flags, H->sm.flag, sizeof(int) * n, cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    return OW3D_OK;
}

int ow3d_test_breaking_state(ow3d_handle* H, double* tan_phi, double* Qr_x) {
    if (!H || !H->brk_on) {
        g_last_error = "ow3d_test_breaking_state: no breaking model on this handle";
        return OW3D_ERR_BAD_INPUT;
    }
    CK(cudaSetDevice(H->dev));
    const size_t n = (size_t)H->brk.nfx;
    if (tan_phi) CK(cudaMemcpyAsync(tan_phi, H->brk.tan_phi, sizeof(double) * n, cudaMemcpyDeviceToHost, H->st));
    if (Qr_x) CK(cudaMemcpyAsync(Qr_x, H->brk.Qr_x, sizeof(double) * n, cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    return OW3D_OK;
}

int ow3d_test_relax_target(const ow3d_handle* H, int zone, double* eta, double* phis) {
    if (!H || zone < 0 || zone >= (int)H->zones.size()) return OW3D_ERR_BAD_INPUT;
    const RelaxZoneDev& z = H->zones[(size_t)zone];
    if (!z.eta || z.nt <= 0) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    const size_t n = (size_t)(z.i1 - z.i0 + 1) * (z.j1 - z.j0 + 1) * (size_t)z.nt * sizeof(double);
    if (eta) CK(cudaMemcpy(eta, z.eta, n, cudaMemcpyDeviceToHost));
    if (phis) CK(cudaMemcpy(phis, z.phis, n, cudaMemcpyDeviceToHost));
    return OW3D_OK;
}

int ow3d_zone_box(const ow3d_handle* H, int zone, int* i0, int* i1, int* j0, int* j1) {
    if (!H || zone < 0 || zone >= (int)H->zones.size()) return OW3D_ERR_BAD_INPUT;
    const RelaxZoneDev& z = H->zones[zone];
    *i0 = z.i0; *i1 = z.i1; *j0 = z.j0; *j1 = z.j1;
    return OW3D_OK;
}

// ------------------------------------------------------------ result files
namespace {
// E and P (fields 0) or h and hx (fields 1) on the host, ghosts included, and
// the grid as the reference's 2-D arrays x(i,j), y(i,j).
int host_fields(ow3d_handle* H, int fields, std::vector<double>& a, std::vector<double>& b, std::vector<double>& x,
                std::vector<double>& y) {
    const GridHost& G = H->G;
    const size_t C = (size_t)G.C;
    a.resize(C); b.resize(C); x.resize(C); y.resize(C);
    if (fields == 0) {
        CK(cudaMemcpyAsync(a.data(), H->E, C * sizeof(double), cudaMemcpyDeviceToHost, H->st));
        CK(cudaMemcpyAsync(b.data(), H->P, C * sizeof(double), cudaMemcpyDeviceToHost, H->st));
        CK(cudaStreamSynchronize(H->st));
    } else {
        a = G.h; b = G.hx;
    }
    for (int j = 0; j < G.Nyg; ++j)
        for (int i = 0; i < G.Nxg; ++i) { x[(size_t)j * G.Nxg + i] = G.x[i]; y[(size_t)j * G.Nxg + i] = G.y[j]; }
    return OW3D_OK;
}
}  // namespace

int ow3d_write_ep(ow3d_handle* H, const char* dir, int nr, int fields) {
    if (!H || nr < 0 || nr > 99999 || fields < 0 || fields > 1) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    std::vector<double> a, b, x, y;
    TRY(host_fields(H, fields, a, b, x, y));
    char name[32];
    std::snprintf(name, sizeof name, "EP_%05d.bin", nr);
    std::string path = (dir && *dir) ? std::string(dir) + "/" + name : std::string(name);
    const int r = ow3d_write_ep_file(path.c_str(), H->G.Nxg, H->G.Nyg, x.data(), y.data(), a.data(), b.data());
    if (r) g_last_error = ow3d_io_last_error();
    return r;
}

int ow3d_write_ascii(ow3d_handle* H, const char* dir, int nr, int fields) {
    // the unit number 100 + nr names the file with three digits (CHOUT3)
    if (!H || nr < 0 || 100 + nr > 999 || fields < 0 || fields > 1) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    std::vector<double> a, b, x, y;
    TRY(host_fields(H, fields, a, b, x, y));
    char name[32];
    std::snprintf(name, sizeof name, "fort.%03d", 100 + nr);
    std::string path = (dir && *dir) ? std::string(dir) + "/" + name : std::string(name);
    const int r = ow3d_write_ascii_file(path.c_str(), H->G.Nxg, H->G.Nyg, x.data(), y.data(), a.data(), b.data());
    if (r) g_last_error = ow3d_io_last_error();
    return r;
}

int ow3d_write_end(ow3d_handle* H, const char* path) {
    if (!H || !path) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    std::vector<double> a, b, x, y;
    TRY(host_fields(H, 0, a, b, x, y));
    const GridHost& G = H->G;
    std::vector<double> E, P;
    for (int j = G.gy; j < G.Ny + G.gy; ++j)
        for (int i = G.gx; i < G.Nx + G.gx; ++i) {
            E.push_back(a[(size_t)j * G.Nxg + i]);
            P.push_back(b[(size_t)j * G.Nxg + i]);
        }
    // domain size as the reference forms it, x(Nx,1) - x(1,1) and
    // y(Nx,1) - y(1,1) of its ghost-including arrays (the second is 0)
    const double xtank = G.x[(size_t)G.Nx - 1] - G.x[0];
    const double ytank = 0.0;
    const int r = ow3d_write_end_file(path, xtank, ytank, G.Nx, G.Ny, H->time, E.data(), P.data());
    if (r) g_last_error = ow3d_io_last_error();
    return r;
}

int ow3d_store_data(ow3d_handle* H, const char* dir, int* files) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    const int S = H->p.StoreDataONOFF;
    const int64_t t = H->tstep;
    int n = 0;
    auto end_path = [&]() { return (dir && *dir) ? std::string(dir) + "/OceanWave3D.end" : std::string("OceanWave3D.end"); };
    if (S > 0) {
        if (t == 0) {
            TRY(ow3d_write_ep(H, dir, 0, 0)); TRY(ow3d_write_ep(H, dir, 99999, 1)); n = 2;
        } else if (t % S == 0) {
            if (t > 99999) { g_last_error = "ow3d_store_data: EP file numbers have five digits"; return OW3D_ERR_BAD_INPUT; }
            TRY(ow3d_write_ep(H, dir, (int)t, 0)); TRY(ow3d_write_end(H, end_path().c_str())); n = 2;
        }
    } else if (S < 0) {
        if (t == 0) {
            TRY(ow3d_write_ascii(H, dir, 0, 0)); TRY(ow3d_write_ascii(H, dir, 899, 1)); n = 2;
        } else if (t % (-S) == 0) {
            const int64_t nr = t / (-S);
            if (100 + nr > 999) { g_last_error = "ow3d_store_data: ASCII file numbers have three digits"; return OW3D_ERR_BAD_INPUT; }
            TRY(ow3d_write_ascii(H, dir, (int)nr, 0)); TRY(ow3d_write_end(H, end_path().c_str())); n = 2;
        }
    }
    if (files) *files = n;
    return OW3D_OK;
}

namespace {
// The 13 kinematics fields of the current state in a device buffer the
// caller frees (cudaFree).
int kinematics_fields(ow3d_handle* H, double** out) {
    const GridHost& G = H->G;
    const size_t N = (size_t)G.N;
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, (13 * N + (size_t)G.Nzg) * sizeof(double));
    if (e != cudaSuccess) {
        cudaGetLastError();
        g_last_error = std::string("ow3d_kinematics: cudaMalloc: ") + cudaGetErrorString(e);
        return OW3D_ERR_OOM;
    }
    double* dz = d + 13 * N;
    e = cudaMemcpyAsync(dz, G.z.data(), (size_t)G.Nzg * sizeof(double), cudaMemcpyHostToDevice, H->st);
    KinArgs a;
    a.Nxg = G.Nxg; a.Nyg = G.Nyg; a.Nzg = G.Nzg;
    a.dox = G.Nx > 1; a.doy = G.three && G.Ny > 1;
    a.chain = H->p.LinearONOFF != 0;
    a.N = G.N;
    a.SX = H->SX; a.SY = H->SY; a.SZ = H->SZ; a.z = dz;
    a.h = H->h; a.hx = H->hx; a.hy = H->hy; a.E = H->E; a.Ex = H->Ex; a.Ey = H->Ey;
    if (e == cudaSuccess) {
        launch_kinematics(a, H->PHI, d, H->st);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(H->st);
    if (e != cudaSuccess) {
        cudaFree(d);
        g_last_error = std::string("ow3d_kinematics: ") + cudaGetErrorString(e);
        return OW3D_ERR_CUDA;
    }
    *out = d;
    return OW3D_OK;
}
}  // namespace

int ow3d_kinematics(ow3d_handle* H, double* u, double* v, double* w, double* grads) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    if (H->G.per) { g_last_error = "ow3d_kinematics: built for wall boundaries, not periodic_x"; return OW3D_ERR_UNSUPPORTED; }
    CK(cudaSetDevice(H->dev));
    double* d = nullptr;
    TRY(kinematics_fields(H, &d));
    const size_t N = (size_t)H->G.N, b = N * sizeof(double);
    cudaError_t e = cudaSuccess;
    if (u && e == cudaSuccess) e = cudaMemcpy(u, d, b, cudaMemcpyDeviceToHost);
    if (v && e == cudaSuccess) e = cudaMemcpy(v, d + N, b, cudaMemcpyDeviceToHost);
    if (w && e == cudaSuccess) e = cudaMemcpy(w, d + 3 * N, b, cudaMemcpyDeviceToHost);
    if (grads && e == cudaSuccess) e = cudaMemcpy(grads, d + 4 * N, 9 * b, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) { g_last_error = std::string("ow3d_kinematics: ") + cudaGetErrorString(e); return OW3D_ERR_CUDA; }
    return OW3D_OK;
}

// StoreKinematicData.f90:98-155 (header, it = 0) and :232-460 (a level).
int ow3d_store_kinematics(ow3d_handle* H, const char* dir, int* files) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    if (files) *files = 0;
    const ow3d_params& p = H->p;
    if (!p.iKinematics || p.nOutFiles <= 0) return OW3D_OK;
    if (p.formattype != 20 && p.formattype != 21) {
        g_last_error = "ow3d_store_kinematics: formattype " + std::to_string(p.formattype) +
                       " kinematics output is not supported (20 and 21 are)";
        return OW3D_ERR_UNSUPPORTED;
    }
    if (p.nOutFiles > OW3D_MAX_KIN_FILES) { g_last_error = "ow3d_store_kinematics: too many slices"; return OW3D_ERR_BAD_INPUT; }
    for (int io = 1; io <= p.nOutFiles; ++io) {
        const int* r = p.kinematics[io - 1];
        if (r[0] < 1 || r[1] > p.Nx || r[0] > r[1] || r[3] < 1 || r[4] > p.Ny || r[3] > r[4] || r[2] < 1 ||
            r[5] < 1 || r[8] < 1 || r[6] > r[7]) {
            g_last_error = "ow3d_store_kinematics: slice " + std::to_string(io) + " is outside the grid or empty";
            return OW3D_ERR_BAD_INPUT;
        }
    }
    CK(cudaSetDevice(H->dev));
    const GridHost& G = H->G;
    const int64_t t = H->tstep;
    const int64_t L = t + 1;   // time level of the current state (level 1 = initial)
    const size_t N = (size_t)G.N, Cn = (size_t)G.C;
    const int nz = G.Nzg;
    auto path_of = [&](int io, int64_t it) {
        char name[48];
        if (p.formattype == 20) std::snprintf(name, sizeof name, "Kinematics%02d.bin", io);
        else std::snprintf(name, sizeof name, "Kinematics_%02d_%05lld.bin", io, (long long)it);
        return (dir && *dir) ? std::string(dir) + "/" + name : std::string(name);
    };
    bool any = false;
    for (int io = 1; io <= p.nOutFiles; ++io) {
        const int* r = p.kinematics[io - 1];
        if (L >= r[6] && L <= r[7] && t % r[8] == 0) any = true;
    }
    // host copies of the fields a level writes
    std::vector<double> E(Cn), Ex(Cn), Ey(Cn, 0.0), phi, kin;
    if (any) {
        if (L > 99999) { g_last_error = "ow3d_store_kinematics: time levels have five digits"; return OW3D_ERR_BAD_INPUT; }
        double* d = nullptr;
        TRY(kinematics_fields(H, &d));
        phi.resize(N); kin.resize(13 * N);
        cudaError_t e = cudaMemcpy(kin.data(), d, 13 * N * sizeof(double), cudaMemcpyDeviceToHost);
        cudaFree(d);
        if (e == cudaSuccess) e = cudaMemcpy(phi.data(), H->PHI, N * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(E.data(), H->E, Cn * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(Ex.data(), H->Ex, Cn * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && G.Nyg > 1) e = cudaMemcpy(Ey.data(), H->Ey, Cn * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { g_last_error = std::string("ow3d_store_kinematics: ") + cudaGetErrorString(e); return OW3D_ERR_CUDA; }
    }
    int written = 0;
    for (int io = 1; io <= p.nOutFiles; ++io) {
        const int* r = p.kinematics[io - 1];
        // slice in ghost-inclusive 0-based indices
        std::vector<size_t> cols;
        for (int j = r[3] + G.gy; j <= r[4] + G.gy; j += r[5])
            for (int i = r[0] + G.gx; i <= r[1] + G.gx; i += r[2]) cols.push_back((size_t)(i - 1) + (size_t)G.Nxg * (j - 1));
        auto put = [&](std::FILE* f, const void* a, size_t nb) {
            const void* parts[1] = {a};
            const size_t sz[1] = {nb};
            return write_record(f, parts, sz, 1);
        };
        auto column_field = [&](const double* F) {
            std::vector<double> s;
            s.reserve(cols.size() * nz);
            for (size_t c : cols) s.insert(s.end(), F + c * nz, F + c * nz + nz);
            return s;
        };
        auto surface_field = [&](const double* F) {
            std::vector<double> s;
            s.reserve(cols.size());
            for (size_t c : cols) s.push_back(F[c]);
            return s;
        };
        if (t == 0) {
            const std::string path = path_of(io, 0);
            std::FILE* f = std::fopen(path.c_str(), "wb");
            if (!f) { g_last_error = "ow3d_store_kinematics: cannot open " + path; return OW3D_ERR_IO; }
            int32_t ints[9];
            for (int m = 0; m < 9; ++m) ints[m] = r[m];
            const double dt = p.dt;
            const int32_t nzi = nz;
            const void* parts[3] = {ints, &dt, &nzi};
            const size_t sz[3] = {sizeof ints, sizeof dt, sizeof nzi};
            bool ok = write_record(f, parts, sz, 3);
            std::vector<double> geo;
            geo.reserve(cols.size() * 5);
            for (size_t c : cols) {
                const size_t i = c % (size_t)G.Nxg, j = c / (size_t)G.Nxg;
                geo.push_back(G.x[i]); geo.push_back(G.y[j]); geo.push_back(G.h[c]);
                geo.push_back(G.hx[c]); geo.push_back(G.three ? G.hy[c] : 0.0);
            }
            ok = ok && put(f, geo.data(), geo.size() * sizeof(double));
            ok = ok && put(f, G.z.data(), (size_t)nz * sizeof(double));
            ok = (std::fclose(f) == 0) && ok;
            if (!ok) { g_last_error = "ow3d_store_kinematics: write failed: " + path; return OW3D_ERR_IO; }
            ++written;
        }
        if (!(L >= r[6] && L <= r[7] && t % r[8] == 0)) continue;
        const std::string path = path_of(io, L);
        std::FILE* f = std::fopen(path.c_str(), p.formattype == 20 ? "ab" : "wb");
        if (!f) { g_last_error = "ow3d_store_kinematics: cannot open " + path; return OW3D_ERR_IO; }
        bool ok = true;
        for (const double* F : {E.data(), Ex.data(), Ey.data()}) {
            const std::vector<double> s = surface_field(F);
            ok = ok && put(f, s.data(), s.size() * sizeof(double));
        }
        // phi, u, v, w, then the 9 gradient fields
        const double* fields[13] = {phi.data(), &kin[0], &kin[N], &kin[3 * N]};
        for (int q = 0; q < 9; ++q) fields[4 + q] = &kin[(4 + q) * N];
        for (const double* F : fields) {
            const std::vector<double> s = column_field(F);
            ok = ok && put(f, s.data(), s.size() * sizeof(double));
        }
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) { g_last_error = "ow3d_store_kinematics: write failed: " + path; return OW3D_ERR_IO; }
        ++written;
    }
    if (files) *files = written;
    return OW3D_OK;
}

int ow3d_step(ow3d_handle* H, int nsteps) {
    if (!H || nsteps < 0) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    int st = OW3D_OK;
    for (int i = 0; i < nsteps; ++i) {
        int r = next_step(H);
        if (r < 0) return r;
        if (r > 0) st = r;
    }
    return st;
}

int ow3d_step_batch(ow3d_handle* const* hs, int n, const int* nsteps, int* status, double* wall_ms) {
    if (!hs || n < 0 || !nsteps) return OW3D_ERR_BAD_INPUT;
    for (int i = 0; i < n; ++i) {
        if (!hs[i] || nsteps[i] < 0) return OW3D_ERR_BAD_INPUT;
        for (int q = 0; q < i; ++q)
            if (hs[q] == hs[i]) { g_last_error = "ow3d_step_batch: a handle appears twice"; return OW3D_ERR_BAD_INPUT; }
    }
    // One host thread, each simulation at its own pace: every handle with
    // steps left has its next step graph in flight on its own stream; the
    // thread polls the streams and, as soon as one step completes, does its
    // bookkeeping and launches that handle's next step. Handles that cannot
    // use graphs (their first step, left GMRES, pressure damping) step
    // directly in between. The simulations' kernels so overlap on the device
    // and a small simulation is not held back by a large one.
    std::vector<int> st(n, OW3D_OK), left(nsteps, nsteps + n);
    std::vector<char> inflight(n, 0);
    std::vector<double> ms(n, 0.0);
    std::vector<std::string> errs(n);
    const auto t0 = std::chrono::steady_clock::now();
    auto done_at = [&](int i) {
        ms[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    auto note = [&](int i, int r) {
        if (r < 0) { st[i] = r; errs[i] = g_last_error; left[i] = 0; done_at(i); return; }
        if (r > 0 && st[i] == OW3D_OK) st[i] = r;
        if (--left[i] == 0) done_at(i);
    };
    for (int i = 0; i < n; ++i) if (left[i] == 0) done_at(i);
    for (;;) {
        // launch the next step of every idle handle; direct steps run here
        bool work = false;
        for (int i = 0; i < n; ++i) {
            if (left[i] <= 0 || inflight[i]) continue;
            work = true;
            if (cudaSetDevice(hs[i]->dev) != cudaSuccess) { note(i, OW3D_ERR_CUDA); continue; }
            const int r = launch_graph_step(hs[i]);
            if (r == OW3D_OK) inflight[i] = 1;
            else if (r == OW3D_ERR_UNSUPPORTED) note(i, rk4_step(hs[i]));
            else note(i, r);
        }
        bool any = false;
        for (int i = 0; i < n; ++i) any = any || inflight[i];
        if (!any) {
            if (!work) break;
            continue;
        }
        // wait for the first in-flight step to complete, then finish it
        for (bool got = false; !got;) {
            for (int i = 0; i < n; ++i) {
                if (!inflight[i]) continue;
                cudaSetDevice(hs[i]->dev);
                const cudaError_t e = cudaStreamQuery(hs[i]->st);
                if (e == cudaErrorNotReady) continue;
                inflight[i] = 0;
                got = true;
                note(i, e == cudaSuccess ? finish_graph_step(hs[i]) : OW3D_ERR_CUDA);
            }
            if (!got) std::this_thread::yield();
        }
    }
    int worst = OW3D_OK;
    for (int i = 0; i < n; ++i) {
        if (status) status[i] = st[i];
        if (wall_ms) wall_ms[i] = ms[i];
        if (st[i] < 0 && (worst >= 0 || st[i] < worst)) { worst = st[i]; g_last_error = errs[i]; }
        else if (st[i] > 0 && worst == OW3D_OK) worst = st[i];
    }
    return worst;
}

int ow3d_step_timed(ow3d_handle* H, int nsteps, double* device_ms) {
    if (!H || nsteps < 0) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a)); CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, H->st));
    int st = OW3D_OK;
    for (int i = 0; i < nsteps; ++i) {
        int r = next_step(H);
        if (r < 0) { cudaEventDestroy(a); cudaEventDestroy(b); return r; }
        if (r > 0) st = r;
    }
    CK(cudaEventRecord(b, H->st));
    CK(cudaEventSynchronize(b));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a); cudaEventDestroy(b);
    if (device_ms) *device_ms = ms;
    return st;
}

int ow3d_get_stats(const ow3d_handle* H, ow3d_stats* s) {
    if (!H || !s) return OW3D_ERR_BAD_INPUT;
    *s = H->stats;
    return OW3D_OK;
}

int ow3d_reset_stats(ow3d_handle* H) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    const double t = H->stats.time;
    const int64_t ts = H->stats.tstep;
    std::memset(&H->stats, 0, sizeof(H->stats));
    H->stats.time = t;
    H->stats.tstep = ts;
    return OW3D_OK;
}

int ow3d_read_paddle_signal(const char* path, int cap, double* dt, int* nt, int* n2, double* y, double* flux) {
    PaddleSignal ps;
    std::string err;
    if (int r = read_paddle_signal(path, ps, &err)) { g_last_error = err; return r; }
    if (dt) *dt = ps.dt;
    if (nt) *nt = ps.nt;
    if (n2) *n2 = ps.n2;
    if (y && flux && cap >= ps.nt * ps.n2) {
        std::copy(ps.y.begin(), ps.y.end(), y);
        std::copy(ps.flux.begin(), ps.flux.end(), flux);
    }
    return OW3D_OK;
}

int ow3d_set_paddle_signal(ow3d_handle* H, int nt, int n2, double dt, const double* y, const double* flux) {
    if (!H || !y || !flux || nt < 5 || n2 < 1 || !(dt > 0)) {
        g_last_error = "ow3d_set_paddle_signal: bad arguments";
        return OW3D_ERR_BAD_INPUT;
    }
    if (!H->pad_on) {
        g_last_error = "ow3d_set_paddle_signal: the handle's IncWaveType is not 3";
        return OW3D_ERR_BAD_INPUT;
    }
    PaddleSignal ps;
    ps.dt = dt; ps.nt = nt; ps.n2 = n2;
    ps.y.assign(y, y + n2);
    ps.flux.assign(flux, flux + (size_t)nt * n2);
    std::vector<double> F, X;
    std::string err;
    if (int r = paddle_tables(H->p, H->G, ps, F, X, &err)) { g_last_error = err; return r; }
    CK(cudaSetDevice(H->dev));
    CK(cudaStreamSynchronize(H->st));
    double *dF, *dX;
    TRY(upload(H, &dF, F));
    TRY(upload(H, &dX, X));
    H->pad.F = dF; H->pad.X = dX; H->pad.nt = nt; H->pad.dt = dt;
    H->pad_set = true;
    drop_step_graphs(H);   // captured wavemaker launches hold the old table
    return OW3D_OK;
}

int ow3d_set_coarse_cluster(ow3d_handle* H, int on) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    const bool c = on != 0;
    if (H->mg64.table.cluster == c && H->mg32.table.cluster == c) return OW3D_OK;
    CK(cudaSetDevice(H->dev));
    CK(cudaStreamSynchronize(H->st));
    H->mg64.table.cluster = c;
    H->mg32.table.cluster = c;
    // the captured launches hold the other coarse kernel
    drop_step_graphs(H);
    for (auto& g : H->iter_graphs) cudaGraphExecDestroy(g.exec);
    H->iter_graphs.clear();
    return OW3D_OK;
}

int ow3d_set_smoother_order(ow3d_handle* H, int order) {
    if (!H || (order != OW3D_SMOOTHER_MULTICOLOUR && order != OW3D_SMOOTHER_LEXICOGRAPHIC)) return OW3D_ERR_BAD_INPUT;
    const bool lx = order == OW3D_SMOOTHER_LEXICOGRAPHIC;
    if (H->mg64.table.lex == lx && H->mg32.table.lex == lx) return OW3D_OK;
    CK(cudaSetDevice(H->dev));
    CK(cudaStreamSynchronize(H->st));
    H->mg64.table.lex = lx;
    H->mg32.table.lex = lx;
    // the captured launches hold the other smoother
    drop_step_graphs(H);
    for (auto& g : H->iter_graphs) cudaGraphExecDestroy(g.exec);
    H->iter_graphs.clear();
    return OW3D_OK;
}

int ow3d_set_graphs(ow3d_handle* H, int on) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    H->graphs = on ? 1 : 0;
    if (!on) drop_step_graphs(H);
    return OW3D_OK;
}

const char* ow3d_strerror(int s) {
    switch (s) {
        case OW3D_OK: return "ok";
        case OW3D_NOT_CONVERGED: return "GMRES reached its matvec limit before the tolerance (solution kept)";
        case OW3D_ERR_BAD_INPUT: return "bad input";
        case OW3D_ERR_CUDA: return "CUDA error";
        case OW3D_ERR_OOM: return "out of device memory";
        case OW3D_ERR_UNSTABLE: return "solution unstable (max|eta| > 10 max h)";
        case OW3D_ERR_TIMEOUT: return "timeout";
        case OW3D_ERR_NO_DEVICE: return "no CUDA device";
        case OW3D_ERR_IO: return "I/O error";
        case OW3D_ERR_UNSUPPORTED: return "unsupported configuration";
        default: return "unknown status";
    }
}

const char* ow3d_version(void) { return "ow3d-b200 0.1 (sm_100a)"; }

const char* ow3d_last_error(void) { return g_last_error.c_str(); }

// --------------------------------------------------------- test hooks
int ow3d_level_count(const ow3d_handle* H) { return H ? H->nlev : -1; }

int ow3d_level_dims(const ow3d_handle* H, int l, int* Nx, int* Ny, int* Nz, int* ncolor) {
    if (!H || l < 0 || l >= H->nlev) return OW3D_ERR_BAD_INPUT;
    const LevelHost& L = H->G.levels[l];
    *Nx = L.Nx; *Ny = L.Ny; *Nz = L.Nz; *ncolor = L.ncolor;
    return OW3D_OK;
}

int ow3d_test_stencils(const ow3d_handle* H, double* SX, double* SY, double* SZ) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    if (SX) std::copy(H->G.SX.w.begin(), H->G.SX.w.end(), SX);
    if (SY) std::copy(H->G.SY.w.begin(), H->G.SY.w.end(), SY);
    if (SZ) std::copy(H->G.SZ.w.begin(), H->G.SZ.w.end(), SZ);
    return OW3D_OK;
}

int ow3d_test_surface_derivs(ow3d_handle* H, double* Ex, double* Ey) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    const size_t cb = sizeof(double) * (size_t)H->G.C;
    if (Ex) CK(cudaMemcpyAsync(Ex, H->Ex, cb, cudaMemcpyDeviceToHost, H->st));
    if (Ey) CK(cudaMemcpyAsync(Ey, H->Ey, cb, cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    return OW3D_OK;
}

int ow3d_test_pdamp_setup(const ow3d_params* p, int* i1, int* nd, double* gamPhi, double* gamEta, double* L,
                          double* Linv) {
    if (!p) return OW3D_ERR_BAD_INPUT;
    std::string e;
    if (check_supported(*p, &e)) { g_last_error = e; return OW3D_ERR_UNSUPPORTED; }
    const size_t C = (size_t)(p->Nx + 2) * (size_t)(p->Ny > 1 ? p->Ny + 2 : 1);
    const std::vector<double> one(C, 1.0), zero(C, 0.0);
    GridHost G;
    if (int r = build_grid(*p, one.data(), zero.data(), zero.data(), zero.data(), zero.data(), G, &e)) {
        g_last_error = e;
        return r;
    }
    PDampHost d;
    if (int r = build_pdamp(*p, G, d, &e)) { g_last_error = e; return r; }
    if (i1) *i1 = d.i1;
    if (nd) *nd = d.nd;
    if (gamPhi) std::copy(d.gamPhi.begin(), d.gamPhi.end(), gamPhi);
    if (gamEta) std::copy(d.gamEta.begin(), d.gamEta.end(), gamEta);
    if (L) std::copy(d.L.begin(), d.L.end(), L);
    if (Linv) std::copy(d.Linv.begin(), d.Linv.end(), Linv);
    return OW3D_OK;
}

int ow3d_test_ran1(int idum, int n, float* out, int* idum_out) {
    if (n < 0 || (n > 0 && !out)) return OW3D_ERR_BAD_INPUT;
    Ran1 r;
    for (int i = 0; i < n; ++i) out[i] = r.next(idum);
    if (idum_out) *idum_out = idum;
    return OW3D_OK;
}

int ow3d_test_level_z(const ow3d_handle* H, int l, double* z) {
    if (!H || l < 0 || l >= H->nlev) return OW3D_ERR_BAD_INPUT;
    std::copy(H->G.levels[l].z.begin(), H->G.levels[l].z.end(), z);
    return OW3D_OK;
}

int ow3d_test_zone_gamma(const ow3d_handle* H, int zone, double* g) {
    if (!H || zone < 0 || zone >= (int)H->zones_h.size()) return OW3D_ERR_BAD_INPUT;
    std::copy(H->zones_h[zone].gam.begin(), H->zones_h[zone].gam.end(), g);
    return OW3D_OK;
}

int ow3d_test_filter_coeffs(const ow3d_handle* H, double* fc, double* F2) {
    if (!H) return OW3D_ERR_BAD_INPUT;
    std::vector<double> a, b;
    filter_coeffs(H->p, a, b);
    std::copy(a.begin(), a.end(), fc);
    std::copy(b.begin(), b.end(), F2);
    return OW3D_OK;
}

int ow3d_test_level_op(ow3d_handle* H, int l, int op, int nu, const double* in1, const double* in2, double* out) {
    if (!H || l < 0 || l >= H->nlev) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    if (!H->mixed) return level_op_t<double>(H, H->mg64, l, op, nu, in1, in2, out);
    return level_op_t<float>(H, H->mg32, l, op, nu, in1, in2, out);
}

int ow3d_bench_kernel(ow3d_handle* H, int which, int reps, double* ms_total) {
    if (!H || reps < 1 || which < 0 || which > 2) return OW3D_ERR_BAD_INPUT;
    if (which == 2 && (H->mixed || H->nlev == 0)) return OW3D_ERR_BAD_INPUT;
    CK(cudaSetDevice(H->dev));
    TRY(ensure_staging(H));
    const size_t nb = sizeof(double) * (size_t)H->G.N;
    std::vector<double> host(H->G.N);
    for (size_t q = 0; q < host.size(); ++q) host[q] = std::sin(0.001 * (double)q);
    CK(cudaMemcpy(H->s_phi, host.data(), nb, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(H->s_rhs, host.data(), nb, cudaMemcpyHostToDevice));
    Surface s{nullptr, nullptr, nullptr, nullptr, nullptr};
    // each timed launch follows a write of the Krylov basis (larger than L2),
    // so that it reads its inputs from DRAM; only the launch itself is timed
    const size_t flush = sizeof(double) * (size_t)(H->m + 1) * (size_t)H->ldv;
    std::vector<cudaEvent_t> ev(2 * (size_t)reps);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    auto once = [&]() {
        if (which == 0) {
            launch_ho_matvec<double>(H->hg, s, H->s_phi, nullptr, nullptr, H->s_rhs, 0, H->st);
        } else if (which == 1) {
            precond_into(H, H->s_phi, nullptr, H->s_rhs);
        } else {
            // one colour pass of the finest multigrid level (x = s_phi, b = s_rhs)
            LevelDev<double> F = H->mg64.lev.back();
            F.xv = H->s_phi;
            F.bv = H->s_rhs;
            launch_lo_pass<double>(F, 0, H->st);
        }
    };
    once();
    for (int r = 0; r < reps; ++r) {
        CK(cudaMemsetAsync(H->V, 0, flush, H->st));
        CK(cudaEventRecord(ev[2 * r], H->st));
        once();
        CK(cudaEventRecord(ev[2 * r + 1], H->st));
    }
    CK(cudaEventSynchronize(ev.back()));
    double tot = 0;
    for (int r = 0; r < reps; ++r) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]));
        tot += ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    *ms_total = tot;
    CK(cudaGetLastError());
    return OW3D_OK;
}

int ow3d_test_sizeof(int which) {
    switch (which) {
        case 0: return (int)sizeof(ow3d_params);
        case 1: return (int)sizeof(ow3d_zone);
        case 2: return (int)sizeof(ow3d_stats);
        default: return -1;
    }
}

}  // extern "C"
