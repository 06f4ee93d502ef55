// GMRES building blocks on the device (FP64 in both precision forms).
//
// The reference drives SPARSKIT2's gmres through reverse communication
// (src/wrappers/iterative_solution.f90:50-134); here the Arnoldi process,
// the Givens rotations and the least-squares update stay on the device:
//   multidot      h_i = s_i <V_i, w>, i < k, and |w|^2      (one pass over V, w)
//   project       w -= sum_i h_i s_i V_i, and |w|^2         (one pass over V, w)
//   arnoldi_finish: Hessenberg column, Givens rotation, residual estimate,
//                   re-orthogonalisation decision and stopping test (1 thread)
// Reductions are deterministic: every block writes a partial sum, the last
// block to finish (atomic ticket) adds the partials in block order.
// Basis vectors are stored unnormalised with a scale factor s_i = 1/|V_i|,
// which saves the normalisation pass.
#include "ow3d_internal.h"
#include <cmath>

namespace ow3d {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxDots = kMaxKrylov + 1;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-reduce `nv` values per thread into partial[v*nblocks + blockIdx.x].
__device__ void block_store_partials(const double* acc, int nv, double* partial, int nblocks) {
    __shared__ double red[kThreads / 32][kMaxDots + 1];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int v = 0; v < nv; ++v) {
        double s = warp_sum(acc[v]);
        if (lane == 0) red[wid][v] = s;
    }
    __syncthreads();
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) s += red[w][v];
        partial[(int64_t)v * nblocks + blockIdx.x] = s;
    }
}

// The last block to finish sums the partials: warp w reduces vectors
// v = w, w + nwarps, ...; lane l adds blocks l, l+32, ... in order and the
// warp tree combines the lanes (a fixed order: deterministic results).
// Returns true in that block.
__device__ bool last_block_reduce(double* partial, int nv, int nblocks, unsigned int* counter, double* out) {
    __shared__ bool amlast;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = atomicAdd(counter, 1u);
        amlast = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!amlast) return false;
    __threadfence();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int v = wid; v < nv; v += nw) {
        const double* pv = partial + (int64_t)v * nblocks;
        double s = 0;
        for (int b = lane; b < nblocks; b += 32) s += __ldcg(pv + b);
        s = warp_sum(s);
        if (lane == 0) out[v] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// Basis vectors are contiguous: V_i = V + i * ldv.
// cond: 0 always run; 1 run only when ks->reorth is set (second CGS pass).
__global__ void __launch_bounds__(kThreads) k_multidot(const double* __restrict__ V, int64_t ldv, int k,
                                                       const double* __restrict__ w, int64_t n, double* partial,
                                                       unsigned int* counter, int nblocks, KrylovState* ks, int cond) {
    if (cond && !ks->reorth) return;
    if (ks->done) return;
    const int nv = k + 1;   // k dot products and |w|^2
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    __shared__ double red[kThreads / 32][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int v0 = 0; v0 < nv; v0 += 8) {
        double acc[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[u] = 0.0;
        for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += stride) {
            const double wt = w[t];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int v = v0 + u;
                if (v < k) acc[u] += V[(int64_t)v * ldv + t] * wt;
                else if (v == k) acc[u] += wt * wt;
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            double sm = warp_sum(acc[u]);
            if (lane == 0) red[wid][u] = sm;
        }
        __syncthreads();
        if (threadIdx.x < 8 && v0 + (int)threadIdx.x < nv) {
            double sm = 0;
            for (int q = 0; q < (int)(blockDim.x / 32); ++q) sm += red[q][threadIdx.x];
            partial[(int64_t)(v0 + threadIdx.x) * nblocks + blockIdx.x] = sm;
        }
        __syncthreads();
    }
    __shared__ double res[kMaxDots];
    if (last_block_reduce(partial, nv, nblocks, counter, res)) {
        if (threadIdx.x == 0) {
            for (int v = 0; v < k; ++v) ks->dots[v] = ks->scale[v] * res[v];
            if (cond) {
                for (int v = 0; v < k; ++v) ks->H[ks->k][v] += ks->dots[v];
            } else {
                for (int v = 0; v < k; ++v) ks->H[ks->k][v] = ks->dots[v];
                ks->w0 = res[k];
            }
        }
    }
}

// w -= sum_v dots[v] * scale[v] * V_v ; |w|^2 -> ks->w1, and decide re-orthogonalisation.
__global__ void __launch_bounds__(kThreads) k_project(const double* __restrict__ V, int64_t ldv, int k,
                                                      double* __restrict__ w, int64_t n,
                                                      double* partial, unsigned int* counter, int nblocks,
                                                      KrylovState* ks, int cond) {
    if (cond && !ks->reorth) return;
    if (ks->done) return;
    __shared__ double coef[kMaxDots];
    for (int v = threadIdx.x; v < k; v += blockDim.x) coef[v] = ks->dots[v] * ks->scale[v];
    __syncthreads();
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += stride) {
        double a = w[t];
#pragma unroll 4
        for (int v = 0; v < k; ++v) a -= coef[v] * V[(int64_t)v * ldv + t];
        w[t] = a;
        acc[0] += a * a;
    }
    block_store_partials(acc, 1, partial, nblocks);
    __shared__ double res[1];
    if (last_block_reduce(partial, 1, nblocks, counter, res)) {
        if (threadIdx.x == 0) {
            ks->w1 = res[0];
            // Daniel-Gragg-Kaufman-Stewart test: re-orthogonalise once when the
            // projection removed more than half of |w|^2.
            ks->reorth = (!cond && res[0] < 0.5 * ks->w0) ? 1 : 0;
        }
    }
}

// Initial residual norm: beta = |v|, tolerance rtol*beta + atol.
__global__ void __launch_bounds__(kThreads) k_norm_init(const double* __restrict__ v, int64_t n, double* partial,
                                                        unsigned int* counter, int nblocks, KrylovState* ks,
                                                        double rtol, double atol) {
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += stride) acc[0] += v[t] * v[t];
    block_store_partials(acc, 1, partial, nblocks);
    __shared__ double res[1];
    if (last_block_reduce(partial, 1, nblocks, counter, res)) {
        if (threadIdx.x == 0) {
            const double beta = sqrt(res[0]);
            ks->beta = beta;
            ks->iters += 1;   // the residual's matvec (iterative_solution.f90:58-60 counts it)
            if (ks->iters == 1) ks->tol = rtol * beta + atol;   // fixed at the first residual
            ks->resid = beta;
            for (int i = 0; i < kMaxKrylov + 2; ++i) ks->g[i] = 0.0;
            ks->g[0] = beta;
            ks->scale[0] = beta > 0 ? 1.0 / beta : 0.0;
            ks->k = 0;
            ks->reorth = 0;
            if (beta <= ks->tol) { ks->done = 1; ks->converged = 1; }
        }
    }
}

// One thread: finish Arnoldi step k (1-based after increment).
__global__ void k_arnoldi_finish(KrylovState* ks, int maxmv, int m) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (ks->done) return;
    const int k = ks->k + 1;           // this step's column index is ks->k (0-based)
    double* hc = ks->H[ks->k];
    const double nrm = sqrt(ks->w1);
    hc[k] = nrm;
    ks->scale[k] = nrm > 0 ? 1.0 / nrm : 0.0;
    for (int i = 0; i < k - 1; ++i) {
        const double a0 = hc[i];
        hc[i] = ks->cs[i] * a0 + ks->sn[i] * hc[i + 1];
        hc[i + 1] = ks->cs[i] * hc[i + 1] - ks->sn[i] * a0;
    }
    double x = hc[k - 1], yv = hc[k];
    const double r = sqrt(x * x + yv * yv);
    double c = 1.0, s = 0.0;
    if (r != 0.0) { c = x / r; s = yv / r; }
    hc[k - 1] = r; hc[k] = 0.0;
    ks->cs[k - 1] = c; ks->sn[k - 1] = s;
    const double al = -s * ks->g[k - 1];
    ks->g[k - 1] = c * ks->g[k - 1];
    ks->g[k] = al;
    ks->resid = fabs(al);
    ks->k = k;
    ks->iters += 1;
    ks->reorth = 0;
    const bool conv = ks->resid <= ks->tol;
    if (conv) ks->converged = 1;
    if (conv || k >= m || ks->iters >= maxmv || nrm == 0.0) ks->done = 1;
}

// Upper-triangular solve H y = g for the current k (1 thread).
__global__ void k_backsolve(KrylovState* ks) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int kk = ks->k;
    while (kk > 0 && ks->H[kk - 1][kk - 1] == 0.0) --kk;
    for (int i = kk - 1; i >= 0; --i) {
        double t = ks->g[i];
        for (int j = i + 1; j < kk; ++j) t -= ks->H[j][i] * ks->y[j];
        ks->y[i] = t / ks->H[i][i];
    }
    for (int i = kk; i <= kMaxKrylov; ++i) ks->y[i] = 0.0;
    ks->k = kk;
}

// x += sum_i y_i * (use_scale ? scale_i : 1) * Z_i
template <typename TZ>
__global__ void __launch_bounds__(kThreads) k_solution_update(double* __restrict__ x, const TZ* __restrict__ Z,
                                                              int64_t ldz, int64_t n,
                                                              const KrylovState* ks, int use_scale) {
    __shared__ double coef[kMaxDots];
    const int k = ks->k;
    for (int v = threadIdx.x; v < k; v += blockDim.x) coef[v] = ks->y[v] * (use_scale ? ks->scale[v] : 1.0);
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += stride) {
        double a = x[t];
        for (int v = 0; v < k; ++v) a += coef[v] * (double)Z[(int64_t)v * ldz + t];
        x[t] = a;
    }
}

__global__ void k_krylov_reset(KrylovState* ks) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    ks->k = 0; ks->done = 0; ks->converged = 0; ks->iters = 0; ks->reorth = 0; ks->status = 0;
    ks->tol = 0; ks->resid = 0; ks->beta = 0;
}

}  // namespace

void launch_multidot(const double* V, int64_t ldv, int k, const double* w, int64_t n, const DotScratch& sc,
                     KrylovState* ks, int cond, cudaStream_t st) {
    k_multidot<<<sc.nblocks, kThreads, 0, st>>>(V, ldv, k, w, n, sc.partial, sc.counter, sc.nblocks, ks, cond);
}

void launch_project(const double* V, int64_t ldv, int k, double* w, int64_t n, const DotScratch& sc, KrylovState* ks,
                    int cond, cudaStream_t st) {
    k_project<<<sc.nblocks, kThreads, 0, st>>>(V, ldv, k, w, n, sc.partial, sc.counter, sc.nblocks, ks, cond);
}

void launch_arnoldi_finish(KrylovState* ks, int maxmv, int m, cudaStream_t st) {
    k_arnoldi_finish<<<1, 32, 0, st>>>(ks, maxmv, m);
}

void launch_norm_init(const double* v, int64_t n, const DotScratch& sc, KrylovState* ks, double rtol, double atol,
                      cudaStream_t st) {
    k_norm_init<<<sc.nblocks, kThreads, 0, st>>>(v, n, sc.partial, sc.counter, sc.nblocks, ks, rtol, atol);
}

void launch_backsolve(KrylovState* ks, cudaStream_t st) { k_backsolve<<<1, 32, 0, st>>>(ks); }

template <typename TZ>
void launch_solution_update(double* x, const TZ* Z, int64_t ldz, int64_t n, const KrylovState* ks, int use_scale,
                            cudaStream_t st) {
    int nb = (int)((n + kThreads - 1) / kThreads);
    if (nb > 148 * 8) nb = 148 * 8;
    if (nb < 1) nb = 1;
    k_solution_update<TZ><<<nb, kThreads, 0, st>>>(x, Z, ldz, n, ks, use_scale);
}
template void launch_solution_update<double>(double*, const double*, int64_t, int64_t, const KrylovState*, int,
                                             cudaStream_t);
template void launch_solution_update<float>(double*, const float*, int64_t, int64_t, const KrylovState*, int,
                                            cudaStream_t);

void launch_krylov_reset(KrylovState* ks, cudaStream_t st) { k_krylov_reset<<<1, 32, 0, st>>>(ks); }

// Restart after a full subspace: keep the matvec count and the tolerance.
__global__ void k_krylov_restart(KrylovState* ks) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    ks->k = 0; ks->done = 0; ks->converged = 0; ks->reorth = 0;
}
void launch_krylov_restart(KrylovState* ks, cudaStream_t st) { k_krylov_restart<<<1, 32, 0, st>>>(ks); }

}  // namespace ow3d
