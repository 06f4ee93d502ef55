// GMRES building blocks on the device (FP64 in both precision forms).
//
// The reference drives SPARSKIT2's gmres through reverse communication
// (src/wrappers/iterative_solution.f90:50-134); here the Arnoldi process,
// the Givens rotations and the least-squares update stay on the device, for
// right (flexible) and left preconditioning alike: each Arnoldi step is one
// reduction pass and one update pass of delayed classical Gram-Schmidt
// (DCGS2, below), whose last block forms the Hessenberg column, the Givens
// rotation, the residual estimate and the stopping test.
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
        int b = lane;
        // eight independent L2 loads in flight per lane, then added in order
        for (; b + 7 * 32 < nblocks; b += 8 * 32) {
            double q[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) q[u] = __ldcg(pv + b + u * 32);
#pragma unroll
            for (int u = 0; u < 8; ++u) s += q[u];
        }
        for (; b < nblocks; b += 32) s += __ldcg(pv + b);
        s = warp_sum(s);
        if (lane == 0) out[v] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// Initial residual norm: beta = |v|, tolerance rtol*beta + atol.
// hnext (nonzero only inside a captured step graph): the condition of the
// graph node that runs the next Arnoldi step, set to "not done".
__global__ void __launch_bounds__(kThreads) k_norm_init(const double* __restrict__ v, int64_t n, double* partial,
                                                        unsigned int* counter, int nblocks, KrylovState* ks,
                                                        double rtol, double atol, cudaGraphConditionalHandle hnext) {
    pdl_entry();
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
            if (hnext) cudaGraphSetConditional(hnext, ks->done ? 0u : 1u);
        }
    }
}

// Upper-triangular solve R y = g for the current k (1 thread); R is the
// in-place rotated H (left GMRES) or the separate rotated copy (FGMRES).
// With in_basis set (left preconditioning), the coefficients of the vectors
// the Arnoldi steps multiplied are taken to the final basis, y <- T y, so
// that the update is x += sum_i y_i v_i.
__global__ void k_backsolve(KrylovState* ks, int rotated_R, int in_basis) {
    pdl_entry();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    auto Rv = [&](int col, int row) -> double { return rotated_R ? ks->R[col][row] : ks->H[col][row]; };
    int kk = ks->k;
    while (kk > 0 && Rv(kk - 1, kk - 1) == 0.0) --kk;
    for (int i = kk - 1; i >= 0; --i) {
        double t = ks->g[i];
        for (int j = i + 1; j < kk; ++j) t -= Rv(j, i) * ks->y[j];
        ks->y[i] = t / Rv(i, i);
    }
    if (in_basis) {
        // T is upper triangular in (i, j): entry i of T y reads y[j >= i]
        // only, so it can replace y[i] in increasing i
        for (int i = 0; i < kk; ++i) {
            double c = 0.0;
            for (int j = i; j < kk; ++j) c += ks->T[j][i] * ks->y[j];
            ks->y[i] = c;
        }
    }
    for (int i = kk; i <= kMaxKrylov; ++i) ks->y[i] = 0.0;
    ks->k = kk;
}

// x += sum_i y_i * (use_scale ? scale_i : 1) * Z_i
template <typename TZ>
__global__ void __launch_bounds__(kThreads) k_solution_update(double* __restrict__ x, const TZ* __restrict__ Z,
                                                              int64_t ldz, int64_t n,
                                                              const KrylovState* ks, int use_scale) {
    pdl_entry();
    __shared__ double coef[kMaxDots];
    const int k = ks->k;
    for (int v = threadIdx.x; v < k; v += blockDim.x) coef[v] = ks->y[v] * (use_scale ? ks->scale[v] : 1.0);
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += stride) {
        double a = x[t];
        for (int v = 0; v < k; ++v) a += coef[v] * (double)__ldcs(Z + (int64_t)v * ldz + t);
        x[t] = a;
    }
}

__global__ void k_krylov_reset(KrylovState* ks) {
    pdl_entry();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    ks->k = 0; ks->done = 0; ks->converged = 0; ks->iters = 0; ks->reorth = 0; ks->status = 0;
    ks->tol = 0; ks->resid = 0; ks->beta = 0;
}

// ---------------------------------------------------------------- DCGS2
// Arnoldi orthogonalisation by delayed classical Gram-Schmidt with
// reorthogonalisation (Swirydowicz, Langou, Ananthan, Yang, Thomas, "Low
// synchronization Gram-Schmidt and generalized minimal residual algorithms",
// NLAA 2021): the second Gram-Schmidt pass of V_j rides on step j's single
// reduction, so each Arnoldi step reads the basis twice (reduce, update)
// instead of four times. V_0..V_{j-1} are final, V_j has had one pass.

// rotate unrotated column col of H with rotations 0..col-1 into R, form
// rotation col, rotate g from its value before rotation col; returns |g[col+1]|
__device__ double dcgs_rotate(KrylovState* ks, int col) {
    for (int r = 0; r <= col + 1; ++r) ks->R[col][r] = ks->H[col][r];
    for (int i = 0; i < col; ++i) {
        const double a0 = ks->R[col][i];
        ks->R[col][i] = ks->cs[i] * a0 + ks->sn[i] * ks->R[col][i + 1];
        ks->R[col][i + 1] = ks->cs[i] * ks->R[col][i + 1] - ks->sn[i] * a0;
    }
    const double x = ks->R[col][col], yv = ks->R[col][col + 1];
    const double r = sqrt(x * x + yv * yv);
    double c = 1.0, sg = 0.0;
    if (r != 0.0) { c = x / r; sg = yv / r; ks->R[col][col] = r; ks->R[col][col + 1] = 0.0; }
    ks->cs[col] = c; ks->sn[col] = sg;
    const double g0 = ks->gsave[col];
    const double al = -sg * g0;
    ks->g[col] = c * g0;
    ks->g[col + 1] = al;
    return fabs(al);
}

// One thread, after step j's reduction: res[2i] = <V_i, V_j>, res[2i+1] = <V_i, W>, i <= j.
// The vector step j multiplied, scale_j V_j with V_j after one pass and
// scale_j its provisional scale, is scale_j (nu q_j + sum sigma_i q_i) in
// the final basis: column j of T (used by left preconditioning, whose
// solution is a combination of those vectors).
__device__ void dcgs_column(KrylovState* ks, int j, const double* res) {
    double ss = 0.0, corr = 0.0;
    if (j >= 1) {
        const double sp = ks->scale[j];
        for (int i = 0; i < j; ++i) {
            const double sig = ks->scale[i] * res[2 * i];
            ks->coefA[i] = sig;          // sigma_i, scaled below
            ks->T[j][i] = sp * sig;
            ss += sig * sig;
        }
        const double nu = sqrt(fmax(res[2 * j] - ss, 0.0));
        ks->T[j][j] = sp * nu;
        // complete column j-1: W_{j-1} = sum (h + sigma) q_i + nu q_j
        for (int i = 0; i < j; ++i) ks->H[j - 1][i] += ks->coefA[i];
        ks->H[j - 1][j] = nu;
        ks->scale[j] = nu > 0 ? 1.0 / nu : 0.0;
        ks->resid = dcgs_rotate(ks, j - 1);
    } else {
        ks->T[0][0] = 1.0;   // scale_0 V_0 is final: v_0
    }
    for (int i = 0; i < j; ++i) {
        const double hq = ks->scale[i] * res[2 * i + 1];
        ks->H[j][i] = hq;
        corr += ks->coefA[i] * hq;
        ks->coefB[i] = hq * ks->scale[i];
        ks->coefA[i] *= ks->scale[i];
    }
    const double hj = (j >= 1) ? (res[2 * j + 1] - corr) * ks->scale[j] : ks->scale[j] * res[2 * j + 1];
    ks->H[j][j] = hj;
    ks->coefB[j] = hj * ks->scale[j];
}

// Reduction: res[2v] = <V_v, V_j>, res[2v+1] = <V_v, W> for v <= j. The
// vectors are cut into chunks of kDotE * blockDim.x element pairs; a block
// takes chunks in turn, keeps its thread's kDotE pairs of V_j and W in
// registers, and streams every V_v of the chunk once (so each vector is read
// from memory once per step). Per vector, each warp adds its sum to its own
// shared-memory slot; the block's slots become partial[u * gridDim.x + b];
// the last block reduces the partials in a fixed order and runs dcgs_column.
constexpr int kDotE = 4;
constexpr int kDotG = 4;   // vectors whose loads are issued together

__global__ void __launch_bounds__(kThreads) k_dcgs_reduce(const double* __restrict__ V, int64_t ldv, int j,
                                                          const double* __restrict__ W, int64_t n, double* partial,
                                                          unsigned int* counter, int nbx, KrylovState* ks) {
    pdl_entry();
    if (ks->done) return;
    __shared__ double acc[2 * kMaxDots][kThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nv = 2 * (j + 1);
    for (int u = threadIdx.x; u < nv * nw; u += blockDim.x) acc[u / nw][u % nw] = 0.0;
    __syncthreads();
    const int64_t n2 = (n + 1) / 2;
    const int64_t chunk = (int64_t)kDotE * blockDim.x;
    const int64_t nchunks = (n2 + chunk - 1) / chunk;
    const double2* q2 = reinterpret_cast<const double2*>(V + (int64_t)j * ldv);
    const double2* w2 = reinterpret_cast<const double2*>(W);
    for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
        const int64_t t0 = ch * chunk + threadIdx.x;
        double2 q[kDotE], w[kDotE];
#pragma unroll
        for (int e = 0; e < kDotE; ++e) {
            const int64_t t = t0 + (int64_t)e * blockDim.x;
            if (t < n2) { q[e] = q2[t]; w[e] = w2[t]; }
            else { q[e] = make_double2(0.0, 0.0); w[e] = make_double2(0.0, 0.0); }
        }
        // vectors in groups of kDotG, all their loads in flight together; the
        // older basis vectors are read once per pass, so they are streamed
        // (evict-first) rather than let them push the multigrid levels and
        // their coefficient tables out of L2 before the next V-cycle
        for (int v0 = 0; v0 <= j; v0 += kDotG) {
            double2 x[kDotG][kDotE];
#pragma unroll
            for (int g = 0; g < kDotG; ++g) {
                const int v = v0 + g;
                const double2* a2 = reinterpret_cast<const double2*>(V + (int64_t)min(v, j) * ldv);
#pragma unroll
                for (int e = 0; e < kDotE; ++e) {
                    const int64_t t = t0 + (int64_t)e * blockDim.x;
                    x[g][e] = (v < j && t < n2) ? __ldcs(a2 + t) : make_double2(0.0, 0.0);
                }
            }
#pragma unroll
            for (int g = 0; g < kDotG; ++g) {
                const int v = v0 + g;
                if (v > j) break;
                double sa = 0, sb = 0;
#pragma unroll
                for (int e = 0; e < kDotE; ++e) {
                    const double2 xe = (v == j) ? q[e] : x[g][e];
                    sa += xe.x * q[e].x + xe.y * q[e].y;
                    sb += xe.x * w[e].x + xe.y * w[e].y;
                }
                sa = warp_sum(sa);
                sb = warp_sum(sb);
                if (lane == 0) { acc[2 * v][wid] += sa; acc[2 * v + 1][wid] += sb; }
            }
        }
    }
    __syncthreads();
    for (int u = threadIdx.x; u < nv; u += blockDim.x) {
        double t = 0;
        for (int w = 0; w < nw; ++w) t += acc[u][w];
        partial[(int64_t)u * gridDim.x + blockIdx.x] = t;
    }
    __shared__ bool amlast;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) amlast = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!amlast) return;
    __threadfence();
    __shared__ double res[2 * kMaxDots];
    const int nb = gridDim.x;
    for (int u = wid; u < nv; u += nw) {
        const double* pv = partial + (int64_t)u * nb;
        double sacc = 0;
        for (int bb = lane; bb < nb; bb += 32) sacc += __ldcg(pv + bb);
        sacc = warp_sum(sacc);
        if (lane == 0) res[u] = sacc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *counter = 0u;
        dcgs_column(ks, j, res);
    }
    (void)nbx;
}

// Update: V_j <- V_j - sum_{i<j} coefA_i V_i,  W <- W - sum_{i<j} coefB_i V_i - coefB_j V_j(new),
// |W|^2; the last block completes column j's provisional norm, its rotation,
// the residual estimate and the stopping test.
__global__ void __launch_bounds__(kThreads) k_dcgs_update(double* __restrict__ V, int64_t ldv, int j,
                                                          double* __restrict__ W, int64_t n, double* partial,
                                                          unsigned int* counter, int nblocks, KrylovState* ks,
                                                          int maxmv, int m, cudaGraphConditionalHandle hnext) {
    pdl_entry();
    if (ks->done) return;
    __shared__ double cA[kMaxDots], cB[kMaxDots + 1];
    for (int v = threadIdx.x; v <= j; v += blockDim.x) { cB[v] = ks->coefB[v]; if (v < j) cA[v] = ks->coefA[v]; }
    __syncthreads();
    const double cBj = cB[j];
    double acc[1] = {0.0};
    const int64_t n2 = (n + 1) / 2;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    double2* vj2 = reinterpret_cast<double2*>(V + (int64_t)j * ldv);
    double2* w2 = reinterpret_cast<double2*>(W);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n2; t += stride) {
        // v_j is next read as an older vector of the following reduction
        // (streamed), so it is written back evict-first too
        double2 q = __ldcs(vj2 + t), a = w2[t];
        for (int v0 = 0; v0 < j; v0 += 8) {
            double2 vv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (v0 + u < j) vv[u] = __ldcs(reinterpret_cast<const double2*>(V + (int64_t)(v0 + u) * ldv) + t);
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (v0 + u < j) {
                    q.x -= cA[v0 + u] * vv[u].x; q.y -= cA[v0 + u] * vv[u].y;
                    a.x -= cB[v0 + u] * vv[u].x; a.y -= cB[v0 + u] * vv[u].y;
                }
        }
        a.x -= cBj * q.x; a.y -= cBj * q.y;
        if (j > 0) __stcs(vj2 + t, q);
        w2[t] = a;
        acc[0] += a.x * a.x + a.y * a.y;
    }
    block_store_partials(acc, 1, partial, nblocks);
    __shared__ double res[1];
    if (last_block_reduce(partial, 1, nblocks, counter, res)) {
        if (threadIdx.x == 0) {
            const double nrm = sqrt(res[0]);
            ks->H[j][j + 1] = nrm;
            ks->scale[j + 1] = nrm > 0 ? 1.0 / nrm : 0.0;
            ks->gsave[j] = ks->g[j];
            ks->resid = dcgs_rotate(ks, j);
            ks->k = j + 1;
            ks->iters += 1;
            const bool conv = ks->resid <= ks->tol;
            if (conv) ks->converged = 1;
            if (conv || j + 1 >= m || ks->iters >= maxmv || nrm == 0.0) ks->done = 1;
            if (hnext) cudaGraphSetConditional(hnext, ks->done ? 0u : 1u);
        }
    }
}

__global__ void k_solve_log(const KrylovState* ks, SolveLog* out) {
    pdl_entry();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    out->iters = ks->iters;
    out->converged = ks->converged;
    out->resid = ks->resid;
    out->beta = ks->beta;
    out->tol = ks->tol;
}

}  // namespace

void launch_dcgs_reduce(const double* V, int64_t ldv, int j, const double* W, int64_t n, const DotScratch& sc,
                        KrylovState* ks, cudaStream_t st) {
    // one block per chunk up to the scratch's blocks; 2(j+1) partial rows
    const int64_t chunks = ((n + 1) / 2 + (int64_t)kDotE * kThreads - 1) / ((int64_t)kDotE * kThreads);
    int nb = sc.nblocks;
    if (nb > chunks) nb = (int)chunks;
    const int cap = (int)(((int64_t)(kMaxKrylov + 2) * sc.nblocks) / (2 * (j + 1)));   // scratch rows
    if (nb > cap) nb = cap;
    if (nb < 1) nb = 1;
    launch_k(k_dcgs_reduce, dim3(nb), dim3(kThreads), 0, st, V, ldv, j, W, n, sc.partial, sc.counter, nb, ks);
}

void launch_dcgs_update(double* V, int64_t ldv, int j, double* W, int64_t n, const DotScratch& sc, KrylovState* ks,
                        int maxmv, int m, cudaStream_t st, cudaGraphConditionalHandle hnext) {
    launch_k(k_dcgs_update, dim3(sc.nblocks), dim3(kThreads), 0, st, V, ldv, j, W, n, sc.partial, sc.counter, sc.nblocks,
                                                                  ks, maxmv, m, hnext);
}
void launch_solve_log(const KrylovState* ks, SolveLog* out, cudaStream_t st) {
    launch_k(k_solve_log, dim3(1), dim3(32), 0, st, ks, out);
}

void launch_norm_init(const double* v, int64_t n, const DotScratch& sc, KrylovState* ks, double rtol, double atol,
                      cudaStream_t st, cudaGraphConditionalHandle hnext) {
    launch_k(k_norm_init, dim3(sc.nblocks), dim3(kThreads), 0, st, v, n, sc.partial, sc.counter, sc.nblocks, ks, rtol, atol,
                                                                hnext);
}

void launch_backsolve(KrylovState* ks, cudaStream_t st, int rotated_R, int in_basis) {
    launch_k(k_backsolve, dim3(1), dim3(32), 0, st, ks, rotated_R, in_basis);
}

template <typename TZ>
void launch_solution_update(double* x, const TZ* Z, int64_t ldz, int64_t n, const KrylovState* ks, int use_scale,
                            cudaStream_t st) {
    int nb = (int)((n + kThreads - 1) / kThreads);
    if (nb > 148 * 8) nb = 148 * 8;
    if (nb < 1) nb = 1;
    launch_k(k_solution_update<TZ>, dim3(nb), dim3(kThreads), 0, st, x, Z, ldz, n, ks, use_scale);
}
template void launch_solution_update<double>(double*, const double*, int64_t, int64_t, const KrylovState*, int,
                                             cudaStream_t);
template void launch_solution_update<float>(double*, const float*, int64_t, int64_t, const KrylovState*, int,
                                            cudaStream_t);

void launch_krylov_reset(KrylovState* ks, cudaStream_t st) { launch_k(k_krylov_reset, dim3(1), dim3(32), 0, st, ks); }

// Restart after a full subspace: keep the matvec count and the tolerance.
__global__ void k_krylov_restart(KrylovState* ks) {
    pdl_entry();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    ks->k = 0; ks->done = 0; ks->converged = 0; ks->reorth = 0;
}
void launch_krylov_restart(KrylovState* ks, cudaStream_t st) { launch_k(k_krylov_restart, dim3(1), dim3(32), 0, st, ks); }

}  // namespace ow3d
