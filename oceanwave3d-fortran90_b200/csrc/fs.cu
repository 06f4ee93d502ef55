// Free-surface update around the Laplace solve (2-D, Nxg*Nyg fields).
//
//   k_fs_stage     rhsFreeSurface3D.f90:12-28 / rhsLinearFreeSurface3D.f90,
//                  Zero_Corners.f90, and the RK4 stage value
//                  (Runge_Kutta_4.f90:61-70,168-175,245-252)
//   k_relax        RelaxationModule_new.f90:52-128 (X/X and Y/Y zones) with
//                  the target lookup of AnalyticWaveMaker2D.f90:21-34
//   k_ghost_x/_y   UpdateGhostLayerX.f90:15-20 / UpdateGhostLayerY.f90
//   k_diff_x/_y    DiffXEven / DiffYEven on 2-D fields (Nz = 1)
//   k_wvel         VerticalFreeSurfaceVelocity.f90:17
//   k_rk_final     Runge_Kutta_4.f90:347-351
//   k_filter_x/_y  FILTERING.f90:17-57
//   k_extrap       Runge_Kutta_4.f90:118-121, 294-303
//   k_pd_*         funPressureTerm.f90:218-311, the pressure-damping terms
#include "ow3d_fs.h"

namespace ow3d {

namespace {

inline int nb(int64_t n, int t = 256) {
    int64_t b = (n + t - 1) / t;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

__global__ void k_fs_stage(FsArgs a, const double* E, const double* P, const double* W, const double* Ex,
                           const double* Px, const double* Ey, const double* Py, const double* E0,
                           const double* P0, double c, double* kE, double* kP, double* tE, double* tP,
                           const double* NuD, const double* Pd, const double* Qr_x) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    const double g = a.g, one = 1.0, half = 0.5;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        double ke, kp;
        if (!a.nonlinear) {
            ke = W[p];
            kp = -g * E[p];
        } else if (!a.three) {
            ke = -Ex[p] * Px[p] + W[p] * (one + Ex[p] * Ex[p]);
            if (Qr_x) ke -= Qr_x[p];   // rhsFreeSurface3D.f90:17, the roller term
            kp = -g * E[p] - half * (Px[p] * Px[p] - W[p] * W[p] * (one + Ex[p] * Ex[p]));
        } else {
            ke = -Ex[p] * Px[p] - Ey[p] * Py[p] + W[p] * (one + Ex[p] * Ex[p] + Ey[p] * Ey[p]);
            kp = -g * E[p] - half * (Px[p] * Px[p] + Py[p] * Py[p] - W[p] * W[p] * (one + Ex[p] * Ex[p] + Ey[p] * Ey[p]));
        }
        if (NuD) { ke += NuD[p]; kp += Pd[p]; }   // rhsFreeSurface3D.f90:27-28
        if (a.three) {
            const int i = (int)(p % a.Nxg), j = (int)(p / a.Nxg);
            if ((i == 0 || i == a.Nxg - 1) && (j == 0 || j == a.Nyg - 1)) { ke = 0.0; kp = 0.0; }
        }
        kE[p] = ke; kP[p] = kp;
        if (tE) { tE[p] = E0[p] + c * ke; tP[p] = P0[p] + c * kp; }
    }
}

// Type 0 (funPressureTerm.f90:238-284): the right-hand side of the zone
// solve, d/dx(gamma_phi d/dx phi) with the Dirichlet row (phi at the first
// point) and the Neumann row (zero), and NuD = -gamma_eta eta over the row.
// One block: the second derivative pass reads the whole zone of the first.
__global__ void k_pd_rhs(PDampDev d, int Nxg, const double* E, const double* P) {
    const int nd = d.nd, R = d.rank, a = (R - 1) / 2;
    const double* p0 = P + (d.i1 - 1);
    for (int i = threadIdx.x; i < nd; i += blockDim.x) {
        const int s = (i < a) ? 0 : (i >= nd - a ? nd - R : i - a);   // DfDx_1D_Uneven.f90:18-29
        const double* w = d.D1 + (size_t)i * R;
        double acc = 0.0;
        for (int m = 0; m < R; ++m) acc += p0[s + m] * w[m];
        // the damping acts on the velocity relative to the constant-flux
        // current, Ur = Q / h at the east wall (funPressureTerm.f90:249-252)
        d.f[i] = d.gamPhi[d.i1 - 1 + i] * (acc - d.Ur);
    }
    for (int i = threadIdx.x; i < Nxg; i += blockDim.x) d.NuD[i] = -d.gamEta[i] * E[i];
    __syncthreads();
    for (int i = threadIdx.x; i < nd; i += blockDim.x) {
        double v = 0.0;
        if (i == 0) {
            v = p0[0];
        } else if (i < nd - 1) {
            const int s = (i < a) ? 0 : (i >= nd - a ? nd - R : i - a);
            const double* w = d.D1 + (size_t)i * R;
            for (int m = 0; m < R; ++m) v += d.f[s + m] * w[m];
        }
        d.r[i] = v;
    }
}

// x = L^-1 r, a warp per row.
__global__ void k_pd_solve(PDampDev d) {
    const int lane = threadIdx.x & 31;
    const int nd = d.nd;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nd; i += nw) {
        const double* row = d.Linv + (size_t)i * nd;
        double acc = 0.0;
        for (int k = lane; k < nd; k += 32) acc += row[k] * d.r[k];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) d.x[i] = acc;
    }
}

// Pd over the zone, zero at its first point (funPressureTerm.f90:286-291);
// Pd stays zero outside the zone.
__global__ void k_pd_apply(PDampDev d) {
    const double x0 = d.x[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.nd; i += gridDim.x * blockDim.x)
        d.Pd[d.i1 - 1 + i] = -(d.x[i] - x0);
}

// Other types (funPressureTerm.f90:299-310): friction on eta and phi.
__global__ void k_pd_friction(PDampDev d, int64_t C, const double* E, const double* P) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        d.NuD[p] = -d.gamEta[p] * E[p];
        d.Pd[p] = -d.gamPhi[p] * P[p];
    }
}

__global__ void k_rk_final(FsArgs a, double* E, double* P, const double* k1E, const double* k2E, const double* k3E,
                           const double* k4E, const double* k1P, const double* k2P, const double* k3P,
                           const double* k4P, double dt) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    const double six = 6.0, two = 2.0;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        E[p] = E[p] + dt / six * (k1E[p] + two * k2E[p] + two * k3E[p] + k4E[p]);
        P[p] = P[p] + dt / six * (k1P[p] + two * k2P[p] + two * k3P[p] + k4P[p]);
    }
}

__global__ void k_relax(FsArgs a, RelaxZoneDev z, double* E, double* P, const StepDev* sd, double off,
                        double transient) {
    const double time = sd->time, RKtime = time + off;
    const double FAC = (RKtime < transient) ? RKtime / transient : 1.0;   // RelaxationModule_new.f90:23-27
    const int bx = z.i1 - z.i0 + 1, by = z.j1 - z.j0 + 1;
    const int64_t box = (int64_t)bx * by;
    const double* te = nullptr; const double* tp = nullptr;
    const double* te2 = nullptr; const double* tp2 = nullptr;
    if (z.wavegen) {
        if (z.nt <= 0 || !z.eta) return;
        if (z.tmode == 1) {
            long it = lround(RKtime / z.tdt); it = it < 0 ? 0 : (it > z.nt - 1 ? z.nt - 1 : it);
            te = z.eta + it * box; tp = z.phis + it * box;
        } else {
            const double diff = (RKtime - time) / z.tdt, tol = 10e-14;
            if (diff < tol || fabs(1.0 - diff) < tol) {
                long it = lround(RKtime / z.tdt); it = it < 0 ? 0 : (it > z.nt - 1 ? z.nt - 1 : it);
                te = z.eta + it * box; tp = z.phis + it * box;
            } else {
                long it = lround(time / z.tdt); it = it < 0 ? 0 : (it > z.nt - 2 ? z.nt - 2 : it);
                te = z.eta + it * box; tp = z.phis + it * box;
                te2 = z.eta + (it + 1) * box; tp2 = z.phis + (it + 1) * box;
            }
        }
    }
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < box; t += (int64_t)gridDim.x * blockDim.x) {
        const int ii = (int)(t % bx), jj = (int)(t / bx);
        const int64_t p = (int64_t)(z.i0 - 1 + ii) + (int64_t)a.Nxg * (z.j0 - 1 + jj);
        const double gm = z.xdir ? z.gam[ii] : z.gam[jj];
        if (!z.wavegen) {
            E[p] = E[p] * gm;
            if (z.phion) P[p] = P[p] * gm;
        } else {
            double ea, pa;
            if (te2) { ea = 0.5 * (te[t] + te2[t]); pa = 0.5 * (tp[t] + tp2[t]); }
            else { ea = te[t]; pa = tp[t]; }
            E[p] = E[p] * gm + FAC * ea * (1.0 - gm);
            P[p] = P[p] * gm + FAC * pa * (1.0 - gm);
        }
    }
}

// Periodic x: the distinct column whose values image column i (1-based)
// carries -- 1 <- Nxg-2, Nxg-1 <- 2, Nxg <- 3 -- or i itself.
__device__ __forceinline__ int src_col(int i, int Nxg) {
    return i == 1 ? Nxg - 2 : (i == Nxg - 1 ? 2 : (i == Nxg ? 3 : i));
}

// Periodic x: image columns of a field with nz values per column copied
// from the distinct columns (zero = 1: set to zero instead).
__global__ void k_images(FsArgs a, double* v, int nz, int zero) {
    const int Nx = a.Nxg;
    const int64_t n = (int64_t)a.Nyg * 3 * nz;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % nz);
        const int64_t q = t / nz;
        const int w = (int)(q % 3), j = (int)(q / 3);
        const int i = w == 0 ? 1 : (w == 1 ? Nx - 1 : Nx);   // 1-based image column
        double* r = v + (int64_t)nz * Nx * j;
        r[(int64_t)nz * (i - 1) + k] = zero ? 0.0 : r[(int64_t)nz * (src_col(i, Nx) - 1) + k];
    }
}

// Ghost values so that the boundary one-sided d/dx equals S: zero for E, the
// current's flux Ul / Ur for P when src is set, else zero
// (UpdateGhostLayerX.f90:15-20); with periodic x, the image columns instead.
__global__ void k_ghost_x(FsArgs a, double* v1, double* v2, int src) {
    const int Nx = a.Nxg;
    if (a.per) {
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.Nyg; j += gridDim.x * blockDim.x) {
            double* r1 = v1 + (int64_t)Nx * j;
            double* r2 = v2 + (int64_t)Nx * j;
            r1[0] = r1[Nx - 3]; r1[Nx - 2] = r1[1]; r1[Nx - 1] = r1[2];
            r2[0] = r2[Nx - 3]; r2[Nx - 2] = r2[1]; r2[Nx - 1] = r2[2];
        }
        return;
    }
    for (int j = blockIdx.x * blockDim.x + threadIdx.x + 1; j <= a.Nyg; j += gridDim.x * blockDim.x) {
        if (a.three && (j == 1 || j == a.Nyg)) continue;
        double* vs[2] = {v1, v2};
        for (int q = 0; q < 2; ++q) {
            double* r = vs[q] + (int64_t)Nx * (j - 1);
            const double* s0 = a.SX + (int64_t)(2 - 1) * kHoRank;          // stencil of point i = 2
            const double* s1 = a.SX + (int64_t)(Nx - 1 - 1) * kHoRank;     // stencil of point i = Nx-1
            double sw = 0.0, se = 0.0;
            if (q == 1 && src) {
                sw = (src == 2 && a.Uw) ? a.Uw[j - 1] + a.Ul : a.Ul;
                se = a.Ur;
            } else if (q == 0 && src == 2 && a.Es) {
                sw = a.Es[j - 1];
            }
            double acc = 0;
            for (int m = 1; m < kHoRank; ++m) acc += s0[m] * r[m];
            r[0] = (sw - acc) / s0[0];
            acc = 0;
            for (int m = 0; m < kHoRank - 1; ++m) acc += s1[m] * r[Nx - kHoRank + m];
            r[Nx - 1] = (se - acc) / s1[kHoRank - 1];
        }
    }
}
__global__ void k_ghost_y(FsArgs a, double* v1, double* v2) {
    const int Nx = a.Nxg, Ny = a.Nyg;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x + 1; i <= Nx; i += gridDim.x * blockDim.x) {
        if (i == 1 || i == Nx) continue;
        double* vs[2] = {v1, v2};
        for (int q = 0; q < 2; ++q) {
            double* c = vs[q] + (i - 1);
            const double* s0 = a.SY + (int64_t)(2 - 1) * kHoRank;
            const double* s1 = a.SY + (int64_t)(Ny - 1 - 1) * kHoRank;
            double acc = 0;
            for (int m = 1; m < kHoRank; ++m) acc += s0[m] * c[(int64_t)Nx * m];
            c[0] = (0.0 - acc) / s0[0];
            acc = 0;
            for (int m = 0; m < kHoRank - 1; ++m) acc += s1[m] * c[(int64_t)Nx * (Ny - kHoRank + m)];
            c[(int64_t)Nx * (Ny - 1)] = (0.0 - acc) / s1[kHoRank - 1];
        }
    }
}

__device__ __forceinline__ int ws7(int i, int n) { return i <= 3 ? 1 : (i <= n - 3 ? i - 3 : n - 6); }

// Ex, Exx from E and Px from P at every point (including ghost rows).
__global__ void k_diff_x(FsArgs a, const double* E, const double* P, double* Ex, double* Exx, double* Px) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    const double* S1 = a.SX;
    const double* S2 = a.SX + (int64_t)a.Nxg * kHoRank;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(p % a.Nxg) + 1;
        const int64_t rb = p - (i - 1);
        double dx = 0, dxx = 0, px = 0;
        if (a.per) {
            // centred on the distinct column the point stands for, cyclic
            const int ic = src_col(i, a.Nxg);
            for (int m = 0; m < kHoRank; ++m) {
                const int64_t q = rb + wrap_x(ic - 3 + m, a.Nxg) - 1;
                dx += S1[(ic - 1) * kHoRank + m] * E[q];
                dxx += S2[(ic - 1) * kHoRank + m] * E[q];
                px += S1[(ic - 1) * kHoRank + m] * P[q];
            }
        } else {
            const int ws = ws7(i, a.Nxg);
            for (int m = 0; m < kHoRank; ++m) {
                const double e = E[rb + ws - 1 + m];
                dx += S1[(i - 1) * kHoRank + m] * e;
                dxx += S2[(i - 1) * kHoRank + m] * e;
                px += S1[(i - 1) * kHoRank + m] * P[rb + ws - 1 + m];
            }
        }
        Ex[p] = dx; Exx[p] = dxx; Px[p] = px;
    }
}
__global__ void k_diff_y(FsArgs a, const double* E, const double* P, double* Ey, double* Eyy, double* Py) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    const double* S1 = a.SY;
    const double* S2 = a.SY + (int64_t)a.Nyg * kHoRank;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(p % a.Nxg) + 1, j = (int)(p / a.Nxg) + 1;
        const int ws = ws7(j, a.Nyg);
        double dy = 0, dyy = 0, py = 0;
        for (int m = 0; m < kHoRank; ++m) {
            const int64_t q = (int64_t)(i - 1) + (int64_t)a.Nxg * (ws - 1 + m);
            dy += S1[(j - 1) * kHoRank + m] * E[q];
            dyy += S2[(j - 1) * kHoRank + m] * E[q];
            py += S1[(j - 1) * kHoRank + m] * P[q];
        }
        Ey[p] = dy; Eyy[p] = dyy; Py[p] = py;
    }
}

// W = (1/d) * dphi/dsigma at the free surface, d = eta + h (or h when linear).
__global__ void k_wvel(FsArgs a, const double* __restrict__ phi, const double* __restrict__ E, double* __restrict__ W) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    const int Nz = a.Nzg;
    const double* S = a.SZ + (int64_t)(Nz - 1) * kHoRank;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        const double* col = phi + p * Nz + (Nz - kHoRank);
        double acc = 0;
        for (int m = 0; m < kHoRank; ++m) acc += S[m] * col[m];
        const double d = (a.nonlinear ? E[p] : 0.0) + a.h[p];
        W[p] = (1.0 / d) * acc;
    }
}

// RHS free-surface row = P at the interior columns (Runge_Kutta_4.f90:106-107);
// the x-ghost columns' Neumann rows = the current's Ul (west) and Ur (east)
// at every level of the interior rows (:108-113), zero without a current.
__global__ void k_set_rhs(FsArgs a, const double* __restrict__ P, double* __restrict__ rhs) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(p % a.Nxg), j = (int)(p / a.Nxg);
        const bool yghost = a.three && (j == 0 || j == a.Nyg - 1);
        if (!a.per && !yghost && (i == 0 || i == a.Nxg - 1)) {
            if (i == 0 && a.Uw) {
                // Uneumann (zero in the bottom row, FAC u above) + the current
                rhs[p * a.Nzg] = 0.0 + a.Ul;
                const double u = a.Uw[j] + a.Ul;
                for (int k = 1; k < a.Nzg; ++k) rhs[p * a.Nzg + k] = u;
            } else {
                const double u = i == 0 ? a.Ul : a.Ur;
                for (int k = 0; k < a.Nzg; ++k) rhs[p * a.Nzg + k] = u;
            }
            continue;
        }
        const bool ghost = i == 0 || i == a.Nxg - 1 || yghost;
        if (ghost) continue;
        if (a.per && i == a.Nxg - 2) continue;   // the repeated column: identity rows, zero
        rhs[p * a.Nzg + a.Nzg - 1] = P[p];
    }
}

__global__ void k_extrap(double* __restrict__ phi, const double* __restrict__ lnew, const double* __restrict__ llast,
                         int64_t n, int stage3, const StepDev* sd) {
    if (stage3 && sd->tstep <= 1) return;   // Runge_Kutta_4.f90:294 (tstep > 1)
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        if (!stage3) phi[p] = 1.5 * lnew[p] - llast[p] * 0.5;
        else phi[p] = 2.66667 * phi[p] - 2.0 * lnew[p] + 0.333333 * llast[p];
    }
}

// Filtering happens on steps that are multiples of `every` (every <= 0:
// always); on the other steps the passes copy src to dst unchanged.
__device__ __forceinline__ bool filter_step(const StepDev* sd, int every) {
    return every <= 0 || (sd->tstep % every) == 0;
}

// FILTERING.f90 x pass over interior rows (reads src, writes dst).
__global__ void k_filter_x(FsArgs a, FilterDev f, const double* __restrict__ src, double* __restrict__ dst,
                           const StepDev* sd, int every) {
    const int Nx = a.Nxg, al = f.alpha, NP = 2 * f.alpha + 1;
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    if (!filter_step(sd, every)) {
        for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x)
            dst[p] = src[p];
        return;
    }
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(p % Nx) + 1, j = (int)(p / Nx) + 1;
        const double* row = src + (p - (i - 1));
        double v = src[p];
        const bool rowok = !a.three || (j >= 2 && j <= a.Nyg - 1);
        if (rowok && a.per) {
            // periodic x: the centred filter at the distinct column the point
            // stands for, cyclic
            const int ic = src_col(i, Nx);
            double acc = 0;
            for (int m = 1; m <= NP; ++m) acc += row[wrap_x(ic - al + m - 1, Nx) - 1] * f.fc[m - 1];
            v = acc;
        } else if (rowok && i >= 2 && i <= Nx - 1) {
            // the reference writes left block, centre, right block in that order
            if (i >= Nx - 1 - al + 1) {  // i = Nx-1-al+ib
                const int ib = i - (Nx - 1 - al);
                double acc = 0;
                for (int m = 1; m <= NP; ++m) acc += row[Nx - 1 - NP + m - 1] * f.F2[(al + 1 - ib - 1) * NP + (NP + 1 - m - 1)];
                v = acc;
            } else if (i - 1 <= al) {  // U(ib+1) = sum_m t(1+m) F2(m, ib), ib = i - 1
                const int ib = i - 1;
                double acc = 0;
                for (int m = 1; m <= NP; ++m) acc += row[1 + m - 1] * f.F2[(ib - 1) * NP + (m - 1)];
                v = acc;
            } else {
                double acc = 0;
                for (int m = 1; m <= NP; ++m) acc += row[i - al + m - 2] * f.fc[m - 1];
                v = acc;
            }
        }
        dst[p] = v;
    }
}
__global__ void k_filter_y(FsArgs a, FilterDev f, const double* __restrict__ src, double* __restrict__ dst,
                           const StepDev* sd, int every) {
    const int Nx = a.Nxg, Ny = a.Nyg, al = f.alpha, NP = 2 * f.alpha + 1;
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    if (!filter_step(sd, every)) {
        for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x)
            dst[p] = src[p];
        return;
    }
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(p % Nx) + 1, j = (int)(p / Nx) + 1;
        auto T = [&](int jj) { return src[(int64_t)(i - 1) + (int64_t)Nx * (jj - 1)]; };
        double v = src[p];
        if (i >= 2 && i <= Nx - 1 && j >= 2 && j <= Ny - 1) {
            if (j >= Ny - 1 - al + 1) {
                const int jb = j - (Ny - 1 - al);
                double acc = 0;
                for (int m = 1; m <= NP; ++m) acc += T(Ny - 1 - NP + m) * f.F2[(al + 1 - jb - 1) * NP + (NP + 1 - m - 1)];
                v = acc;
            } else if (j - 1 <= al) {
                const int jb = j - 1;
                double acc = 0;
                for (int m = 1; m <= NP; ++m) acc += T(1 + m) * f.F2[(jb - 1) * NP + (m - 1)];
                v = acc;
            } else {
                double acc = 0;
                for (int m = 1; m <= NP; ++m) acc += T(j - al + m - 1) * f.fc[m - 1];
                v = acc;
            }
        }
        dst[p] = v;
    }
}

// waveGenerationFromPaddleSignal.f90:43-111 at RK time t = (device time) +
// off: the signal levels itime and itime + 1 around t (1-based, itime =
// floor(t / dt) + 1; kept inside the table, where the reference would read
// past its end), their linear weights, the cubic ramp over the first `ramp`
// seconds, and per interior row the west wall's flux FAC u and eta_x.
__global__ void k_paddle(PaddleDev d, const StepDev* sd, double off) {
    const double t = sd->time + off;
    int it = (int)floor(t / d.dt) + 1;
    if (it < 1) it = 1;
    if (it > d.nt - 1) it = d.nt - 1;
    const double dl1 = t - (it - 1) * d.dt, dl2 = it * d.dt - t;
    const double w1 = dl2 / (dl1 + dl2), w2 = dl1 / (dl1 + dl2);
    double fac = 1.0;
    if (t < d.ramp) fac = -2.0 / (d.ramp * d.ramp * d.ramp) * (t * t * t) + 3.0 / (d.ramp * d.ramp) * (t * t);
    for (int j = d.j0 + (int)(blockIdx.x * blockDim.x + threadIdx.x); j <= d.j1; j += gridDim.x * blockDim.x) {
        const int64_t r0 = (int64_t)(it - 1) * d.Nyg + (j - 1), r1 = (int64_t)it * d.Nyg + (j - 1);
        const double flux = w1 * d.F[r0] + w2 * d.F[r1];
        const double etax = w1 * d.X[r0] + w2 * d.X[r1];
        d.Uw[j - 1] = fac * flux;
        d.Es[j - 1] = etax;
    }
}

__global__ void k_step_begin(StepDev* sd) {
    if (blockIdx.x == 0 && threadIdx.x == 0) sd->tstep += 1;
}
__global__ void k_step_end(StepDev* sd, double dt) {
    if (blockIdx.x == 0 && threadIdx.x == 0) sd->time = sd->time + dt;
}

// max |E| for the instability test; writes flag = 1 when max|E| > 10 max h.
__global__ void k_unstable(FsArgs a, const double* __restrict__ E, double hmax10, int* flag) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x)
        if (!(fabs(E[p]) <= hmax10)) atomicExch(flag, 1);
}

}  // namespace

void fs_stage(const FsArgs& a, const double* E, const double* P, const double* W, const double* Ex, const double* Px,
              const double* Ey, const double* Py, const double* E0, const double* P0, double c, double* kE,
              double* kP, double* tE, double* tP, const double* NuD, const double* Pd, const double* Qr_x,
              cudaStream_t st) {
    int64_t C = (int64_t)a.Nxg * a.Nyg;
    note_launch(), k_fs_stage<<<nb(C), 256, 0, st>>>(a, E, P, W, Ex, Px, Ey, Py, E0, P0, c, kE, kP, tE, tP, NuD, Pd,
                                                     Qr_x);
}
void fs_pdamp(const FsArgs& a, const PDampDev& d, const double* E, const double* P, cudaStream_t st) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    if (d.type != 0) {
        note_launch(), k_pd_friction<<<nb(C), 256, 0, st>>>(d, C, E, P);
        return;
    }
    note_launch(), k_pd_rhs<<<1, 256, 0, st>>>(d, a.Nxg, E, P);
    const int blocks = (int)((d.nd + 7) / 8 < 148 * 4 ? (d.nd + 7) / 8 : 148 * 4);   // 8 rows (warps) a block
    note_launch(), k_pd_solve<<<blocks, 256, 0, st>>>(d);
    note_launch(), k_pd_apply<<<nb(d.nd), 256, 0, st>>>(d);
}
void fs_rk_final(const FsArgs& a, double* E, double* P, double* const* kE, double* const* kP, double dt,
                 cudaStream_t st) {
    int64_t C = (int64_t)a.Nxg * a.Nyg;
    note_launch(), k_rk_final<<<nb(C), 256, 0, st>>>(a, E, P, kE[0], kE[1], kE[2], kE[3], kP[0], kP[1], kP[2], kP[3], dt);
}
void fs_relax(const FsArgs& a, const RelaxZoneDev* zones, int nz, double* E, double* P, const StepDev* sd, double off,
              double transient, cudaStream_t st) {
    for (int z = 0; z < nz; ++z) {
        int64_t box = (int64_t)(zones[z].i1 - zones[z].i0 + 1) * (zones[z].j1 - zones[z].j0 + 1);
        note_launch(), k_relax<<<nb(box), 256, 0, st>>>(a, zones[z], E, P, sd, off, transient);
    }
}
void fs_step_begin(StepDev* sd, cudaStream_t st) { note_launch(), k_step_begin<<<1, 32, 0, st>>>(sd); }
void fs_step_end(StepDev* sd, double dt, cudaStream_t st) { note_launch(), k_step_end<<<1, 32, 0, st>>>(sd, dt); }
void fs_paddle(const PaddleDev& d, const StepDev* sd, double off, cudaStream_t st) {
    note_launch(), k_paddle<<<nb(d.j1 - d.j0 + 1, 128), 128, 0, st>>>(d, sd, off);
}
void fs_derivs(const FsArgs& a, double* E, double* P, double* Ex, double* Exx, double* Px, double* Ey, double* Eyy,
               double* Py, int src, cudaStream_t st) {
    int64_t C = (int64_t)a.Nxg * a.Nyg;
    note_launch(), k_ghost_x<<<nb(a.Nyg, 128), 128, 0, st>>>(a, E, P, src);
    note_launch(), k_diff_x<<<nb(C), 256, 0, st>>>(a, E, P, Ex, Exx, Px);
    if (a.three) {
        note_launch(), k_ghost_y<<<nb(a.Nxg, 128), 128, 0, st>>>(a, E, P);
        note_launch(), k_diff_y<<<nb(C), 256, 0, st>>>(a, E, P, Ey, Eyy, Py);
    }
}
void fs_wvel(const FsArgs& a, const double* phi, const double* E, double* W, cudaStream_t st) {
    int64_t C = (int64_t)a.Nxg * a.Nyg;
    note_launch(), k_wvel<<<nb(C), 256, 0, st>>>(a, phi, E, W);
    if (a.per) fs_images(a, W, 1, 0, st);
}
void fs_images(const FsArgs& a, double* v, int nz, int zero, cudaStream_t st) {
    const int64_t n = (int64_t)a.Nyg * 3 * nz;
    note_launch(), k_images<<<nb(n), 256, 0, st>>>(a, v, nz, zero);
}
void fs_set_rhs(const FsArgs& a, const double* P, double* rhs, cudaStream_t st) {
    int64_t C = (int64_t)a.Nxg * a.Nyg;
    note_launch(), k_set_rhs<<<nb(C), 256, 0, st>>>(a, P, rhs);
}
void fs_extrap(double* phi, const double* lnew, const double* llast, int64_t n, int stage3, const StepDev* sd,
               cudaStream_t st) {
    note_launch(), k_extrap<<<nb(n), 256, 0, st>>>(phi, lnew, llast, n, stage3, sd);
}
void fs_filter(const FsArgs& a, const FilterDev& f, double* U, double* tmp, const StepDev* sd, int every,
               cudaStream_t st) {
    int64_t C = (int64_t)a.Nxg * a.Nyg;
    note_launch(), k_filter_x<<<nb(C), 256, 0, st>>>(a, f, U, tmp, sd, every);
    if (a.three) note_launch(), k_filter_y<<<nb(C), 256, 0, st>>>(a, f, tmp, U, sd, every);
    else cudaMemcpyAsync(U, tmp, sizeof(double) * C, cudaMemcpyDeviceToDevice, st);
}
void fs_unstable(const FsArgs& a, const double* E, double hmax10, int* flag, cudaStream_t st) {
    int64_t C = (int64_t)a.Nxg * a.Nyg;
    note_launch(), k_unstable<<<nb(C), 256, 0, st>>>(a, E, hmax10, flag);
}

}  // namespace ow3d
