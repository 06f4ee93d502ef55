// Local smoothing by the vertical acceleration of the surface
// (LocalSmoothing2D.f90:37-145 for x flumes, LocalSmoothing3D.f90 for 3-D
// grids), run after each step as OceanWave3DTakeATimeStep.f90:33-39 calls it.
//
// From the third step on, the Lagrangian vertical acceleration of the
// surface particles,
//   dw/dt = (3 W^n - 4 W^(n-1) + W^(n-2)) / (2 dt) - w_z eta_t
//           + u w_x (+ v w_y) + w w_z,
// is formed at every surface point from the step's last solution: w = phi_s
// / d, u = phi_x + sigma_x w, w_z = (w)_s / d, w_x = (w)_x + sigma_x w_z
// (sigma_x = ((1 - sigma) h_x - sigma eta_x) / d at the surface, the
// reference's chain rule over the whole grid evaluated here only where it is
// used), eta_t = (k1 + 2 k2 + 2 k3 + k4) / 6 of the step. As in the
// reference, the 3-D v is the x derivative of phi plus sigma_y w (its
// DiffXEven call with the y half-width). Where -dw/dt >= accel_tol_fact g at
// a point i = 6..Nxg-5 of a row, the points i-5..i+5 of the row take the
// weight 1/4; if any point did, eta and the surface potential of every row
// are filtered with [a, 1 - 2a, a] over i = 2..Nxg-1.
//
// k_accel: one thread per surface point (7 sigma derivatives of its column,
// 7 + 7 of the neighbour columns at the surface); it also files W in the
// three-step history ring. k_smooth_apply: the weights from the flags of the
// row (a window of 11 points) and the filter into scratch fields, which a
// device copy returns to eta and phi.
#include "ow3d_fs.h"

namespace ow3d {

namespace {

inline int nb(int64_t n, int t = 256) {
    int64_t b = (n + t - 1) / t;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

__device__ __forceinline__ int win7(int i, int n) { return i <= 3 ? 1 : (i <= n - 3 ? i - 3 : n - 6); }

// d/dsigma of the column at row k (1-based), DiffZArbitrary.f90's window
__device__ __forceinline__ double dsig_row(const double* __restrict__ SZ, const double* col, int k, int Nz) {
    const int ws = win7(k, Nz);
    const double* S = SZ + (int64_t)(k - 1) * kHoRank;
    double acc = 0;
    for (int m = 0; m < kHoRank; ++m) acc += S[m] * col[ws - 1 + m];
    return acc;
}

__global__ void k_accel(FsArgs a, SmoothDev s, const double* __restrict__ phi, const double* __restrict__ E,
                        const double* __restrict__ Ex, const double* __restrict__ Ey, const double* __restrict__ W,
                        const double* __restrict__ k1, const double* __restrict__ k2, const double* __restrict__ k3,
                        const double* __restrict__ k4, const StepDev* sd) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    const int Nz = a.Nzg;
    const long long t = sd->tstep;
    double* const slot = s.WH[t % 3];
    const double* const W1 = s.WH[(t + 2) % 3];   // W after step t - 1
    const double* const W2 = s.WH[(t + 1) % 3];   // W after step t - 2
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        const double w0 = W[p];
        int flag = 0;
        if (t >= 3) {
            const int i = (int)(p % a.Nxg) + 1, j = (int)(p / a.Nxg) + 1;
            const double d = a.h[p] + E[p];
            const double* col = phi + p * Nz;
            // w = phi_s / d on the seven rows of the surface window
            double wr[kHoRank];
            for (int r = 0; r < kHoRank; ++r) wr[r] = dsig_row(a.SZ, col, Nz - kHoRank + 1 + r, Nz) / d;
            const double* Ss = a.SZ + (int64_t)(Nz - 1) * kHoRank;
            double wz = 0;
            for (int m = 0; m < kHoRank; ++m) wz += Ss[m] * wr[m];
            wz = wz / d;
            const double zs = s.z[Nz - 1];
            // x derivatives at the surface: phi_x and (phi_s / d)_x
            const int ws = win7(i, a.Nxg);
            const double* Sx = a.SX + (int64_t)(i - 1) * kHoRank;
            const int64_t rb = p - (i - 1);
            double ux = 0, wx = 0;
            for (int m = 0; m < kHoRank; ++m) {
                const int64_t q = rb + ws - 1 + m;
                const double* cq = phi + q * Nz;
                ux += Sx[m] * cq[Nz - 1];
                wx += Sx[m] * (dsig_row(a.SZ, cq, Nz, Nz) / (a.h[q] + E[q]));
            }
            const double sx = (1.0 - zs) * s.hx[p] - zs * Ex[p];
            const double u = ux + sx * wr[kHoRank - 1];
            wx = wx + sx * wz;
            const double etat = 1.0 / 6.0 * (k1[p] + 2.0 * k2[p] + 2.0 * k3[p] + k4[p]);
            double wt = 0.5 * s.dt_inv * (3.0 * w0 - 4.0 * W1[p] + W2[p]) - wz * etat;
            if (a.three) {
                const int wsy = win7(j, a.Nyg);
                const double* Sy = a.SY + (int64_t)(j - 1) * kHoRank;
                double wy = 0;
                for (int m = 0; m < kHoRank; ++m) {
                    const int64_t q = (int64_t)(wsy - 1 + m) * a.Nxg + (i - 1);
                    wy += Sy[m] * (dsig_row(a.SZ, phi + q * Nz, Nz, Nz) / (a.h[q] + E[q]));
                }
                const double sy = (1.0 - zs) * s.hy[p] - zs * Ey[p];
                const double v = ux + sy * wr[kHoRank - 1];
                wy = wy + sy * wz;
                wt = wt + u * wx + v * wy + wr[kHoRank - 1] * wz;
            } else {
                wt = wt + u * wx + wr[kHoRank - 1] * wz;
            }
            s.Wt[p] = wt;
            if (i >= 6 && i <= a.Nxg - 5 && -wt >= s.tol) {
                flag = 1;
                atomicOr(s.any, 1);
            }
        }
        s.flag[p] = flag;
        slot[p] = w0;   // the slot of step t - 3, read by no point of this step
    }
}

__global__ void k_smooth_apply(FsArgs a, SmoothDev s, const double* __restrict__ E, const double* __restrict__ P) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    const bool on = *s.any != 0;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < C; p += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(p % a.Nxg) + 1;
        double e = E[p], f = P[p];
        if (on && i >= 2 && i <= a.Nxg - 1) {
            double al = 0.0;
            const int lo = i - 5 < 6 ? 6 : i - 5, hi = i + 5 > a.Nxg - 5 ? a.Nxg - 5 : i + 5;
            for (int q = lo; q <= hi; ++q)
                if (s.flag[p + (q - i)]) { al = 0.25; break; }
            e = al * E[p - 1] + (1.0 - 2.0 * al) * E[p] + al * E[p + 1];
            f = al * P[p - 1] + (1.0 - 2.0 * al) * P[p] + al * P[p + 1];
        }
        s.sE[p] = e;
        s.sP[p] = f;
    }
}

}  // namespace

int fs_local_smoothing(const FsArgs& a, const SmoothDev& s, const double* phi, double* E, double* P,
                       const double* Ex, const double* Ey, const double* W, double* const* kE, const StepDev* sd,
                       cudaStream_t st) {
    const int64_t C = (int64_t)a.Nxg * a.Nyg;
    if (cudaMemsetAsync(s.any, 0, sizeof(int), st) != cudaSuccess) return OW3D_ERR_CUDA;
    note_launch(), k_accel<<<nb(C), 256, 0, st>>>(a, s, phi, E, Ex, Ey, W, kE[0], kE[1], kE[2], kE[3], sd);
    note_launch(), k_smooth_apply<<<nb(C), 256, 0, st>>>(a, s, E, P);
    if (cudaMemcpyAsync(E, s.sE, sizeof(double) * (size_t)C, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(P, s.sP, sizeof(double) * (size_t)C, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return OW3D_ERR_CUDA;
    return OW3D_OK;
}

}  // namespace ow3d
