// Fluid kinematics of the current state on the whole grid, ghost points
// included (src/IO/StoreKinematicData.f90:256-460): the velocities
//   u = phi_x + s_x phi_s,  v = phi_y + s_y phi_s,  w = phi_s / d
// and the nine gradient fields the reference writes beside them. phi_s is
// the sigma derivative (DiffZArbitrary, order 1), phi_x and phi_y the 7-point
// x and y derivatives (DiffXEven, DiffYEven) with the per-position stencils
// of the operator, d = h + eta, and s_x = ((1 - z) h_x - z eta_x) / d with the
// sigma levels z including the ghost level z(1) = -z(3); the s_x, s_y terms
// are added only when LinearONOFF is nonzero. Two point-wise passes: the
// first writes u, v, phi_s and w, the second differentiates phi_s, u and v.
// This is an output path (called at output times), memory-bound and launched
// on the handle's stream.
#include "ow3d_internal.h"

#define OW3D_GRID_STRIDE(var, n) \
    for (int64_t var = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; var < (n); var += (int64_t)gridDim.x * blockDim.x)

namespace ow3d {
namespace {

// 1-based start of the 7-point window at position i of n (DiffXEven.f90:16-38,
// DiffZArbitrary.f90:15-34).
__device__ __forceinline__ int win7(int i, int n) { return i <= 3 ? 1 : (i <= n - 3 ? i - 3 : n - 6); }

struct Point {
    int k, i, j;
    int64_t col;           // offset of (1, i, j)
    double d, sx, sy, z;
};

__device__ __forceinline__ Point point_of(const KinArgs& a, int64_t p) {
    Point q;
    const int64_t c = p / a.Nzg;
    q.k = (int)(p - c * a.Nzg) + 1;
    const int64_t jj = c / a.Nxg;
    q.i = (int)(c - jj * a.Nxg) + 1;
    q.j = (int)jj + 1;
    q.col = c * a.Nzg;
    q.d = a.h[c] + a.E[c];
    q.z = a.z[q.k - 1];
    // ((1-z)/d*hx - z/d*etax) as StoreKinematicData.f90:281 evaluates it
    q.sx = a.chain ? (1.0 - q.z) / q.d * a.hx[c] - q.z / q.d * a.Ex[c] : 0.0;
    q.sy = a.chain && a.doy ? (1.0 - q.z) / q.d * a.hy[c] - q.z / q.d * a.Ey[c] : 0.0;
    return q;
}

__device__ __forceinline__ double dz(const KinArgs& a, const Point& q, const double* F) {
    const double* w = a.SZ + (size_t)(q.k - 1) * 7;
    const double* f = F + q.col + (win7(q.k, a.Nzg) - 1);
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < 7; ++m) s += w[m] * f[m];
    return s;
}
__device__ __forceinline__ double dx(const KinArgs& a, const Point& q, const double* F) {
    const double* w = a.SX + (size_t)(q.i - 1) * 7;
    const double* f = F + q.col + (int64_t)(win7(q.i, a.Nxg) - q.i) * a.Nzg + (q.k - 1);
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < 7; ++m) s += w[m] * f[(int64_t)m * a.Nzg];
    return s;
}
__device__ __forceinline__ double dy(const KinArgs& a, const Point& q, const double* F) {
    const double* w = a.SY + (size_t)(q.j - 1) * 7;
    const int64_t oy = (int64_t)a.Nzg * a.Nxg;
    const double* f = F + q.col + (int64_t)(win7(q.j, a.Nyg) - q.j) * oy + (q.k - 1);
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < 7; ++m) s += w[m] * f[(int64_t)m * oy];
    return s;
}

// u, v, phi_s, w (StoreKinematicData.f90:256-300)
__global__ void k_kin_velocity(KinArgs a, const double* __restrict__ phi, double* __restrict__ u,
                               double* __restrict__ v, double* __restrict__ ps, double* __restrict__ w) {
    OW3D_GRID_STRIDE(p, a.N) {
        const Point q = point_of(a, p);
        const double s = dz(a, q, phi);
        u[p] = a.dox ? dx(a, q, phi) + q.sx * s : 0.0;
        v[p] = a.doy ? dy(a, q, phi) + q.sy * s : 0.0;
        ps[p] = s;
        w[p] = s / q.d;
    }
}

// D_s F / d, D_x F + s_x D_s F, D_y F + s_y D_s F (StoreKinematicData.f90:330-460)
__global__ void k_kin_gradient(KinArgs a, const double* __restrict__ F, double* __restrict__ gz,
                               double* __restrict__ gx, double* __restrict__ gy) {
    OW3D_GRID_STRIDE(p, a.N) {
        const Point q = point_of(a, p);
        const double s = dz(a, q, F);
        gz[p] = s / q.d;
        gx[p] = a.dox ? dx(a, q, F) + q.sx * s : 0.0;
        gy[p] = a.doy ? dy(a, q, F) + q.sy * s : 0.0;
    }
}

int blocks_for(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

void launch_kinematics(const KinArgs& a, const double* phi, double* out, cudaStream_t st) {
    const int64_t N = a.N;
    double* f[13];
    for (int q = 0; q < 13; ++q) f[q] = out + (int64_t)q * N;
    const int nb = blocks_for(N);
    note_launch(), k_kin_velocity<<<nb, 256, 0, st>>>(a, phi, f[0], f[1], f[2], f[3]);
    // phi_s, u, v in the reference's order: d/ds, d/dx, d/dy of each
    note_launch(), k_kin_gradient<<<nb, 256, 0, st>>>(a, f[2], f[4], f[5], f[6]);
    note_launch(), k_kin_gradient<<<nb, 256, 0, st>>>(a, f[0], f[7], f[8], f[9]);
    note_launch(), k_kin_gradient<<<nb, 256, 0, st>>>(a, f[1], f[10], f[11], f[12]);
}

}  // namespace ow3d
