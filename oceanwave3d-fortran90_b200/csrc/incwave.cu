// The incident wave of a generation zone, synthesised on the device.
//
// The reference builds it on the host before the time loop
// (OceanWave3DT0Setup.f90:176-255): the mono-chromatic wave in closed form
// (random_wave_signal.f90:151-172), and random waves as an inverse real
// Fourier transform of seeded complex amplitudes moved to each point by the
// dispersion relation (random_wave_signal.f90:48-150, random_wave_signal_3D.f90
// for waves at a heading and spread seas). The amplitudes, wavenumbers and
// headings come from the sequential generator and are set up on the host
// (incident_wave_setup in setup.cpp, a few thousand numbers); the series
// itself -- every sample at every point of the zone, the bulk of the work --
// is formed here and stays on the device as the zone's relaxation target.
//
// Random waves: at point p and sample n,
//   eta_n(p) = sum_{k=1}^{kmax-1} Re(A_k(p) W^(k n)),   W = e^(-2 pi i / N),
// with A_k(p) = c_k e^(i nu_k d_k(p)), and the surface potential likewise
// with B_k(p) = (g / omega_k) (Im A_k, -Re A_k). This is the transform the
// host evaluates with an FFT over the N samples, summed here directly (the
// results agree to rounding) from a table of the N twiddle factors.
#include "ow3d_internal.h"

namespace ow3d {

namespace {

// A_k(p), B_k(p) for every evaluation point p (i fastest, then j) and mode k.
__global__ void k_incwave_modes(const double2* __restrict__ c, const double* __restrict__ nus,
                                const double* __restrict__ kcos, const double* __restrict__ ksin, int kmax,
                                double cosb, double sinb, const double* __restrict__ dx,
                                const double* __restrict__ dy, int bx, int npts, double g, double domega,
                                double2* __restrict__ A, double2* __restrict__ B) {
    const int64_t total = (int64_t)npts * kmax;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % kmax);
        const int p = (int)(t / kmax);
        const int i = p % bx, j = p / bx;
        double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
        if (k >= 1) {
            const double dist = kcos ? kcos[k] * dx[i] + ksin[k] * dy[j] : cosb * dx[i] + sinb * dy[j];
            double sn, cs;
            sincos(nus[k] * dist, &sn, &cs);
            const double2 ck = c[k];
            a = make_double2(ck.x * cs - ck.y * sn, ck.x * sn + ck.y * cs);
            const double f = g / (k * domega);
            b = make_double2(f * a.y, -f * a.x);
        }
        A[t] = a;
        B[t] = b;
    }
}

// eta and the surface potential at sample n of evaluation point p, written to
// every row the point stands for (all rows for a long-crested wave).
__global__ void k_incwave_sum(const double2* __restrict__ A, const double2* __restrict__ B,
                              const double2* __restrict__ W, int N, int kmax, int nt, int bx, int by, int npts,
                              int heading, double* __restrict__ eta, double* __restrict__ phis) {
    const int64_t total = (int64_t)nt * npts;
    const int64_t box = (int64_t)bx * by;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(t % npts);
        const int n = (int)(t / npts);
        const double2* a = A + (int64_t)p * kmax;
        const double2* b = B + (int64_t)p * kmax;
        double e = 0.0, f = 0.0;
        int idx = 0;
        for (int k = 1; k < kmax; ++k) {
            idx += n;
            if (idx >= N) idx -= N;   // (k n) mod N, n < N
            const double2 w = __ldg(W + idx);
            const double2 ak = a[k], bk = b[k];
            e += ak.x * w.x - ak.y * w.y;
            f += bk.x * w.x - bk.y * w.y;
        }
        const int i = p % bx, j = p / bx;
        if (heading) {
            eta[(int64_t)n * box + (int64_t)j * bx + i] = e;
            phis[(int64_t)n * box + (int64_t)j * bx + i] = f;
        } else {
            for (int jj = 0; jj < by; ++jj) {
                eta[(int64_t)n * box + (int64_t)jj * bx + i] = e;
                phis[(int64_t)n * box + (int64_t)jj * bx + i] = f;
            }
        }
    }
}

// The mono-chromatic wave: amp cos(nu d - omega t), (g / omega) amp sin(...).
__global__ void k_incwave_mono(double amp, double nu, double omega, double phifact, double t0, double dt, double cosb,
                               double sinb, const double* __restrict__ dx, const double* __restrict__ dy, int bx,
                               int by, int nt, double* __restrict__ eta, double* __restrict__ phis) {
    const int64_t box = (int64_t)bx * by;
    const int64_t total = (int64_t)nt * box;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = t % box;
        const int n = (int)(t / box);
        const int i = (int)(q % bx), j = (int)(q / bx);
        const double dist = cosb * dx[i] + sinb * dy[j];
        const double arg = nu * dist - omega * (t0 + n * dt);
        eta[t] = amp * cos(arg);
        phis[t] = phifact * amp * sin(arg);
    }
}

inline int blocks_for(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

int launch_incident_wave(const IncidentWaveDev& w, double* eta, double* phis, cudaStream_t st) {
    const int npts = w.bx * w.ny_eval;
    if (w.mono) {
        // dy holds one value per row for waves at a heading, else zeros
        note_launch(), k_incwave_mono<<<blocks_for((int64_t)w.nt * w.bx * w.by), 256, 0, st>>>(
            w.amp, w.nu, w.omega, w.phifact, w.t0, w.dt, w.cosb, w.sinb, w.dx, w.dy_rows, w.bx, w.by, w.nt, eta, phis);
    } else {
        note_launch(), k_incwave_modes<<<blocks_for((int64_t)npts * w.kmax), 256, 0, st>>>(
            w.c, w.nus, w.kcos, w.ksin, w.kmax, w.cosb, w.sinb, w.dx, w.dy, w.bx, npts, w.g, w.domega, w.A, w.B);
        note_launch(), k_incwave_sum<<<blocks_for((int64_t)w.nt * npts), 256, 0, st>>>(
            w.A, w.B, w.W, w.N, w.kmax, w.nt, w.bx, w.by, npts, w.heading, eta, phis);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? OW3D_OK : OW3D_ERR_CUDA;
}

}  // namespace ow3d
