// The roller breaking model of x flumes (DetectBreaking.f90:72-211), on the
// device.
//
// Rollers are searched from the right end of the flume: a toe lies between
// columns j-1 and j (1-based, ghosts included, nfx = Nxg) where the surface
// slope, eta_x at j+1/2 by forward differences, crosses -tan(phi(j)) and no
// roller found so far covers column j. The toe's sub-grid position xr and
// elevation sr come from the local quadratic; the roller extends back from
// the column ahead of the toe while the surface stays above the tangent line
// from the toe, with thickness del_fac times that height (capped at
// eta - sr). Qr_x, the 1-2-1 smoothed g * thickness, is subtracted from the
// kinematic condition when i_breaking is 1 (rhsFreeSurface3D.f90:17). The
// call after a step (update) also relaxes the roller angle: tan(phi) is
// tan(phi_b) everywhere except from three columns ahead of each toe to the
// back of its roller, where it moves by dt / T_half of the way from the
// toe's previous value toward tan(phi_0) (DetectBreaking.f90:175-186), and it
// records the rollers as the reference writes them to roller.dat (:205-211).
//
// The search is sequential (a toe is skipped where an earlier roller already
// lies), so it runs in one warp: 32 candidate toes are tested at a time and
// the toes of a chunk taken in order; each roller's extent is found 32
// columns at a time. The per-column passes (slopes, Qr_x, the angle reset)
// use the whole block. A flume has a few thousand columns at most, so one
// block covers it; the kernel costs a few microseconds per call.
#include "ow3d_fs.h"

namespace ow3d {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__global__ void __launch_bounds__(256) k_breaking(BreakDev b, const double* __restrict__ E, int update) {
    const int nfx = b.nfx;
    const int tid = threadIdx.x, nth = blockDim.x;
    // 1-based column j is E[j - 1]; thick and eta_x are indexed 1-based
    for (int j = tid; j <= nfx; j += nth) {
        b.thick[j] = 0.0;
        b.eta_x[j] = (j >= 2 && j <= nfx - 2) ? b.dx_inv * (E[j] - E[j - 1]) : 0.0;
        if (j < nfx) {
            b.Qr_x[j] = 0.0;
            b.tan_old[j] = b.tan_phi[j];
        }
    }
    __syncthreads();
    __shared__ int s_n;
    if (tid < 32) {
        const int lane = tid;
        int n = 0;
        for (int base = nfx - 2; base >= 3; base -= 32) {
            const int j = base - lane;
            bool cand = false;
            if (j >= 3) {
                const double t = b.tan_phi[j - 1];
                cand = b.eta_x[j - 1] < -t && b.eta_x[j] >= -t;
            }
            unsigned m = __ballot_sync(kFull, cand);
            while (m) {
                const int jj = base - (__ffs(m) - 1);
                m &= m - 1;
                __syncwarp();   // thickness written by the previous roller
                if (!(b.thick[jj] <= 0.0)) continue;
                const double tphib = b.tan_phi[jj - 1];
                const double ea = b.eta_x[jj - 1], eb = b.eta_x[jj];
                const double a = 0.5 * b.dx_inv * (eb - ea);
                const double bb = 0.5 * (eb + ea);
                const double c = E[jj - 1];
                const double dxr = -(tphib + bb) / (2.0 * a);
                const double xr = (double)(jj - 1) * b.dx + dxr;
                const int jr = (int)(xr * b.dx_inv) + 2;
                const double sr = a * dxr * dxr + bb * dxr + c;
                int cnt = 0;
                for (int i0 = jr - 1; i0 >= 3; i0 -= 32) {
                    const int i = i0 - lane;
                    double d = 0.0;
                    bool stop = true;
                    if (i >= 3) {
                        const double ei = E[i - 1];
                        d = b.del_fac * (ei - (sr + tphib * (xr - (double)(i - 1) * b.dx)));
                        stop = d < 0.0;
                        if (d > ei - sr) d = ei - sr;
                    }
                    const unsigned sm = __ballot_sync(kFull, stop);
                    const int first = sm ? __ffs(sm) - 1 : 32;
                    if (lane < first) b.thick[i] = d;
                    cnt += first;
                    if (first < 32) break;
                }
                if (lane == 0 && n < b.cap) {
                    b.npts[n] = cnt;
                    b.toe[n] = jr;
                    b.xr[n] = xr;
                    b.sr[n] = sr;
                }
                ++n;
            }
        }
        if (lane == 0) s_n = n;
    }
    __syncthreads();
    const int n = s_n < b.cap ? s_n : b.cap;
    if (update) {
        for (int j = tid; j < nfx; j += nth) b.tan_phi[j] = b.tan_b;
        __syncthreads();
        if (tid < 32) {
            // rollers in the order found: where two overlap, the later one's value stands
            for (int r = 0; r < n; ++r) {
                const int toe = b.toe[r];
                const double tphib = b.tan_old[toe - 1];
                const double v = tphib + b.dt / b.T_half * (b.tan_0 - tphib);
                for (int i = 1 + tid; i <= b.npts[r] + 3; i += 32) {
                    const int idx = toe + 4 - i;
                    if (idx >= 1 && idx <= nfx) b.tan_phi[idx - 1] = v;
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (int r = tid; r < n; r += nth) {
            b.r_thick[r] = b.thick[b.toe[r] - 1];
            b.r_tan[r] = b.tan_phi[b.toe[r] - 1];
        }
        if (tid == 0) *b.n_rollers = s_n;
    }
    if (s_n > 0 && b.dynamics) {
        const double g = b.g;
        for (int j = 3 + tid; j <= nfx - 2; j += nth)
            b.Qr_x[j - 1] = 0.25 * (g * b.thick[j + 1]) + 0.5 * (g * b.thick[j]) + 0.25 * (g * b.thick[j - 1]);
    }
}

}  // namespace

void fs_breaking(const BreakDev& b, const double* E, int update, cudaStream_t st) {
    note_launch(), k_breaking<<<1, 256, 0, st>>>(b, E, update);
}

}  // namespace ow3d
