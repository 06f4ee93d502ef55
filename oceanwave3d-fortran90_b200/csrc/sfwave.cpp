// The stream-function (Fourier) solution of a steady periodic wave on
// constant depth, the incident wave of IncWaveType 1. It is Fenton's method
// in the form the reference uses (src/utilities/stream_func_set_up.f90:1-59,
// stream_func_coeffs.f:1-153, init.f:1-72, eqns.f:1-74): 2N+10 unknowns
// (kd, kH, T sqrt(gk), c sqrt(k/g), the two mean currents, the mean fluid
// speed, the volume flux, the Bernoulli constant, k eta at the N+1
// collocation points over half a wavelength and the N stream-function
// coefficients), Newton's method with a forward-difference Jacobian
// (step 1% of the unknown, 1e-5 near zero), the height reached in nsteps
// steps with the solution extrapolated from the last two, convergence when
// the summed correction is below 1e-6 (1e-8 on the last step). The surface
// elevation and potential at (x, t) follow stream_func_wave_finite
// (stream_func_wave_finite.f:3-71).
#include <cmath>
#include <string>
#include <vector>

#include "setup.h"

namespace ow3d {
namespace {

struct SFProblem {
    int n = 0, num = 0;
    bool finite = true, period = false, euler = true;
    double hoverd = 0, height = 0, value = 0, pi = 0;
    std::vector<double> cosa, sina, coeff;   // cosa, sina: 0..2N; coeff: 1..N
};

// init.f: the linear solution as the first guess; z is 1-based (z[0] unused)
void sf_init(SFProblem& P, std::vector<double>& z, std::vector<double>& s1, std::vector<double>& s2) {
    const int n = P.n, num = P.num;
    const double pi = P.pi;
    if (P.finite) {
        if (P.period) {
            const double A = 4.0 * pi * pi * P.height / P.hoverd;
            const double B = A / std::sqrt(std::tanh(A));
            const double T = std::tanh(B);
            z[1] = B + (A - B * T) / (T + B * (1.0 - T * T));
        } else {
            z[1] = 2.0 * pi * P.height / P.hoverd;
        }
        z[2] = z[1] * P.hoverd;
        z[4] = std::sqrt(std::tanh(z[1]));
    } else {
        z[1] = -1.0;
        z[4] = 1.0;
        z[2] = P.period ? 4.0 * pi * pi * P.height : 2.0 * pi * P.height;
    }
    z[3] = 2.0 * pi / z[4];
    if (P.euler) { z[5] = P.value * std::sqrt(z[2]); z[6] = 0.0; }
    else { z[5] = 0.0; z[6] = P.value * std::sqrt(z[2]); }
    z[7] = z[4];
    z[8] = 0.0;
    z[9] = 0.5 * z[7] * z[7];
    z[10] = 0.5 * z[2];
    P.cosa[0] = 1.0;
    P.sina[0] = 0.0;
    for (int i = 1; i <= n; ++i) {
        P.cosa[i] = std::cos(i * pi / n);
        P.cosa[i + n] = std::cos((i + n) * pi / n);
        P.sina[i] = std::sin(i * pi / n);
        P.sina[i + n] = std::sin((i + n) * pi / n);
        z[n + i + 10] = 0.0;
        z[i + 10] = 0.5 * z[2] * P.cosa[i];
    }
    z[n + 11] = 0.5 * z[2] / z[7];
    for (int i = 1; i <= 9; ++i) s1[i] = z[i];
    for (int i = 10; i <= num; ++i) s1[i] = 0.0;
    for (int i = 1; i <= num; ++i) s2[i] = 0.0;
}

// eqns.f: the residuals of the 2N+10 equations
void sf_eqns(SFProblem& P, const std::vector<double>& z, std::vector<double>& rhs) {
    const int n = P.n;
    rhs[1] = P.finite ? z[2] - z[1] * P.hoverd : z[1] + 1.0;
    rhs[2] = P.period ? z[2] - P.height * z[3] * z[3] : z[2] - 2.0 * P.pi * P.height;
    rhs[3] = z[4] * z[3] - P.pi - P.pi;
    rhs[4] = z[5] + z[7] - z[4];
    rhs[5] = z[6] + z[7] - z[4];
    if (P.finite) {
        rhs[5] = rhs[5] - z[8] / z[1];
        for (int i = 1; i <= n; ++i) P.coeff[i] = z[n + i + 10] / std::cosh(i * z[1]);
    }
    const int it = P.euler ? 5 : 6;
    rhs[6] = z[it] - P.value * std::sqrt(z[2]);
    rhs[7] = z[10] + z[n + 10];
    for (int i = 1; i <= n - 1; ++i) rhs[7] = rhs[7] + z[10 + i] + z[10 + i];
    rhs[8] = z[10] - z[n + 10] - z[2];
    for (int m = 0; m <= n; ++m) {
        double psi = 0.0, u = 0.0, v = 0.0;
        if (P.finite) {
            for (int j = 1; j <= n; ++j) {
                const int nm = (m * j) % (n + n);
                const double e = std::exp(j * (z[1] + z[10 + m]));
                const double s = 0.5 * (e - 1.0 / e), c = 0.5 * (e + 1.0 / e);
                psi = psi + P.coeff[j] * s * P.cosa[nm];
                u = u + j * P.coeff[j] * c * P.cosa[nm];
                v = v + j * P.coeff[j] * s * P.sina[nm];
            }
        } else {
            for (int j = 1; j <= n; ++j) {
                const int nm = (m * j) % (n + n);
                const double e = std::exp(j * z[10 + m]);
                psi = psi + z[n + j + 10] * e * P.cosa[nm];
                u = u + j * z[n + j + 10] * e * P.cosa[nm];
                v = v + j * z[n + j + 10] * e * P.sina[nm];
            }
        }
        rhs[m + 9] = psi - z[8] - z[7] * z[m + 10];
        rhs[n + m + 10] = 0.5 * ((-z[7] + u) * (-z[7] + u) + v * v) + z[m + 10] - z[9];
    }
}

// A x = b for a dense column-major matrix (Gaussian elimination with partial
// pivoting); 1-based b, 0-based A(i, j) = A[(j-1)*n + (i-1)]. false when singular.
bool dense_solve(int n, std::vector<double>& A, std::vector<double>& b) {
    auto a = [&](int i, int j) -> double& { return A[(size_t)(j - 1) * n + (i - 1)]; };
    for (int k = 1; k <= n; ++k) {
        int piv = k;
        for (int i = k + 1; i <= n; ++i) if (std::fabs(a(i, k)) > std::fabs(a(piv, k))) piv = i;
        if (a(piv, k) == 0.0) return false;
        if (piv != k) {
            for (int j = 1; j <= n; ++j) std::swap(a(k, j), a(piv, j));
            std::swap(b[k], b[piv]);
        }
        for (int i = k + 1; i <= n; ++i) {
            const double f = a(i, k) / a(k, k);
            if (f == 0.0) continue;
            for (int j = k + 1; j <= n; ++j) a(i, j) -= f * a(k, j);
            b[i] -= f * b[k];
        }
    }
    for (int k = n; k >= 1; --k) {
        double s = b[k];
        for (int j = k + 1; j <= n; ++j) s -= a(k, j) * b[j];
        b[k] = s / a(k, k);
    }
    return true;
}

}  // namespace

// stream_func_set_up.f90:21-57 and stream_func_coeffs.f:15-80.
int stream_function_solve(const ow3d_params& p, SFWave& w, std::string* err) {
    auto fail = [&](const std::string& m) { if (err) *err = m; return OW3D_ERR_BAD_INPUT; };
    const int n = p.sf_nmodes;
    if (n < 2 || n > 1000 || p.sf_nsteps < 1 || !(p.sf_H > 0) || !(p.sf_h > 0) || !(p.sf_L > 0) || !(p.g > 0))
        return fail("stream_function_wave: line 8 needs H, h, L > 0, nsteps >= 1 and at least 2 Fourier modes");
    if (p.sf_wavel_or_per != 0 && !(p.sf_T > 0)) return fail("stream_function_wave: the period must be positive");
    const double grav = p.g, depth = p.sf_h;
    double wavenum = 2.0 * std::acos(-1.0) / p.sf_L;   // ReadInputFileParameters.f90:293
    SFProblem P;
    P.n = n;
    P.num = 2 * n + 10;
    P.pi = 4.0 * std::atan(1.0);
    P.finite = !(wavenum * depth > 9.0);
    P.period = p.sf_wavel_or_per != 0;
    P.euler = p.sf_euler_or_stokes == 0;
    const double hoverd0 = P.finite ? p.sf_H / depth : 0.0;
    const double height0 = P.period ? p.sf_H / (grav * p.sf_T * p.sf_T) : p.sf_H / p.sf_L;
    P.value = p.sf_uEorS / std::sqrt(grav * p.sf_H);
    const int num = P.num;
    P.cosa.assign((size_t)num + 1, 0.0);
    P.sina.assign((size_t)num + 1, 0.0);
    P.coeff.assign((size_t)num + 1, 0.0);
    std::vector<double> z((size_t)num + 1, 0.0), s1(z), s2(z), rhs1(z), rhs2(z), b(z);
    std::vector<double> A((size_t)num * num);
    const double crit = 1e-6;
    const int nstep = p.sf_nsteps, number = 256;
    const double dhe = height0 / nstep, dho = hoverd0 / nstep;
    for (int ns = 1; ns <= nstep; ++ns) {
        P.height = ns * dhe;
        P.hoverd = ns * dho;
        if (ns <= 1) sf_init(P, z, s1, s2);
        else for (int i = 1; i <= num; ++i) z[i] = 2.0 * s2[i] - s1[i];
        bool done = false;
        for (int iter = 1; iter <= number && !done; ++iter) {
            sf_eqns(P, z, rhs1);
            for (int i = 1; i <= num; ++i) {
                double h = 0.01 * z[i];
                if (std::fabs(z[i]) < 1e-4) h = 1e-5;
                z[i] = z[i] + h;
                sf_eqns(P, z, rhs2);
                z[i] = z[i] - h;
                b[i] = -rhs1[i];
                for (int j = 1; j <= num; ++j) A[(size_t)(i - 1) * num + (j - 1)] = (rhs2[j] - rhs1[j]) / h;
            }
            if (!dense_solve(num, A, b)) return fail("stream_function_wave: singular Newton matrix");
            double sum = 0.0;
            for (int i = 1; i <= num; ++i) { sum += std::fabs(b[i]); z[i] = z[i] + b[i]; }
            const double criter = (ns == nstep) ? 0.01 * crit : crit;
            if (sum < criter) done = true;
        }
        if (!done) return fail("stream_function_wave: the solution did not converge in 256 iterations");
        if (ns == 1) { for (int i = 1; i <= num; ++i) s2[i] = z[i]; }
        else { for (int i = 1; i <= num; ++i) { s1[i] = s2[i]; s2[i] = z[i]; } }
    }
    // Fourier coefficients of the elevation (stream_func_coeffs.f:72-78)
    std::vector<double> y((size_t)num + 1, 0.0);
    for (int j = 1; j <= n; ++j) {
        double sum = 0.5 * (z[10] + z[n + 10] * ((j % 2) ? -1.0 : 1.0));
        for (int m = 1; m <= n - 1; ++m) sum = sum + z[10 + m] * P.cosa[(m * j) % (n + n)];
        y[j] = 2.0 * sum / n;
    }
    double period = p.sf_T;
    if (!P.period) period = z[3] / std::sqrt(grav * wavenum);
    else wavenum = z[1] / depth;
    w.n = n;
    w.k = wavenum;
    w.T = period;
    w.L = 2.0 * std::acos(-1.0) / wavenum;
    w.c = w.L / w.T;
    w.g = grav;
    w.z = z;
    w.y = y;
    return OW3D_OK;
}

// stream_func_wave_finite.f:10-66: elevation and surface potential at x, t.
void stream_function_eval(const SFWave& w, int nx, const double* x, double t, double* eta, double* phis) {
    const int n = w.n;
    const std::vector<double>& zz = w.z;
    const std::vector<double>& yy = w.y;
    const double kinv = 1.0 / w.k;
    const double ufactor = std::sqrt(w.g * kinv), pfactor = ufactor * kinv;
    const double omega_t = w.k * ufactor * zz[4] * t;
    for (int j = 0; j < nx; ++j) {
        const double kx = w.k * x[j] - omega_t;
        double km = (double)n;
        double e_j = 0.5 * yy[n] * std::cos(km * kx);
        for (int m = 1; m <= n - 1; ++m) {
            km = (double)m;
            e_j = e_j + yy[m] * std::cos(km * kx);
        }
        double ph = (zz[4] - zz[7]) * x[j] * w.k;
        for (int m = 1; m <= n; ++m) {
            km = (double)m;
            const double e = std::exp(km * (zz[1] + e_j));
            const double b = zz[n + m + 10] * 0.5 * (e + 1.0 / e) / std::cosh(km * zz[1]);
            ph = ph + b * std::sin(km * kx);
        }
        if (eta) eta[j] = kinv * e_j;
        if (phis) phis[j] = ph * pfactor;
    }
}

// Initial geometry and surface of the deck's IC for the cases built from
// formulas (SetupInitialConditions.f90): 0 (flat, depth Lz > 0, still water),
// 1 (the deep-water standing wave of nonlinearstandingwave1D.f90), 3 (the
// Whalin shoal of bottomWhalin.f90), 4 and 5 (flat deep / shallow water with a cosine surface along x, or y in
// a y-only basin), 7 (flat, depth of the stream-function wave, that wave over
// the whole basin at t = time0 when relaxation is on, then the relaxation
// weights of the non-generating zones applied three times). Outputs are
// Nxg*Nyg, ghosts included.
int initial_condition(const ow3d_params& p, double* h, double* hx, double* hxx, double* hy, double* hyy, double* E,
                      double* P, std::string* err) {
    auto fail = [&](const std::string& m, int code) { if (err) *err = m; return code; };
    if (!h || !E || !P) return fail("initial_condition: h, E and P are required", OW3D_ERR_BAD_INPUT);
    GridHost G;
    const int Nxg = p.Nx + (p.Nx > 1 ? 2 : 0), Nyg = p.Ny + (p.Ny > 1 ? 2 : 0);
    const size_t C = (size_t)Nxg * Nyg;
    std::vector<double> ones(C, 1.0), zeros(C, 0.0);
    int r = build_grid(p, ones.data(), zeros.data(), zeros.data(), zeros.data(), zeros.data(), G, err);
    if (r) return r;
    for (double* a : {hx, hxx, hy, hyy}) if (a) std::fill(a, a + C, 0.0);
    std::fill(E, E + C, 0.0);
    std::fill(P, P + C, 0.0);
    const double pi = std::acos(-1.0), two = 2.0;
    const bool alongx = p.Nx > 1;
    auto coord = [&](size_t c) { return alongx ? G.x[c % (size_t)Nxg] : G.y[c / (size_t)Nxg]; };
    switch (p.IC) {
        case 0:   // :18-114 with Lz > 0 and no pressure forcing: still water
            if (!(p.Lz > 0)) return fail("initial_condition: IC 0 with Lz <= 0 reads a bathymetry file", OW3D_ERR_UNSUPPORTED);
            std::fill(h, h + C, p.Lz);
            return OW3D_OK;
        case 1: {   // :116-129, nonlinearstandingwave1D.f90: deep-water standing wave (Agnon and Glozman)
            // the series' coefficients carry the reference's single-precision
            // literals (0.5243 and 10.0**(-2) are REAL there)
            std::fill(h, h + C, two);   // wavenumber pi, wavelength 2: L/h = 1, deep water
            const float a[8] = {0.0f, 0.5243f, 0.4978f, 0.6542f, 0.1007f, 0.1653f, 0.2753f, 0.4522f};
            const int e10[8] = {-1, -2, -3, -4, -4, -5, -6, -7};
            double coef[8];
            for (int n = 0; n < 8; ++n) {
                float pw = 1.0f;
                for (int q = 0; q < -e10[n]; ++q) pw *= 10.0f;
                const float tenpow = 1.0f / pw;
                coef[n] = n == 0 ? 0.8867 * (double)tenpow
                                 : std::sqrt(std::sqrt((double)(n + 1))) * (double)a[n] * (double)tenpow;
            }
            for (size_t c = 0; c < C; ++c) {
                const double X = coord(c);
                double s = 0.0;
                for (int n = 0; n < 8; ++n) s += coef[n] * std::cos((n + 1) * pi * X);
                E[c] = 0.5 * s;
            }
            return OW3D_OK;
        }
        case 3: {   // :155-161, bottomWhalin.f90: the Whalin shoal (flat surface)
            const bool xlong = p.Nx > p.Ny;
            const double y0 = xlong ? (G.y.size() > 1 ? (G.y[1] - G.y[0]) / two : 0.0)
                                    : (G.x.size() > 1 ? (G.x[1] - G.x[0]) / two : 0.0);
            // the single-precision 10.67 and 18.29 of the x-long branch are kept
            const double lo = xlong ? (double)10.67f : 10.67, hi = xlong ? (double)18.29f : 18.29;
            for (int j = 1; j <= Nyg; ++j)
                for (int i = 1; i <= Nxg; ++i) {
                    const size_t c = (size_t)(i - 1) + (size_t)Nxg * (j - 1);
                    double across = xlong ? G.y[(size_t)(j - 1)] : G.x[(size_t)(i - 1)];
                    const double along = xlong ? G.x[(size_t)(i - 1)] : G.y[(size_t)(j - 1)];
                    if (across < y0) across = y0;
                    const double sg = std::sqrt(6.096 * across - across * across);
                    const double sgd = -0.04 * (6.096 - two * across) * 0.5 / sg;
                    const double sgdd = 0.04 * 6.096 * 6.096 / (4.0 * sg * sg * sg);
                    double vh, valong = 0, vacross = 0, vaa = 0, vcc = 0;
                    if (along <= lo - sg) vh = 0.4572;
                    else if (along >= hi - sg) vh = 0.1524;
                    else { vh = 0.4572 + 0.04 * (10.67 - sg - along); valong = -0.04; vacross = sgd; vcc = sgdd; }
                    h[c] = vh;
                    if (xlong) {
                        if (hx) hx[c] = valong; if (hxx) hxx[c] = vaa; if (hy) hy[c] = vacross; if (hyy) hyy[c] = vcc;
                    } else {
                        if (hy) hy[c] = valong; if (hyy) hyy[c] = vaa; if (hx) hx[c] = vacross; if (hxx) hxx[c] = vcc;
                    }
                }
            return OW3D_OK;
        }
        case 4:
        case 5: {   // :183-234
            const double L = alongx ? p.Lx : p.Ly;
            const double kw = two * pi / L;
            const double kh = p.IC == 4 ? two * pi : 0.5;
            const double depth = kh / kw;
            const double HH = p.IC == 4 ? L / 10.0 : depth * 0.75;
            std::fill(h, h + C, depth);
            for (size_t c = 0; c < C; ++c) E[c] = HH / two * std::cos(kw * coord(c));
            return OW3D_OK;
        }
        case 7: {   // :303-385 (Cartesian grids)
            std::fill(h, h + C, p.sf_h);
            if (p.relaxONOFF != 1) return OW3D_OK;
            SFWave w;
            r = stream_function_solve(p, w, err);
            if (r) return r;
            const bool xdir = (p.relaxXorY == 'X' || p.relaxXorY == 'x');
            const double rd = p.relaxDegrees / 180.0 * pi;
            const int n1 = xdir ? Nxg : Nyg, n2 = xdir ? Nyg : Nxg;
            std::vector<double> pos((size_t)n1), e((size_t)n1), f((size_t)n1);
            for (int b = 0; b < n2; ++b) {
                for (int a = 0; a < n1; ++a) {
                    const double xa = xdir ? G.x[(size_t)a] : G.y[(size_t)a];
                    const double yb = xdir ? G.y[(size_t)b] : G.x[(size_t)b];
                    pos[(size_t)a] = rd == 0.0 ? xa : (xdir ? xa * std::cos(rd) + yb * std::sin(rd)
                                                            : -xa * std::sin(rd) + yb * std::cos(rd));
                }
                if (rd == 0.0 && b > 0) {
                    // the line is the same for every row
                } else {
                    stream_function_eval(w, n1, pos.data(), p.time0, e.data(), f.data());
                }
                for (int a = 0; a < n1; ++a) {
                    const size_t c = xdir ? (size_t)a + (size_t)Nxg * b : (size_t)b + (size_t)Nxg * a;
                    E[c] = e[(size_t)a];
                    P[c] = f[(size_t)a];
                }
            }
            // the relaxation three times (:364-366): generation zones relax
            // towards the same wave (no change), the others damp
            const std::vector<ZoneHost> Z = build_zones(p, G);
            for (int pass = 0; pass < 3; ++pass)
                for (const ZoneHost& z : Z) {
                    if (z.wavegen) continue;
                    for (int j = z.j0; j <= z.j1; ++j)
                        for (int i = z.i0; i <= z.i1; ++i) {
                            const double gm = z.xdir ? z.gam[(size_t)(i - z.i0)] : z.gam[(size_t)(j - z.j0)];
                            const size_t c = (size_t)(i - 1) + (size_t)Nxg * (j - 1);
                            E[c] *= gm;
                            if (z.phion) P[c] *= gm;
                        }
                }
            return OW3D_OK;
        }
        default:
            return fail("initial_condition: IC " + std::to_string(p.IC) +
                            " is not built (0, 1, 3, 4, 5 and 7 are; -1 reads OceanWave3D.init)",
                        OW3D_ERR_UNSUPPORTED);
    }
}

}  // namespace ow3d
