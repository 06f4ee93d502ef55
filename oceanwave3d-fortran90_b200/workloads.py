"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No external dataset is involved: every input is generated here from a seed.

  irregular_sea   3-D flat 1 m depth, linear JONSWAP sea (Hs, Tp, gamma) with
                  cos^2 directional spreading and uniform random phases,
                  1025 x 257 x 17 by default (also the 2049 x 513 x 9 case)
  shoal           3-D 35 m x 6 m basin, 0.45 m depth rising to 0.15 m over a
                  semi-elliptic shoal with a cos^2 taper, 257 x 33 x 9
  standing_2d     2-D flume with a cosine free surface (2-D x-sigma cases)
  stream_function_2d
                  2-D stream-function wave, kh = 1, H/L half the breaking
                  limit, 64 points per wavelength, 9 sigma levels: the wave
                  over the whole flume at t = 0 (the reference's IC 7),
                  generated in the first wavelength, absorbed in the last
"""
import numpy as np

from .capi import default_params, dims

G = 9.81


def dispersion_k(omega, h, g=G):
    """Wavenumber of linear waves: omega^2 = g k tanh(k h) (Newton iteration)."""
    omega = np.asarray(omega, dtype=np.float64)
    k = omega ** 2 / g
    for _ in range(50):
        f = g * k * np.tanh(k * h) - omega ** 2
        df = g * np.tanh(k * h) + g * k * h / np.cosh(k * h) ** 2
        k = k - f / df
    return k


def jonswap(f, Hs, Tp, gamma=3.3):
    """One-sided JONSWAP variance density S(f) scaled to the significant wave height Hs."""
    fp = 1.0 / Tp
    sig = np.where(f <= fp, 0.07, 0.09)
    r = np.exp(-((f - fp) ** 2) / (2 * sig ** 2 * fp ** 2))
    S = f ** -5.0 * np.exp(-1.25 * (fp / f) ** 4) * gamma ** r
    df = np.gradient(f)
    m0 = np.sum(S * df)
    return S * (Hs / 4.0) ** 2 / m0


def linear_sea(x, y, h, Hs=0.05, Tp=1.5, gamma=3.3, nfreq=48, ndir=9, theta0=0.0, fmax_fac=3.0, seed=0):
    """Surface elevation eta and surface potential phis of a linear directional
    sea on the grid x (nx) by y (ny); returns arrays of shape (ny, nx)."""
    rng = np.random.default_rng(seed)
    fp = 1.0 / Tp
    f = np.linspace(0.5 * fp, fmax_fac * fp, nfreq)
    S = jonswap(f, Hs, Tp, gamma)
    df = f[1] - f[0]
    th = np.linspace(-np.pi / 2, np.pi / 2, ndir + 2)[1:-1] + theta0
    D = np.cos(th - theta0) ** 2
    D = D / D.sum()
    amp = np.sqrt(2 * S[:, None] * df * D[None, :])        # (nfreq, ndir)
    om = 2 * np.pi * f
    k = dispersion_k(om, h)
    ph = rng.uniform(0, 2 * np.pi, size=amp.shape)
    X, Y = np.meshgrid(x, y)
    eta = np.zeros_like(X)
    phis = np.zeros_like(X)
    for a in range(nfreq):
        for b in range(ndir):
            arg = k[a] * (np.cos(th[b]) * X + np.sin(th[b]) * Y) + ph[a, b]
            eta += amp[a, b] * np.cos(arg)
            phis += amp[a, b] * G / om[a] * np.sin(arg)
    return eta, phis


def grid_xy(p):
    Nxg, Nyg, _ = dims(p)
    x = (np.arange(Nxg) - 1) / (p.Nx - 1) * p.Lx
    gy = 1 if p.Ny > 1 else 0
    y = (np.arange(Nyg) - gy) / max(p.Ny - 1, 1) * p.Ly if p.Ny > 1 else np.array([p.Ly])
    return x, y


def irregular_sea(Nx=1025, Ny=257, Nz=17, dx=0.05, Hs=0.05, Tp=1.5, gamma=3.3, courant=0.5, seed=1234,
                  precision=0, reltol=1e-8, **kw):
    """The irregular-sea configuration: flat 1 m depth, walls, no zones; the
    initial state is a seeded linear JONSWAP sea (eta, surface potential)."""
    h0 = 1.0
    p = default_params(Nx=Nx, Ny=Ny, Nz=Nz, Lx=(Nx - 1) * dx, Ly=(Ny - 1) * dx, Lz=h0, GridZ=1,
                       reltol=reltol, precision=precision, **kw)
    p.dt = courant * dx / np.sqrt(G * h0)
    p.g = G
    Nxg, Nyg, _ = dims(p)
    x, y = grid_xy(p)
    eta, phis = linear_sea(x, y, h0, Hs=Hs, Tp=Tp, gamma=gamma, seed=seed)
    geo = dict(h=np.full(Nxg * Nyg, h0))
    return p, geo, eta.ravel(), phis.ravel()


def shoal(Nx=257, Ny=33, Nz=9, courant=0.5, precision=0, **kw):
    """35 m x 6 m basin, 0.45 m deep, shoaling to 0.15 m over a semi-elliptic
    shoal (semi-axes 4 m x 3 m) with a cos^2 taper; analytic depth derivatives."""
    Lx, Ly, hd, hs = 35.0, 6.0, 0.45, 0.15
    p = default_params(Nx=Nx, Ny=Ny, Nz=Nz, Lx=Lx, Ly=Ly, Lz=hd, GridZ=1, precision=precision, **kw)
    p.dt = courant * (Lx / (Nx - 1)) / np.sqrt(G * hd)
    x, y = grid_xy(p)
    X, Y = np.meshgrid(x, y)
    xc, yc, a, b = 17.0, 3.0, 4.0, 3.0
    r2 = ((X - xc) / a) ** 2 + ((Y - yc) / b) ** 2
    inside = r2 < 1.0
    c = np.cos(0.5 * np.pi * np.sqrt(np.minimum(r2, 1.0)))
    bump = (hd - hs) * np.where(inside, c ** 2, 0.0)
    h = hd - bump
    # derivatives of (hd-hs) cos^2(pi/2 sqrt(r2)) by finite differences of the
    # analytic field on a fine local stencil (smooth: C1 at the rim)
    e = 1e-5
    def hf(XX, YY):
        rr = ((XX - xc) / a) ** 2 + ((YY - yc) / b) ** 2
        cc = np.cos(0.5 * np.pi * np.sqrt(np.minimum(rr, 1.0)))
        return hd - (hd - hs) * np.where(rr < 1.0, cc ** 2, 0.0)
    hx = (hf(X + e, Y) - hf(X - e, Y)) / (2 * e)
    hy = (hf(X, Y + e) - hf(X, Y - e)) / (2 * e)
    hxx = (hf(X + e, Y) - 2 * h + hf(X - e, Y)) / e ** 2
    hyy = (hf(X, Y + e) - 2 * h + hf(X, Y - e)) / e ** 2
    geo = dict(h=h.ravel(), hx=hx.ravel(), hxx=hxx.ravel(), hy=hy.ravel(), hyy=hyy.ravel())
    return p, geo


def standing_2d(Nx=65, Nz=9, L=2 * np.pi, h0=1.0, amp=0.05, courant=0.5, **kw):
    p = default_params(Nx=Nx, Ny=1, Nz=Nz, Lx=L, Ly=1.0, Lz=h0, GridZ=1, **kw)
    p.dt = courant * (L / (Nx - 1)) / np.sqrt(G * h0)
    x, _ = grid_xy(p)
    E0 = amp * np.cos(2 * np.pi * x / L)
    return p, dict(h=np.full(x.size, h0)), E0, np.zeros_like(E0)


def breaking_steepness(kh):
    """Limiting steepness H/L of a periodic wave at relative depth kh
    (Miche's criterion, 0.142 tanh(kh))."""
    return 0.142 * np.tanh(kh)


def stream_function_2d(n_waves=8, ppw=64, Nz=9, kh=1.0, h0=1.0, steepness=0.5, courant=0.5, sponge_waves=3, **kw):
    """The 2-D stream-function wave case: a flume of n_waves wavelengths
    (L = 2 pi h0 / kh) with ppw points per wavelength, the wave of height
    steepness x the breaking limit everywhere at t = 0 (IC 7 of the
    reference), a generation zone over the first wavelength fed with the
    exact wave at every RK stage time (relaxation target mode 1) and a sponge
    over the last. Returns params, geometry, E0, P0 and the targets
    {zone: (mode, nt, dt_sample, eta, phis)} for `steps` time steps."""
    from . import stream_function_wave
    L = 2 * np.pi * h0 / kh
    Nx = n_waves * ppw + 1
    steps = kw.pop("steps", 200)
    p = default_params(Nx=Nx, Ny=1, Nz=Nz, Lx=n_waves * L, Ly=1.0, Lz=h0, GridZ=1,
                       relaxONOFF=1, relaxNo=2, relaxTransientTime=0.0,
                       zones=[dict(x1=0.0, x2=L, ftype=10, param=3.5, wavegen=1),
                              dict(x1=(n_waves - sponge_waves) * L, x2=n_waves * L, ftype=9, param=3.5)], **kw)
    p.IncWaveType = 1
    p.g = G
    p.sf_H, p.sf_h, p.sf_L = steepness * breaking_steepness(kh) * L, h0, L
    p.sf_T, p.sf_wavel_or_per, p.sf_uEorS, p.sf_euler_or_stokes = 0.0, 0, 0.0, 0
    p.sf_nsteps, p.sf_nmodes = 6, 24
    _, _, (k, Lw, T, c) = stream_function_wave(p, np.zeros(1))
    p.dt = courant * (L / ppw) / c
    Nxg, Nyg, _ = dims(p)
    x = (np.arange(Nxg) - 1) * (p.Lx / (Nx - 1))
    E0, P0, _ = stream_function_wave(p, x, 0.0)
    geo = dict(h=np.full(Nxg * Nyg, h0))
    # zone 0 box: the first wavelength (1-based ghost-inclusive indices)
    i0, i1 = 2, 2 + ppw
    nt = 2 * steps + 2
    tt = np.arange(nt) * (0.5 * p.dt)
    eta = np.array([stream_function_wave(p, x[i0 - 1:i1], t)[0] for t in tt])
    phis = np.array([stream_function_wave(p, x[i0 - 1:i1], t)[1] for t in tt])
    return p, geo, E0, P0, {0: (1, nt, 0.5 * p.dt, eta, phis)}


def periodic_wave_2d(Nx=65, Nz=9, kh=1.0, h0=1.0, steepness=0.5, courant=0.5, **kw):
    """The 2-D periodic stream-function wave: one wavelength L = 2 pi h0 / kh
    (kh = 1, depth 1 m) periodic in x with Nx points including both ends
    (x_1 = 0 and x_Nx = L hold the same value), Nz sin-clustered sigma
    levels, the nonlinear stream-function wave of height steepness x the
    breaking limit at t = 0, flat bottom, time step at Courant number
    `courant` on the phase speed. Returns params, geometry, E0, P0 and the
    wave's (k, L, T, c); the exact solution at time t is the same wave
    translated, stream_function_wave(params, x, t)."""
    from . import stream_function_wave
    L = 2 * np.pi * h0 / kh
    p = default_params(Nx=Nx, Ny=1, Nz=Nz, Lx=L, Ly=1.0, Lz=h0, GridZ=1, periodic_x=1, **kw)
    p.IncWaveType = 1
    p.g = G
    p.sf_H, p.sf_h, p.sf_L = steepness * breaking_steepness(kh) * L, h0, L
    p.sf_T, p.sf_wavel_or_per, p.sf_uEorS, p.sf_euler_or_stokes = 0.0, 0, 0.0, 0
    p.sf_nsteps, p.sf_nmodes = 6, 24
    _, _, info = stream_function_wave(p, np.zeros(1))
    p.dt = courant * (L / (Nx - 1)) / info[3]
    Nxg, Nyg, _ = dims(p)
    x = (np.arange(Nxg) - 1) * (L / (Nx - 1))
    E0, P0, _ = stream_function_wave(p, x, 0.0)
    return p, dict(h=np.full(Nxg * Nyg, h0)), E0, P0, info
