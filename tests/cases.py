"""Small synthetic cases shared by the tests (seeded, analytic bathymetry)."""
import numpy as np


def capi():
    from conftest import load_package
    return load_package().capi


def flat_2d(Nx=17, Nz=9, L=2.0, h0=1.0, **kw):
    c = capi()
    p = c.default_params(Nx=Nx, Ny=1, Nz=Nz, Lx=L, Ly=1.0, Lz=h0, GridZ=1, **kw)
    Nxg, Nyg, _ = c.dims(p)
    h = np.full(Nxg * Nyg, h0)
    return p, dict(h=h)


def bump_3d(Nx=17, Ny=9, Nz=9, Lx=2.0, Ly=1.0, h0=1.0, amp=0.2, **kw):
    """Depth h0 minus a Gaussian bump; analytic h_x, h_xx, h_y, h_yy (ghosts included)."""
    c = capi()
    p = c.default_params(Nx=Nx, Ny=Ny, Nz=Nz, Lx=Lx, Ly=Ly, Lz=h0, GridZ=1, **kw)
    Nxg, Nyg, _ = c.dims(p)
    x = (np.arange(Nxg) - 1) / (Nx - 1) * Lx
    y = (np.arange(Nyg) - (1 if Ny > 1 else 0)) / max(Ny - 1, 1) * Ly
    X, Y = np.meshgrid(x, y)          # (Nyg, Nxg): i fastest when raveled
    sx, sy, x0, y0 = 0.3 * Lx, 0.4 * Ly, 0.55 * Lx, 0.45 * Ly
    G = amp * np.exp(-((X - x0) ** 2 / (2 * sx ** 2) + (Y - y0) ** 2 / (2 * sy ** 2)))
    h = h0 - G
    hx = G * (X - x0) / sx ** 2
    hxx = G * (1 / sx ** 2 - (X - x0) ** 2 / sx ** 4)
    hy = G * (Y - y0) / sy ** 2
    hyy = G * (1 / sy ** 2 - (Y - y0) ** 2 / sy ** 4)
    if Ny == 1:
        hy[:] = 0; hyy[:] = 0
    return p, dict(h=h.ravel(), hx=hx.ravel(), hxx=hxx.ravel(), hy=hy.ravel(), hyy=hyy.ravel())


def slope_2d(Nx=33, Nz=9, L=4.0, h0=1.0, h1=0.6, **kw):
    c = capi()
    p = c.default_params(Nx=Nx, Ny=1, Nz=Nz, Lx=L, Ly=1.0, Lz=h0, GridZ=1, **kw)
    Nxg, _, _ = c.dims(p)
    x = (np.arange(Nxg) - 1) / (Nx - 1) * L
    # smooth monotone transition h0 -> h1 (tanh), analytic derivatives
    a, xm = 3.0 / L, 0.5 * L
    t = np.tanh(a * (x - xm))
    h = 0.5 * (h0 + h1) - 0.5 * (h0 - h1) * t
    hx = -0.5 * (h0 - h1) * a * (1 - t ** 2)
    hxx = -0.5 * (h0 - h1) * a * (-2 * t * a * (1 - t ** 2))
    return p, dict(h=h, hx=hx, hxx=hxx)


def surface(p, amp=0.02, seed=0):
    """A smooth synthetic free surface and its exact horizontal derivatives."""
    c = capi()
    Nxg, Nyg, _ = c.dims(p)
    rng = np.random.default_rng(seed)
    x = (np.arange(Nxg) - 1) / (p.Nx - 1) * p.Lx
    y = (np.arange(Nyg) - (1 if p.Ny > 1 else 0)) / max(p.Ny - 1, 1) * p.Ly
    X, Y = np.meshgrid(x, y)
    E = np.zeros_like(X); Ex = np.zeros_like(X); Exx = np.zeros_like(X); Ey = np.zeros_like(X); Eyy = np.zeros_like(X)
    for _ in range(3):
        kx = 2 * np.pi * rng.integers(1, 3) / p.Lx
        ky = (2 * np.pi * rng.integers(0, 2) / p.Ly) if p.Ny > 1 else 0.0
        ph = rng.uniform(0, 2 * np.pi)
        a = amp * rng.uniform(0.3, 1.0)
        arg = kx * X + ky * Y + ph
        E += a * np.cos(arg); Ex += -a * kx * np.sin(arg); Exx += -a * kx ** 2 * np.cos(arg)
        Ey += -a * ky * np.sin(arg); Eyy += -a * ky ** 2 * np.cos(arg)
    return [v.ravel() for v in (E, Ex, Exx, Ey, Eyy)]


def field3(p, seed=1):
    c = capi()
    Nxg, Nyg, Nzg = c.dims(p)
    return np.random.default_rng(seed).standard_normal(Nxg * Nyg * Nzg)


def fs_rhs(p, P):
    """RHS with the free-surface Dirichlet row = P on the interior columns."""
    c = capi()
    Nxg, Nyg, Nzg = c.dims(p)
    gy = 1 if p.Ny > 1 else 0
    r = np.zeros((Nyg, Nxg, Nzg))
    P2 = np.asarray(P).reshape(Nyg, Nxg)
    r[gy:Nyg - gy, 1:Nxg - 1, -1] = P2[gy:Nyg - gy, 1:Nxg - 1]
    return r.ravel()


def shoal_generation(W, nsteps, **kw):
    """The 257 x 33 x 9 shoal basin with its generation zone (0-3 m, the
    linear regular wave T = 1 s, H = 0.01 m at the 0.45 m depth, sampled
    every half step) and its sponge (30-35 m); GMRES reltol 1e-8 with the
    example decks' abstol 1e-6. Returns params, geometry and a function of
    the zone-0 box (i0, i1, j0, j1) that gives the zone's target
    (mode, nt, dt_sample, eta, phis) for nsteps steps."""
    zones = [dict(x1=0.0, x2=3.0, y1=0.0, y2=6.0, ftype=-10, param=3.5, wavegen=1),
             dict(x1=30.0, x2=35.0, y1=0.0, y2=6.0, ftype=9, param=3.5)]
    p, geo = W.shoal(relaxONOFF=1, relaxNo=2, relaxTransientTime=1.0, zones=zones, reltol=1e-8, abstol=1e-6, **kw)
    x, _ = W.grid_xy(p)

    def target(box):
        i0, i1, j0, j1 = box
        xs = x[i0 - 1:i1]
        T, H, h = 1.0, 0.01, 0.45
        om = 2 * np.pi / T
        k = W.dispersion_k(om, h)
        nt = 2 * nsteps + 2
        tt = np.arange(nt) * (0.5 * p.dt)
        ny = j1 - j0 + 1
        eta = np.array([np.tile(0.5 * H * np.cos(k * xs - om * t), ny) for t in tt])
        phis = np.array([np.tile(0.5 * H * W.G / om * np.sin(k * xs - om * t), ny) for t in tt])
        return (0, nt, 0.5 * p.dt, eta, phis)
    return p, geo, target


def run_steps(sim, nsteps):
    """Step one step at a time; returns the matvec count of each step."""
    its = []
    for _ in range(nsteps):
        a = sim.stats()["total_iterations"]
        st = sim.step(1)
        assert st >= 0, st
        its.append(sim.stats()["total_iterations"] - a)
    return np.array(its, dtype=np.int64)
