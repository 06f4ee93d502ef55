"""CPU checks of the oracle itself: known-answer and physics tests.

The reference ships no tests or stored outputs for this path, so the oracle is
pinned by (1) the multigrid hierarchy its coarsening rules give at the
documented grid sizes, (2) analytic answers (harmonic polynomials, the linear
wave potential, the linear standing wave, Savitzky-Golay polynomial
reproduction), (3) agreement between the reference-ordered and the
device-ordered algorithms, and (4) the committed golden vectors
(tests/golden, checked in test_golden.py).
"""
import numpy as np
import pytest

import cases


def oracle_for(oracle, p, geo, mode=None):
    return oracle.Oracle(p, **geo, mode=oracle.MODE_REFERENCE if mode is None else mode)


# --- multigrid hierarchy (MGPreProcess.f90:31,95-215) -----------------------

HIERARCHY = [
    ((65, 1, 9), [(3, 1, 3), (5, 1, 5), (9, 1, 9), (17, 1, 9), (33, 1, 9), (65, 1, 9)], 2.06),
    ((257, 33, 9), [(3, 3, 3), (5, 5, 5), (9, 9, 9), (17, 9, 9), (33, 9, 9), (65, 9, 9), (129, 17, 9),
                    (257, 33, 9)], 1.44),
    ((129, 33, 13), [(5, 5, 7), (9, 9, 7), (9, 9, 13), (17, 9, 13), (33, 9, 13), (65, 17, 13),
                     (129, 33, 13)], 1.45),
]


@pytest.mark.parametrize("dims,levels,ratio", HIERARCHY, ids=["65x1x9", "257x33x9", "129x33x13"])
def test_mg_hierarchy(ow3d, oracle, dims, levels, ratio):
    nx, ny, nz = dims
    p = ow3d.default_params(Nx=nx, Ny=ny, Nz=nz, Lx=1.0, Ly=1.0, GridZ=1)
    Nxg, Nyg, _ = ow3d.dims(p)
    o = oracle.Oracle(p, h=np.ones(Nxg * Nyg))
    got = [o.level_dims(l)[:3] for l in range(o.nlevels)]
    assert got == levels
    tot = sum(o.level_size(l) for l in range(o.nlevels)) / o.N
    assert abs(tot - ratio) < 0.01


# --- operator exactness ------------------------------------------------------

def _grid(p, o):
    Nxg, Nyg, Nzg = o.Nxg, o.Nyg, o.Nzg
    x = (np.arange(Nxg) - 1) / (p.Nx - 1) * p.Lx
    y = (np.arange(Nyg) - (1 if p.Ny > 1 else 0)) / max(p.Ny - 1, 1) * p.Ly
    s = o.fine_z()
    return x, y, s


@pytest.mark.parametrize("three", [False, True], ids=["2d", "3d"])
def test_matvec_harmonic_polynomial(ow3d, oracle, three):
    """Flat bottom, flat surface: sigma = (z+h)/h and the 7-point stencils are
    exact for polynomials of degree <= 6, so a harmonic cubic gives zero
    interior residual."""
    if three:
        p, geo = cases.bump_3d(Nx=17, Ny=13, Nz=9, amp=0.0)
    else:
        p, geo = cases.flat_2d(Nx=17, Nz=9)
    o = oracle_for(oracle, p, geo)
    x, y, s = _grid(p, o)
    h0 = 1.0
    Y, X, S = np.meshgrid(y, x, s, indexing="ij")          # (j, i, k): k fastest when raveled
    Z = S * h0 - h0
    phi = X ** 3 - 3 * X * Z ** 2 + (Y ** 2 - Z ** 2 if three else 0.0)
    o.set_surface(np.zeros(o.C))
    r = o.matvec(phi.ravel()).reshape(o.Nyg, o.Nxg, o.Nzg)
    gy = 1 if three else 0
    js = slice(2, o.Nyg - 2) if three else slice(0, 1)
    inner = r[js, 2:o.Nxg - 2, 2:o.Nzg - 1]
    assert np.max(np.abs(inner)) < 1e-9 * np.max(np.abs(phi))
    # free-surface rows are the identity
    assert np.allclose(r[gy:o.Nyg - gy, 1:o.Nxg - 1, -1], phi.reshape(r.shape)[gy:o.Nyg - gy, 1:o.Nxg - 1, -1])


def _wave_solve(ow3d, oracle, Nx, Nz, mode):
    L, h0 = 2.0, 1.0
    p, geo = cases.flat_2d(Nx=Nx, Nz=Nz, L=L, h0=h0, reltol=1e-12, abstol=1e-14, GMRESmaxiterations=60)
    o = oracle_for(oracle, p, geo, mode)
    x, _, s = _grid(p, o)
    k = 2 * np.pi / L
    exact = (np.cosh(k * s[None, :] * h0) * np.cos(k * x)[:, None]).ravel()
    o.set_surface(np.zeros(o.C))
    P = np.cosh(k * h0) * np.cos(k * x)
    phi, it, res, st = o.solve(cases.fs_rhs(p, P), np.zeros(o.N))
    e = (phi - exact).reshape(o.Nxg, o.Nzg)[1:-1, 1:]
    return np.max(np.abs(e)) / np.max(np.abs(exact)), it


@pytest.mark.parametrize("mode", [0, 1], ids=["reference", "device"])
def test_solve_linear_wave_potential(ow3d, oracle, mode):
    """phi = cosh(k(z+h)) cos(kx) solves the Laplace problem with a flat bottom
    and walls at x = 0, L (k = 2 pi / L); sixth-order convergence in x."""
    e1, it1 = _wave_solve(ow3d, oracle, 17, 17, mode)
    e2, it2 = _wave_solve(ow3d, oracle, 33, 17, mode)
    assert e2 < 1e-4
    assert e1 / e2 > 2 ** 4, (e1, e2)


def test_reference_and_device_orderings_agree(ow3d, oracle):
    """Lexicographic GS + left GMRES and multicolour GS + right FGMRES solve
    the same system: solutions agree to the solver tolerance."""
    p, geo = cases.bump_3d(Nx=33, Ny=17, Nz=9, reltol=1e-10, GMRESmaxiterations=60)
    surf = cases.surface(p, amp=0.03, seed=4)
    rhs = cases.fs_rhs(p, np.sin(np.linspace(0, 3, (p.Nx + 2) * (p.Ny + 2))))
    out = []
    for mode in (oracle.MODE_REFERENCE, oracle.MODE_DEVICE):
        o = oracle_for(oracle, p, geo, mode)
        o.set_surface(*surf)
        phi, it, res, st = o.solve(rhs, np.zeros(o.N))
        assert st == 0 and 3 <= it <= p.GMRESmaxiterations
        out.append(phi)
    assert np.max(np.abs(out[0] - out[1])) < 1e-6 * np.max(np.abs(out[0]))


def test_gmres_stops_at_matvec_limit(ow3d, oracle):
    """The reference accepts a non-converged solve after GMRESmaxiterations
    matvecs (iterative_solution.f90:43,117-134)."""
    p, geo = cases.bump_3d(Nx=17, Ny=9, Nz=9, reltol=1e-30, abstol=0.0, GMRESmaxiterations=5)
    o = oracle_for(oracle, p, geo)
    o.set_surface(*cases.surface(p))
    phi, it, res, st = o.solve(cases.fs_rhs(p, np.ones(o.C)), np.zeros(o.N))
    assert it == 5 and st == 1


# --- time stepping -----------------------------------------------------------

def test_linear_standing_wave_period(ow3d, oracle):
    """Linear standing wave in a closed basin: eta = A cos(kx) cos(wt),
    w^2 = g k tanh(kh) (the reference's linearstandingwave2D solution)."""
    L, h0, A = 2.0, 1.0, 1e-3
    Nx = 33
    k = 2 * np.pi / L
    g = 9.81
    w = np.sqrt(g * k * np.tanh(k * h0))
    T = 2 * np.pi / w
    nsteps = 64
    p, geo = cases.flat_2d(Nx=Nx, Nz=13, L=L, h0=h0, LinearONOFF=0, dt=T / nsteps, g=g, reltol=1e-10)
    o = oracle_for(oracle, p, geo)
    x = (np.arange(o.Nxg) - 1) / (Nx - 1) * L
    o.set_state(A * np.cos(k * x), np.zeros(o.Nxg))
    assert o.step(nsteps // 2) >= 0
    E, P, W, phi, t = o.get_state()
    assert abs(t - T / 2) < 1e-12
    err = np.max(np.abs(E[1:-1] - A * np.cos(k * x[1:-1]) * np.cos(w * t)))
    assert err < 1e-3 * A, err


# --- filter and relaxation tables -------------------------------------------

@pytest.mark.parametrize("alpha,order", [(3, 4), (6, 10), (4, 6)])
def test_sg_filter_reproduces_polynomials(ow3d, oracle, alpha, order):
    """Savitzky-Golay smoothing (FilterInit.f90, savgol.f90) is exact on
    polynomials up to its order on the centred rows. The first and last
    alpha rows use the boundary table the reference stores (read through its
    (2 alpha+1) x alpha view), which is not polynomial-exact, so they are
    checked only for being finite and changed."""
    p, geo = cases.flat_2d(Nx=33, Nz=9, L=4.0, filteringONOFF=1, filterALPHA=alpha, filterORDER=order)
    o = oracle_for(oracle, p, geo)
    c, b = o.filter_coeffs()
    j = np.arange(-alpha, alpha + 1)
    for q in range(order + 1):
        assert abs(np.dot(c, j.astype(float) ** q) - (1.0 if q == 0 else 0.0)) < 1e-11 * float(alpha) ** q
    x = np.linspace(-1.0, 1.2, o.Nxg)
    U = 0.3 + x - 0.7 * x ** 2 + 0.2 * x ** order
    F = o.filter(U)
    centred = slice(1 + alpha, o.Nxg - 1 - alpha)
    assert np.max(np.abs(F[centred] - U[centred])) < 1e-9
    assert np.all(np.isfinite(F)) and F[0] == U[0] and F[-1] == U[-1]


def test_relaxation_gamma_profiles(ow3d, oracle):
    """Relaxation ramps of GammaFunctions.f90 over the zone's own x points:
    ftype 9 is 1 - xi^p, ftype 10 is 3 xi^2 - 2 xi^3, and a negative ftype
    reverses the profile."""
    p, geo = cases.flat_2d(Nx=65, Nz=9, L=8.0, relaxONOFF=1, relaxNo=2,
                           zones=[dict(x1=0.0, x2=2.0, ftype=-10, param=3.5, wavegen=1),
                                  dict(x1=6.0, x2=8.0, ftype=9, param=3.5)])
    o = oracle_for(oracle, p, geo)
    x = (np.arange(o.Nxg) - 1) / (p.Nx - 1) * p.Lx
    for z, f in ((0, lambda t: (3 * t ** 2 - 2 * t ** 3)[::-1]), (1, lambda t: 1 - t ** 3.5)):
        i0, i1, _, _ = o.zone_box(z)
        xs = x[i0 - 1:i1]
        t = (xs - xs[0]) / (xs[-1] - xs[0])
        assert np.max(np.abs(o.zone_gamma(z) - f(t))) < 1e-14
