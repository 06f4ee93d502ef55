"""Periodic lateral boundary in x (params.periodic_x): the 2-D stream-function
wave of the first benchmark configuration -- one wavelength (kh = 1, depth
1 m, half the breaking steepness) with Nx = 65 points including both ends, 9
sigma levels, RK4 at Courant 0.5 for 200 steps, GMRES reltol 1e-8.

The reference has no periodic boundary (its lateral rows are walls,
BuildLinearSystem.f90:149-216, and its ghost-layer update is
UpdateGhostLayerX.f90:15,20); the oracle and the device implement the same
periodic form: distinct columns 2..Nxg-2 coupled cyclically in every stencil
(operator, smoother, residual, restriction, prolongation, surface
derivatives, filter), the ghost columns and the repeated column Nxg-1 as
identity rows that stay zero inside the solves, and image columns filled for
the surface fields and on output.

CPU: the oracle against exact answers -- a periodic harmonic potential, and
the steady stream-function wave translating at its phase speed -- plus the
parameter checks. GPU: the device against the oracle (1e-12 on the operator,
1e-10 on the preconditioner and after the 200 steps, matvec counts within
one per solve) and against the translated wave.
"""
import ctypes as C

import numpy as np
import pytest

import cases  # noqa: F401


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _xgrid(p, Nxg):
    return (np.arange(Nxg) - 1) * (p.Lx / (p.Nx - 1))


def _translation_errors(ow3d, p, E, P, t, Nxg):
    """Distance of (E, P) from the exact wave translated to time t: E in units
    of the wave height; P relative, after removing its mean offset (the
    Bernoulli constant makes the surface potential drift by a constant)."""
    x = _xgrid(p, Nxg)
    Ee, Pe, _ = ow3d.stream_function_wave(p, x, t)
    d = (P - Pe)[1:-2]
    return float(np.max(np.abs(E - Ee)) / p.sf_H), float(np.max(np.abs(d - d.mean())) / np.max(np.abs(Pe)))


@pytest.mark.parametrize("mode", [0, 1], ids=["reference_ordering", "device_ordering"])
def test_oracle_periodic_wave_translates(ow3d, oracle, mode):
    """200 steps (about 1.6 periods) of the steep periodic wave: the surface
    stays the exactly translated wave to within 1% of its height."""
    p, geo, E0, P0, info = ow3d.workloads.periodic_wave_2d()
    o = oracle.Oracle(p, **geo, mode=mode)
    o.set_state(E0, P0)
    assert o.step(200) >= 0
    E, P, W, phi, t = o.get_state()
    eE, eP = _translation_errors(ow3d, p, E, P, t, o.Nxg)
    assert eE < 0.01 and eP < 0.01, (eE, eP)
    # image columns: 1 <- Nxg-2, Nxg-1 <- 2, Nxg <- 3 (on E, P, W and phi)
    n, Nz = o.Nxg, o.Nzg
    for f in (E, P, W):
        assert f[0] == f[n - 3] and f[n - 2] == f[1] and f[n - 1] == f[2]
    ph = phi.reshape(n, Nz)
    assert np.array_equal(ph[0], ph[n - 3]) and np.array_equal(ph[n - 2], ph[1])


def test_oracle_periodic_harmonic_solve(ow3d, oracle):
    """phi = cosh(k(z+h)) cos(kx) / cosh(kh), harmonic and periodic, from its
    free-surface values with the kinematic bottom condition: the solve
    recovers it to the 6th-order truncation error."""
    p, geo, E0, P0, info = ow3d.workloads.periodic_wave_2d(Nx=65, Nz=17)
    p.reltol, p.abstol = 1e-12, 0.0
    o = oracle.Oracle(p, **geo, mode=1)
    n, Nz = o.Nxg, o.Nzg
    x = _xgrid(p, n)
    z = o.fine_z()
    k = 2 * np.pi / p.Lx
    h = 1.0
    exact = np.cosh(k * (z[None, :] * h - h + h)) * np.cos(k * x[:, None]) / np.cosh(k * h)   # sigma: z = sigma h - h
    rhs = np.zeros((n, Nz))
    rhs[1:n - 2, -1] = exact[1:n - 2, -1]
    sol, it, res, st = o.solve(rhs.ravel(), np.zeros(o.N))
    s = sol.reshape(n, Nz)
    err = np.max(np.abs(s[1:n - 2, 1:] - exact[1:n - 2, 1:]))
    assert err < 1e-6, err
    # identity rows of the image columns stay zero inside the solve
    assert np.all(s[0] == 0) and np.all(s[n - 2] == 0) and np.all(s[n - 1] == 0)


def test_periodic_params_checked(ow3d):
    L = ow3d.lib()
    b = C.c_size_t()
    p, geo, E0, P0, info = ow3d.workloads.periodic_wave_2d()
    assert L.ow3d_estimate_bytes(C.byref(p), C.byref(b)) == 0
    q = ow3d.default_params(Nx=5, Nz=9, periodic_x=1)
    assert L.ow3d_estimate_bytes(C.byref(q), C.byref(b)) == ow3d.capi.ERR_BAD_INPUT
    q = ow3d.default_params(Nx=65, Nz=9, periodic_x=1, iKinematics=1, nOutFiles=1)
    assert L.ow3d_estimate_bytes(C.byref(q), C.byref(b)) == ow3d.capi.ERR_BAD_INPUT
    assert b"periodic_x" in L.ow3d_last_error()


def test_periodic_sloping_bottom_refused(ow3d):
    """The periodic multigrid levels carry no mixed-derivative terms: a
    bottom with h_x != 0 is refused before any device work."""
    L = ow3d.lib()
    p, geo, E0, P0, info = ow3d.workloads.periodic_wave_2d()
    Nxg, Nyg, _ = ow3d.dims(p)
    h = np.ones(Nxg * Nyg)
    hx = np.full(Nxg * Nyg, 0.01)
    d = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    out = C.c_void_p()
    assert L.ow3d_create(C.byref(p), d(h), d(hx), None, None, None, C.byref(out)) == ow3d.capi.ERR_UNSUPPORTED
    assert b"flat bottom" in L.ow3d_last_error()


# ----------------------------------------------------------------- device


@pytest.mark.gpu
def test_periodic_operator_and_preconditioner_match_oracle(ow3d, oracle):
    p, geo, E0, P0, info = ow3d.workloads.periodic_wave_2d()
    sim = ow3d.Simulation(p, **geo)
    o = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    n, Nz = sim.Nxg, sim.Nzg
    rng = np.random.default_rng(5)
    phi = rng.standard_normal((n, Nz))
    phi[[0, n - 2, n - 1]] = 0.0
    x = _xgrid(p, n)
    k = 2 * np.pi / p.Lx
    E = 0.05 * np.cos(k * x); Ex = -0.05 * k * np.sin(k * x); Exx = -0.05 * k * k * np.cos(k * x)
    o.set_surface(E, Ex, Exx)
    assert rel(sim.matvec(phi.ravel(), E, Ex, Exx), o.matvec(phi.ravel())) < 1e-12
    r = rng.standard_normal((n, Nz))
    r[[0, n - 2, n - 1]] = 0.0
    assert rel(sim.precondition(r.ravel()), o.precond(r.ravel())) < 1e-10


@pytest.mark.gpu
def test_periodic_wave_200_steps_matches_oracle(ow3d, oracle):
    """The first benchmark configuration as specified (periodic, 65 x 9, 200
    RK4 steps, FP64) against the device-ordered oracle: 1e-10 on eta, P and
    phi after the whole run, matvec counts within one per solve; and within
    1% of the wave height of the exactly translated wave."""
    p, geo, E0, P0, info = ow3d.workloads.periodic_wave_2d()
    sim = ow3d.Simulation(p, **geo)
    o = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    for s in (sim, o):
        s.set_state(E0, P0)
    its = cases.run_steps(sim, 200)
    its_o = cases.run_steps(o, 200)
    E, P, W, phi, t = sim.get_state()
    Eo, Po, Wo, phio, to = o.get_state()
    assert abs(t - to) < 1e-12
    errs = {"E": rel(E, Eo), "P": rel(P, Po), "phi": rel(phi, phio), "W": rel(W, Wo)}
    assert max(errs.values()) < 1e-10, errs
    assert np.all(np.abs(its - its_o) <= 4), (its - its_o)
    eE, eP = _translation_errors(ow3d, p, E, P, t, sim.Nxg)
    assert eE < 0.01 and eP < 0.01, (eE, eP)
