"""Local smoothing by the vertical acceleration of the surface
(LocalSmoothing2D.f90 for x flumes, LocalSmoothing3D.f90 for 3-D grids,
called after every step from OceanWave3DTakeATimeStep.f90:33-39; on for
accel_tol_fact <= 100 of deck line 2).

CPU: the oracle's Lagrangian dw/dt against linear theory (a small standing
wave: dw/dt = -omega^2 eta at the surface), and its filter against a numpy
restatement of the weights and the [a, 1-2a, a] filter applied to the same
run without smoothing (the two runs are the same up to the first smoothed
step, so the smoothed state must be exactly the filtered one).
GPU: the device's dw/dt, flags and state against the device-ordered oracle
over runs where the filter fires (x flume and 3-D), direct and captured steps.
"""
import numpy as np
import pytest

import cases

G = 9.81


def _oracle(oracle, p, geo, E0, P0):
    o = oracle.Oracle(p, geo["h"], geo.get("hx"), geo.get("hxx"), geo.get("hy"), geo.get("hyy"),
                      mode=oracle.MODE_DEVICE)
    o.set_state(E0, P0)
    return o


def test_oracle_acceleration_matches_linear_theory(ow3d, oracle):
    """A standing wave of steepness ka = 1e-3 over kh = 1: the surface's
    vertical acceleration is -omega^2 eta to O((omega dt)^2) and O(ka)."""
    p, geo, E0, P0 = ow3d.workloads.standing_2d(Nx=65, Nz=9, amp=1e-3, accel_tol_fact=100.0)
    p.g = G
    o = _oracle(oracle, p, geo, E0, P0)
    assert o.accel_state() is not None
    k = 2 * np.pi / p.Lx
    om2 = G * k * np.tanh(k * p.Lz)
    for step in range(1, 7):
        o.step(1)
        Wt, cols = o.accel_state()
        if step < 3:
            continue
        E = o.get_state()[0]
        err = np.max(np.abs(Wt[2:-2] + om2 * E[2:-2])) / np.max(np.abs(om2 * E))
        assert err < 1e-2, (step, err)
        assert cols.size == 0                 # 100 g is never reached


def _steep_flume(ow3d, accel):
    W = ow3d.workloads
    p, geo, E0, P0, targets = W.stream_function_2d(n_waves=4, ppw=32, steepness=0.8, steps=12,
                                                   accel_tol_fact=accel)
    return p, geo, E0, P0, targets


def _bump(ow3d, accel):
    p, geo = cases.bump_3d(Nx=33, Ny=17, Nz=9, Lx=2.0, Ly=1.0, accel_tol_fact=accel)
    Nxg, Nyg = p.Nx + 2, p.Ny + 2
    x = (np.arange(Nxg) - 1) / (p.Nx - 1) * p.Lx
    y = (np.arange(Nyg) - 1) / (p.Ny - 1) * p.Ly
    X, Y = np.meshgrid(x, y)
    E0 = (0.06 * np.exp(-((X - 0.8) ** 2 + (Y - 0.5) ** 2) / 0.02)).ravel()
    return p, geo, E0, np.zeros_like(E0), None


def _make(ow3d, case, accel):
    return _steep_flume(ow3d, accel) if case == "flume" else _bump(ow3d, accel)


def _limit_that_fires(ow3d, oracle, case, steps=3):
    """An acceleration limit half the largest -dw/dt of the third step."""
    p, geo, E0, P0, tg = _make(ow3d, case, 100.0)
    o = _oracle(oracle, p, geo, E0, P0)
    if tg:
        o.set_relax_target(0, *tg[0])
    o.step(steps)
    Wt, _ = o.accel_state()
    Wt = Wt.reshape(o.Nyg, o.Nxg)[:, 5:o.Nxg - 5]      # the points the test reads, i = 6..Nxg-5
    return 0.5 * np.max(-Wt) / p.g


@pytest.mark.parametrize("case", ["flume", "bump"])
def test_oracle_filter_is_the_restated_filter(ow3d, oracle, case):
    threads = oracle.set_threads(0)
    oracle.set_threads(1)                     # bitwise reproducible runs
    try:
        fact = _limit_that_fires(ow3d, oracle, case)
        runs = {}
        for name, accel in (("on", fact), ("off", 1000.0)):
            p, geo, E0, P0, tg = _make(ow3d, case, accel)
            o = _oracle(oracle, p, geo, E0, P0)
            if tg:
                o.set_relax_target(0, *tg[0])
            o.step(3)
            runs[name] = o
    finally:
        oracle.set_threads(threads)
    on, off = runs["on"], runs["off"]
    assert off.accel_state() is None
    Wt, cols = on.accel_state()
    Nx, Ny = on.Nxg, on.Nyg
    tol = fact * p.g
    want = [j * Nx + (i - 1) for j in range(Ny) for i in range(6, Nx - 4) if -Wt[j * Nx + i - 1] >= tol]
    assert list(cols) == want and len(want) > 0
    alpha = np.zeros((Ny, Nx))
    for c in want:
        j, i = divmod(c, Nx)
        alpha[j, i - 5:i + 6] = 0.25
    Eo, Po = off.get_state()[:2]
    for got, f in ((on.get_state()[0], Eo), (on.get_state()[1], Po)):
        f = f.reshape(Ny, Nx)
        ref = f.copy()
        a = alpha[:, 1:-1]
        ref[:, 1:-1] = a * f[:, :-2] + (1.0 - 2.0 * a) * f[:, 1:-1] + a * f[:, 2:]
        assert np.array_equal(got, ref.ravel())


def test_smoothing_parameters(ow3d):
    import ctypes as C
    L = ow3d.lib()
    b = C.c_size_t()
    q = ow3d.default_params(Nx=65, Nz=9, Lx=2.0, accel_tol_fact=0.5)
    assert L.ow3d_estimate_bytes(C.byref(q), C.byref(b)) == 0
    q = ow3d.default_params(Nx=65, Nz=9, Lx=2.0, accel_tol_fact=0.5, periodic_x=1)
    assert L.ow3d_estimate_bytes(C.byref(q), C.byref(b)) == ow3d.capi.ERR_BAD_INPUT


# ------------------------------------------------------------------ GPU

@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [0, 1], ids=["direct", "graphs"])
@pytest.mark.parametrize("case", ["flume", "bump"])
def test_device_smoothing_matches_oracle(ow3d, oracle, case, graphs):
    fact = _limit_that_fires(ow3d, oracle, case)
    p, geo, E0, P0, tg = _make(ow3d, case, fact)
    o = _oracle(oracle, p, geo, E0, P0)
    sim = ow3d.Simulation(p, **geo)
    assert ow3d.lib().ow3d_set_graphs(sim.h, graphs) == 0
    sim.set_state(E0, P0)
    if tg:
        o.set_relax_target(0, *tg[0])
        sim.set_relax_target(0, *tg[0])
    fired = 0
    for step in range(1, 9):
        assert o.step(1) >= 0 and sim.step(1) >= 0
        if step < 3:
            continue
        Wo, co = o.accel_state()
        Wd, cd = sim.accel_state()
        assert np.max(np.abs(Wd - Wo)) <= 1e-9 * np.max(np.abs(Wo)), step
        assert np.array_equal(cd, co), step
        fired += len(co)
    assert fired > 0
    for a, b in zip(sim.get_state()[:4], o.get_state()[:4]):
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b))
