"""The constant-flux current of IncWaveType 4 (ReadInputFileParameters.f90:42-49,
655-690; OceanWave3DT0Setup.f90:325-326; Runge_Kutta_4.f90:82-88,108-113):
u = Q/h on the west and east walls' Neumann rows and in the surface
potential's ghost points.

CPU: the deck reading (4 becomes the stream-function wave 1 with the current
flag, and the flux Q from the line after the curvilinear line), the
refusals, and the oracle's uniform current: eta = -U^2 / (2g), phi = U x is
kept by the scheme with the current on (to the small waves of the first
step) and not without it.
GPU: the device against the device-ordered oracle on that state and on a
stream-function wave riding the current (1e-10), direct and captured steps.
"""
import numpy as np
import pytest

import cases

DECK = """stream-function wave on a following current (synthetic)
-1  4 1000.
10. 1. 0.5 641 1 10 0 0 1 1 1 1
3 3 3 1 1 1
5121 .2 1 0.5 1
9.81
1 1 0 23 1e-8 1e-6 1 V 1 1 2
.08 0.5 1. .7206986 0  0.1 0 6 32
-256  20 1 1
1 641 1 1 1 1 1 5121 1
1 0
1 6 10 0.08 0.08 0.4
1 0. 2 X 0
0.    1.  0. 1.  9 3.5 X 1 X 0. 1
1.    2.  0. 1. 10 3.5 X 1 X 0. 1
1  1
9. 10. 0. 0. 1. 1. 0
0 2.0 2 0 0 1 0
0
0.05
"""


def test_deck_current_line(ow3d, tmp_path):
    f = tmp_path / "c.inp"
    f.write_text(DECK)
    p = ow3d.read_deck(f)
    assert (p.IncWaveType, p.current_flag, p.current_Q) == (1, 1, 0.05)
    assert (p.sf_H, p.sf_h, p.sf_uEorS) == (0.08, 0.5, 0.1)
    f.write_text(DECK.replace("-1  4 1000.", "-1  1 1000."))
    p = ow3d.read_deck(f)
    assert (p.IncWaveType, p.current_flag, p.current_Q) == (1, 0, 0.0)
    # IncWaveType 5: the flux wavemaker (3) with a current; the wavemaker's
    # line comes first, then the flux (tests/test_flux_wavemaker.py)
    import ctypes as C
    f.write_text(DECK.replace("-1  4 1000.", "-1  5 1000.").replace("0\n0.05\n", "0\n3. 4 paddle.dat\n0.05\n"))
    p = ow3d.read_deck(f)
    assert (p.IncWaveType, p.current_flag, p.current_Q, p.flux_order) == (3, 1, 0.05, 4)
    assert ow3d.lib().ow3d_estimate_bytes(C.byref(p), C.byref(C.c_size_t())) == 0
    q = ow3d.default_params(Nx=65, Nz=9, Lx=2.0, periodic_x=1, current_flag=1, current_Q=0.1)
    assert ow3d.lib().ow3d_estimate_bytes(C.byref(q), C.byref(C.c_size_t())) == ow3d.capi.ERR_BAD_INPUT


def uniform_current(U=0.2, h0=0.5, Nx=65, L=4.0, on=True, **kw):
    p, geo = cases.flat_2d(Nx=Nx, Nz=9, L=L, h0=h0, current_flag=1 if on else 0, current_Q=U * h0 if on else 0.0,
                           **kw)
    p.dt = 0.5 * (L / (Nx - 1)) / np.sqrt(9.81 * h0)
    x = (np.arange(Nx + 2) - 1) * (L / (Nx - 1))
    E0 = np.full(Nx + 2, -U * U / (2 * p.g))
    P0 = U * x
    return p, geo, E0, P0


@pytest.mark.parametrize("on", [True, False], ids=["current", "walls"])
def test_oracle_uniform_current_is_steady(oracle, on):
    """The uniform current eta = -U^2/(2g), phi = U x is a steady state of the
    scheme with the current's wall fluxes: it only sheds the small waves of
    the first step, whose surface derivatives the set-up takes with a zero
    ghost source as the reference's does (OceanWave3DT0Setup.f90:444, the
    source is still zero there). With closed walls the flow must stop and
    the state departs by orders of magnitude more."""
    U = 0.2
    p, geo, E0, P0 = uniform_current(U=U, on=on)
    o = oracle.Oracle(p, geo["h"], mode=oracle.MODE_DEVICE)
    o.set_state(E0, P0)
    assert o.step(20) >= 0
    E, P = o.get_state()[:2]
    dev = max(np.max(np.abs(E[1:-1] - E0[1:-1])), np.max(np.abs(P[1:-1] - P0[1:-1])) / U)
    if on:
        assert dev < 2e-3, dev
    else:
        assert dev > 3e-2, dev


DAMP = dict(PDampingONOFF=1, NDampZones=1, pd_type=0, pd_x0=3.0, pd_x1=4.0, pd_y0=0.0, pd_y1=1.0,
            pd_g0Phi=1.0, pd_g0Eta=0.0)


def test_oracle_pressure_damping_acts_relative_to_the_current(oracle):
    """funPressureTerm.f90:249-252 damps the velocity relative to the
    current: the uniform current passes a pressure-damping zone unchanged
    (to the small waves of the first step), where damping the whole velocity
    would brake it."""
    U = 0.2
    p, geo, E0, P0 = uniform_current(U=U, **DAMP)
    o = oracle.Oracle(p, geo["h"], mode=oracle.MODE_DEVICE)
    o.set_state(E0, P0)
    assert o.step(20) >= 0
    E, P = o.get_state()[:2]
    dev = max(np.max(np.abs(E[1:-1] - E0[1:-1])), np.max(np.abs(P[1:-1] - P0[1:-1])) / U)
    assert dev < 1e-2, dev     # 3.5e-3 measured; damping the whole velocity gives 0.99


def sf_on_current(ow3d, U=0.1, steps=20, krylov=0):
    W = ow3d.workloads
    p, geo, E0, P0, targets = W.stream_function_2d(n_waves=4, ppw=32, steps=steps, krylov=krylov)
    # the same wave with a mean Eulerian current U, and the current's flux
    p.sf_uEorS = U
    p.sf_euler_or_stokes = 0
    p.current_flag = 1
    p.current_Q = U * p.sf_h
    Nxg = p.Nx + 2
    x = (np.arange(Nxg) - 1) * (p.Lx / (p.Nx - 1))
    E0, P0, _ = ow3d.stream_function_wave(p, x, 0.0)
    mode, nt, dts, _, _ = targets[0]
    i0, i1 = 2, 2 + 32
    tt = np.arange(nt) * dts
    eta = np.array([ow3d.stream_function_wave(p, x[i0 - 1:i1], t)[0] for t in tt])
    phis = np.array([ow3d.stream_function_wave(p, x[i0 - 1:i1], t)[1] for t in tt])
    return p, geo, E0, P0, (mode, nt, dts, eta, phis)


def test_oracle_wave_on_current_runs(ow3d, oracle):
    p, geo, E0, P0, tg = sf_on_current(ow3d)
    o = oracle.Oracle(p, geo["h"], mode=oracle.MODE_DEVICE)
    o.set_state(E0, P0)
    o.set_relax_target(0, *tg)
    assert o.step(20) >= 0
    E = o.get_state()[0]
    assert np.all(np.isfinite(E)) and np.max(np.abs(E)) < 2 * p.sf_H


# ------------------------------------------------------------------ GPU

@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [0, 1], ids=["direct", "graphs"])
def test_device_current_matches_oracle(ow3d, oracle, graphs):
    for case in ("uniform", "damped", "wave"):
        if case in ("uniform", "damped"):
            p, geo, E0, P0 = uniform_current(**(DAMP if case == "damped" else {}))
            tg = None
        else:
            p, geo, E0, P0, tg = sf_on_current(ow3d)
        o = oracle.Oracle(p, geo["h"], mode=oracle.MODE_DEVICE)
        sim = ow3d.Simulation(p, **geo)
        assert ow3d.lib().ow3d_set_graphs(sim.h, graphs) == 0
        o.set_state(E0, P0)
        sim.set_state(E0, P0)
        if tg:
            o.set_relax_target(0, *tg)
            sim.set_relax_target(0, *tg)
        assert o.step(20) >= 0 and sim.step(20) >= 0
        # interior columns: the ghost columns' W and phi are the Neumann rows'
        # unknowns, where the nonzero wall flux leaves the two solves' tolerance-
        # level differences larger relative to the small interior W
        Nz = sim.Nzg
        for name, a, b in zip("EPW", sim.get_state()[:3], o.get_state()[:3]):
            assert np.max(np.abs(a - b)[1:-1]) <= 1e-10 * np.max(np.abs(b)), (case, name)
        a, b = sim.get_state()[3].reshape(-1, Nz)[1:-1], o.get_state()[3].reshape(-1, Nz)[1:-1]
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b)), (case, "phi")
