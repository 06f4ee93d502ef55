"""The flux wavemaker of IncWaveType 3 (and 5, with a constant-flux current):
a paddle signal u(t, y) read from a file (setupWavePaddle.f90) imposed on
the west wall (waveGenerationFromPaddleSignal.f90, called from
Runge_Kutta_4.f90:83-85,264-266,385-387): the Neumann rows of every level
above the bottom carry the ramped flux, interpolated linearly in time and
with flux_order points in y; at the end of each step the ghost points of
the surface potential and elevation carry the flux and eta_x = -u_t / g.

CPU: the file reader and the deck line; the oracle's wave generation against
continuity (the volume the wall lets in is the integral of u h); the refusals.
GPU: the device against the device-ordered oracle (1e-10) in a 2-D flume,
with the current of IncWaveType 5, and in 3-D with a signal of 5 points in y
interpolated with 3, direct and captured steps.
"""
import numpy as np
import pytest

import cases
from conftest import reference_decks

G = 9.81


def write_signal(path, dt, y, flux, header="synthetic paddle signal"):
    nt, n2 = flux.shape
    with open(path, "w") as f:
        f.write(header + "\n")
        f.write(f"{dt:.6e} {nt} {n2}\n")
        f.write(" ".join(f"{v:.6e}" for v in y) + "\n")
        for i in range(nt):
            f.write(f"{i * dt:.6e} " + " ".join(f"{v:.15e}" for v in flux[i]) + "\n")


def signal(nt=400, dt=0.02, n2=1, U0=0.01, T=1.25, Ly=1.0):
    t = np.arange(nt) * dt
    y = (np.arange(n2) + 0.5) * (Ly / n2)
    shape = 1.0 + 0.2 * np.cos(np.pi * y / Ly)          # varies across the wall in 3-D
    flux = U0 * np.sin(2 * np.pi * t / T)[:, None] * (shape[None, :] if n2 > 1 else 1.0)
    return dt, y, flux


def test_read_paddle_signal(ow3d, tmp_path):
    dt, y, flux = signal(nt=50, n2=3)
    f = tmp_path / "paddle.dat"
    write_signal(f, dt, y, flux)
    d2, y2, f2 = ow3d.read_paddle_signal(f)
    assert d2 == dt and np.allclose(y2, y, rtol=1e-6) and np.allclose(f2, flux, rtol=1e-14, atol=0)
    with pytest.raises(ow3d.OW3DError):
        ow3d.read_paddle_signal(tmp_path / "missing.dat")
    ref = (reference_decks() or tmp_path / "none") / "Mono2D_T1.25Eps05.wavemaker"
    if ref.exists():
        d3, y3, f3 = ow3d.read_paddle_signal(ref)
        assert (d3, f3.shape, float(y3[0])) == (0.02, (3126, 1), 1.0)


DECK = """flux wavemaker (synthetic)
0 3 1000.
30. 1 0.85 401 1 9 0 0 1 1 1 1
3 3 3 1 1 1
3001 0.02 1 0. 1
9.81
1 3 0 23 1e-8 1e-6 1 V 1 1 2
0.0 0.85 1. 1. 0 0. 1 6 24
0 0
1 0
0 6 10 0.08 0.08 0.4
1 0.0 1 X 0
25. 30. 0. 1. 9 3.5 X 0 X 0.
0 2.0 2 0 0 1 0
0
0 1 Mono2D_T1.25Eps05.wavemaker
"""


def test_deck_flux_wavemaker_line(ow3d, tmp_path):
    f = tmp_path / "fw.inp"
    f.write_text(DECK)
    p = ow3d.read_deck(f)
    assert (p.IncWaveType, p.flux_ramp, p.flux_order, p.flux_file) == (3, 0.0, 1, b"Mono2D_T1.25Eps05.wavemaker")
    assert p.current_flag == 0
    f.write_text(DECK.replace("0 3 1000.", "0 5 1000.") + "0.05\n")
    p = ow3d.read_deck(f)
    assert (p.IncWaveType, p.current_flag, p.current_Q) == (3, 1, 0.05)
    import ctypes as C
    L = ow3d.lib()
    q = ow3d.default_params(Nx=65, Nz=9, Lx=4.0, IncWaveType=3, flux_order=11)
    assert L.ow3d_estimate_bytes(C.byref(q), C.byref(C.c_size_t())) == ow3d.capi.ERR_BAD_INPUT
    q = ow3d.default_params(Nx=65, Nz=9, Lx=4.0, IncWaveType=3, flux_order=1, periodic_x=1)
    assert L.ow3d_estimate_bytes(C.byref(q), C.byref(C.c_size_t())) == ow3d.capi.ERR_BAD_INPUT


def flume(ramp=0.5, order=1, Nx=129, L=8.0, h0=0.5, **kw):
    p, geo = cases.flat_2d(Nx=Nx, Nz=9, L=L, h0=h0, IncWaveType=3, flux_ramp=ramp, flux_order=order, **kw)
    p.g = G
    p.dt = 0.02
    p.Nsteps = 200
    return p, geo


def ramp_fac(t, r):
    return np.where(t < r, -2.0 / r ** 3 * t ** 3 + 3.0 / r ** 2 * t ** 2, 1.0)


def test_oracle_wavemaker_continuity(oracle):
    """The west wall lets in u(t) h per unit width: the elevation's volume
    follows the integral of the ramped flux times the depth."""
    p, geo = flume()
    dt_s, y, flux = signal(nt=400, dt=0.02, n2=1, U0=0.005)
    o = oracle.Oracle(p, geo["h"], mode=oracle.MODE_DEVICE)
    o.set_paddle(dt_s, y, flux)
    o.set_state(np.zeros(o.C), np.zeros(o.C))
    dx = p.Lx / (p.Nx - 1)
    vols, ts = [], []
    for n in range(1, 61):
        assert o.step(1) >= 0
        E = o.get_state()[0]
        vols.append(np.trapezoid(E[1:-1], dx=dx))
        ts.append(n * p.dt)
    tt = np.linspace(0.0, ts[-1], 6001)
    u = 0.005 * np.sin(2 * np.pi * tt / 1.25) * ramp_fac(tt, p.flux_ramp)
    cum = np.concatenate([[0.0], np.cumsum(0.5 * (u[1:] + u[:-1]) * np.diff(tt))]) * 0.5
    want = np.interp(ts, tt, cum)
    err = np.max(np.abs(np.array(vols) - want)) / np.max(np.abs(want))
    assert err < 0.02, err     # 0.7% measured


def test_wavemaker_parameters_accepted(ow3d):
    """A flux-wavemaker deck's parameters pass the checks; the signal is a
    run-time requirement (a handle refuses to step without it, on the GPU)."""
    import ctypes as C
    p, geo = flume()
    assert ow3d.lib().ow3d_estimate_bytes(C.byref(p), C.byref(C.c_size_t())) == 0


# ------------------------------------------------------------------ GPU

def _case(kind):
    if kind == "flume":
        p, geo = flume(ramp=0.5)
        sig = signal(nt=400, n2=1)
    elif kind == "current":
        p, geo = flume(ramp=0.5, current_flag=1, current_Q=0.02)
        sig = signal(nt=400, n2=1)
    else:
        p, geo = cases.bump_3d(Nx=33, Ny=17, Nz=9, Lx=4.0, Ly=1.0, IncWaveType=3, flux_ramp=0.3, flux_order=3)
        p.g = G
        p.dt = 0.02
        p.Nsteps = 100
        sig = signal(nt=200, n2=5, Ly=1.0)
    return p, geo, sig


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [0, 1], ids=["direct", "graphs"])
@pytest.mark.parametrize("kind", ["flume", "current", "3d"])
def test_device_wavemaker_matches_oracle(ow3d, oracle, kind, graphs):
    p, geo, (dt_s, y, flux) = _case(kind)
    o = oracle.Oracle(p, geo["h"], geo.get("hx"), geo.get("hxx"), geo.get("hy"), geo.get("hyy"),
                      mode=oracle.MODE_DEVICE)
    o.set_paddle(dt_s, y, flux)
    sim = ow3d.Simulation(p, **geo)
    with pytest.raises(ow3d.OW3DError):
        sim.step(1)                       # no signal installed yet
    sim.set_paddle_signal(dt_s, y, flux)
    assert ow3d.lib().ow3d_set_graphs(sim.h, graphs) == 0
    Z = np.zeros(sim.C)
    o.set_state(Z, Z)
    sim.set_state(Z, Z)
    assert o.step(30) >= 0 and sim.step(30) >= 0
    for a, b in zip(sim.get_state()[:4], o.get_state()[:4]):
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b)), kind
    assert np.max(np.abs(sim.get_state()[0])) > 1e-4            # a wave was made
