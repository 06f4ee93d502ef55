"""Parity of the CUDA path with the CPU oracle (device-matched mode) on the
benchmark configurations' own grids, a few time steps each:

* the 3-D shoal basin at its full 257 x 33 x 9 grid, with the incident-wave
  generation zone (0-3 m) and the sponge (30-35 m), FP64;
* the 2-D x-sigma wave at 65 x 9 (one wavelength, kh = 1, steep), FP64;
* a 129 x 33 x 17 sub-basin of the irregular sea (same dx, Nz and spectrum),
  FP64 and mixed precision;
* the 2-D stream-function wave (kh = 1, half the breaking steepness) in a
  flume with stream-function generation and a sponge, 257 x 9, FP64.

Tolerances as in test_gpu_parity: 1e-10 relative L-infinity on eta, P and phi
for FP64 (reduction order and fused multiply-adds only), iteration totals
within one per solve; 1e-6 on eta for the mixed path against the FP64 oracle.
"""
import numpy as np
import pytest

import cases  # noqa: F401  (puts tests/ on the path for the package loader)

pytestmark = pytest.mark.gpu

RTOL_RUN = 1e-10


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _compare(sim, orc, tol=RTOL_RUN, phi_tol=None):
    E, P, W, phi, t = sim.get_state()
    Eo, Po, Wo, phio, to = orc.get_state()
    assert abs(t - to) < 1e-12
    assert rel(E, Eo) < tol, rel(E, Eo)
    assert rel(P, Po) < tol, rel(P, Po)
    assert rel(phi, phio) < (phi_tol or tol), rel(phi, phio)
    return E, Eo


def _iterations_match(sim, orc):
    s, so = sim.stats(), orc.stats()
    assert s["solves"] == so["solves"]
    assert abs(s["total_iterations"] - so["total_iterations"]) <= s["solves"], (s, so)


def test_shoal_257x33x9_generation_and_sponge(ow3d, oracle):
    W = ow3d.workloads
    zones = [dict(x1=0.0, x2=3.0, y1=0.0, y2=6.0, ftype=-10, param=3.5, wavegen=1),
             dict(x1=30.0, x2=35.0, y1=0.0, y2=6.0, ftype=9, param=3.5)]
    p, geo = W.shoal(relaxONOFF=1, relaxNo=2, relaxTransientTime=1.0, zones=zones)
    nsteps = 4
    sim = ow3d.Simulation(p, **geo)
    orc = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    # linear regular incident wave, T = 1 s, H = 0.01 m, at the 0.45 m depth
    i0, i1, j0, j1 = sim.zone_box(0)
    x, _ = W.grid_xy(p)
    xs = x[i0 - 1:i1]
    T, H, h = 1.0, 0.01, 0.45
    om = 2 * np.pi / T
    k = W.dispersion_k(om, h)
    nt = 2 * nsteps + 2
    tt = np.arange(nt) * (0.5 * p.dt)
    ny = j1 - j0 + 1
    eta = np.array([np.tile(0.5 * H * np.cos(k * xs - om * t), ny) for t in tt])
    phis = np.array([np.tile(0.5 * H * W.G / om * np.sin(k * xs - om * t), ny) for t in tt])
    for s in (sim, orc):
        s.set_relax_target(0, 0, nt, 0.5 * p.dt, eta, phis)
        s.set_state(np.zeros(sim.C), np.zeros(sim.C))
    assert sim.step(nsteps) >= 0
    assert orc.step(nsteps) >= 0
    E, Eo = _compare(sim, orc)
    assert np.max(np.abs(Eo)) > 1e-5          # the wave has entered the basin
    _iterations_match(sim, orc)


def test_wave_2d_65x9_steep(ow3d, oracle):
    W = ow3d.workloads
    p, geo, E0, P0 = W.standing_2d(Nx=65, Nz=9, amp=0.08)
    sim = ow3d.Simulation(p, **geo)
    orc = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    sim.set_state(E0, P0)
    orc.set_state(E0, P0)
    assert sim.step(20) >= 0
    assert orc.step(20) >= 0
    _compare(sim, orc)
    _iterations_match(sim, orc)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_irregular_sea_129x33x17(ow3d, oracle, precision):
    W = ow3d.workloads
    p, geo, E0, P0 = W.irregular_sea(Nx=129, Ny=33, Nz=17, precision=precision, seed=7)
    q, geo_o, _, _ = W.irregular_sea(Nx=129, Ny=33, Nz=17, precision=0, seed=7)
    sim = ow3d.Simulation(p, **geo)
    orc = oracle.Oracle(q, **geo_o, mode=oracle.MODE_DEVICE)
    sim.set_state(E0, P0)
    orc.set_state(E0, P0)
    assert sim.step(3) >= 0
    assert orc.step(3) >= 0
    if precision == 0:
        _compare(sim, orc)
        _iterations_match(sim, orc)
    else:
        # FP32 preconditioner inside FP64 FGMRES: eta within 1e-6 of the FP64 oracle
        _compare(sim, orc, tol=1e-6)


def test_stream_function_flume_2d(ow3d, oracle):
    """The 2-D stream-function case (kh = 1, H/L half the breaking limit, 32
    points per wavelength, 9 sigma levels) as the reference can run it: the
    wave over the flume at t = 0, generated in the first wavelength from
    targets at every RK stage time (mode 1), absorbed in the last three."""
    W = ow3d.workloads
    p, geo, E0, P0, targets = W.stream_function_2d(ppw=32, steps=12)
    sim = ow3d.Simulation(p, **geo)
    orc = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    for s in (sim, orc):
        s.set_state(E0, P0)
        s.set_relax_target(0, *targets[0])
    assert sim.step(12) >= 0
    assert orc.step(12) >= 0
    _compare(sim, orc)
    _iterations_match(sim, orc)
