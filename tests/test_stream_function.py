"""Stream-function wave of IncWaveType 1 (ow3d_stream_function_wave): the
reference's Fenton solution, host-only.

Pinned by theory: the linear limit (Airy dispersion and profile), the
third-order Stokes phase speed c^2 = g/k tanh(kd) (1 + (ka)^2 (9 - 10 s^2 +
9 s^4) / (8 s^4)), s = tanh(kd), which the solution must follow up to
(ka)^4 terms; and exact properties of a steady wave: crest-to-trough height,
zero mean elevation, translation at the phase speed. The reference's
example decks with IncWaveType 1 all solve.
"""
import os
import pathlib

import numpy as np
import pytest
from conftest import reference_decks


def _params(ow3d, kd, kH, nmodes=20, nsteps=4, period=None):
    p = ow3d.default_params(Nx=65, Nz=9, Lx=2 * np.pi, Ly=1.0, Lz=kd)
    p.g = 9.81
    p.sf_h, p.sf_L, p.sf_H = kd, 2 * np.pi, kH
    p.sf_wavel_or_per, p.sf_nsteps, p.sf_nmodes = 0, nsteps, nmodes
    if period is not None:
        p.sf_wavel_or_per, p.sf_T = 1, period
    return p


def test_line_8_parsed(ow3d, tmp_path):
    from test_deck import DECK_3D
    f = tmp_path / "a.inp"
    f.write_text(DECK_3D)
    p = ow3d.read_deck(f)
    assert (p.sf_H, p.sf_h, p.sf_L, p.sf_T) == (0.1, 1.0, 3.0, 2.0)
    assert (p.sf_wavel_or_per, p.sf_uEorS, p.sf_euler_or_stokes, p.sf_nsteps, p.sf_nmodes) == (0, 0.0, 1, 6, 24)


def test_linear_limit(ow3d):
    p = _params(ow3d, 1.0, 1e-5)
    x = np.linspace(0, 2 * np.pi, 41)
    t = 0.37
    eta, phis, (k, L, T, c) = ow3d.stream_function_wave(p, x, t)
    om = np.sqrt(p.g * np.tanh(1.0))
    assert abs(T - 2 * np.pi / om) < 1e-9 * T and abs(c - L / T) < 1e-12 * c and k == 1.0
    a = 0.5e-5
    assert np.max(np.abs(eta - a * np.cos(x - om * t))) < 1e-3 * a
    # the surface potential of the linear wave, g/omega a sin(kx - omega t)
    assert np.max(np.abs(phis - p.g / om * a * np.sin(x - om * t))) < 1e-3 * p.g / om * a


@pytest.mark.parametrize("kd,ka", [(3.0, 0.1), (1.0, 0.05), (3.0, 0.05)])
def test_stokes_third_order_phase_speed(ow3d, kd, ka):
    _, _, (k, L, T, c) = ow3d.stream_function_wave(_params(ow3d, kd, 2 * ka), np.zeros(1))
    s = np.tanh(kd)
    c0 = np.sqrt(9.81 * s)
    pred = 1 + 0.5 * ka ** 2 * (9 - 10 * s ** 2 + 9 * s ** 4) / (8 * s ** 4)
    assert abs(c / c0 - pred) < 3 * ka ** 4


def test_steep_wave_exact_properties(ow3d):
    """kd = 1 and H/L at half the breaking limit (about 0.054 at kd = 1):
    height, mean level and steady translation."""
    p = _params(ow3d, 1.0, 0.054 * 2 * np.pi, nmodes=24, nsteps=6)
    H = p.sf_H
    x = np.linspace(0, 2 * np.pi, 257)[:-1]
    eta, phis, (k, L, T, c) = ow3d.stream_function_wave(p, x, 0.0)
    crest, trough = ow3d.stream_function_wave(p, np.array([0.0, np.pi]), 0.0)[0]
    assert abs((crest - trough) - H) < 1e-10 * H
    assert abs(eta.mean()) < 1e-12 * H
    assert crest > 0.55 * H and -trough < 0.45 * H          # crests sharper than troughs
    t = 0.3
    eta_t, _, _ = ow3d.stream_function_wave(p, x + c * t, t)
    assert np.max(np.abs(eta_t - eta)) < 1e-10 * H


def test_period_given(ow3d):
    """With the period given (WAVELorPER = 1) the wavelength follows from the
    solution; in the linear limit it is the Airy wavelength."""
    om = 2 * np.pi / 2.0
    p = _params(ow3d, 1.0, 1e-5, period=2.0)
    _, _, (k, L, T, c) = ow3d.stream_function_wave(p, np.zeros(1))
    assert T == 2.0 and abs(om ** 2 - p.g * k * np.tanh(k * p.sf_h)) < 1e-6 * om ** 2
    assert abs(c - L / T) < 1e-12 * c


def test_errors(ow3d):
    p = _params(ow3d, 1.0, 0.1, nmodes=1)
    with pytest.raises(ow3d.OW3DError, match="Fourier modes"):
        ow3d.stream_function_wave(p, np.zeros(3))


REF_DECKS = reference_decks() or pathlib.Path("/nonexistent")


@pytest.mark.skipif(not REF_DECKS.is_dir(), reason="reference example decks not on this machine")
def test_reference_stream_function_decks_solve(ow3d):
    solved = 0
    for f in sorted(REF_DECKS.iterdir()):
        if not f.name.startswith("OceanWave3D.inp"):
            continue
        try:
            p = ow3d.read_deck(f)
        except ow3d.OW3DError:
            continue
        if p.IncWaveType != 1:
            continue
        L = ow3d.stream_function_wave(p, np.zeros(1))[2][1]     # the solution's wavelength
        x = np.linspace(0, L, 257)
        eta, phis, (k, L, T, c) = ow3d.stream_function_wave(p, x)
        assert abs((eta.max() - eta.min()) - p.sf_H) < 1e-3 * p.sf_H, f.name
        assert np.all(np.isfinite(phis)) and abs(c - L / T) < 1e-12 * c, f.name
        solved += 1
    assert solved >= 3


def test_flume_propagation_oracle(ow3d, oracle):
    """The 2-D stream-function case (workloads.stream_function_2d: the wave
    over the flume at t = 0, generated in the first wavelength with
    relaxation targets of mode 1, absorbed in the last three) stepped one
    period by the oracle: over the second to fourth wavelengths the
    elevation stays within 3% of H of the exact translating wave, and inside
    the generation zone within 0.5% (the exact wave is steady in its own
    frame, so any other change is the flume's error)."""
    W = ow3d.workloads
    ppw = 32
    steps = 2 * ppw                                    # Courant 0.5: one period
    p, geo, E0, P0, targets = W.stream_function_2d(ppw=ppw, steps=steps)
    orc = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    assert orc.zone_box(0) == (2, 2 + ppw, 1, 1)
    orc.set_state(E0, P0)
    orc.set_relax_target(0, *targets[0])
    assert orc.step(steps) >= 0
    E, P, W_, phi, t = orc.get_state()
    x = (np.arange(p.Nx + 2) - 1) * p.Lx / (p.Nx - 1)
    Ee, Pe, (k, L, T, c) = ow3d.stream_function_wave(p, x, t)
    assert abs(t - T) < 0.02 * T
    mid = (x >= L) & (x <= 4 * L)
    gen = (x >= 0) & (x <= 0.5 * L)
    assert np.max(np.abs(E[mid] - Ee[mid])) < 0.03 * p.sf_H
    assert np.max(np.abs(E[gen] - Ee[gen])) < 0.005 * p.sf_H


def test_initial_conditions(ow3d):
    """ow3d_initial_condition for the ICs built from formulas
    (SetupInitialConditions.f90): 4 and 5 (cosine surface on flat deep and
    shallow water), 7 (the stream-function wave over the basin, the sponge's
    weights applied three times), 0 (still water) and an unsupported one."""
    W = ow3d.workloads
    p = ow3d.default_params(Nx=33, Nz=9, Lx=4.0, Ly=1.0, Lz=1.0)
    x = (np.arange(p.Nx + 2) - 1) * p.Lx / (p.Nx - 1)
    for ic, kh, hh in ((4, 2 * np.pi, p.Lx / 10), (5, 0.5, None)):
        p.IC = ic
        geo, E, P = ow3d.initial_condition(p)
        kw = 2 * np.pi / p.Lx
        depth = kh / kw
        H = hh if hh is not None else 0.75 * depth
        assert np.allclose(geo["h"], depth, rtol=1e-15) and not geo["hx"].any()
        assert np.allclose(E, H / 2 * np.cos(kw * x), rtol=0, atol=1e-15 * H) and not P.any()
    p.IC = 0
    geo, E, P = ow3d.initial_condition(p)
    assert np.all(geo["h"] == 1.0) and not E.any() and not P.any()
    p.IC = 2
    with pytest.raises(ow3d.OW3DError) as e:
        ow3d.initial_condition(p)
    assert e.value.status == ow3d.capi.ERR_UNSUPPORTED
    # IC 7 on the stream-function flume: the wave everywhere, damped in the sponge
    q, geo_w, E0, P0, _ = W.stream_function_2d(ppw=32, steps=2)
    q.IC = 7
    geo, E, P = ow3d.initial_condition(q)
    assert np.all(geo["h"] == q.sf_h)
    xq = (np.arange(q.Nx + 2) - 1) * q.Lx / (q.Nx - 1)
    Ee, Pe, _ = ow3d.stream_function_wave(q, xq, q.time0)
    L = q.sf_L
    free = xq < (8 - 3) * L
    assert np.array_equal(E[free], Ee[free]) and np.array_equal(P[free], Pe[free])
    sponge = xq > 5.5 * L
    assert np.max(np.abs(E[sponge])) < np.max(np.abs(Ee[sponge]))
    q.relaxONOFF = 0
    geo, E, P = ow3d.initial_condition(q)
    assert not E.any() and not P.any()                  # the reference sets the wave only with relaxation on


def test_initial_conditions_standing_wave_and_whalin(ow3d):
    """IC 1 (nonlinearstandingwave1D.f90: h = 2 and the eight-term series with
    the reference's single-precision coefficients) and IC 3 (bottomWhalin.f90:
    the shoal's depth and slopes; the x-long basin compares with the
    single-precision 10.67 and 18.29)."""
    p = ow3d.default_params(Nx=65, Nz=9, Lx=2.0, Ly=1.0, Lz=2.0)
    p.IC = 1
    geo, E, P = ow3d.initial_condition(p)
    x = (np.arange(p.Nx + 2) - 1) * p.Lx / (p.Nx - 1)
    a = [0.8867 * float(np.float32(0.1))] + [
        np.sqrt(np.sqrt(n + 1)) * float(np.float32(c)) * float(np.float32(1) / np.float32(10.0 ** e))
        for n, (c, e) in enumerate(zip([0.5243, 0.4978, 0.6542, 0.1007, 0.1653, 0.2753, 0.4522],
                                       [2, 3, 4, 4, 5, 6, 7]), start=1)]
    want = 0.5 * sum(a[n] * np.cos((n + 1) * np.pi * x) for n in range(8))
    assert np.all(geo["h"] == 2.0) and np.max(np.abs(E - want)) < 1e-15 and not P.any()
    q = ow3d.default_params(Nx=129, Ny=17, Nz=9, Lx=35.0, Ly=3.048, Lz=0.4572)   # the reference's Whalin basin (Nz 9)
    q.IC = 3
    geo, E, P = ow3d.initial_condition(q)
    xg = (np.arange(q.Nx + 2) - 1) * q.Lx / (q.Nx - 1)
    yg = (np.arange(q.Ny + 2) - 1) * q.Ly / (q.Ny - 1)
    h = geo["h"].reshape(q.Ny + 2, q.Nx + 2)
    hx = geo["hx"].reshape(q.Ny + 2, q.Nx + 2)
    y0 = (yg[1] - yg[0]) / 2
    for j in (1, 9, 18):
        y = max(yg[j], y0)
        s = np.sqrt(6.096 * y - y * y)
        for i in range(q.Nx + 2):
            if xg[i] <= float(np.float32(10.67)) - s:
                assert h[j, i] == 0.4572 and hx[j, i] == 0.0
            elif xg[i] >= float(np.float32(18.29)) - s:
                assert h[j, i] == 0.1524
            else:
                assert abs(h[j, i] - (0.4572 + 0.04 * (10.67 - s - xg[i]))) < 1e-15 and hx[j, i] == -0.04
    assert not E.any() and h.min() == 0.1524 and h.max() == 0.4572
