"""Incident linear wave of IncWaveType 2 (ow3d_incident_wave) and the deck
lines after the relaxation zones (pressure damping, SWENSE, curvilinear, the
wave line) -- host-only, no device.

The mono-chromatic wave of random_wave_signal.f90:151-172 is
eta = H/2 cos(nu (x - x0) - omega t), phiS = g/omega H/2 sin(...), with nu from
fdwvnum.f90. The checks: the samples against that closed form evaluated
here with nu from a converged Newton solve of omega^2 = g nu tanh(nu h) (the
reference's explicit formula agrees with the exact root to about 1e-10);
the zone box and the rows; the error paths; and the wave lines of the
reference's own example decks when they are on this machine.
"""
import os
import pathlib

import numpy as np
import pytest

DECK = """incident wave, mono-chromatic, x-directed generation zone
0 2
20. 2. 1. 129 9 9 0 0 1 1 1 1
3 3 3 1 1 1
400 0.02 1 0 1 0.3
9.81
1 3 0 23 1e-8 1e-6 1 V 1 1 20 12
0.1 1. 3. 2. 0 0. 1 6 24
0 0
1 0
0 6 10 0.08 0.08 0.4
1 2.0 2 X 0
0. 4. 0. 2. -10 3.5 X 1 X 0.
16. 20. 0. 2. 9 3.5 X 0 X 0.
0 0                 <- pressure damping off
0 2.0 2 0 0 1 0     <- SWENSE
0                   <- curvilinear
-1 1.25 0.04 0.8 35. 4 -34 1.5 0. run06.el 0.0
"""


def _deck(tmp_path, text=DECK):
    f = tmp_path / "wave.inp"
    f.write_text(text)
    return f


def test_wave_line_parsed(ow3d, tmp_path):
    p = ow3d.read_deck(_deck(tmp_path))
    assert p.IncWaveType == 2 and p.ispec == -1
    assert (p.Tp, p.Hs, p.h0, p.kh_max, p.x0, p.y0) == (1.25, 0.04, 0.8, 35.0, 1.5, 0.0)
    assert (p.seed, p.seed2) == (-4, -34)          # made negative (ReadInputFileParameters.f90:632-647)
    assert p.gamma_jonswap == 3.3 and p.time0 == 0.3
    # without the pressure-damping line the SWENSE line is not taken for one
    q = ow3d.read_deck(_deck(tmp_path, DECK.replace("0 0                 <- pressure damping off\n", "")))
    assert (q.ispec, q.Tp, q.x0) == (-1, 1.25, 1.5)
    # directional lines: file name, then beta0 s0 gamma
    d = ow3d.read_deck(_deck(tmp_path, DECK.replace("-1 1.25 0.04 0.8 35. 4 -34 1.5 0. run06.el 0.0",
                                                    "34 1.25 0.04 0.8 20. -1 -34 0 7.5 run06.el 10 80.0 2.5")))
    assert (d.ispec, d.beta0, d.s0, d.gamma_jonswap) == (34, 10.0, 80.0, 2.5)
    with pytest.raises(ow3d.OW3DError, match="incident-wave line"):
        ow3d.read_deck(_deck(tmp_path, DECK.replace("-1 1.25 0.04 0.8 35. 4 -34 1.5 0. run06.el 0.0", "-1 1.25")))


def _newton_k(omega, h, g):
    k = omega ** 2 / g
    for _ in range(60):
        f = g * k * np.tanh(k * h) - omega ** 2
        k -= f / (g * np.tanh(k * h) + g * k * h / np.cosh(k * h) ** 2)
    return k


def test_monochromatic_wave_closed_form(ow3d, tmp_path):
    p = ow3d.read_deck(_deck(tmp_path))
    eta, phis, (i0, i1, j0, j1) = ow3d.incident_wave(p, 0)
    assert eta.shape == (p.Nsteps, j1 - j0 + 1, i1 - i0 + 1)
    # the zone box: x in [0, 4] of a 20 m basin with dx = 20/128, y in [0, 2]:
    # the interior rows (PreprocessRelaxationZones.f90 traces the positions)
    dx = p.Lx / (p.Nx - 1)
    x = (np.arange(p.Nx + 2) - 1) * dx
    assert i0 == 2 and abs(x[i1 - 1] - 4.0) <= dx and j0 == 2 and j1 == p.Ny + 1
    omega = 2 * np.pi / p.Tp
    nu = _newton_k(omega, p.h0, p.g)
    t = p.time0 + np.arange(p.Nsteps) * p.dt
    arg = nu * (x[i0 - 1:i1][None, :] - p.x0) - omega * t[:, None]
    want_e = 0.5 * p.Hs * np.cos(arg)
    want_p = p.g / omega * 0.5 * p.Hs * np.sin(arg)
    # the reference's explicit wavenumber is within ~1e-10 of the root; over
    # Nsteps * dt = 8 s of phase that moves the samples by far less than 1e-7 H
    assert np.max(np.abs(eta - want_e[:, None, :])) < 1e-7 * p.Hs
    assert np.max(np.abs(phis - want_p[:, None, :])) < 1e-7 * p.Hs * p.g / omega
    # the x-directed wave is the same on every row of the zone
    assert np.array_equal(eta, np.broadcast_to(eta[:, :1, :], eta.shape))


def test_wavenumber_formula_close_to_root(ow3d, tmp_path):
    """The explicit formula (fdwvnum) against the exact root over shallow to
    deep water: the samples of a wave with kh in [0.05, 12]."""
    base = ow3d.read_deck(_deck(tmp_path))
    for h0 in (0.02, 0.3, 0.8, 3.0, 30.0):
        base.h0 = h0
        eta, phis, _ = ow3d.incident_wave(base, 0, nt=2)
        omega = 2 * np.pi / base.Tp
        nu = _newton_k(omega, h0, base.g)
        x = (np.arange(base.Nx + 2) - 1) * base.Lx / (base.Nx - 1)
        want = 0.5 * base.Hs * np.cos(nu * (x[1:eta.shape[2] + 1] - base.x0) - omega * base.time0)
        assert np.max(np.abs(eta[0, 0] - want)) < 1e-8 * base.Hs, h0


def test_incident_wave_errors(ow3d, tmp_path):
    p = ow3d.read_deck(_deck(tmp_path))
    with pytest.raises(ow3d.OW3DError, match="not an x-directed generation zone"):
        ow3d.incident_wave(p, 1)
    with pytest.raises(ow3d.OW3DError, match="no such relaxation zone"):
        ow3d.incident_wave(p, 5)
    p.ispec = 1
    with pytest.raises(ow3d.OW3DError) as e:
        ow3d.incident_wave(p, 0)
    assert e.value.status == ow3d.capi.ERR_UNSUPPORTED
    p.ispec = -1
    p.IncWaveType = 0
    with pytest.raises(ow3d.OW3DError, match="IncWaveType"):
        ow3d.incident_wave(p, 0)


REF_DECKS = pathlib.Path(os.environ.get("OW3D_REFERENCE_DECKS", "/root/reference/examples/inputfiles"))


@pytest.mark.skipif(not REF_DECKS.is_dir(), reason="reference example decks not on this machine")
def test_reference_wave_lines(ow3d):
    """Every example deck with IncWaveType 2: the parsed wave parameters are
    the first items of its last non-blank line that starts with ispec."""
    seen = 0
    for f in sorted(REF_DECKS.iterdir()):
        if not f.name.startswith("OceanWave3D.inp"):
            continue
        try:
            p = ow3d.read_deck(f)
        except ow3d.OW3DError:
            continue
        if p.IncWaveType != 2:
            continue
        lines = [ln.split() for ln in f.read_text(errors="replace").splitlines() if ln.strip()]
        cand = [ln for ln in lines if ln and ln[0].lstrip("-").isdigit() and int(ln[0]) == p.ispec and len(ln) >= 9]
        assert cand, f.name
        ln = cand[-1]
        assert float(ln[1]) == p.Tp and float(ln[2]) == p.Hs and float(ln[3]) == p.h0, f.name
        assert -abs(int(float(ln[5]))) == p.seed and float(ln[7]) == p.x0, f.name
        seen += 1
    assert seen >= 5
