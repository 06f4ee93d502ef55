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
from conftest import reference_decks

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
        t = np.tanh(k * h)
        k -= f / (g * t + g * k * h * (1 - t * t))
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
    p.ispec = 2                                    # waves from a file: not built
    with pytest.raises(ow3d.OW3DError) as e:
        ow3d.incident_wave(p, 0)
    assert e.value.status == ow3d.capi.ERR_UNSUPPORTED
    p.ispec = -1
    p.IncWaveType = 0
    with pytest.raises(ow3d.OW3DError, match="IncWaveType"):
        ow3d.incident_wave(p, 0)


REF_DECKS = reference_decks() or pathlib.Path("/nonexistent")


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


def test_generator_park_miller_check(ow3d):
    """The generator's underlying sequence is Park and Miller's minimal
    standard: from x0 = 1, x10000 = 1043618065 (their published check). A
    restart (idum <= 0) takes 40 steps to fill the shuffle table, so 9960
    deviates later idum is x10000."""
    import ctypes as C
    L = ow3d.lib()
    out = (C.c_float * 9960)()
    idum = C.c_int()
    assert L.ow3d_test_ran1(-1, 9960, out, C.byref(idum)) == 0
    assert idum.value == 1043618065
    v = np.frombuffer(out, dtype=np.float32)
    assert v.min() > 0 and v.max() < 1 and abs(v.mean() - 0.5) < 0.02


def _random_deck(tmp_path, ispec):
    text = DECK.replace("400 0.02 1 0 1 0.3", "4000 0.02 1 0 1 0.")
    text = text.replace("-1 1.25 0.04 0.8 35. 4 -34 1.5 0. run06.el 0.0", f"{ispec} 1.25 0.04 0.8 20. 4 -34 0. 0. run06.el")
    return ow3d_read(tmp_path, text)


def ow3d_read(tmp_path, text):
    from conftest import load_package
    return load_package().read_deck(_deck(tmp_path, text))


def _jonswap(f, Hs, Tp, gamma):
    fp = 1 / Tp
    A = 3.32285 * Hs ** 2 * fp ** 4 * 9.82 ** 2 / (2 * np.pi) ** 4
    B = 1.25 * fp ** 4
    sigma = np.where(f <= fp, 0.07, 0.09)
    return A / f ** 5 * np.exp(-B / f ** 4) * gamma ** np.exp(-0.5 * ((f - fp) / (sigma * fp)) ** 2)


def _pm(f, Hs, Tp):
    T02 = float(np.float32(0.71)) * Tp
    return Hs ** 2 / (4 * np.pi * T02 ** 4) / f ** 5 * np.exp(-1 / (np.pi * T02 ** 4) / f ** 4)


@pytest.mark.parametrize("ispec", [1, 0])
def test_random_wave_spectrum_phases_and_dispersion(ow3d, tmp_path, ispec):
    """JONSWAP (1) and P-M (0): at x = x0 the Fourier coefficients of the
    generated series are sqrt(2 S(f_k) df) e^(2 pi i psi_k) with psi_k the
    generator's deviates from seed2 (phases rounded to single precision),
    zero from the kh_max cut-off on; downstream they carry e^(i nu_k d) with
    nu_k the dispersion root; phiS has the coefficients g/omega (-i) c_k; and
    the variance is sum S(f_k) df (Parseval)."""
    import ctypes as C
    p = _random_deck(tmp_path, ispec)
    eta, phis, (i0, i1, j0, j1) = ow3d.incident_wave(p, 0)
    N = eta.shape[0]
    assert N == 4096
    dt = p.dt
    df = 1 / (N * dt)
    k = np.arange(1, N // 2)
    f = k * df
    S = _jonswap(f, p.Hs, p.Tp, 3.3) if ispec == 1 else _pm(f, p.Hs, p.Tp)
    n_cut = int(np.floor(np.sqrt(p.g * p.kh_max / p.h0 * np.tanh(p.kh_max)) / (2 * np.pi * df) + 0.5)) + 1
    keep = k < n_cut - 1
    psi = (C.c_float * (N // 2 - 1))()
    assert ow3d.lib().ow3d_test_ran1(-34, N // 2 - 1, psi, None) == 0
    ph = 2 * np.pi * np.frombuffer(psi, dtype=np.float32).astype(np.float64)
    want = np.sqrt(2 * S * df) * (np.cos(ph).astype(np.float32) + 1j * np.sin(ph).astype(np.float32))
    want = np.where(keep, want, 0)
    x = (np.arange(p.Nx + 2) - 1) * p.Lx / (p.Nx - 1)
    omega = 2 * np.pi * f
    nu = _newton_k(omega, p.h0, p.g)
    for col in (0, 7):                         # x = x0 = 0, and 7 columns downstream
        d = x[i0 - 1 + col] - p.x0
        ce = np.conj(np.fft.fft(eta[:, 0, col])[1:N // 2]) * 2 / N
        cp = np.conj(np.fft.fft(phis[:, 0, col])[1:N // 2]) * 2 / N
        w = want * np.exp(1j * nu * d)
        scale = np.abs(want).max()
        assert np.max(np.abs(ce - w)) < 1e-6 * scale, col
        assert np.max(np.abs(cp - p.g / omega * (-1j) * w)) < 1e-6 * scale * p.g / omega.min(), col
    var = np.sum(np.where(keep, S, 0) * df)
    assert abs(np.var(eta[:, 0, 0]) / var - 1) < 1e-6     # |phase| = 1 to single precision
    assert abs(4 * np.sqrt(var) / p.Hs - 1) < 0.1       # the spectrum's H_s, before truncation effects


def test_random_wave_limits(ow3d, tmp_path):
    p = _random_deck(tmp_path, 1)
    with pytest.raises(ow3d.OW3DError, match="samples"):
        ow3d.incident_wave(p, 0, nt=5000)
    p.ispec = 2
    with pytest.raises(ow3d.OW3DError) as e:
        ow3d.incident_wave(p, 0)
    assert e.value.status == ow3d.capi.ERR_UNSUPPORTED


def _heading_deck(tmp_path, line, nsteps="400"):
    text = DECK.replace("400 0.02 1 0 1 0.3", f"{nsteps} 0.02 1 0 1 0.3")
    return ow3d_read(tmp_path, text.replace("-1 1.25 0.04 0.8 35. 4 -34 1.5 0. run06.el 0.0", line))


def _xy(p):
    x = (np.arange(p.Nx + 2) - 1) * p.Lx / (p.Nx - 1)
    y = (np.arange(p.Ny + 2) - 1) * p.Ly / (p.Ny - 1)
    return x, y


def test_monochromatic_wave_at_heading(ow3d, tmp_path):
    """ispec -30 (random_wave_signal_3D.f90:150-171): the wave at beta0 to
    the x-axis on every point of the zone, phase nu ((x-x0) cos b + (y-y0) sin b)."""
    p = _heading_deck(tmp_path, "-30 1.25 0.04 0.8 35. 4 -34 1.5 0.5 run06.el 22.5 1.0 3.3")
    assert (p.ispec, p.beta0) == (-30, 22.5)
    eta, phis, (i0, i1, j0, j1) = ow3d.incident_wave(p, 0)
    x, y = _xy(p)
    b = np.deg2rad(p.beta0)
    omega = 2 * np.pi / p.Tp
    nu = _newton_k(omega, p.h0, p.g)
    X, Y = np.meshgrid(x[i0 - 1:i1], y[j0 - 1:j1])
    d = np.cos(b) * (X - p.x0) + np.sin(b) * (Y - p.y0)
    t = p.time0 + np.arange(eta.shape[0]) * p.dt
    arg = nu * d[None] - omega * t[:, None, None]
    assert np.max(np.abs(eta - 0.5 * p.Hs * np.cos(arg))) < 1e-7 * p.Hs
    assert np.max(np.abs(phis - p.g / omega * 0.5 * p.Hs * np.sin(arg))) < 1e-7 * p.Hs * p.g / omega
    assert not np.array_equal(eta[:, 0, :], eta[:, -1, :])      # rows differ at a heading


def test_random_wave_at_heading(ow3d, tmp_path):
    """ispec 31: the JONSWAP coefficients of the long-crested case, moved to
    each point along the heading."""
    import ctypes as C
    p = _heading_deck(tmp_path, "31 1.25 0.04 0.8 20. 4 -34 0. 0. run06.el 30.0 1.0 3.3", nsteps="1000")
    eta, phis, (i0, i1, j0, j1) = ow3d.incident_wave(p, 0)
    N = eta.shape[0]
    assert N == 1024
    df = 1 / (N * p.dt)
    k = np.arange(1, N // 2)
    S = _jonswap(k * df, p.Hs, p.Tp, p.gamma_jonswap)
    n_cut = int(np.floor(np.sqrt(p.g * p.kh_max / p.h0 * np.tanh(p.kh_max)) / (2 * np.pi * df) + 0.5)) + 1
    psi = (C.c_float * (N // 2 - 1))()
    ow3d.lib().ow3d_test_ran1(-34, N // 2 - 1, psi, None)
    ph = 2 * np.pi * np.frombuffer(psi, dtype=np.float32).astype(np.float64)
    want = np.where(k < n_cut - 1, np.sqrt(2 * S * df) * (np.cos(ph).astype(np.float32) + 1j * np.sin(ph).astype(np.float32)), 0)
    nu = _newton_k(2 * np.pi * k * df, p.h0, p.g)
    x, y = _xy(p)
    b = np.deg2rad(p.beta0)
    for (ci, cj) in ((0, 0), (5, 3)):
        d = np.cos(b) * (x[i0 - 1 + ci] - p.x0) + np.sin(b) * (y[j0 - 1 + cj] - p.y0)
        ce = np.conj(np.fft.fft(eta[:, cj, ci])[1:N // 2]) * 2 / N
        assert np.max(np.abs(ce - want * np.exp(1j * nu * d))) < 1e-6 * np.abs(want).max(), (ci, cj)


def test_heading_needs_zone_without_rotation(ow3d, tmp_path):
    p = _heading_deck(tmp_path, "-30 1.25 0.04 0.8 35. 4 -34 1.5 0.5 run06.el 22.5 1.0 3.3")
    p.zones[0].degrees = 10.0
    with pytest.raises(ow3d.OW3DError, match="degrees"):
        ow3d.incident_wave(p, 0)


def _spread_headings(draws, s0, beta0, ncta):
    """Headings drawn by the inverse of the tabulated cos^(2 s0) distribution
    (spreading.f90): the first grid heading whose cumulative value reaches the
    deviate."""
    ipow = 2 * s0
    cmin, cmax = beta0 - np.pi / 2, beta0 + np.pi / 2
    d1 = (cmax - cmin) / float(np.float32(ncta - 1))
    cc1 = cmin + np.arange(ncta) * d1
    spm = 1.0 / np.sum(np.cos((cc1 - beta0) / 2) ** ipow * d1)
    dc = np.pi / float(np.float32(ncta))
    cta = cmin + np.arange(ncta) * dc
    cosint = np.cumsum(np.cos((cta - beta0) / 2) ** ipow * dc) * spm
    idx = np.minimum(np.searchsorted(cosint, draws, side="left"), ncta - 1)
    return cta[idx]


def test_spread_sea_cos2s(ow3d, tmp_path):
    """ispec 34 (build_coeff_3D_Cos.f90, spreading.f90): N/2 headings drawn
    first from the generator, then the phases; every component travels along
    its own heading."""
    import ctypes as C
    p = _heading_deck(tmp_path, "34 1.25 0.04 0.8 20. 4 -34 0. 0.5 run06.el 0 8.0 3.3", nsteps="1000")
    assert (p.ispec, p.beta0, p.s0) == (34, 0.0, 8.0)
    eta, phis, (i0, i1, j0, j1) = ow3d.incident_wave(p, 0)
    N = eta.shape[0]
    draws = (C.c_float * (N - 1))()
    ow3d.lib().ow3d_test_ran1(-34, N - 1, draws, None)
    d = np.frombuffer(draws, dtype=np.float32).astype(np.float64)
    beta = _spread_headings(d[:N // 2], p.s0, p.beta0, N // 2)      # beta0 enters as the deck gives it
    assert np.all(np.abs(beta) <= np.pi / 2) and abs(np.mean(beta)) < 0.1
    ph = 2 * np.pi * d[N // 2:]
    df = 1 / (N * p.dt)
    k = np.arange(1, N // 2)
    S = _jonswap(k * df, p.Hs, p.Tp, p.gamma_jonswap)
    n_cut = int(np.floor(np.sqrt(p.g * p.kh_max / p.h0 * np.tanh(p.kh_max)) / (2 * np.pi * df) + 0.5)) + 1
    want = np.where(k < n_cut - 1, np.sqrt(2 * S * df) * (np.cos(ph).astype(np.float32) + 1j * np.sin(ph).astype(np.float32)), 0)
    nu = _newton_k(2 * np.pi * k * df, p.h0, p.g)
    bk = beta[1:N // 2]                                   # heading of component k is beta(k + 1)
    x, y = _xy(p)
    for (ci, cj) in ((0, 0), (6, 4)):
        dx, dy = x[i0 - 1 + ci] - p.x0, y[j0 - 1 + cj] - p.y0
        ce = np.conj(np.fft.fft(eta[:, cj, ci])[1:N // 2]) * 2 / N
        w = want * np.exp(1j * nu * (np.cos(bk) * dx + np.sin(bk) * dy))
        assert np.max(np.abs(ce - w)) < 1e-6 * np.abs(want).max(), (ci, cj)


def test_normally_spread_sea(ow3d, tmp_path):
    """ispec 33 (build_coeff_3D.f90): each component's heading from its phase
    deviate psi, beta = beta0 + sqrt(2 sigma) erf^-1((2 psi - 1) erf(pi /
    (2 sqrt(2 sigma)))) with sigma = 0.2 (f / fp)^2.5, and -1 in place of the
    inverse for psi < 1/2, which is what the reference's inverse returns
    for a negative argument."""
    import ctypes as C
    from scipy.special import erf, erfinv
    p = _heading_deck(tmp_path, "33 1.25 0.04 0.8 20. 4 -34 0. 0.5 run06.el 0 1.0 3.3", nsteps="1000")
    eta, phis, (i0, i1, j0, j1) = ow3d.incident_wave(p, 0)
    N = eta.shape[0]
    draws = (C.c_float * (N // 2 - 1))()
    ow3d.lib().ow3d_test_ran1(-34, N // 2 - 1, draws, None)
    psi = np.frombuffer(draws, dtype=np.float32).astype(np.float64)
    df = 1 / (N * p.dt)
    k = np.arange(1, N // 2)
    f = k * df
    sigma = 0.2 * (f * p.Tp) ** 2.5
    arg = (2 * psi - 1) * erf(np.pi / (2 * np.sqrt(2 * sigma)))
    e2 = np.where(arg >= 0, erfinv(np.maximum(arg, 0)), -1.0)
    beta = np.deg2rad(p.beta0 + np.rad2deg(np.sqrt(2 * sigma) * e2))
    S = _jonswap(f, p.Hs, p.Tp, p.gamma_jonswap)
    n_cut = int(np.floor(np.sqrt(p.g * p.kh_max / p.h0 * np.tanh(p.kh_max)) / (2 * np.pi * df) + 0.5)) + 1
    ph = 2 * np.pi * psi
    want = np.where(k < n_cut - 1, np.sqrt(2 * S * df) * (np.cos(ph).astype(np.float32) + 1j * np.sin(ph).astype(np.float32)), 0)
    nu = _newton_k(2 * np.pi * f, p.h0, p.g)
    x, y = _xy(p)
    for (ci, cj) in ((0, 0), (6, 4)):
        dx, dy = x[i0 - 1 + ci] - p.x0, y[j0 - 1 + cj] - p.y0
        ce = np.conj(np.fft.fft(eta[:, cj, ci])[1:N // 2]) * 2 / N
        w = want * np.exp(1j * nu * (np.cos(beta) * dx + np.sin(beta) * dy))
        assert np.max(np.abs(ce - w)) < 1e-6 * np.abs(want).max(), (ci, cj)


# ----------------------------------------------------------------- device

_DEVICE_CASES = {
    "mono": ("-1 1.25 0.04 0.8 35. 4 -34 1.5 0. run06.el 0.0", "400"),
    "jonswap": ("1 1.25 0.04 0.8 20. 4 -34 0. 0. run06.el", "1000"),
    "pm": ("0 1.25 0.04 0.8 20. 4 -34 0. 0. run06.el", "1000"),
    "mono_heading": ("-30 1.25 0.04 0.8 35. 4 -34 1.5 0.5 run06.el 22.5 1.0 3.3", "400"),
    "jonswap_heading": ("31 1.25 0.04 0.8 20. 4 -34 0. 0. run06.el 30.0 1.0 3.3", "1000"),
    "normal_spread": ("33 1.25 0.04 0.8 20. 4 -34 0. 0.5 run06.el 0 1.0 3.3", "1000"),
    "cos2s_spread": ("34 1.25 0.04 0.8 20. 4 -34 0. 0.5 run06.el 0 8.0 3.3", "1000"),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(_DEVICE_CASES))
def test_device_incident_wave_matches_host(ow3d, tmp_path, case):
    """ow3d_incident_wave_device forms the series on the device (closed form
    for the mono-chromatic wave, the direct sum over the modes for random
    waves) and installs it as the zone's target: the same samples as the
    host synthesis (ow3d_incident_wave, an FFT for random waves) to 1e-12 of
    the wave's amplitude, and the same RK4 steps to 1e-12."""
    line, nsteps = _DEVICE_CASES[case]
    p = _heading_deck(tmp_path, line, nsteps=nsteps)
    eta, phis, box = ow3d.incident_wave(p, 0)
    nt = eta.shape[0]
    Nxg, Nyg, _ = ow3d.dims(p)
    geo = dict(h=np.full(Nxg * Nyg, p.h0))
    dev = ow3d.Simulation(p, **geo)
    dev.incident_wave_device(0, nt)
    de, dp = dev.relax_target(0, nt)
    he, hp = eta.reshape(nt, -1), phis.reshape(nt, -1)
    assert np.max(np.abs(de - he)) <= 1e-12 * np.max(np.abs(he)), np.max(np.abs(de - he))
    assert np.max(np.abs(dp - hp)) <= 1e-12 * np.max(np.abs(hp)), np.max(np.abs(dp - hp))
    # the same steps with the host-built target
    host = ow3d.Simulation(p, **geo)
    host.set_relax_target(0, 0, nt, p.dt, eta, phis)
    for s in (dev, host):
        s.set_state(np.zeros(Nxg * Nyg), np.zeros(Nxg * Nyg))
        assert s.step(6) >= 0
    E1, E2 = dev.get_state()[0], host.get_state()[0]
    assert np.max(np.abs(E2)) > 0
    assert np.max(np.abs(E1 - E2)) <= 1e-12 * np.max(np.abs(E2))
    dev.close(); host.close()
