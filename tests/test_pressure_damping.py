"""Pressure-damping zones of 2-D decks (PreprocessPDampingZones.f90,
BuildPDampMatrices.f90, funPressureTerm.f90:218-311, rhsFreeSurface3D.f90:27-28).

CPU: the deck's zone line; the host set-up (zone points, the Gaussian gamma,
the zone matrix and the inverse the device applies) against a numpy
restatement; the decks the device refuses; the oracle's damping of a
standing wave.
GPU: the device against the oracle with a type-0 zone (velocity damping
through the zone solve) and a friction zone, a few steps each.
"""
import ctypes as C
import os
import pathlib

import numpy as np
import pytest

import cases
from test_driver import DECK
from conftest import reference_decks

REF = reference_decks() or pathlib.Path("/nonexistent")


def _zone(p, typ=0, x0=6.0, x1=8.0, g0=1.0):
    p.PDampingONOFF, p.NDampZones, p.pd_type = 1, 1, typ
    p.pd_x0, p.pd_x1, p.pd_y0, p.pd_y1, p.pd_g0Phi, p.pd_g0Eta = x0, x1, 0.0, 0.0, g0, g0
    return p


def _case(typ=0, Nx=129):
    p, geo = cases.flat_2d(Nx=Nx, Nz=9, L=8.0, dt=0.02)
    return _zone(p, typ), geo


def _setup(ow3d, p):
    L = ow3d.lib()
    L.ow3d_test_pdamp_setup.argtypes = [C.c_void_p] + [C.c_void_p] * 6
    i1, nd = C.c_int(), C.c_int()
    r = L.ow3d_test_pdamp_setup(C.byref(p), C.byref(i1), C.byref(nd), None, None, None, None)
    if r != 0:
        return r, None
    n, Nxg = nd.value, p.Nx + 2
    gp, ge = np.zeros(Nxg), np.zeros(Nxg)
    A, Ai = np.zeros(n * n), np.zeros(n * n)
    assert L.ow3d_test_pdamp_setup(C.byref(p), None, None, *[a.ctypes.data for a in (gp, ge, A, Ai)]) == 0
    return 0, (i1.value, n, gp, ge, A.reshape(n, n), Ai.reshape(n, n))


def _standing(p):
    x = (np.arange(p.Nx + 2) - 1) * (p.Lx / (p.Nx - 1))
    return 0.02 * np.cos(2 * np.pi * x / 2.0)


def test_deck_zone_line(ow3d, tmp_path):
    f = tmp_path / "pd.inp"
    f.write_text(DECK.replace("0 0\n0 2.0 2", "1 1 <- Damping pressure zone\n12. 16. 0. 0. 0.5 0.25 0\n0 2.0 2"))
    p = ow3d.read_deck(f)
    assert (p.PDampingONOFF, p.NDampZones, p.pd_type) == (1, 1, 0)
    assert (p.pd_x0, p.pd_x1, p.pd_y0, p.pd_y1, p.pd_g0Phi, p.pd_g0Eta) == (12.0, 16.0, 0.0, 0.0, 0.5, 0.25)
    # the lines after the zone are still read: the incident-wave line of IncWaveType 2
    assert (p.ispec, p.Tp, p.Hs) == (-1, 1.2, 0.02)
    assert _setup(ow3d, p)[0] == 0


@pytest.mark.skipif(not REF.is_dir(), reason="reference example decks not on this machine")
@pytest.mark.parametrize("name", ["OceanWave3D.inp", "OceanWave3D.inp.StreamFuncWave", "OceanWave3D.inp.RandomWave2D"])
def test_reference_decks_set_up(ow3d, name):
    p = ow3d.read_deck(REF / name)
    assert p.PDampingONOFF == 1 and p.NDampZones == 1 and p.pd_type == 0
    r, s = _setup(ow3d, p)
    assert r == 0
    i1, nd, gp, ge, A, Ai = s
    x = (np.arange(p.Nx + 2) - 1) * (p.Lx / (p.Nx - 1))
    assert x[i1 - 1] >= p.pd_x0 and x[i1 - 2] < p.pd_x0
    assert np.abs(Ai @ A - np.eye(nd)).max() < 1e-9


def test_setup_matches_restatement(ow3d):
    p, _ = _case(0)
    r, (i1, nd, gp, ge, A, Ai) = _setup(ow3d, p)
    assert r == 0
    dx = p.Lx / (p.Nx - 1)
    x = (np.arange(p.Nx + 2) - 1) * dx
    # TracePosition: the first node at or beyond the box edges
    assert i1 == int(np.argmax(x >= p.pd_x0 - 1e-12)) + 1
    assert nd == int(np.argmax(x >= p.pd_x1 - 1e-12)) + 2 - i1
    # GammaFunctions type 12 (parameter 0.25), times 2 pi g0
    xz = x[i1 - 1:i1 - 1 + nd]
    g = 2 * np.pi * np.exp(-((xz - xz[-1]) / (xz[-1] - xz[0])) ** 2 / (2 * 0.25 ** 2))
    assert np.abs(gp[i1 - 1:i1 - 1 + nd] - g).max() < 1e-14 and np.array_equal(gp, ge)
    assert not gp[:i1 - 1].any() and not gp[i1 - 1 + nd:].any()
    # the zone matrix on t^2 and t^3 (exact for the 7-point stencils): value,
    # second derivatives, first derivative at the last point
    t = np.arange(nd) * dx
    for v, d1, d2 in ((t ** 2, 2 * t, 2 + 0 * t), (t ** 3, 3 * t ** 2, 6 * t)):
        Lv = A @ v
        assert abs(Lv[0] - v[0]) < 1e-14
        assert np.abs(Lv[1:-1] - d2[1:-1]).max() < 1e-8 * np.abs(d2).max() + 1e-9
        assert abs(Lv[-1] - d1[-1]) < 1e-9 * abs(d1[-1])
    # every row has 2*alpha+1 entries (the Dirichlet row one)
    assert (A[0] != 0).sum() == 1 and all((A[r] != 0).sum() <= 7 for r in range(1, nd))
    assert np.abs(Ai @ A - np.eye(nd)).max() < 1e-10
    assert np.abs(Ai - np.linalg.inv(A)).max() < 1e-10 * np.abs(Ai).max()
    # a friction zone has gamma only
    p1, _ = _case(1)
    r, (j1, n1, gp1, _, _, _) = _setup(ow3d, p1)
    assert r == 0 and (j1, n1) == (i1, nd) and np.array_equal(gp1, gp)


def test_refused_and_bad_zones(ow3d):
    ERR_BAD, ERR_UNS = ow3d.capi.ERR_BAD_INPUT, ow3d.capi.ERR_UNSUPPORTED
    p, _ = _case(0)
    p.NDampZones = 2
    assert _setup(ow3d, p)[0] == ERR_UNS
    p3, _ = cases.bump_3d(Nx=17, Ny=9, Nz=9)
    assert _setup(ow3d, _zone(p3, 1, 1.0, 2.0))[0] == ERR_UNS
    # a type-0 zone needs 2*alpha+1 points
    p, _ = _case(0)
    p.pd_x0, p.pd_x1 = 7.7, 8.0
    assert _setup(ow3d, p)[0] == ERR_BAD
    p.pd_type = 1
    assert _setup(ow3d, p)[0] == 0


@pytest.mark.parametrize("typ", [0, 1])
def test_oracle_damps_a_standing_wave(ow3d, oracle, typ):
    """Peak wave energy over 4 s of a 2 m standing wave in an 8 m tank, with
    and without a zone over the last 2 m: without it stays near its start,
    with it the late peaks fall well below."""
    p, geo = _case(typ)
    E0 = _standing(p)
    peaks = []
    for on in (0, 1):
        q = ow3d.capi.Params.from_buffer_copy(p)
        q.PDampingONOFF = on
        orc = oracle.Oracle(q, **geo, mode=oracle.MODE_DEVICE)
        orc.set_state(E0, np.zeros_like(E0))
        e = []
        for _ in range(10):
            assert orc.step(20) >= 0
            e.append(np.sum(orc.get_state()[0][1:-1] ** 2))
        peaks.append(max(e[-4:]))
    assert peaks[1] < 0.8 * peaks[0], peaks


@pytest.mark.gpu
@pytest.mark.parametrize("typ", [0, 1])
def test_device_matches_oracle(ow3d, oracle, typ):
    """1e-10 relative on eta, P and phi after 6 steps: the device applies the
    inverse of the zone matrix where the oracle solves with its LU factors;
    the matrix's condition number (about 1.4e4 here) keeps the two within
    about 1e-13."""
    p, geo = _case(typ)
    E0 = _standing(p)
    sim = ow3d.Simulation(p, **geo)
    try:
        sim.set_state(E0, np.zeros_like(E0))
        assert sim.step(6) >= 0
        E, P, W, phi, t = sim.get_state()
    finally:
        sim.close()
    orc = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    orc.set_state(E0, np.zeros_like(E0))
    assert orc.step(6) >= 0
    Eo, Po, Wo, phio, to = orc.get_state()
    rel = lambda a, b: np.max(np.abs(a - b)) / np.max(np.abs(b))
    assert abs(t - to) < 1e-12
    assert rel(E, Eo) < 1e-10 and rel(P, Po) < 1e-10 and rel(phi, phio) < 1e-10, (rel(E, Eo), rel(P, Po))
    # the zone acted: the undamped oracle differs
    q = ow3d.capi.Params.from_buffer_copy(p)
    q.PDampingONOFF = 0
    und = oracle.Oracle(q, **geo, mode=oracle.MODE_DEVICE)
    und.set_state(E0, np.zeros_like(E0))
    und.step(6)
    assert rel(und.get_state()[0], Eo) > 1e-6
