"""The deck driver (oceanwave3d-fortran90_b200/driver.py): host set-up of a
deck and the reference's time loop with its output schedule.

CPU: prepare() on synthetic decks and on the reference's own example decks
(when present), and whole runs with the oracle as the backend.
GPU: a run of a synthetic deck on the device, its files, and its state
against the same run on the oracle.
"""
import os
import pathlib

import numpy as np
import pytest
from conftest import reference_decks

DECK = """driver test: 2-D flume, mono-chromatic incident wave, sponge
0 2
16. 1. 1. 129 1 9 0 0 1 1 1 1
3 3 3 1 1 1
40 0.05 1 0.5 1
9.81
1 3 0 23 1e-8 1e-6 1 V 1 1 20 12
0.02 1. 2. 1.2 1 0. 0 4 20
5 20 1 1
1 129 8 1 1 1 1 40 2
1 0
0 6 10 0.08 0.08 0.4
1 0. 2 X 0
0. 2. 0. 1. 10 3.5 X 1 X 0.
12. 16. 0. 1. 9 3.5 X 0 X 0.
0 0
0 2.0 2 0 0 1 0
0
-1 1.2 0.02 1. 35. 4 -34 0. 0. run06.el 0.0
"""


def _deck(tmp_path, text=DECK):
    f = tmp_path / "case.inp"
    f.write_text(text)
    return f


def _oracle_backend(oracle):
    return lambda p, **g: oracle.Oracle(p, **g, mode=oracle.MODE_DEVICE)


def test_prepare_synthetic(ow3d, tmp_path):
    from ow3d_b200 import driver
    s = driver.prepare(_deck(tmp_path))
    p = s.params
    # dt from the Courant number and the incident wave's speed g Tp / (2 pi)
    assert abs(p.dt - 0.5 * (16.0 / 128) / (p.g * p.Tp / (2 * np.pi))) < 1e-15
    (mode, nt, dts, eta, phis), = s.targets.values()
    i0, i1, j0, j1 = driver.zone_box(p, 0)
    assert (mode, nt, dts) == (0, p.Nsteps, p.dt) and eta.shape == (nt, j1 - j0 + 1, i1 - i0 + 1)
    assert np.abs(eta).max() <= 0.5 * p.Hs * (1 + 1e-12)
    assert not s.E0.any() and np.all(s.geometry["h"] == 1.0)


def test_run_with_oracle_and_hot_start(ow3d, oracle, tmp_path):
    from ow3d_b200 import driver
    sim, s, st = driver.run(_deck(tmp_path), steps=8, backend=_oracle_backend(oracle))
    E, P, W, phi, t = sim.get_state()
    assert st >= 0 and 0 < np.max(np.abs(E)) < s.params.Hs
    assert abs(t - 8 * s.params.dt) < 1e-12
    # IC -1: the state comes back from OceanWave3D.init (written as the reference writes it)
    Nx = s.params.Nx
    Ei, Pi = E[1:-1], P[1:-1]
    assert ow3d.lib().ow3d_write_end_file(str(tmp_path / "OceanWave3D.init").encode(), 16.0, 0.0, Nx, 1, t,
                                          ow3d._d(np.ascontiguousarray(Ei)), ow3d._d(np.ascontiguousarray(Pi))) == 0
    s2 = driver.prepare(_deck(tmp_path, DECK.replace("0 2\n16.", "-1 2\n16.")))
    assert s2.params.time0 == t and np.array_equal(s2.E0[1:-1], Ei) and np.array_equal(s2.P0[1:-1], Pi)


REF = reference_decks() or pathlib.Path("/nonexistent")


@pytest.mark.skipif(not REF.is_dir(), reason="reference example decks not on this machine")
@pytest.mark.parametrize("name", ["LinearTravellingWave", "RandomWave2D", "NLStanding", "RandomWave2DShoaling",
                                  "ObliqueRegular1Beach", "StreamFuncWave", "FluxWavemaker2D",
                                  "RollerBreakingModel2D", "FilterBreakingModel2D"])
def test_reference_decks_run_on_oracle(ow3d, oracle, name):
    """The reference's own example decks set up and step (two steps on the
    oracle) with bounded surfaces: incident waves of several kinds, a
    formula IC, a bathymetry file, directional generation zones, pressure
    damping, the flux wavemaker with its paddle-signal file, the roller
    breaking model and the local smoothing."""
    from ow3d_b200 import driver
    sim, s, st = driver.run(REF / f"OceanWave3D.inp.{name}", steps=2, backend=_oracle_backend(oracle))
    E = sim.get_state()[0]
    p = s.params
    H = max(p.Hs, p.sf_H, 0.1)
    assert st >= 0 and np.all(np.isfinite(E)) and np.max(np.abs(E)) < 5 * H, (name, np.max(np.abs(E)))


@pytest.mark.skipif(not REF.is_dir(), reason="reference example decks not on this machine")
@pytest.mark.parametrize("name", ["SFWaveAndFollowingCurrent", "SFWaveAndOpposingCurrent"])
def test_reference_current_decks_run_on_oracle(ow3d, oracle, tmp_path, name):
    """The stream-function wave on a following and an opposing current
    (IncWaveType 4): a hot start from the deck's own .init file (copied to
    the OceanWave3D.init the reference reads), the current's flux, the
    pressure-damping zone relative to it and the local smoothing (deck line
    2 gives 1 g), two steps on the oracle with bounded surfaces."""
    import shutil
    from ow3d_b200 import driver
    shutil.copy(REF / f"OceanWave3D.inp.{name}", tmp_path / "case.inp")
    shutil.copy(REF / f"{name}.init", tmp_path / "OceanWave3D.init")
    sim, s, st = driver.run(tmp_path / "case.inp", steps=2, backend=_oracle_backend(oracle))
    p = s.params
    assert (p.IncWaveType, p.current_flag, p.PDampingONOFF) == (1, 1, 1) and p.accel_tol_fact == 1.0
    E = sim.get_state()[0]
    assert st >= 0 and np.all(np.isfinite(E)) and np.max(np.abs(E)) < 5 * p.sf_H


@pytest.mark.gpu
def test_run_on_device_matches_oracle_and_writes_files(ow3d, oracle, tmp_path):
    from ow3d_b200 import driver
    deck = _deck(tmp_path)
    out = tmp_path / "out"
    sim, s, st = driver.run(deck, outdir=out, steps=6)
    E, P, W, phi, t = sim.get_state()
    sim.close()
    orc, _, _ = driver.run(deck, steps=6, backend=_oracle_backend(oracle))
    Eo, Po, Wo, phio, to = orc.get_state()
    assert abs(t - to) < 1e-12
    assert np.max(np.abs(E - Eo)) <= 1e-10 * np.max(np.abs(Eo))
    assert np.max(np.abs(phi - phio)) <= 1e-10 * np.max(np.abs(phio))
    # StoreDataONOFF 5: EP files at steps 0 and 5 (and the bathymetry file);
    # kinematics slice every 2 levels from level 1
    assert (out / "EP_00000.bin").exists() and (out / "EP_00005.bin").exists() and (out / "EP_99999.bin").exists()
    k = ow3d.load_kinematics(out / "Kinematics01.bin")
    assert [len(k["levels"])] == [4]          # levels 1, 3, 5, 7
