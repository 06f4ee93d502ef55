"""Input-deck parser (ow3d_read_deck), the positional format of
ReadInputFileParameters.f90: synthetic decks with known values, the optional
fields, and the error paths. When the reference's example decks are present
on this machine they are parsed as extra fixtures (skipped elsewhere)."""
import os
import pathlib

import pytest
from conftest import reference_decks

DECK_3D = """synthetic 3-D basin with two relaxation zones
-1 0                                   <- IC, IncWaveType
40. 10. 1. 129 33 9 0 0 1 1 1 1         <- Lx Ly Lz Nx Ny Nz GridX GridY GridZ ghosts
3 3 3 1 1 1                            <- stencil half-widths
500 0.05 1 0 1                         <- Nsteps dt timemethod CFL extrapolation
9.81                                   <- g
1 3 0 23 1e-8 1e-6 1 V 1 1 20 12       <- solver Precond strategy m reltol abstol maxit cyclet nu1 nu2 MGmaxgrids
0.1 1. 3. 2. 0 0. 1 6 24               <- stream function line
0 0                                    <- no output
1 0                                    <- nonlinear
1 6 10 0.08 0.08 0.4                   <- filter
1 2.0 2 X 0                            <- relaxation: on, ramp, zones
0. 5. 0. 10. -10 3.5 X 1 X 0.
35. 40. 0. 10. 9 3.5 X 0 X 0.
"""

DECK_2D_CFL = """synthetic flume, solver field omitted, dt from CFL
0 1
8. 1. 1. 65 1 9 0 0 1 1 1 1
3 3 3 1 1 1
100 0.1 1 0.5 1 2.5
9.82 1000.
3 0 30 1e-9 1e-7 2 W 2 3 0
0.05 1. 2. 1. 0 0. 1 6 24
-5 20 1 2                              <- formattype 20: two output-file lines follow
1 65 1 1 1 1 1 100 1
1 65 2 1 1 1 1 100 2
0 1
0 6 10 0.08 0.08 0.4
0.1 0.2 0.3 0.4 0.5 0.6 1              <- optional breaking line
0 0. 0 X 0
"""


def write(tmp_path, name, text):
    f = tmp_path / name
    f.write_text(text)
    return f


def test_deck_3d(ow3d, tmp_path):
    p = ow3d.read_deck(write(tmp_path, "a.inp", DECK_3D))
    assert (p.IC, p.IncWaveType) == (-1, 0)
    assert (p.Lx, p.Ly, p.Lz, p.Nx, p.Ny, p.Nz) == (40.0, 10.0, 1.0, 129, 33, 9)
    assert (p.GridX, p.GridY, p.GridZ, p.GhostGridX, p.GhostGridY, p.GhostGridZ) == (0, 0, 1, 1, 1, 1)
    assert (p.alpha, p.beta, p.gamma, p.alphaprecond, p.betaprecond, p.gammaprecond) == (3, 3, 3, 1, 1, 1)
    assert (p.Nsteps, p.dt, p.timemethod, p.CFL, p.extrapolationONOFF) == (500, 0.05, 1, 0.0, 1)
    assert p.g == 9.81
    assert (p.solver, p.Precond, p.MGCoarseningStrategy, p.GMRESmaxiterations) == (1, 3, 0, 23)
    assert (p.reltol, p.abstol, p.maxit, p.cyclet, p.nu1, p.nu2, p.MGmaxgrids) == (1e-8, 1e-6, 1, b"V", 1, 1, 20)
    assert (p.LinearONOFF, p.filteringONOFF, p.filterALPHA, p.filterORDER) == (1, 1, 6, 10)
    assert list(p.sigma_filt) == [0.08, 0.08, 0.4]
    assert (p.relaxONOFF, p.relaxTransientTime, p.relaxNo, p.relaxXorY) == (1, 2.0, 2, b"X")
    z0, z1 = p.zones[0], p.zones[1]
    assert (z0.x1, z0.x2, z0.y1, z0.y2, z0.ftype, z0.param, z0.XorY, z0.WavegenONOFF) == (0, 5, 0, 10, -10, 3.5, b"X", 1)
    assert (z1.x1, z1.x2, z1.ftype, z1.WavegenONOFF) == (35, 40, 9, 0)


def test_deck_2d_optional_fields(ow3d, tmp_path):
    p = ow3d.read_deck(write(tmp_path, "b.inp", DECK_2D_CFL))
    assert (p.Nx, p.Ny, p.Nz) == (65, 1, 9)
    # 2-D: no y ghosts, no y stencil (ReadInputFileParameters.f90)
    assert p.GhostGridY == 0 and p.beta == 0 and p.betaprecond == 0
    # CFL != 0 overrides dt with CFL * dx
    assert abs(p.dt - 0.5 * 8.0 / 64) < 1e-15
    assert p.time0 == 2.5
    assert p.g == 9.82
    # solver field omitted: GMRES is implied, the line starts at Precond
    assert (p.solver, p.Precond, p.MGCoarseningStrategy, p.GMRESmaxiterations) == (1, 3, 0, 30)
    assert (p.reltol, p.abstol, p.maxit, p.cyclet, p.nu1, p.nu2, p.MGmaxgrids) == (1e-9, 1e-7, 2, b"W", 2, 3, 0)
    # kinematics output lines (ReadInputFileParameters.f90:300-336), then the breaking line is skipped
    assert (p.StoreDataONOFF, p.formattype, p.iKinematics, p.nOutFiles) == (-5, 20, 1, 2)
    assert list(p.kinematics[0]) == [1, 65, 1, 1, 1, 1, 1, 100, 1]
    assert list(p.kinematics[1]) == [1, 65, 2, 1, 1, 1, 1, 100, 2]
    assert p.LinearONOFF == 0 and p.PressureTermOnOff == 1
    assert p.filteringONOFF == 0 and p.relaxONOFF == 0


def test_deck_breaking_line(ow3d, tmp_path):
    """Line 12 (ReadInputFileParameters.f90:478-479): i_breaking, T_1/2,
    phi_b, phi_0, f_delta, f_cel, gamma_break, as the roller-breaking decks
    of the reference write it."""
    text = DECK_2D_CFL.replace("0.1 0.2 0.3 0.4 0.5 0.6 1", "1 .8 32. 20. 1.5 1.3 1.0")
    p = ow3d.read_deck(write(tmp_path, "rb.inp", text))
    assert (p.i_breaking, p.T_half, p.phi_b, p.phi_0) == (1, 0.8, 32.0, 20.0)
    assert (p.del_fac, p.cel_fac, p.gamma_break) == (1.5, 1.3, 1.0)
    assert p.relaxONOFF == 0
    p = ow3d.read_deck(write(tmp_path, "nb.inp", DECK_3D))
    assert (p.i_breaking, p.T_half) == (0, 0.0)


def test_deck_errors(ow3d, tmp_path):
    with pytest.raises(ow3d.OW3DError) as e:
        ow3d.read_deck(tmp_path / "missing.inp")
    assert e.value.status == ow3d.capi.ERR_IO
    bad = DECK_3D.replace("40. 10. 1. 129 33 9 0 0 1 1 1 1", "40. 10. 1. 129 33")
    with pytest.raises(ow3d.OW3DError) as e:
        ow3d.read_deck(write(tmp_path, "bad.inp", bad))
    assert e.value.status == ow3d.capi.ERR_BAD_INPUT
    many = DECK_3D.replace("1 2.0 2 X 0", "1 2.0 9 X 0")
    with pytest.raises(ow3d.OW3DError):
        ow3d.read_deck(write(tmp_path, "many.inp", many))
    # kinematics ranges outside the grid or the run (ReadInputFileParameters.f90:318-330)
    for old, new, what in (("1 65 2 1 1 1 1 100 2", "1 66 2 1 1 1 1 100 2", "x coordinate range"),
                           ("1 65 2 1 1 1 1 100 2", "1 65 2 1 2 1 1 100 2", "y coordinate range"),
                           ("1 65 2 1 1 1 1 100 2", "1 65 2 1 1 1 5 101 2", "time range"),
                           ("-5 20 1 2 ", "-5 20 1 21 ", "too many")):
        with pytest.raises(ow3d.OW3DError, match=what):
            ow3d.read_deck(write(tmp_path, "kin.inp", DECK_2D_CFL.replace(old, new)))


def test_parsed_deck_builds_a_valid_estimate(ow3d, tmp_path):
    import ctypes as C
    p = ow3d.read_deck(write(tmp_path, "a.inp", DECK_3D))
    b = C.c_size_t()
    assert ow3d.lib().ow3d_estimate_bytes(C.byref(p), C.byref(b)) == 0 and b.value > 0


REF_DECKS = reference_decks() or pathlib.Path("/nonexistent")


@pytest.mark.skipif(not REF_DECKS.is_dir(), reason="reference example decks not on this machine")
def test_reference_example_decks_parse(ow3d):
    decks = sorted(f for f in REF_DECKS.iterdir() if f.name.startswith("OceanWave3D.inp"))
    assert decks
    parsed = 0
    for f in decks:
        try:
            p = ow3d.read_deck(f)
        except ow3d.OW3DError:
            continue
        parsed += 1
        assert p.Nx >= 1 and p.Ny >= 1 and p.Nz >= 2
        assert p.GMRESmaxiterations >= 1 and p.reltol > 0
        assert p.cyclet in (b"V", b"W", b"F")
        if p.formattype in (20, 21):
            # the kinematics lines follow line 9 (counted without blank lines)
            lines = [ln for ln in f.read_text(errors="replace").splitlines()]
            i9 = next(i for i, ln in enumerate(lines[1:], 1)
                      if ln.split()[:2] == [str(p.StoreDataONOFF), str(p.formattype)])
            for q in range(p.nOutFiles):
                want = [int(float(v)) for v in lines[i9 + 1 + q].replace(",", " ").split()[:9]]
                assert list(p.kinematics[q]) == want, (f.name, q)
    assert parsed >= 0.8 * len(decks), (parsed, len(decks))


def test_decks_needing_unbuilt_features_are_refused(ow3d, tmp_path):
    """A deck that turns on a feature outside this library's path (pressure
    damping in 3-D, SWENSE, flux wave generation, a constant-flux current) is
    refused with OW3D_ERR_UNSUPPORTED by ow3d_create and
    ow3d_estimate_bytes instead of running without it."""
    import ctypes as C
    L = ow3d.lib()
    base = DECK_3D + "0 0\n0 2.0 2 0 0 1 0\n0\n"

    def status(text):
        p = ow3d.read_deck(write(tmp_path, "f.inp", text))
        return L.ow3d_estimate_bytes(C.byref(p), C.byref(C.c_size_t())), p

    st, p = status(base)
    assert st == 0 and (p.PDampingONOFF, p.swenseONOFF, p.curvilinearONOFF, p.i_breaking) == (0, 0, 0, 0)
    cases_ = {
        "pressure": base.replace("0 0\n0 2.0 2", "1 1\n0. 5. 0. 10. 0.1 0.1 0\n0 2.0 2"),
        "SWENSE": base.replace("0 2.0 2 0 0 1 0", "1 2.0 2 0 0 1 0"),
    }
    for what, text in cases_.items():
        st, p = status(text)
        assert st == ow3d.capi.ERR_UNSUPPORTED, (what, st)
    # IncWaveType 3, the flux wavemaker, with its line after the curvilinear
    # line (its signal is installed at run time, tests/test_flux_wavemaker.py)
    st, p = status(base.replace("-1 0  ", "-1 3  ") + "2. 3 paddle.dat\n")
    assert st == 0 and (p.IncWaveType, p.flux_ramp, p.flux_order) == (3, 2.0, 3)
    # IncWaveType 4, the stream-function wave on a current, is read as 1 with
    # the current flag (tests/test_current.py)
    st, p = status(base.replace("-1 0  ", "-1 4  "))
    assert st == 0 and (p.IncWaveType, p.current_flag) == (1, 1)
    st, p = status(base.replace("-1 0  ", "-1 0 1000. "))
    assert st == 0 and p.accel_from_deck == 1
    # the breaking model acts on x flumes only (Runge_Kutta_4.f90:55): a 3-D
    # deck with it on runs without it, as in the reference
    st, p = status(base.replace("1 6 10 0.08 0.08 0.4", "1 6 10 0.08 0.08 0.4\n1 1.0 32. 20. 1.5 1.3 1.0"))
    assert st == 0 and p.i_breaking == 1
    # local smoothing by the vertical acceleration is built: every limit up to
    # 100 g that a deck gives turns it on (LocalSmoothing2D.f90:37), 0 and
    # negative values included
    for text in ("-1 0 0.5 ", "-1 0 100. ", "-1 0 0. ", "-1 0 -5. "):
        st, p = status(base.replace("-1 0  ", text))
        assert st == 0 and p.accel_from_deck == 1, text
