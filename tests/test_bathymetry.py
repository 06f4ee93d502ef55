"""Bathymetry files of decks with Lz <= 0 (ow3d_read_bathymetry,
SetupInitialConditions.f90:51-111 and OceanWave3DT0Setup.f90:346-364),
host-only: the file name on deck line 3, both gradient flags, the ghost
extension, and derivatives exact for a polynomial depth (the 7-point stencils
differentiate degree <= 6 exactly away from the copied ghost values).
"""
import os
import pathlib

import numpy as np
import pytest
from conftest import reference_decks

DECK = """bathymetry from a file
0 0
20. 1. -1. 33 9 9 0 0 1 1 1 1 bottom.dat   <- Lz <= 0: file
3 3 3 1 1 1
100 0.02 1 0 1
9.81
1 3 0 23 1e-8 1e-6 1 V 1 1 20 12
0.1 1. 3. 2. 0 0. 1 6 24
0 0
1 0
0 6 10 0.08 0.08 0.4
0 2.0 0 X 0
"""


def _write(tmp_path, flag, rows):
    f = tmp_path / "bottom.dat"
    body = "\n".join(" ".join(f"{v:.17e}" for v in r) for r in rows)
    f.write_text(f"% test bottom\n{flag}  <- gradient flag\n{body}\n")
    return f


def _interior_xy(p):
    x = np.arange(p.Nx) * p.Lx / (p.Nx - 1)
    y = np.arange(p.Ny) * p.Ly / (p.Ny - 1)
    return np.meshgrid(x, y)


def test_file_name_on_line_3(ow3d, tmp_path):
    d = tmp_path / "deck.inp"
    d.write_text(DECK)
    p = ow3d.read_deck(d)
    assert p.Lz == -1.0 and p.bathymetry_file == b"bottom.dat"
    with pytest.raises(ow3d.OW3DError, match="bathymetry file name"):
        d.write_text(DECK.replace(" bottom.dat   <- Lz <= 0: file", ""))
        ow3d.read_deck(d)


def test_flag_0_values_and_ghosts(ow3d, tmp_path):
    (tmp_path / "deck.inp").write_text(DECK)
    p = ow3d.read_deck(tmp_path / "deck.inp")
    X, Y = _interior_xy(p)
    h = 1 + 0.01 * X + 0.02 * Y
    rows = [(h[j, i], 0.01, 0.0, 0.02, 0.0) for j in range(p.Ny) for i in range(p.Nx)]
    _write(tmp_path, 0, rows)
    geo, flag = ow3d.read_bathymetry(p, deck_dir=tmp_path)
    assert flag == 0
    H = geo["h"].reshape(p.Ny + 2, p.Nx + 2)
    assert np.array_equal(H[1:-1, 1:-1], h)
    assert np.array_equal(H[:, 0], H[:, 1]) and np.array_equal(H[:, -1], H[:, -2])
    assert np.array_equal(H[0, :], H[1, :]) and np.array_equal(H[-1, :], H[-2, :])
    assert np.all(geo["hx"] == 0.01) and np.all(geo["hy"] == 0.02) and not geo["hxx"].any()


def test_flag_1_numerical_derivatives(ow3d, tmp_path):
    (tmp_path / "deck.inp").write_text(DECK)
    p = ow3d.read_deck(tmp_path / "deck.inp")
    X, Y = _interior_xy(p)
    h = 1 + 0.002 * X ** 2 + 0.01 * Y ** 3
    _write(tmp_path, 1, [(h[j, i],) for j in range(p.Ny) for i in range(p.Nx)])
    geo, flag = ow3d.read_bathymetry(p, deck_dir=tmp_path)
    assert flag == 1
    HX = geo["hx"].reshape(p.Ny + 2, p.Nx + 2)
    HXX = geo["hxx"].reshape(p.Ny + 2, p.Nx + 2)
    HY = geo["hy"].reshape(p.Ny + 2, p.Nx + 2)
    # interior points whose 7-point windows avoid the copied ghost values
    sx, sy = slice(5, p.Nx - 3), slice(5, p.Ny - 3)
    Xi, Yi = X[sy.start - 1:sy.stop - 1, sx.start - 1:sx.stop - 1], Y[sy.start - 1:sy.stop - 1, sx.start - 1:sx.stop - 1]
    assert np.max(np.abs(HX[sy, sx] - 0.004 * Xi)) < 1e-10
    assert np.max(np.abs(HXX[sy, sx] - 0.004)) < 1e-9
    assert np.max(np.abs(HY[sy, sx] - 0.03 * Yi ** 2)) < 1e-10


def test_errors(ow3d, tmp_path):
    (tmp_path / "deck.inp").write_text(DECK)
    p = ow3d.read_deck(tmp_path / "deck.inp")
    with pytest.raises(ow3d.OW3DError):
        ow3d.read_bathymetry(p, path=tmp_path / "missing.dat")
    _write(tmp_path, 0, [(1.0, 0.0)] * (p.Nx * p.Ny))
    with pytest.raises(ow3d.OW3DError, match="needs 5 values"):
        ow3d.read_bathymetry(p, deck_dir=tmp_path)


REF = reference_decks() or pathlib.Path("/nonexistent")


@pytest.mark.skipif(not (REF / "beach_137").exists(), reason="reference example files not on this machine")
def test_reference_beach_file(ow3d):
    """The reference's own bathymetry example with the deck that names it."""
    p = ow3d.read_deck(REF / "OceanWave3D.inp.RandomWave2DShoaling")
    assert p.bathymetry_file == b"beach_137"
    geo, flag = ow3d.read_bathymetry(p, deck_dir=REF)
    assert flag == 0
    rows = [ln.split() for ln in (REF / "beach_137").read_text().splitlines()[2:] if ln.strip()]
    h = np.array([float(r[0]) for r in rows])
    assert np.array_equal(geo["h"][1:-1], h) and geo["h"][0] == h[0] and geo["h"][-1] == h[-1]
    assert np.array_equal(geo["hx"][1:-1], [float(r[1]) for r in rows])
