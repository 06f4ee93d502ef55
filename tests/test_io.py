"""Result and hot-start files of the reference (io.cpp):

* EP_#####.bin: Fortran unformatted records with 32-bit length markers,
  as StoreData writes them (src/IO/StoreData.f90:11-29);
* fort.NNN: "x y E P" per point in the edit descriptor 4e16.6e3 with an empty
  line after each row (src/IO/StoreDataAscii.f90:21-31);
* OceanWave3D.end / .init: header, "Lx Ly Nx Ny time", "E P" per interior
  point (OceanWave3DTakeATimeStep.f90:146-162, ReadInputFileParameters.f90:113-125).

The host-only functions run on CPU; the handle forms (state copied off the
device, the StoreDataONOFF schedule) are marked gpu.
"""
import decimal
import pathlib

import numpy as np
import pytest

import cases  # noqa: F401  (puts tests/ on the path for the package loader)
from conftest import reference_decks

REF_INPUTS = reference_decks() or pathlib.Path("/nonexistent")


def fortran_e16_6e3(v):
    """Fortran E16.6E3 from its definition: 0.dddddd x 10^e with the six
    digits correctly rounded (half to even on the exact binary value), the
    exponent signed with three digits, right-justified in 16 columns."""
    if v == 0.0:
        return f"{'0.000000E+000':>16}"
    d = decimal.Decimal(abs(v))
    e = d.adjusted() + 1                                   # 10^(e-1) <= |v| < 10^e
    m = (d.scaleb(-e)).quantize(decimal.Decimal("0.000001"), rounding=decimal.ROUND_HALF_EVEN)
    if m >= 1:                                             # rounding carried to 1.000000
        m, e = decimal.Decimal("0.100000"), e + 1
    body = f"{'-' if v < 0 else ''}0.{str(m)[2:]}E{'-' if e < 0 else '+'}{abs(e):03d}"
    return f"{body:>16}"


def test_fortran_edit_descriptor_known_answers():
    assert fortran_e16_6e3(1.5) == "   0.150000E+001"
    assert fortran_e16_6e3(-0.00123) == "  -0.123000E-002"
    assert fortran_e16_6e3(0.0) == "   0.000000E+000"
    assert fortran_e16_6e3(123456789.0) == "   0.123457E+009"
    assert fortran_e16_6e3(9.9999996) == "   0.100000E+002"


def _arrays(nx, ny, seed=3):
    rng = np.random.default_rng(seed)
    x = np.tile(np.linspace(-0.1, 5.0, nx), ny)
    y = np.repeat(np.linspace(0.0, 2.0, ny), nx)
    E = rng.standard_normal(nx * ny) * 10.0 ** rng.integers(-12, 4, nx * ny)
    P = rng.standard_normal(nx * ny)
    E[3] = 0.0
    P[5] = 9.9999996
    return x, y, E, P


def test_ep_file_records(ow3d, tmp_path):
    L = ow3d.lib()
    nx, ny = 13, 5
    x, y, E, P = _arrays(nx, ny)
    path = tmp_path / "EP_00007.bin"
    assert L.ow3d_write_ep_file(str(path).encode(), nx, ny, *[ow3d._d(np.ascontiguousarray(a)) for a in (x, y, E, P)]) == 0
    raw = path.read_bytes()
    n = nx * ny
    # record 1: two int32 framed by markers 8; records 2, 3: 2n doubles framed by 16n
    assert np.frombuffer(raw, "<i4", 4, 0).tolist() == [8, nx, ny, 8]
    assert np.frombuffer(raw, "<i4", 1, 16)[0] == 16 * n
    assert len(raw) == 16 + 2 * (16 * n + 8)
    got = ow3d.load_ep(path)
    assert got[0] == nx and got[1] == ny
    for a, b in zip(got[2:], (x, y, E, P)):
        assert np.array_equal(a.ravel(), b)


def test_ascii_file_format(ow3d, tmp_path):
    L = ow3d.lib()
    nx, ny = 7, 3
    x, y, E, P = _arrays(nx, ny, seed=5)
    path = tmp_path / "fort.105"
    assert L.ow3d_write_ascii_file(str(path).encode(), nx, ny, *[ow3d._d(np.ascontiguousarray(a)) for a in (x, y, E, P)]) == 0
    lines = path.read_text().split("\n")
    assert len(lines) == ny * (nx + 1) + 1 and lines[-1] == ""
    for j in range(ny):
        for i in range(nx):
            k = j * nx + i
            want = "".join(fortran_e16_6e3(v) for v in (x[k], y[k], E[k], P[k]))
            assert lines[j * (nx + 1) + i] == want, (j, i)
        assert lines[j * (nx + 1) + nx] == ""


def test_end_file_round_trip_and_grid_check(ow3d, tmp_path):
    L = ow3d.lib()
    Nx, Ny = 9, 4
    rng = np.random.default_rng(1)
    E = rng.standard_normal(Nx * Ny) * 1e-3
    P = rng.standard_normal(Nx * Ny)
    path = tmp_path / "OceanWave3D.end"
    assert L.ow3d_write_end_file(str(path).encode(), 8.0, 0.0, Nx, Ny, 12.375, ow3d._d(E), ow3d._d(P)) == 0
    E2, P2, t = ow3d.read_init_file(path, Nx, Ny)
    assert np.array_equal(E, E2) and np.array_equal(P, P2) and t == 12.375
    with pytest.raises(ow3d.OW3DError, match="grids must agree"):
        ow3d.read_init_file(path, Nx + 1, Ny)


@pytest.mark.skipif(not REF_INPUTS.exists(), reason="reference example files not mounted")
@pytest.mark.parametrize("name,nx,ny", [("SFWaveAndFollowingCurrent.init", 641, 1),
                                        ("SFWaveAndOpposingCurrent.init", 641, 1)])
def test_reads_reference_hot_start_files(ow3d, name, nx, ny):
    """The reference's own hot-start examples parse, with their grid sizes."""
    path = REF_INPUTS / name
    E, P, t = ow3d.read_init_file(path, nx, ny)
    rows = [ln.split() for ln in path.read_text().splitlines()[2:] if ln.strip()]
    assert len(rows) == nx * ny
    assert np.allclose(E, [float(r[0]) for r in rows]) and np.allclose(P, [float(r[1]) for r in rows])


@pytest.mark.gpu
def test_handle_writes_state_and_schedule(ow3d, tmp_path):
    p, geo = cases.bump_3d(Nx=17, Ny=9, Nz=9, dt=0.02)
    p.StoreDataONOFF = 2
    sim = ow3d.Simulation(p, **geo)
    x = (np.arange(p.Nx + 2) - 1) / (p.Nx - 1) * p.Lx
    E0 = np.tile(0.01 * np.cos(np.pi * x / p.Lx), p.Ny + 2)
    sim.set_state(E0, np.zeros_like(E0))
    assert sim.store_data(str(tmp_path)) == 2                 # step 0: EP_00000 and the bathymetry file
    assert (tmp_path / "EP_00000.bin").exists() and (tmp_path / "EP_99999.bin").exists()
    sim.step(1)
    assert sim.store_data(str(tmp_path)) == 0                 # step 1: not a multiple of 2
    sim.step(1)
    assert sim.store_data(str(tmp_path)) == 2                 # step 2: EP_00002 and OceanWave3D.end
    E, P, W, phi, t = sim.get_state()
    nx, ny, X, Y, Ef, Pf = ow3d.load_ep(tmp_path / "EP_00002.bin")
    assert (nx, ny) == (p.Nx + 2, p.Ny + 2)
    assert np.array_equal(Ef.ravel(), E) and np.array_equal(Pf.ravel(), P)
    assert np.allclose(X[0], x)
    Ei, Pi, ti = ow3d.read_init_file(tmp_path / "OceanWave3D.end", p.Nx, p.Ny)
    inner = E.reshape(p.Ny + 2, p.Nx + 2)[1:-1, 1:-1].ravel()
    assert np.array_equal(Ei, inner) and abs(ti - t) < 1e-15
    sim.write_ascii(str(tmp_path), 5)
    assert (tmp_path / "fort.105").exists()
    nb, _, _, _, hb, hxb = ow3d.load_ep(tmp_path / "EP_99999.bin")
    assert np.array_equal(hb.ravel(), geo["h"])
