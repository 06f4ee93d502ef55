"""Fluid kinematics (StoreKinematicData.f90:256-460): u, v, w and the nine
gradient fields, and the Kinematics files.

CPU: the numpy restatement (oracle/kinematics.py) on fields whose
derivatives the 7-point stencils give exactly (polynomials of degree <= 6 in
x and sigma), with and without the chain-rule terms.
GPU: ow3d_kinematics against the restatement on the GPU's own state after a
few steps (3-D bump, nonlinear; 2-D flat, linear), and ow3d_store_kinematics
(formattype 20 and 21) read back record by record.
"""
import numpy as np
import pytest

import cases
from conftest import load_oracle

O = load_oracle()
import kinematics as K  # noqa: E402  (oracle restatement: the checker; on the path with the oracle)

# the device's x/y stencil weights come from exact grid offsets and agree
# with the oracle's to about 1e-13 relative; derivatives of smooth fields
# amplify that by the ratio of a field to its variation over a stencil
TOL = 1e-10


def _oracle(ow3d, p, geo):
    return O.Oracle(p, **geo, mode=O.MODE_DEVICE)


def _xz(orc, p):
    x = (np.arange(orc.Nxg) - 1) / (p.Nx - 1) * p.Lx
    X = np.broadcast_to(x.reshape(1, orc.Nxg, 1), (orc.Nyg, orc.Nxg, orc.Nzg)).ravel()
    Z = np.broadcast_to(orc.fine_z().reshape(1, 1, orc.Nzg), (orc.Nyg, orc.Nxg, orc.Nzg)).ravel()
    return X, Z


def _tables(orc):
    SX, SY, SZ = orc.stencils()
    return SX[0], SY[0], SZ[0]


def test_restatement_exact_on_polynomials(ow3d):
    """phi = x^2 sigma + sigma^3 on a bump: phi_x = 2 x sigma, phi_s = x^2 +
    3 sigma^2 (both exact for the 7-point stencils), so every output field
    has a closed form given s_x = (1 - sigma) h_x / h (eta = 0)."""
    p, geo = cases.bump_3d(Nx=17, Ny=9, Nz=9)
    orc = _oracle(ow3d, p, geo)
    X, Z = _xz(orc, p)
    C, N = orc.C, orc.N
    h, hx, hy = geo["h"], geo["hx"], geo["hy"]
    phi = X ** 2 * Z + Z ** 3
    zero = np.zeros(C)
    SX, SY, SZ = _tables(orc)
    Hn, HXn, HYn = (np.repeat(a, orc.Nzg) for a in (h, hx, hy))
    for nonlinear in (True, False):
        (u, v, w), g = K.kinematics(zero, zero, zero, phi, h, hx, hy, SX, SY, SZ, orc.fine_z(),
                                    orc.Nxg, orc.Nyg, orc.Nzg, nonlinear)
        ps = X ** 2 + 3 * Z ** 2
        sx = (1 - Z) / Hn * HXn if nonlinear else 0.0
        sy = (1 - Z) / Hn * HYn if nonlinear else 0.0
        scale = np.max(np.abs(phi)) + 1
        assert np.max(np.abs(u - (2 * X * Z + sx * ps))) < 1e-10 * scale
        assert np.max(np.abs(v - sy * ps)) < 1e-10 * scale
        assert np.max(np.abs(w - ps / Hn)) < 1e-10 * scale
        # d/ds, d/dx, d/dy of phi_s = x^2 + 3 sigma^2: 6 sigma, 2 x, 0
        assert np.max(np.abs(g[0] - 6 * Z / Hn)) < 1e-9 * scale
        assert np.max(np.abs(g[1] - (2 * X + sx * 6 * Z))) < 1e-9 * scale
        assert np.max(np.abs(g[2] - sy * 6 * Z)) < 1e-9 * scale
    assert N == len(u)


def test_restatement_2d_has_no_v(ow3d):
    p, geo = cases.flat_2d(Nx=17, Nz=9)
    orc = _oracle(ow3d, p, geo)
    X, Z = _xz(orc, p)
    SX, SY, SZ = _tables(orc)
    zero = np.zeros(orc.C)
    (u, v, w), g = K.kinematics(zero, zero, zero, X * Z, geo["h"], zero, zero, SX, SY, SZ, orc.fine_z(),
                                orc.Nxg, orc.Nyg, orc.Nzg, True)
    assert np.max(np.abs(u - Z)) < 1e-12 and np.max(np.abs(w - X)) < 1e-12
    assert not v.any() and not g[2].any() and not g[5].any() and not g[6:].any()


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _gpu_case(ow3d, p, geo, steps):
    sim = ow3d.Simulation(p, **geo)
    E0 = cases.surface(p, amp=0.02, seed=3)[0]
    sim.set_state(E0, np.zeros_like(E0))
    assert sim.step(steps) >= 0
    return sim


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["bump3d_nonlinear", "flat2d_linear"])
def test_kinematics_matches_restatement(ow3d, case):
    """The restatement gets the GPU's own state: phi, eta and the eta
    derivatives the device holds (on the ghost rows these are taken before
    the other direction's ghost update, so an oracle that recomputed them
    from the final eta would differ there), with the oracle's stencils."""
    if case == "bump3d_nonlinear":
        p, geo = cases.bump_3d(Nx=33, Ny=17, Nz=9, dt=0.02)
    else:
        p, geo = cases.flat_2d(Nx=65, Nz=9, dt=0.02)
        p.LinearONOFF = 0
    sim = _gpu_case(ow3d, p, geo, 3)
    try:
        E, P, W, phi, t = sim.get_state()
        Ex, Ey = sim.surface_derivs()
        u, v, w, g = sim.kinematics()
    finally:
        sim.close()
    orc = _oracle(ow3d, p, geo)
    SX, SY, SZ = _tables(orc)
    z = np.zeros(orc.C)
    (uo, vo, wo), go = K.kinematics(E, Ex, Ey if p.Ny > 1 else z, phi, geo["h"], geo.get("hx", z), geo.get("hy", z),
                                    SX, SY, SZ, orc.fine_z(), orc.Nxg, orc.Nyg, orc.Nzg, p.LinearONOFF != 0)
    assert _rel(u, uo) < TOL and _rel(w, wo) < TOL
    if p.Ny > 1:
        assert _rel(v, vo) < TOL
    else:
        assert not v.any()
    for q in range(9):
        if np.any(go[q]):
            assert _rel(g[q], go[q]) < TOL, q
        else:
            assert not g[q].any(), q


@pytest.mark.gpu
@pytest.mark.parametrize("formattype", [20, 21])
def test_store_kinematics_files(ow3d, tmp_path, formattype):
    p, geo = cases.bump_3d(Nx=33, Ny=17, Nz=9, dt=0.02)
    p.formattype, p.iKinematics, p.nOutFiles = formattype, 1, 2
    p.Nsteps = 10
    p.kinematics[0][:] = [3, 30, 3, 2, 15, 4, 1, 10, 2]   # levels 1, 3, 5, ...
    p.kinematics[1][:] = [5, 5, 1, 9, 9, 1, 2, 3, 1]     # one column, levels 2 and 3
    sim = ow3d.Simulation(p, **geo)
    E0 = cases.surface(p, amp=0.02, seed=4)[0]
    sim.set_state(E0, np.zeros_like(E0))
    written = [sim.store_kinematics(str(tmp_path))]       # step 0: headers, level 1 of slice 1
    snaps = {1: sim.kinematics() + (sim.get_state(),)}
    for level in (2, 3):
        sim.step(1)
        written.append(sim.store_kinematics(str(tmp_path)))
        snaps[level] = sim.kinematics() + (sim.get_state(),)
    sim.close()
    assert written == [3, 1, 2]
    Nxg, Nyg, Nzg = p.Nx + 2, p.Ny + 2, p.Nz + 1

    def check(rec, slice_, level):
        u, v, w, g, (E, P, W, phi, t) = snaps[level]
        xb, xe, xs, yb, ye, ys = slice_[:6]
        cols = [(i - 1) + Nxg * (j - 1) for j in range(yb + 1, ye + 2, ys) for i in range(xb + 1, xe + 2, xs)]
        col = lambda F: np.stack([F[c * Nzg:(c + 1) * Nzg] for c in cols])
        assert np.array_equal(rec["eta"], E[cols])
        assert np.array_equal(rec["phi"], col(phi))
        assert np.array_equal(rec["u"], col(u)) and np.array_equal(rec["v"], col(v))
        assert np.array_equal(rec["w"], col(w))
        for q, name in enumerate(ow3d.KINEMATICS_FIELDS[7:]):
            assert np.array_equal(rec[name], col(g[q])), name

    levels = {0: [1, 3], 1: [2, 3]}
    for io in (1, 2):
        r = list(p.kinematics[io - 1])
        if formattype == 20:
            k = ow3d.load_kinematics(tmp_path / f"Kinematics{io:02d}.bin")
            assert k["range"] == r and k["nz"] == Nzg and abs(k["dt"] - p.dt) < 1e-15
            npts = len(range(r[0], r[1] + 1, r[2])) * len(range(r[3], r[4] + 1, r[5]))
            assert k["geometry"].shape == (npts, 5) and len(k["z"]) == Nzg
            assert [len(k["levels"])] == [len(levels[io - 1])]
            for rec, level in zip(k["levels"], levels[io - 1]):
                check(rec, r, level)
        else:
            k0 = ow3d.load_kinematics(tmp_path / f"Kinematics_{io:02d}_00000.bin")
            assert k0["range"] == r and not k0["levels"]
            for level in levels[io - 1]:
                k = ow3d.load_kinematics(tmp_path / f"Kinematics_{io:02d}_{level:05d}.bin")
                assert len(k["levels"]) == 1
                check(k["levels"][0], r, level)
