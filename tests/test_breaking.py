"""The roller breaking model of x flumes (DetectBreaking.f90, called at every
RK stage from Runge_Kutta_4.f90:55,164,241,336 and after the step from
OceanWave3DTakeATimeStep.f90:45-49; its Qr_x enters the kinematic condition,
rhsFreeSurface3D.f90:17).

CPU: the oracle's restatement against a second, pure-Python restatement of
the same lines on seeded synthetic surfaces with many rollers (several per
32-column chunk, rollers that overlap, the roller-angle state carried from
call to call), and the oracle's runs: rollers form on a steep wave, the
roller term changes the run with i_breaking = 1 and leaves it bitwise
unchanged with i_breaking = 2 (geometry only).
GPU: the device kernel against the oracle on the same surfaces (roller
counts, toes and extents exact; positions, elevations, thicknesses, angles
and Qr_x to 1e-12), and the device's runs with the model on against the
device-ordered oracle (1e-10 after the run, the rollers of every checked
step exact), direct and captured steps alike.
"""
import math

import numpy as np
import pytest

import cases

DEG = math.acos(-1.0) / 180.0


def detect_breaking_py(E, tan_phi, prm, update):
    """DetectBreaking.f90:72-201, restated with the reference's 1-based loops
    (pure Python; small cases only). Returns (rollers, tan_phi after the
    call, Qr_x); each roller is [npts, toe, x, eta] plus, with update,
    [thickness behind the toe, tan(phi) at the toe]."""
    nfx = len(E)
    dx = prm["dx"]
    dx_inv = 1.0 / dx
    et = lambda j: float(E[j - 1])
    tan_old = [float(t) for t in tan_phi]
    thick = [0.0] * (nfx + 2)
    Qr = [0.0] * (nfx + 2)
    eta_x = [0.0] * (nfx + 2)
    for j in range(2, nfx - 1):
        eta_x[j] = dx_inv * (et(j + 1) - et(j))
    rollers = []
    for j in range(nfx - 2, 2, -1):
        tphib = tan_old[j - 1]
        if eta_x[j - 1] < -tphib and eta_x[j] >= -tphib and thick[j] <= 0.0:
            a = 0.5 * dx_inv * (eta_x[j] - eta_x[j - 1])
            b = 0.5 * (eta_x[j] + eta_x[j - 1])
            c = et(j)
            dxr = -(tphib + b) / (2.0 * a)
            xr = (j - 1) * dx + dxr
            jr = int(xr * dx_inv) + 2
            sr = a * dxr * dxr + b * dxr + c
            n = 0
            for i in range(jr - 1, 2, -1):
                d = prm["del_fac"] * (et(i) - (sr + tphib * (xr - (i - 1) * dx)))
                if d < 0.0:
                    break
                if d > et(i) - sr:
                    d = et(i) - sr
                thick[i] = d
                n += 1
                Qr[i] = prm["g"] * thick[i]
            rollers.append([n, jr, xr, sr])
    new_tan = list(tan_old)
    if update:
        new_tan = [prm["tan_b"]] * nfx
        for n, jr, _, _ in rollers:
            t = tan_old[jr - 1]
            for i in range(1, n + 4):
                idx = jr + 4 - i
                if 1 <= idx <= nfx:
                    new_tan[idx - 1] = t + prm["dt"] / prm["T_half"] * (prm["tan_0"] - t)
        for r in rollers:
            r += [thick[r[1] - 1], new_tan[r[1] - 1]]
    Qr_x = [0.0] * nfx
    if rollers and prm["i_breaking"] == 1:
        for j in range(3, nfx - 1):
            Qr_x[j - 1] = 0.25 * Qr[j + 1] + 0.5 * Qr[j] + 0.25 * Qr[j - 1]
    return rollers, np.array(new_tan), np.array(Qr_x)


BREAK = dict(i_breaking=1, T_half=0.8, phi_b=20.0, phi_0=10.0, del_fac=1.5, cel_fac=1.3, gamma_break=1.0)


def flume(Nx=257, L=8.0, **kw):
    args = dict(BREAK)
    args.update(kw)
    p, geo = cases.flat_2d(Nx=Nx, Nz=9, L=L, **args)
    prm = dict(dx=L / (Nx - 1), g=p.g, del_fac=p.del_fac, dt=p.dt, T_half=p.T_half,
               tan_b=math.tan(DEG * p.phi_b), tan_0=math.tan(DEG * p.phi_0), i_breaking=p.i_breaking)
    return p, geo, prm


def profiles(p, n=6, seed=3):
    """Seeded surfaces with steep fronts: a gentle swell plus fronts of
    random height and width, some packed closer than 32 columns, some
    overlapping another front's roller."""
    rng = np.random.default_rng(seed)
    Nxg = p.Nx + 2
    x = (np.arange(Nxg) - 1) * (p.Lx / (p.Nx - 1))
    out = []
    for _ in range(n):
        E = 0.02 * np.sin(2 * np.pi * x / p.Lx * rng.integers(1, 4) + rng.uniform(0, 6.3))
        for _ in range(int(rng.integers(4, 12))):
            x0 = rng.uniform(0.1, 0.95) * p.Lx
            A, w = rng.uniform(0.01, 0.1), rng.uniform(0.02, 0.15)
            E += -A * np.tanh((x - x0) / w) + A * np.exp(-((x - x0 + 2 * w) / (2 * w)) ** 2)
        out.append(E)
    return out


def _same_rollers(got, want, tol=1e-12):
    n = len(want)
    assert len(got["npts"]) == n
    if n == 0:
        return
    w = np.array(want, dtype=float)
    assert np.array_equal(got["npts"], w[:, 0].astype(int))
    assert np.array_equal(got["toe"], w[:, 1].astype(int))
    for k, name in enumerate(("x", "eta", "thickness", "tan_phi"), start=2):
        np.testing.assert_allclose(got[name], w[:, k], rtol=0, atol=tol, err_msg=name)


def test_oracle_detection_matches_python_restatement(oracle):
    p, geo, prm = flume()
    o = oracle.Oracle(p, geo["h"], mode=oracle.MODE_DEVICE)
    tan = np.full(o.C, prm["tan_b"])
    total = 0
    for k, E in enumerate(profiles(p)):
        update = k % 3 != 1     # calls without the update keep the angle state
        rollers, tan, qx = detect_breaking_py(E, tan, prm, update)
        o.detect_breaking(E, update)
        t_o, q_o = o.breaking_state()
        np.testing.assert_allclose(t_o, tan, rtol=0, atol=1e-14)
        np.testing.assert_allclose(q_o, qx, rtol=0, atol=1e-12)
        if update:
            _same_rollers(o.rollers(), rollers)
        total += len(rollers)
    assert total >= 20                     # the surfaces do break


def test_oracle_rollers_overlap_and_pack():
    """The seeded surfaces exercise the cases the warp-parallel search
    handles specially: toes closer than 32 columns and toes skipped because
    an earlier roller covers them."""
    p, geo, prm = flume()
    packed = skipped = 0
    tan = np.full(p.Nx + 2, prm["tan_b"])
    for E in profiles(p):
        rollers, tan, _ = detect_breaking_py(E, tan, prm, True)
        toes = sorted(r[1] for r in rollers)
        packed += sum(1 for a, b in zip(toes, toes[1:]) if b - a < 32)
        # candidates that the thickness test rejected
        nfx = len(E)
        ex = np.zeros(nfx + 2)
        ex[2:nfx - 1] = (E[2:nfx - 1] - E[1:nfx - 2]) / prm["dx"]
        cands = sum(1 for j in range(3, nfx - 1) if ex[j - 1] < -prm["tan_b"] <= ex[j])
        skipped += cands - len(rollers)
    assert packed >= 5
    assert skipped >= 1


def _steep_flume(ow3d, i_breaking, steps, **kw):
    W = ow3d.workloads
    args = dict(BREAK, i_breaking=i_breaking)
    args.update(kw)
    p, geo, E0, P0, targets = W.stream_function_2d(n_waves=4, ppw=32, steepness=0.8, steps=steps, **args)
    return p, geo, E0, P0, targets


def _oracle_run(oracle, p, geo, E0, P0, targets, steps, mode):
    o = oracle.Oracle(p, geo["h"], mode=mode)
    o.set_state(E0, P0)
    mode_t, nt, dts, eta, phis = targets[0]
    o.set_relax_target(0, mode_t, nt, dts, eta, phis)
    rollers = []
    for _ in range(steps):
        assert o.step(1) >= 0
        rollers.append(o.rollers())
    return o, rollers


def test_oracle_breaking_changes_the_run_only_with_the_roller_term(ow3d, oracle):
    steps = 30
    runs = {}
    threads = oracle.set_threads(0)
    oracle.set_threads(1)       # one thread: the runs are bitwise reproducible
    try:
        for ib in (0, 1, 2):
            p, geo, E0, P0, targets = _steep_flume(ow3d, ib, steps)
            o, rollers = _oracle_run(oracle, p, geo, E0, P0, targets, steps, oracle.MODE_DEVICE)
            runs[ib] = (o.get_state(), rollers)
    finally:
        oracle.set_threads(threads)
    E0s, E1s, E2s = (runs[k][0][0] for k in (0, 1, 2))
    assert sum(len(r["npts"]) for r in runs[1][1]) > 0        # rollers on the steep fronts
    assert np.array_equal(E2s, E0s)                            # geometry only: the run is unchanged
    assert np.array_equal(runs[2][0][1], runs[0][0][1])
    assert np.max(np.abs(E1s - E0s)) > 1e-6                    # the roller term acts
    assert len(runs[0][1][-1]["npts"]) == 0                    # off: no rollers reported


def test_breaking_parameters_checked(ow3d):
    """T_half > 0 (the angle update divides by it), f_delta >= 0, and wall
    boundaries are required of an x flume with the model on; a 3-D deck with
    i_breaking set is accepted and runs without it, as in the reference
    (Runge_Kutta_4.f90:55 tests FineGrid%ny == 1)."""
    import ctypes as C
    L = ow3d.lib()
    b = C.c_size_t()
    bad = (dict(T_half=0.0), dict(T_half=-1.0), dict(del_fac=-0.5), dict(periodic_x=1))
    for change in bad:
        args = dict(BREAK)
        args.update(change)
        q = ow3d.default_params(Nx=33, Nz=9, Lx=2.0, **args)
        assert L.ow3d_estimate_bytes(C.byref(q), C.byref(b)) == ow3d.capi.ERR_BAD_INPUT, change
    q = ow3d.default_params(Nx=33, Nz=9, Lx=2.0, **BREAK)
    assert L.ow3d_estimate_bytes(C.byref(q), C.byref(b)) == 0
    q = ow3d.default_params(Nx=17, Ny=17, Nz=9, Lx=2.0, Ly=2.0, **dict(BREAK, T_half=0.0))
    assert L.ow3d_estimate_bytes(C.byref(q), C.byref(b)) == 0


# ------------------------------------------------------------------ GPU

@pytest.mark.gpu
def test_device_detection_matches_oracle(ow3d, oracle):
    p, geo, prm = flume()
    o = oracle.Oracle(p, geo["h"], mode=oracle.MODE_DEVICE)
    sim = ow3d.Simulation(p, **geo)
    for k, E in enumerate(profiles(p, n=8, seed=11)):
        update = k % 3 != 1
        o.detect_breaking(E, update)
        sim.detect_breaking(E, update)
        t_o, q_o = o.breaking_state()
        t_d, q_d = sim.breaking_state()
        np.testing.assert_allclose(t_d, t_o, rtol=0, atol=1e-14)
        np.testing.assert_allclose(q_d, q_o, rtol=0, atol=1e-12)
        if update:
            want = o.rollers()
            got = sim.rollers()
            for name in ("npts", "toe"):
                assert np.array_equal(got[name], want[name]), name
            for name in ("x", "eta", "thickness", "tan_phi"):
                np.testing.assert_allclose(got[name], want[name], rtol=0, atol=1e-12, err_msg=name)


@pytest.mark.gpu
@pytest.mark.parametrize("i_breaking", [1, 2])
@pytest.mark.parametrize("graphs", [0, 1], ids=["direct", "graphs"])
def test_device_breaking_run_matches_oracle(ow3d, oracle, i_breaking, graphs):
    steps = 40
    p, geo, E0, P0, targets = _steep_flume(ow3d, i_breaking, steps)
    o, rollers_o = _oracle_run(oracle, p, geo, E0, P0, targets, steps, oracle.MODE_DEVICE)
    sim = ow3d.Simulation(p, **geo)
    assert ow3d.lib().ow3d_set_graphs(sim.h, graphs) == 0
    sim.set_state(E0, P0)
    mode_t, nt, dts, eta, phis = targets[0]
    sim.set_relax_target(0, mode_t, nt, dts, eta, phis)
    seen = 0
    for s in range(steps):
        assert sim.step(1) >= 0
        got, want = sim.rollers(), rollers_o[s]
        assert np.array_equal(got["npts"], want["npts"]) and np.array_equal(got["toe"], want["toe"]), s
        np.testing.assert_allclose(got["x"], want["x"], rtol=0, atol=1e-9)
        seen += len(got["npts"])
    assert seen > 0
    Ed, Pd, _, phid, _ = sim.get_state()
    Eo, Po, _, phio, _ = o.get_state()
    for a, b in ((Ed, Eo), (Pd, Po), (phid, phio)):
        assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < 1e-10
