"""Parity of the CUDA path with the CPU oracle (device-matched mode).

Tolerances: operators and multigrid components agree to rounding (1e-12
relative); solves and time steps to 1e-10 relative L-infinity on eta and phi
(the differences come only from reduction order and fused multiply-adds);
GMRES iteration counts within one.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

RTOL_OP = 1e-12
RTOL_RUN = 1e-10


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def make(ow3d, oracle, case, **kw):
    p, geo = case(**kw)
    sim = ow3d.Simulation(p, **geo)
    orc = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    return p, geo, sim, orc


CASES = [
    (cases.flat_2d, dict(Nx=17, Nz=9)),
    (cases.slope_2d, dict(Nx=33, Nz=9)),
    (cases.bump_3d, dict(Nx=17, Ny=9, Nz=9)),
    (cases.bump_3d, dict(Nx=33, Ny=17, Nz=9)),
]
IDS = ["flat2d", "slope2d", "bump3d-17x9", "bump3d-33x17"]


@pytest.mark.parametrize("case,kw", CASES, ids=IDS)
def test_stencils_match(ow3d, oracle, case, kw):
    p, geo, sim, orc = make(ow3d, oracle, case, **kw)
    SX, SY, SZ = sim.stencils()
    oX, oY, oZ = orc.stencils()
    # same Fornberg recurrence; host compilers may contract multiply-adds differently
    assert np.allclose(SX, oX, rtol=1e-13, atol=1e-13 * np.abs(oX).max())
    assert np.allclose(SZ, oZ, rtol=1e-13, atol=1e-13 * np.abs(oZ).max())
    if p.Ny > 1:
        assert np.allclose(SY, oY, rtol=1e-13, atol=1e-13 * np.abs(oY).max())


@pytest.mark.parametrize("case,kw", CASES, ids=IDS)
def test_matvec_random(ow3d, oracle, case, kw):
    p, geo, sim, orc = make(ow3d, oracle, case, **kw)
    surf = cases.surface(p, amp=0.05)
    phi = cases.field3(p)
    y = sim.matvec(phi, *surf)
    orc.set_surface(*surf)
    yo = orc.matvec(phi)
    assert rel(y, yo) < RTOL_OP


def test_matvec_unit_probe_3d(ow3d, oracle):
    """Assemble A column by column (the reference's A.bin probe) on a tiny grid."""
    p, geo, sim, orc = make(ow3d, oracle, cases.bump_3d, Nx=9, Ny=9, Nz=9)
    surf = cases.surface(p, amp=0.05, seed=3)
    orc.set_surface(*surf)
    n = sim.N
    rng = np.random.default_rng(0)
    for c in rng.choice(n, size=60, replace=False):
        e = np.zeros(n); e[c] = 1.0
        assert rel(sim.matvec(e, *surf), orc.matvec(e)) < RTOL_OP


@pytest.mark.parametrize("case,kw", CASES, ids=IDS)
def test_mg_components(ow3d, oracle, case, kw):
    p, geo, sim, orc = make(ow3d, oracle, case, **kw)
    L = sim.level_count()
    assert L == orc.nlevels
    rng = np.random.default_rng(5)
    for l in range(L):
        assert sim.level_dims(l) == orc.level_dims(l)
        n = sim.level_size(l)
        x = rng.standard_normal(n); b = rng.standard_normal(n)
        assert rel(sim.level_op(l, 0, x), orc.level_matvec(l, x)) < RTOL_OP, f"A_l, level {l}"
        if l > 0:
            assert rel(sim.level_op(l, 1, x, b, nu=2), orc.level_smooth(l, x, b, nu=2)) < 1e-11, f"smoother, level {l}"
            assert rel(sim.level_op(l, 2, x), orc.restrict(l, x)) < RTOL_OP, f"restriction, level {l}"
            xc = rng.standard_normal(sim.level_size(l - 1))
            assert rel(sim.level_op(l, 3, xc), orc.prolong(l, xc)) < RTOL_OP, f"prolongation, level {l}"
    b0 = rng.standard_normal(sim.level_size(0))
    assert rel(sim.level_op(0, 4, b0), orc.coarse_solve(b0)) < 1e-10


@pytest.mark.parametrize("case,kw", CASES, ids=IDS)
def test_vcycle(ow3d, oracle, case, kw):
    p, geo, sim, orc = make(ow3d, oracle, case, **kw)
    r = cases.field3(p, seed=7)
    assert rel(sim.precondition(r), orc.precond(r)) < 1e-10


@pytest.mark.parametrize("krylov", [0, 1], ids=["fgmres", "lgmres"])
@pytest.mark.parametrize("case,kw", CASES, ids=IDS)
def test_solve(ow3d, oracle, case, kw, krylov):
    p, geo = case(**kw)
    p.krylov = krylov
    sim = ow3d.Simulation(p, **geo)
    orc = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    surf = cases.surface(p, amp=0.03, seed=11)
    P = np.cos(np.linspace(0, 2 * np.pi, sim.C))
    rhs = cases.fs_rhs(p, P)
    phi0 = np.zeros(sim.N)
    phi, it, st = sim.solve(rhs, phi0, *surf)
    orc.set_surface(*surf)
    phio, ito, res, sto = orc.solve(rhs, phi0)
    assert abs(it - ito) <= 1, (it, ito)
    assert rel(phi, phio) < RTOL_RUN


def _run_both(ow3d, oracle, p, geo, E0, P0, nsteps, targets=None):
    sim = ow3d.Simulation(p, **geo)
    orc = oracle.Oracle(p, **geo, mode=oracle.MODE_DEVICE)
    sim.set_state(E0, P0)
    orc.set_state(E0, P0)
    for z, (mode, nt, dts, eta, phis) in (targets or {}).items():
        sim.set_relax_target(z, mode, nt, dts, eta, phis)
        orc.set_relax_target(z, mode, nt, dts, eta, phis)
    assert sim.step(nsteps) >= 0
    assert orc.step(nsteps) >= 0
    return sim, orc


@pytest.mark.parametrize("nonlinear", [1, 0], ids=["nonlinear", "linear"])
def test_rk4_2d_standing(ow3d, oracle, nonlinear):
    p, geo = cases.flat_2d(Nx=33, Nz=9, L=2.0, LinearONOFF=nonlinear, dt=0.02)
    Nxg = p.Nx + 2
    x = (np.arange(Nxg) - 1) / (p.Nx - 1) * p.Lx
    E0 = 0.02 * np.cos(np.pi * x / p.Lx)
    P0 = np.zeros(Nxg)
    sim, orc = _run_both(ow3d, oracle, p, geo, E0, P0, 10)
    E, P, W, phi, t = sim.get_state()
    Eo, Po, Wo, phio, to = orc.get_state()
    assert abs(t - to) < 1e-14
    assert rel(E, Eo) < RTOL_RUN and rel(P, Po) < RTOL_RUN and rel(phi, phio) < RTOL_RUN
    so = orc.stats(); s = sim.stats()
    assert s["solves"] == so["solves"]
    assert abs(s["total_iterations"] - so["total_iterations"]) <= s["solves"]


def test_rk4_3d_bump_filter_sponge(ow3d, oracle):
    p, geo = cases.bump_3d(Nx=33, Ny=17, Nz=9, Lx=4.0, Ly=2.0, dt=0.02, filteringONOFF=2, filterALPHA=3,
                           filterORDER=4, relaxONOFF=1, relaxNo=1, relaxTransientTime=0.0,
                           zones=[dict(x1=3.0, x2=4.0, y1=0.0, y2=2.0, ftype=9, param=3.5)])
    Nxg, Nyg, _ = p.Nx + 2, p.Ny + 2, p.Nz + 1
    x = (np.arange(Nxg) - 1) / (p.Nx - 1) * p.Lx
    y = (np.arange(Nyg) - 1) / (p.Ny - 1) * p.Ly
    X, Y = np.meshgrid(x, y)
    E0 = (0.01 * np.exp(-((X - 1.5) ** 2 + (Y - 1.0) ** 2) / 0.1)).ravel()
    P0 = np.zeros_like(E0)
    sim, orc = _run_both(ow3d, oracle, p, geo, E0, P0, 6)
    E, P, W, phi, t = sim.get_state()
    Eo, Po, Wo, phio, to = orc.get_state()
    assert rel(E, Eo) < RTOL_RUN and rel(P, Po) < RTOL_RUN and rel(phi, phio) < RTOL_RUN


def test_rk4_2d_generation_zone(ow3d, oracle):
    """Relaxation-zone generation from a tabulated target (linear wave)."""
    p, geo = cases.flat_2d(Nx=65, Nz=9, L=8.0, dt=0.025, relaxONOFF=1, relaxNo=2, relaxTransientTime=0.5,
                           zones=[dict(x1=0.0, x2=2.0, ftype=-10, param=3.5, wavegen=1),
                                  dict(x1=6.0, x2=8.0, ftype=9, param=3.5)])
    sim = ow3d.Simulation(p, **geo)
    i0, i1, j0, j1 = sim.zone_box(0)
    Nxg = p.Nx + 2
    x = (np.arange(Nxg) - 1) / (p.Nx - 1) * p.Lx
    xs = x[i0 - 1:i1]
    k = 2 * np.pi / 2.0; om = np.sqrt(9.81 * k * np.tanh(k)); H = 0.01
    nt = 40
    tt = np.arange(nt) * p.dt
    eta = np.array([0.5 * H * np.cos(k * xs - om * t) for t in tt])
    phis = np.array([0.5 * H * 9.81 / om * np.sin(k * xs - om * t) for t in tt])
    sim.close()
    sim, orc = _run_both(ow3d, oracle, p, geo, np.zeros(Nxg), np.zeros(Nxg), 20,
                         targets={0: (0, nt, p.dt, eta, phis)})
    E, P, W, phi, t = sim.get_state()
    Eo, Po, Wo, phio, to = orc.get_state()
    assert np.max(np.abs(Eo)) > 1e-4
    assert rel(E, Eo) < RTOL_RUN and rel(P, Po) < RTOL_RUN


def test_mixed_precision_error(ow3d, oracle):
    """FP32 multigrid + FP64 FGMRES/RK4 vs the FP64 oracle: eta error <= 1e-6 relative."""
    p, geo = cases.bump_3d(Nx=33, Ny=17, Nz=9, Lx=4.0, Ly=2.0, dt=0.02)
    p.precision = 1
    Nxg, Nyg = p.Nx + 2, p.Ny + 2
    x = (np.arange(Nxg) - 1) / (p.Nx - 1) * p.Lx
    y = (np.arange(Nyg) - 1) / (p.Ny - 1) * p.Ly
    X, Y = np.meshgrid(x, y)
    E0 = (0.01 * np.cos(np.pi * X / p.Lx) * np.cos(np.pi * Y / p.Ly)).ravel()
    sim = ow3d.Simulation(p, **geo)
    q, geo2 = cases.bump_3d(Nx=33, Ny=17, Nz=9, Lx=4.0, Ly=2.0, dt=0.02)
    orc = oracle.Oracle(q, **geo2, mode=oracle.MODE_DEVICE)
    sim.set_state(E0, np.zeros_like(E0)); orc.set_state(E0, np.zeros_like(E0))
    sim.step(10); orc.step(10)
    E, P, W, phi, t = sim.get_state()
    Eo, Po, Wo, phio, to = orc.get_state()
    assert rel(E, Eo) < 1e-6
    assert rel(phi, phio) < 1e-6


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_graph_launched_steps_match_direct_launches(ow3d, precision):
    """FGMRES steps replayed as CUDA graphs (the default from the second solve
    on) give bitwise the same state and launch count as direct launches."""
    # large enough that the finest multigrid level runs outside the fused
    # coarse kernel (the graph path's case; on smaller grids it falls back)
    p, geo = cases.bump_3d(Nx=257, Ny=33, Nz=17, Lx=16.0, Ly=2.0, dt=0.02)
    p.precision = precision
    Nxg, Nyg = p.Nx + 2, p.Ny + 2
    x = (np.arange(Nxg) - 1) / (p.Nx - 1) * p.Lx
    E0 = np.tile(0.01 * np.cos(np.pi * x / p.Lx), Nyg)
    L = ow3d.lib()
    out = []
    for graphs in (1, 0):
        sim = ow3d.Simulation(p, **geo)
        assert L.ow3d_set_graphs(sim.h, graphs) == 0
        sim.set_state(E0, np.zeros_like(E0))
        n0 = L.ow3d_launch_count()
        assert sim.step(3) >= 0
        out.append((sim.get_state(), L.ow3d_launch_count() - n0, sim.stats()["total_iterations"]))
        ng_cached = L.ow3d_test_graph_count(sim.h)
        assert (ng_cached > 0) if graphs else (ng_cached == 0), ng_cached
        sim.close()
    (sg, ng, ig), (sd, nd, idd) = out
    for a, b in zip(sg[:4], sd[:4]):
        assert np.array_equal(a, b)
    # the whole-step graphs of steps 2 and 3 add one record kernel per solve
    # and always run the back-substitution and update
    assert ig == idd and 0 <= ng - nd <= 3 * 4 * 3


def _step_case(ow3d, name):
    """Cases for the whole-step graphs: 3-D bump (FP64 and mixed; finest
    level outside the fused coarse kernel), the shoal basin with its
    generation zone, sponge and a filter every other step (sloping bottom:
    four colours and the level-1 passes), the periodic wave (finest level
    inside the fused coarse kernel) and the stream-function flume
    (relaxation targets at every stage time)."""
    W = ow3d.workloads
    if name.startswith("bump3d"):
        p, geo = cases.bump_3d(Nx=129, Ny=33, Nz=17, Lx=8.0, Ly=2.0, dt=0.02)
        p.precision = 1 if "mixed" in name else 0
        p.krylov = 1 if name.endswith("left") else 0
        x = (np.arange(p.Nx + 2) - 1) / (p.Nx - 1) * p.Lx
        E0 = np.tile(0.01 * np.cos(np.pi * x / p.Lx), p.Ny + 2)
        return p, geo, E0, np.zeros_like(E0), None
    if name.startswith("shoal_filter"):
        p, geo, target = cases.shoal_generation(W, 8, filteringONOFF=2, krylov=1 if name.endswith("left") else 0)
        return p, geo, np.zeros((p.Nx + 2) * (p.Ny + 2)), np.zeros((p.Nx + 2) * (p.Ny + 2)), target
    if name == "periodic":
        p, geo, E0, P0, info = W.periodic_wave_2d()
        return p, geo, E0, P0, None
    p, geo, E0, P0, targets = W.stream_function_2d(ppw=16, steps=8)
    return p, geo, E0, P0, (lambda box: targets[0])


@pytest.mark.parametrize("name", ["bump3d_fp64", "bump3d_mixed", "shoal_filter", "periodic", "sfwave",
                                  "bump3d_fp64_left", "bump3d_mixed_left", "shoal_filter_left"])
def test_step_graphs_match_direct_steps(ow3d, name):
    """Steps replayed as one CUDA graph each (the default from the second
    step on: each solve's Arnoldi steps as conditional nodes that the device
    enables, the time level read on the device) give bitwise the state, the
    matvec counts and the solver records of direct launches, for FGMRES and
    for left-preconditioned GMRES."""
    L = ow3d.lib()
    out = []
    for graphs in (1, 0):
        p, geo, E0, P0, target = _step_case(ow3d, name)
        sim = ow3d.Simulation(p, **geo)
        assert L.ow3d_set_graphs(sim.h, graphs) == 0
        if target is not None:
            sim.set_relax_target(0, *target(sim.zone_box(0)))
        sim.set_state(E0, P0)
        its = cases.run_steps(sim, 6)
        st = sim.stats()
        out.append((sim.get_state(), its, st))
        n = L.ow3d_test_step_graph_count(sim.h)
        assert (n == 2) if graphs else (n == 0), n
        sim.close()
    (sg, ig, tg), (sd, idd, td) = out
    for a, b in zip(sg[:4], sd[:4]):
        assert np.array_equal(a, b)
    assert sg[4] == sd[4]
    assert np.array_equal(ig, idd)
    for k in ("solves", "total_iterations", "min_iterations", "max_iterations", "not_converged",
              "last_residual", "last_initial_residual", "last_tolerance"):
        assert tg[k] == td[k], k


def test_step_batch_matches_single_steps(ow3d):
    """ow3d_step_batch (one host thread, the handles' step graphs launched
    together each round) gives each simulation bitwise the state of stepping
    it alone."""
    import ctypes as C
    L = ow3d.lib()
    W = ow3d.workloads
    specs = [W.periodic_wave_2d(), W.periodic_wave_2d(Nx=129, Nz=9)]
    alone, sims = [], []
    for p, geo, E0, P0, info in specs:
        s = ow3d.Simulation(p, **geo)
        s.set_state(E0, P0)
        assert s.step(5) >= 0
        alone.append(s.get_state())
        s.close()
    for p, geo, E0, P0, info in specs:
        s = ow3d.Simulation(p, **geo)
        s.set_state(E0, P0)
        sims.append(s)
    hs = (C.c_void_p * 2)(*[s.h.value for s in sims])
    ns = (C.c_int * 2)(5, 3)
    stv = (C.c_int * 2)()
    assert L.ow3d_step_batch(hs, 2, ns, stv, None) >= 0
    ns2 = (C.c_int * 2)(0, 2)
    assert L.ow3d_step_batch(hs, 2, ns2, stv, None) >= 0
    for s, a in zip(sims, alone):
        b = s.get_state()
        for x, y in zip(a[:4], b[:4]):
            assert np.array_equal(x, y)
        s.close()
