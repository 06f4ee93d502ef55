"""The device's Gauss-Seidel smoother in the reference's lexicographic row order
(ow3d_set_smoother_order(h, OW3D_SMOOTHER_LEXICOGRAPHIC)) against the
reference-ordered oracle (MODE_REFERENCE): the special rows, then per
smoothing step a sweep over all rows in index order and the special rows
again (GaussSeidel.f90:15-26, GaussSeidelSpecialPoints.f90:43-53,
MultiGridSolver.f90:118-126,174-181), and left-preconditioned GMRES with the
reference's stopping test (iterative_solution.f90:23-24,58-60).

The device runs the sweep as wavefronts and the special rows in three
parallel phases; the results are those of the sequential order up to
rounding: 1e-11 relative on a smoothing, 1e-10 on a preconditioner
application and after whole runs, and GMRES matvec counts within one per
solve. The whole-run comparisons against the committed reference-ordered
fixtures (tests/golden/run_*_ref.npz) are in test_gpu_fullrun.py.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

RTOL_SMOOTH = 1e-11
RTOL_RUN = 1e-10


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


CASES = [
    (cases.flat_2d, dict(Nx=17, Nz=9)),
    (cases.slope_2d, dict(Nx=33, Nz=9)),
    (cases.bump_3d, dict(Nx=17, Ny=9, Nz=9)),
    (cases.bump_3d, dict(Nx=33, Ny=17, Nz=9)),
    (cases.bump_3d, dict(Nx=65, Ny=33, Nz=9, amp=0.0)),
    # finest level above the shared-memory size: a thread-block cluster
    (cases.bump_3d, dict(Nx=129, Ny=33, Nz=9)),
    # finest level whose window does not fit a cluster block, and a long 2-D
    # level: one block from global memory
    (cases.bump_3d, dict(Nx=1025, Ny=9, Nz=9)),
    (cases.flat_2d, dict(Nx=4097, Nz=9, L=64.0)),
]
IDS = ["flat2d", "slope2d", "bump3d-17x9", "bump3d-33x17", "flat3d-65x33", "bump3d-129x33-cluster",
       "bump3d-1025x9-global", "flat2d-4097-global"]


def make(ow3d, oracle, case, **kw):
    p, geo = case(**kw)
    sim = ow3d.Simulation(p, **geo)
    sim.set_smoother_order(ow3d.capi.SMOOTHER_LEXICOGRAPHIC)
    orc = oracle.Oracle(p, **geo, mode=oracle.MODE_REFERENCE)
    return p, sim, orc


@pytest.mark.parametrize("case,kw", CASES, ids=IDS)
def test_lexicographic_smoothing_matches_reference_order(ow3d, oracle, case, kw):
    p, sim, orc = make(ow3d, oracle, case, **kw)
    rng = np.random.default_rng(11)
    for l in range(1, sim.level_count()):
        n = sim.level_size(l)
        x = rng.standard_normal(n); b = rng.standard_normal(n)
        for nu in (1, 2):
            assert rel(sim.level_op(l, 1, x, b, nu=nu), orc.level_smooth(l, x, b, nu=nu)) < RTOL_SMOOTH, \
                f"level {l}, nu {nu}"


def test_lexicographic_differs_from_multicolour(ow3d, oracle):
    """The two orders are different smoothers: the check above would not pass
    with the multicolour order."""
    p, sim, orc = make(ow3d, oracle, cases.bump_3d, Nx=17, Ny=9, Nz=9)
    l = sim.level_count() - 1
    rng = np.random.default_rng(3)
    n = sim.level_size(l)
    x = rng.standard_normal(n); b = rng.standard_normal(n)
    ref = orc.level_smooth(l, x, b, nu=1)
    sim.set_smoother_order(ow3d.capi.SMOOTHER_MULTICOLOUR)
    assert rel(sim.level_op(l, 1, x, b, nu=1), ref) > 1e-3
    sim.set_smoother_order(ow3d.capi.SMOOTHER_LEXICOGRAPHIC)
    assert rel(sim.level_op(l, 1, x, b, nu=1), ref) < RTOL_SMOOTH


@pytest.mark.parametrize("case,kw", CASES, ids=IDS)
def test_lexicographic_vcycle_matches_reference_order(ow3d, oracle, case, kw):
    p, sim, orc = make(ow3d, oracle, case, **kw)
    r = cases.field3(p, seed=7)
    assert rel(sim.precondition(r), orc.precond(r)) < RTOL_RUN


def test_smoother_order_rejects_unknown(ow3d):
    p, geo = cases.flat_2d()
    sim = ow3d.Simulation(p, **geo)
    assert ow3d.lib().ow3d_set_smoother_order(sim.h, 2) == ow3d.capi.ERR_BAD_INPUT
    assert ow3d.lib().ow3d_set_smoother_order(sim.h, -1) == ow3d.capi.ERR_BAD_INPUT


def test_periodic_wave_200_steps_matches_reference_order(ow3d, oracle):
    """The periodic 65 x 9 wave, 200 RK4 steps in FP64 with left GMRES and the
    lexicographic smoother, against the reference-ordered oracle run here."""
    p, geo, E0, P0, info = ow3d.workloads.periodic_wave_2d(krylov=ow3d.capi.KRYLOV_LGMRES)
    sim = ow3d.Simulation(p, **geo)
    sim.set_smoother_order(ow3d.capi.SMOOTHER_LEXICOGRAPHIC)
    o = oracle.Oracle(p, **geo, mode=oracle.MODE_REFERENCE)
    for s in (sim, o):
        s.set_state(E0, P0)
    its = cases.run_steps(sim, 200)
    its_o = cases.run_steps(o, 200)
    E, P, W, phi, t = sim.get_state()
    Eo, Po, Wo, phio, to = o.get_state()
    assert abs(t - to) < 1e-12
    errs = {"E": rel(E, Eo), "P": rel(P, Po), "phi": rel(phi, phio)}
    assert max(errs.values()) < RTOL_RUN, errs
    assert np.all(np.abs(its - its_o) <= 4), (its - its_o)


def test_mixed_precision_lexicographic_steps(ow3d, oracle):
    """The lexicographic smoother in the FP32 hierarchy of the mixed form:
    five steps of the 3-D bump with left GMRES against the reference-ordered
    FP64 oracle, to the FP32 preconditioner's level (the left-preconditioned
    solution carries its rounding), and the same matvec counts within one per
    solve."""
    p, geo = cases.bump_3d(Nx=33, Ny=17, Nz=9, dt=0.02)
    p.krylov = ow3d.capi.KRYLOV_LGMRES
    p.precision = ow3d.capi.PREC_MIXED
    sim = ow3d.Simulation(p, **geo)
    sim.set_smoother_order(ow3d.capi.SMOOTHER_LEXICOGRAPHIC)
    o = oracle.Oracle(p, **geo, mode=oracle.MODE_REFERENCE)
    E0 = cases.surface(p, amp=0.02, seed=4)[0]
    for s in (sim, o):
        s.set_state(E0, np.zeros_like(E0))
    its = cases.run_steps(sim, 5)
    its_o = cases.run_steps(o, 5)
    E, P, W, phi, t = sim.get_state()
    Eo, Po, Wo, phio, to = o.get_state()
    errs = {"E": rel(E, Eo), "P": rel(P, Po), "phi": rel(phi, phio)}
    assert max(errs.values()) < 1e-5, errs
    assert np.all(np.abs(its - its_o) <= 4), (its - its_o)
