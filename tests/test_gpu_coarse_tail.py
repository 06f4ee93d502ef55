"""The fused coarse cycle with its small levels in one thread-block cluster
(the tail kernel) against the same cycle on the whole cooperative grid: the
same device functions run on the same points in the same colour order, so
the solves and steps are bitwise identical whichever kernel runs a level."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(ow3d, make, tail, cluster, steps=3):
    L = ow3d.lib()
    old_t = L.ow3d_test_set_tail_max_points(tail)
    old_c = L.ow3d_test_set_tail_cluster(cluster)
    try:
        p, geo, E0, P0 = make()
        sim = ow3d.Simulation(p, **geo)
        sim.set_state(E0, P0)
        sim.step(steps)
        out = sim.get_state()
        sim.close()
        return out
    finally:
        L.ow3d_test_set_tail_max_points(old_t)
        L.ow3d_test_set_tail_cluster(old_c)


def _shoal(ow3d, prec):
    def make():
        p, geo = ow3d.workloads.shoal(Nx=257, Ny=33, Nz=9, precision=prec)
        C = (p.Nx + 2) * (p.Ny + 2)
        x = np.linspace(0.0, 1.0, C)
        return p, geo, 0.01 * np.sin(40 * x), np.zeros(C)
    return make


def _sea(ow3d, prec):
    def make():
        return ow3d.workloads.irregular_sea(Nx=257, Ny=65, Nz=17, precision=prec, seed=7)[:4]
    return make


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("case", ["shoal", "sea"])
def test_tail_cluster_is_bitwise_the_grid_cycle(ow3d, case, prec):
    make = (_shoal if case == "shoal" else _sea)(ow3d, prec)
    ref = _run(ow3d, make, 0, 16)                 # every coarse level on the grid
    for tail, cluster in ((8192, 16), (8192, 8), (1 << 40, 16)):
        got = _run(ow3d, make, tail, cluster)    # 1 << 40: the whole fused cycle in the cluster
        for a, b in zip(got[:4], ref[:4]):
            assert np.array_equal(a, b), (tail, cluster)


def test_coarse_cluster_mode_per_handle(ow3d):
    """ow3d_set_coarse_cluster: the whole fused coarse cycle of one handle in
    a cluster, switched on and off between steps (the captured graphs are
    dropped and captured again), bitwise the grid cycle throughout."""
    make = _sea(ow3d, 0)
    runs = []
    for schedule in ((0, 0, 0), (1, 1, 1), (1, 0, 1)):
        p, geo, E0, P0 = make()
        sim = ow3d.Simulation(p, **geo)
        sim.set_state(E0, P0)
        for on in schedule:
            assert ow3d.lib().ow3d_set_coarse_cluster(sim.h, on) == 0
            sim.step(2)
        runs.append(sim.get_state())
        sim.close()
    for got in runs[1:]:
        for a, b in zip(got[:4], runs[0][:4]):
            assert np.array_equal(a, b)
