"""The tiled colour pass (columns away from the walls solved from shared-memory
tiles, wall columns in the leading blocks of the same launch) against the
per-column colour pass: both run the same arithmetic per column on the same
values, so the results must agree bitwise, in FP64 and in FP32 (where tile
rows start off the 16-byte boundary), for 17 and 9 sigma levels (8 and 4
lanes per column), for single colour passes, whole smoothing steps and RK4
steps.
"""
import numpy as np
import pytest

import cases  # noqa: F401  (puts tests/ on the path for the package loader)

pytestmark = pytest.mark.gpu


def _tiles(ow3d, min_tiles):
    """Tiled pass on every level it covers (1) or on none (0); returns the
    previous setting."""
    return ow3d.lib().ow3d_test_set_colour_tiles(min_tiles)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("nz", [17, 9])
def test_colour_passes_tiled_equal_per_column(ow3d, precision, nz):
    p, geo, E0, P0 = ow3d.workloads.irregular_sea(Nx=129, Ny=33, Nz=nz, precision=precision)
    sim = ow3d.Simulation(p, **geo)
    rng = np.random.default_rng(7 + nz)
    nl = sim.level_count()
    checked = 0
    prev = _tiles(ow3d, 1)
    try:
        for l in range(nl - 1, 0, -1):
            nx, ny, _, ncolor = sim.level_dims(l)
            if nx + 2 < 12 or ny + 2 < 12:
                break
            n = sim.level_size(l)
            x = rng.standard_normal(n)
            b = rng.standard_normal(n)
            got = {}
            for on in (1, 0):
                _tiles(ow3d, on)
                got[on] = ([sim.level_op(l, 5, x, b, nu=c) for c in range(ncolor)],
                           sim.level_op(l, 1, x, b, nu=2))
            for a, c in zip(got[1][0], got[0][0]):
                assert np.array_equal(a, c), f"colour pass, level {l}"
            assert np.array_equal(got[1][1], got[0][1]), f"smoothing, level {l}"
            assert not np.array_equal(got[1][1], x)
            checked += 1
    finally:
        _tiles(ow3d, prev)
        sim.close()
    assert checked >= 2


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_steps_tiled_equal_per_column(ow3d, precision):
    """257 x 65 x 17: the finest multigrid level runs outside the fused coarse
    kernel, so its smoothing takes the tiled pass inside the solves."""
    p, geo, E0, P0 = ow3d.workloads.irregular_sea(Nx=257, Ny=65, Nz=17, precision=precision)
    out = []
    prev = _tiles(ow3d, 1)
    try:
        for on in (1, 0):
            _tiles(ow3d, on)
            sim = ow3d.Simulation(p, **geo)
            sim.set_state(E0, P0)
            assert sim.step(3) >= 0
            out.append((sim.get_state(), sim.stats()["total_iterations"]))
            sim.close()
    finally:
        _tiles(ow3d, prev)
    (st, it), (sp, ip) = out
    for a, b in zip(st[:4], sp[:4]):
        assert np.array_equal(a, b)
    assert it == ip
