"""The schedule of the device's lexicographic smoother, checked on the CPU
against the reference-ordered oracle's own level matrices (the low-order
operator as the reference assembles it, BuildLinearSystemMatrix.f90).

The device sweeps a level as wavefronts: row (k, i, j) in wave
(k-1) + 2 (i-1) + B (j-1), with B = 6 on levels with mixed-derivative terms
(4 colour classes) and B = 2 otherwise. That reproduces the sequential
sweep in index order (GaussSeidel.f90:15-26) exactly when, for every nonzero
a_rc off the diagonal, the wave of c is below the wave of r if and only if
c < r. The special rows (MGPreProcess.f90:376-439) run in three phases --
ghost columns at i = 1 / j = 1, bottom rows, ghost columns at i = Nxg /
j = Nyg -- which reproduces GaussSeidelSpecialPoints.f90:43-53 when no two
special rows of one phase are coupled and every coupling between special
rows of different phases points from the lower phase to the higher index.
"""
import numpy as np
import pytest

import cases


def _coords(n, Nxg, Nzg):
    r = np.arange(n)
    k = r % Nzg + 1
    i = (r // Nzg) % Nxg + 1
    j = r // (Nzg * Nxg) + 1
    return k, i, j


def _levels(ow3d, oracle, case, kw):
    if case == "periodic":
        p, geo, _, _, _ = ow3d.workloads.periodic_wave_2d()
    elif case == "shoal":
        p, geo = ow3d.workloads.shoal(Nx=65, Ny=17)
    else:
        p, geo = getattr(cases, case)(**kw)
    o = oracle.Oracle(p, **geo, mode=oracle.MODE_REFERENCE)
    three = p.Ny > 1
    out = []
    for l in range(1, o.nlevels):
        nx, ny, nz, ncolor = o.level_dims(l)
        A = o.level_csr(l).tocoo()
        n = A.shape[0]
        gx = p.GhostGridX
        gy = p.GhostGridY if three else 0
        Nxg, Nyg, Nzg = nx + 2 * gx, ny + 2 * gy, nz + p.GhostGridZ
        assert Nxg * Nyg * Nzg == n
        out.append((A, Nxg, Nyg, Nzg, three, ncolor))
    return out


CASES = [("flat_2d", dict(Nx=17, Nz=9)), ("slope_2d", dict(Nx=33, Nz=9)),
         ("bump_3d", dict(Nx=17, Ny=9, Nz=9)), ("bump_3d", dict(Nx=33, Ny=17, Nz=9)),
         ("bump_3d", dict(Nx=33, Ny=17, Nz=9, amp=0.0)), ("periodic", {}), ("shoal", {})]
IDS = ["flat2d", "slope2d", "bump3d-17x9", "bump3d-33x17", "flat3d-33x17", "periodic65", "shoal65x17"]


@pytest.mark.parametrize("case,kw", CASES, ids=IDS)
def test_wavefronts_keep_the_index_order(ow3d, oracle, case, kw):
    for A, Nxg, Nyg, Nzg, three, ncolor in _levels(ow3d, oracle, case, kw):
        k, i, j = _coords(A.shape[0], Nxg, Nzg)
        B = (6 if ncolor == 4 else 2) if three else 0
        T = (k - 1) + 2 * (i - 1) + B * (j - 1)
        off = (A.row != A.col) & (A.data != 0)
        r, c = A.row[off], A.col[off]
        assert np.all(np.sign(T[c] - T[r]) == np.sign(c - r)), (Nxg, Nyg, Nzg)


@pytest.mark.parametrize("case,kw", CASES, ids=IDS)
def test_special_phases_keep_the_index_order(ow3d, oracle, case, kw):
    for A, Nxg, Nyg, Nzg, three, ncolor in _levels(ow3d, oracle, case, kw):
        k, i, j = _coords(A.shape[0], Nxg, Nzg)
        lo = (i == 1) | (three & (j == 1))
        hi = (i == Nxg) | (three & (j == Nyg))
        special = (k == 1) | lo | hi
        phase = np.where(lo, 0, np.where(hi, 2, 1))
        off = (A.row != A.col) & (A.data != 0)
        r, c = A.row[off], A.col[off]
        both = special[r] & special[c]
        r, c = r[both], c[both]
        assert np.all(phase[r] != phase[c])
        assert np.all((phase[c] < phase[r]) == (c < r))
