"""The allocation-free residual entry point (ow3d_residual_device_noalloc)
against the existing host-pointer matvec (ow3d_matvec): d_res = rhs - A phi
and its 2-norm, two calls in a row on the same handle (the second call reuses
the fixed device scratch the first one left with its finish counter reset).

Collected last on purpose: it must pass alone and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def _dev(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("case,kw", [(cases.bump_3d, dict(Nx=33, Ny=17, Nz=9)), (cases.slope_2d, dict(Nx=33, Nz=9))],
                         ids=["bump3d", "slope2d"])
def test_residual_noalloc_matches_matvec(ow3d, case, kw):
    import torch
    p, geo = case(**kw)
    sim = ow3d.Simulation(p, **geo)
    L = ow3d.lib()
    rng = np.random.default_rng(21)
    surf = cases.surface(p, amp=0.03, seed=2)
    dsurf = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in surf]
    for call in range(2):
        phi = rng.standard_normal(sim.N)
        rhs = rng.standard_normal(sim.N)
        ref_res = rhs - sim.matvec(phi, *surf)
        ref_norm = float(np.linalg.norm(ref_res))
        d_phi = torch.from_numpy(phi).cuda()
        d_rhs = torch.from_numpy(rhs).cuda()
        d_res = torch.empty(sim.N, dtype=torch.float64, device="cuda")
        norm = C.c_double()
        ptrs = [_dev(t) for t in dsurf]
        st = L.ow3d_residual_device_noalloc(sim.h, _dev(d_rhs), _dev(d_phi), *ptrs, _dev(d_res), C.byref(norm))
        assert st == 0, (call, L.ow3d_last_error())
        torch.cuda.synchronize()
        res = d_res.cpu().numpy()
        assert np.max(np.abs(res - ref_res)) <= 1e-12 * np.max(np.abs(ref_res)), call
        assert abs(norm.value - ref_norm) <= 1e-12 * ref_norm, (call, norm.value, ref_norm)


def test_residual_noalloc_rejects_null(ow3d):
    p, geo = cases.bump_3d(Nx=17, Ny=9, Nz=9)
    sim = ow3d.Simulation(p, **geo)
    L = ow3d.lib()
    norm = C.c_double()
    assert L.ow3d_residual_device_noalloc(sim.h, None, None, None, None, None, None, None, None,
                                          C.byref(norm)) == ow3d.capi.ERR_BAD_INPUT
