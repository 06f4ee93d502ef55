"""ORACLE -- test infrastructure only.

Python handle on the CPU restatement of the OceanWave3D hot path
(oracle/ow3d_oracle.cpp). Only tests/, __graft_entry__.smoke() and the CPU
baseline / reference arm of bench.py use it, and only as the checker or the
timed CPU baseline; the product path never calls it.
"""
import ctypes as C
import importlib.util
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
LIB = HERE / "_build" / "libow3d_oracle.so"

MODE_REFERENCE = 0   # lexicographic GS + left GMRES (the reference's algorithm)
MODE_DEVICE = 1      # multicolour GS + right FGMRES (what the CUDA path runs)


def capi():
    # share the ctypes classes with the package when it is loaded
    if "ow3d_b200.capi" in sys.modules:
        return sys.modules["ow3d_b200.capi"]
    name = "ow3d_capi"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, ROOT / "oceanwave3d-fortran90_b200" / "capi.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        D, I, V = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
        P = C.c_void_p  # a Params instance passed by address
        L.orc_create.restype = V
        L.orc_create.argtypes = [P, D, D, D, D, D, C.c_int]
        L.orc_destroy.argtypes = [V]
        L.orc_set_mode.argtypes = [V, C.c_int]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_dims.argtypes = [V, I, I, I, I]
        L.orc_level_dims.argtypes = [V, C.c_int, I, I, I, I]
        L.orc_level_z.argtypes = [V, C.c_int, D]
        L.orc_fine_z.argtypes = [V, D]
        L.orc_level_nnz.argtypes = [V, C.c_int]
        L.orc_level_csr.argtypes = [V, C.c_int, I, I, D]
        L.orc_level_matvec.argtypes = [V, C.c_int, D, D]
        L.orc_level_smooth.argtypes = [V, C.c_int, D, D, C.c_int]
        L.orc_level_pass.argtypes = [V, C.c_int, C.c_int, D, D]
        L.orc_restrict.argtypes = [V, C.c_int, D, D]
        L.orc_prolong.argtypes = [V, C.c_int, D, D]
        L.orc_coarse_solve.argtypes = [V, D]
        L.orc_stencils.argtypes = [V, D, D, D]
        L.orc_set_surface.argtypes = [V, D, D, D, D, D]
        L.orc_matvec.argtypes = [V, D, D]
        L.orc_precond.argtypes = [V, D, D]
        L.orc_solve.argtypes = [V, D, D, I, D]
        L.orc_set_state.argtypes = [V, D, D, D, D, C.c_double]
        L.orc_get_state.argtypes = [V, D, D, D, D, D]
        L.orc_get_derivs.argtypes = [V, D, D, D, D, D, D]
        L.orc_set_relax_target.argtypes = [V, C.c_int, C.c_int, C.c_int, C.c_double, D, D]
        L.orc_zone_box.argtypes = [V, C.c_int, I, I, I, I]
        L.orc_zone_gamma.argtypes = [V, C.c_int, D]
        L.orc_filter_coeffs.argtypes = [V, D, D]
        L.orc_filter.argtypes = [V, D]
        L.orc_step.argtypes = [V, C.c_int]
        L.orc_stats.argtypes = [V, C.POINTER(C.c_int64), C.POINTER(C.c_int64), I, I, I, D, C.POINTER(C.c_int64)]
        L.orc_reset_stats.argtypes = [V]
        L.orc_rollers.argtypes = [V, C.c_int, I, I, D, D, D, D]
        L.orc_breaking_state.argtypes = [V, D, D]
        L.orc_detect_breaking.argtypes = [V, D, C.c_int]
        L.orc_accel_state.argtypes = [V, D, C.c_int, I]
        L.orc_set_paddle.argtypes = [V, C.c_int, C.c_int, C.c_double, D, D]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """One simulation in the CPU oracle. Arrays use the reference's Fortran
    layout flattened in column-major order: 3-D (k,i,j) -> k fastest,
    2-D (i,j) -> i fastest."""

    def __init__(self, params, h, hx=None, hxx=None, hy=None, hyy=None, mode=MODE_REFERENCE):
        self.params = params
        L = lib()
        z = np.zeros_like(_c(h))
        self._keep = [_c(h), _c(hx) if hx is not None else z, _c(hxx) if hxx is not None else z,
                      _c(hy) if hy is not None else z, _c(hyy) if hyy is not None else z]
        self.h = L.orc_create(C.addressof(params), *[_p(a) for a in self._keep], mode)
        if not self.h:
            raise ValueError("oracle: set-up failed (grid not coarsenable?)")
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        L.orc_dims(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        self.Nxg, self.Nyg, self.Nzg, self.nlevels = a.value, b.value, c.value, d.value
        self.C = self.Nxg * self.Nyg
        self.N = self.C * self.Nzg

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def set_mode(self, mode):
        lib().orc_set_mode(self.h, mode)

    # --- set-up tables
    def level_dims(self, l):
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        lib().orc_level_dims(self.h, l, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        return a.value, b.value, c.value, d.value

    def level_size(self, l):
        nx, ny, nz, _ = self.level_dims(l)
        gx = self.params.GhostGridX if self.params.Nx > 1 else 0
        gy = self.params.GhostGridY if self.params.Ny > 1 else 0
        return (nx + 2 * gx) * (ny + 2 * gy) * (nz + self.params.GhostGridZ)

    def level_csr(self, l):
        import scipy.sparse as sp
        n = self.level_size(l)
        nnz = lib().orc_level_nnz(self.h, l)
        rp = np.zeros(n + 1, np.int32); ci = np.zeros(nnz, np.int32); v = np.zeros(nnz)
        lib().orc_level_csr(self.h, l, rp.ctypes.data_as(C.POINTER(C.c_int)), ci.ctypes.data_as(C.POINTER(C.c_int)), _p(v))
        return sp.csr_matrix((v, ci, rp), shape=(n, n))

    def level_z(self, l):
        nz = self.level_dims(l)[2] + self.params.GhostGridZ
        z = np.zeros(nz); lib().orc_level_z(self.h, l, _p(z)); return z

    def fine_z(self):
        z = np.zeros(self.Nzg); lib().orc_fine_z(self.h, _p(z)); return z

    def stencils(self):
        r = 2 * self.params.alpha + 1
        SX = np.zeros((2, self.Nxg, r)); SY = np.zeros((2, self.Nyg, 2 * self.params.beta + 1))
        SZ = np.zeros((2, self.Nzg, 2 * self.params.gamma + 1))
        lib().orc_stencils(self.h, _p(SX), _p(SY), _p(SZ))
        return SX, SY, SZ

    def level_matvec(self, l, x):
        x = _c(x); y = np.zeros_like(x); lib().orc_level_matvec(self.h, l, _p(x), _p(y)); return y

    def level_smooth(self, l, x, b, nu=1):
        x = _c(x).copy(); b = _c(b); lib().orc_level_smooth(self.h, l, _p(x), _p(b), nu); return x

    def level_pass(self, l, colour, x, b):
        """One device-ordering smoother phase: colour pass, or the bottom-row pass (colour < 0)."""
        x = _c(x).copy(); b = _c(b); lib().orc_level_pass(self.h, l, colour, _p(x), _p(b)); return x

    def restrict(self, lf, rf):
        rc = np.zeros(self.level_size(lf - 1)); lib().orc_restrict(self.h, lf, _p(_c(rf)), _p(rc)); return rc

    def prolong(self, lf, pc):
        pf = np.zeros(self.level_size(lf)); lib().orc_prolong(self.h, lf, _p(pf), _p(_c(pc))); return pf

    def coarse_solve(self, b):
        x = _c(b).copy(); lib().orc_coarse_solve(self.h, _p(x)); return x

    # --- the hot path
    def set_surface(self, E=None, Ex=None, Exx=None, Ey=None, Eyy=None):
        arrs = [None if a is None else _c(a) for a in (E, Ex, Exx, Ey, Eyy)]
        lib().orc_set_surface(self.h, *[_p(a) for a in arrs])

    def matvec(self, phi):
        phi = _c(phi); y = np.zeros_like(phi); lib().orc_matvec(self.h, _p(phi), _p(y)); return y

    def precond(self, r):
        r = _c(r); u = np.zeros_like(r); lib().orc_precond(self.h, _p(r), _p(u)); return u

    def solve(self, rhs, phi0):
        phi = _c(phi0).copy(); it = C.c_int(); res = C.c_double()
        st = lib().orc_solve(self.h, _p(_c(rhs)), _p(phi), C.byref(it), C.byref(res))
        return phi, it.value, res.value, st

    def set_state(self, E, P, W=None, phi=None, t=0.0):
        arrs = [_c(E), _c(P), None if W is None else _c(W), None if phi is None else _c(phi)]
        lib().orc_set_state(self.h, *[_p(a) for a in arrs], t)

    def get_state(self):
        E = np.zeros(self.C); P = np.zeros(self.C); W = np.zeros(self.C); phi = np.zeros(self.N); t = C.c_double()
        lib().orc_get_state(self.h, _p(E), _p(P), _p(W), _p(phi), C.byref(t))
        return E, P, W, phi, t.value

    def get_derivs(self):
        out = [np.zeros(self.C) for _ in range(6)]
        lib().orc_get_derivs(self.h, *[_p(a) for a in out])
        return out

    def set_relax_target(self, zone, mode, nt, dts, eta, phis):
        return lib().orc_set_relax_target(self.h, zone, mode, nt, dts, _p(_c(eta)), _p(_c(phis)))

    def zone_box(self, zone):
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        r = lib().orc_zone_box(self.h, zone, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        if r != 0:
            raise IndexError(zone)
        return a.value, b.value, c.value, d.value

    def zone_gamma(self, zone):
        i0, i1, j0, j1 = self.zone_box(zone)
        n = (i1 - i0 + 1) if self.params.zones[zone].XorY == b"X" else (j1 - j0 + 1)
        g = np.zeros(n); lib().orc_zone_gamma(self.h, zone, _p(g)); return g

    def filter_coeffs(self):
        al = self.params.filterALPHA; NP = 2 * al + 1
        c = np.zeros(NP); b = np.zeros(NP * al)
        lib().orc_filter_coeffs(self.h, _p(c), _p(b))
        return c, b.reshape(al, NP)

    def filter(self, U):
        U = _c(U).copy(); lib().orc_filter(self.h, _p(U)); return U

    def step(self, n=1):
        return lib().orc_step(self.h, n)

    def stats(self):
        s, t, mn, mx, last, res, nc = C.c_int64(), C.c_int64(), C.c_int(), C.c_int(), C.c_int(), C.c_double(), C.c_int64()
        lib().orc_stats(self.h, C.byref(s), C.byref(t), C.byref(mn), C.byref(mx), C.byref(last), C.byref(res), C.byref(nc))
        return dict(solves=s.value, total_iterations=t.value, min=mn.value, max=mx.value, last=last.value,
                    last_residual=res.value, not_converged=nc.value)

    def reset_stats(self):
        lib().orc_reset_stats(self.h)

    def rollers(self):
        """The rollers of the last step (DetectBreaking.f90:205-211), as
        Simulation.rollers returns them."""
        cap = self.Nxg
        ints = [np.zeros(cap, dtype=np.int32) for _ in range(2)]
        dbl = [np.zeros(cap) for _ in range(4)]
        I = C.POINTER(C.c_int)
        n = lib().orc_rollers(self.h, cap, *(a.ctypes.data_as(I) for a in ints), *(_p(a) for a in dbl))
        names = ("npts", "toe", "x", "eta", "thickness", "tan_phi")
        return {nm: a[:n].copy() for nm, a in zip(names, ints + dbl)}

    def detect_breaking(self, E, update=False):
        """One detect_breaking call on the surface E (DetectBreaking.f90);
        update: the call after a step (roller-angle update, roller record)."""
        E = _c(E)
        if lib().orc_detect_breaking(self.h, _p(E), 1 if update else 0) != 0:
            raise ValueError("oracle: no breaking model in this simulation")

    def set_paddle(self, dt, y, flux):
        """The flux wavemaker's signal (setupWavePaddle.f90): flux (nt, n2) at
        the n2 positions y every dt."""
        y, flux = _c(y), _c(flux)
        nt, n2 = flux.shape
        if lib().orc_set_paddle(self.h, nt, n2, float(dt), _p(y), _p(flux)) != 0:
            raise ValueError("oracle: not a flux-wavemaker simulation, or a signal shorter than 5 times")

    set_paddle_signal = set_paddle

    def accel_state(self):
        """The last local-smoothing call (LocalSmoothing2D/3D.f90): the surface
        dw/dt per column and the 0-based columns where -dw/dt reached the
        limit; None when the filter is off."""
        Wt = np.zeros(self.C)
        cols = np.zeros(self.C, dtype=np.int32)
        n = lib().orc_accel_state(self.h, _p(Wt), self.C, cols.ctypes.data_as(C.POINTER(C.c_int)))
        return None if n < 0 else (Wt, cols[:n].copy())

    def breaking_state(self):
        t, q = np.zeros(self.C), np.zeros(self.C)
        lib().orc_breaking_state(self.h, _p(t), _p(q))
        return t, q


def set_threads(n):
    return lib().orc_set_threads(n)
