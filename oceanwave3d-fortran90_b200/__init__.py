"""B200-native OceanWave3D hot path: the per-stage sigma-grid Laplace solve and
the RK4 free-surface update, as CUDA kernels for sm_100a behind the C ABI of
include/ow3d.h.

This module is the Python host side of that ABI (the reference's driver is
Fortran; a Fortran host binds the same symbols through the iso_c_binding
module include/ow3d_iface.f90). It mirrors the reference's split into a set-up call
(OceanWave3DT0Setup) and a time-step call (OceanWave3DTakeATimeStep) and
exposes the drop-in Laplace solve (iterative_solution).

Arrays follow the reference's Fortran layout, flattened column-major:
3-D fields PHI(k,i,j) with k fastest, 2-D fields E(i,j) with i fastest, ghost
points included. numpy arrays of shape (Nyg, Nxg, Nzg) / (Nyg, Nxg) in C order
have exactly that memory layout.
"""
import ctypes as _C
import os as _os
import pathlib as _pathlib

import numpy as _np

from . import capi
from . import workloads  # noqa: F401
from .capi import Params, Zone, Stats, default_params, dims, set_zone  # noqa: F401

# libow3d.so exports the functions of include/ow3d.h; the testing build,
# libow3d_dev.so (same objects), also the probes of include/ow3d_test.h that
# the parity tests call. OW3D_TEST_BUILD=1 selects the testing build.
LIB_PATH = _pathlib.Path(__file__).resolve().parent / (
    "libow3d_dev.so" if _os.environ.get("OW3D_TEST_BUILD") == "1" else "libow3d.so")
_lib = None


class OW3DError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = f"{what}: status {status}"
        if _lib is not None:
            msg += f" ({_lib.ow3d_strerror(status).decode()}; {_lib.ow3d_last_error().decode()})"
        super().__init__(msg)


def lib():
    """The loaded CUDA library. There is no CPU fallback: a missing library is an error."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise OW3DError(-8, f"{LIB_PATH} is missing; build it with build.py (there is no CPU fallback)")
        L = _C.CDLL(str(LIB_PATH))
        capi.declare(L)
        D = _C.POINTER(_C.c_double)
        L.ow3d_bench_kernel.argtypes = [_C.c_void_p, _C.c_int, _C.c_int, D]
        L.ow3d_launch_count.argtypes = []
        L.ow3d_launch_count.restype = _C.c_ulonglong
        L.ow3d_level_count.argtypes = [_C.c_void_p]
        L.ow3d_level_dims.argtypes = [_C.c_void_p, _C.c_int] + [_C.POINTER(_C.c_int)] * 4
        if not hasattr(L, "ow3d_test_stencils"):   # the product build: no probes
            _lib = L
            return _lib
        L.ow3d_test_stencils.argtypes = [_C.c_void_p, D, D, D]
        L.ow3d_test_surface_derivs.argtypes = [_C.c_void_p, D, D]
        L.ow3d_test_ran1.argtypes = [_C.c_int, _C.c_int, _C.POINTER(_C.c_float), _C.POINTER(_C.c_int)]
        L.ow3d_test_level_z.argtypes = [_C.c_void_p, _C.c_int, D]
        L.ow3d_test_zone_gamma.argtypes = [_C.c_void_p, _C.c_int, D]
        L.ow3d_test_filter_coeffs.argtypes = [_C.c_void_p, D, D]
        L.ow3d_test_level_op.argtypes = [_C.c_void_p, _C.c_int, _C.c_int, _C.c_int, D, D, D]
        L.ow3d_test_sizeof.argtypes = [_C.c_int]
        L.ow3d_test_set_coarse_blocks.argtypes = [_C.c_int]
        L.ow3d_test_set_coop_max_points.argtypes = [_C.c_longlong]
        L.ow3d_test_set_coop_max_points.restype = _C.c_longlong
        L.ow3d_test_set_colour_tiles.argtypes = [_C.c_int]
        L.ow3d_test_set_tail_max_points.argtypes = [_C.c_longlong]
        L.ow3d_test_set_tail_max_points.restype = _C.c_longlong
        L.ow3d_test_set_tail_cluster.argtypes = [_C.c_int]
        L.ow3d_test_set_pdl.argtypes = [_C.c_int]
        L.ow3d_test_set_colour_prefetch.argtypes = [_C.c_int]
        L.ow3d_test_graph_count.argtypes = [_C.c_void_p]
        L.ow3d_test_step_graph_count.argtypes = [_C.c_void_p]
        L.ow3d_test_relax_target.argtypes = [_C.c_void_p, _C.c_int, D, D]
        L.ow3d_test_breaking_state.argtypes = [_C.c_void_p, D, D]
        L.ow3d_test_detect_breaking.argtypes = [_C.c_void_p, D, _C.c_int]
        L.ow3d_test_accel_state.argtypes = [_C.c_void_p, D, _C.POINTER(_C.c_int)]
        _lib = L
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(_C.POINTER(_C.c_double))


def _f64(a):
    return None if a is None else _np.ascontiguousarray(a, dtype=_np.float64)


def _check(st, what):
    if st < 0:
        raise OW3DError(st, what)
    return st


def read_deck(path):
    """Parse an OceanWave3D input deck (ReadInputFileParameters.f90) into Params."""
    p = Params()
    _check(lib().ow3d_read_deck(str(path).encode(), _C.byref(p)), "ow3d_read_deck")
    return p


def _b(path):
    return str(path).encode()


def initial_condition(params):
    """Geometry dict (h, hx, hxx, hy, hyy) and initial E, P of the deck's IC
    (0, 4, 5, 7; include/ow3d.h ow3d_initial_condition)."""
    Nxg, Nyg, _ = dims(params)
    geo = {k: _np.zeros(Nxg * Nyg) for k in ("h", "hx", "hxx", "hy", "hyy")}
    E, P = _np.zeros(Nxg * Nyg), _np.zeros(Nxg * Nyg)
    _check(lib().ow3d_initial_condition(_C.byref(params), *[_d(geo[k]) for k in geo], _d(E), _d(P)),
           "ow3d_initial_condition")
    return geo, E, P


def read_bathymetry(params, path=None, deck_dir=None):
    """The bathymetry file of a deck with Lz <= 0: a dict of h, hx, hxx, hy,
    hyy (Nxg*Nyg, ghosts included) for Simulation, and the file's gradient
    flag. path defaults to the deck's file name, taken relative to deck_dir."""
    if path is None:
        name = params.bathymetry_file.decode()
        path = _pathlib.Path(deck_dir or ".") / name
    Nxg, Nyg, _ = dims(params)
    out = {k: _np.zeros(Nxg * Nyg) for k in ("h", "hx", "hxx", "hy", "hyy")}
    flag = _C.c_int()
    _check(lib().ow3d_read_bathymetry(_C.byref(params), str(path).encode(), *[_d(out[k]) for k in out],
                                      _C.byref(flag)), "ow3d_read_bathymetry")
    return out, flag.value


def stream_function_wave(params, x, t=0.0):
    """The stream-function wave of the deck's line 8 at positions x and time t:
    eta, surface phi and (k, L, T, c)."""
    x = _np.ascontiguousarray(x, dtype=_np.float64)
    eta, phis, info = _np.zeros_like(x), _np.zeros_like(x), _np.zeros(4)
    _check(lib().ow3d_stream_function_wave(_C.byref(params), x.size, _d(x), float(t), _d(eta), _d(phis), _d(info)),
           "ow3d_stream_function_wave")
    return eta, phis, tuple(info)


def read_paddle_signal(path):
    """The flux wavemaker's paddle-signal file (ow3d_read_paddle_signal):
    (dt, y (n2,), flux (nt, n2))."""
    dt, nt, n2 = _C.c_double(), _C.c_int(), _C.c_int()
    _check(lib().ow3d_read_paddle_signal(_b(path), 0, _C.byref(dt), _C.byref(nt), _C.byref(n2), None, None),
           "ow3d_read_paddle_signal")
    y, flux = _np.zeros(n2.value), _np.zeros(nt.value * n2.value)
    _check(lib().ow3d_read_paddle_signal(_b(path), flux.size, _C.byref(dt), _C.byref(nt), _C.byref(n2), _d(y),
                                         _d(flux)), "ow3d_read_paddle_signal")
    return dt.value, y, flux.reshape(nt.value, n2.value)


def incident_wave(params, zone, nt=None):
    """The incident wave of IncWaveType 2 on generation zone `zone` (0-based):
    eta and surface phi as (nt, rows, columns) arrays every dt (nt defaults
    to the reference's sample count), and the zone's ghost-inclusive 1-based
    box (i0, i1, j0, j1). Pass them to Simulation.set_relax_target with mode
    0 and dt_sample = dt."""
    L = lib()
    box = (_C.c_int * 5)()
    _check(L.ow3d_incident_wave(_C.byref(params), zone, 1, None, None, box), "ow3d_incident_wave")
    i0, i1, j0, j1, nref = list(box)
    nt = int(nref if nt is None else nt)
    eta = _np.zeros((nt, j1 - j0 + 1, i1 - i0 + 1))
    phis = _np.zeros_like(eta)
    _check(L.ow3d_incident_wave(_C.byref(params), zone, nt, _d(eta), _d(phis), box), "ow3d_incident_wave")
    return eta, phis, (i0, i1, j0, j1)


def read_init_file(path, Nx, Ny):
    """Read a hot-start file (OceanWave3D.init format): interior E, P (Nx*Ny
    each, x fastest) and the start time."""
    E = _np.zeros(Nx * Ny); P = _np.zeros(Nx * Ny); t = _C.c_double()
    st = lib().ow3d_read_init_file(_b(path), Nx, Ny, _d(E), _d(P), _C.byref(t))
    if st:
        raise OW3DError(st, "ow3d_read_init_file: " + lib().ow3d_io_last_error().decode())
    return E, P, t.value


def load_ep(path):
    """Read an EP_#####.bin file (Fortran unformatted records with 32-bit
    length markers, as StoreData writes it): nx, ny and x, y, E, P as
    (ny, nx) arrays."""
    raw = _pathlib.Path(path).read_bytes()
    recs, pos = [], 0
    while pos < len(raw):
        n = int(_np.frombuffer(raw, "<i4", 1, pos)[0])
        body = raw[pos + 4:pos + 4 + n]
        if int(_np.frombuffer(raw, "<i4", 1, pos + 4 + n)[0]) != n:
            raise ValueError(f"{path}: record markers disagree")
        recs.append(body)
        pos += n + 8
    nx, ny = (int(v) for v in _np.frombuffer(recs[0], "<i4"))
    xy = _np.frombuffer(recs[1], "<f8").reshape(2, ny, nx)
    ep = _np.frombuffer(recs[2], "<f8").reshape(2, ny, nx)
    return nx, ny, xy[0], xy[1], ep[0], ep[1]


def load_records(path):
    """The records of a Fortran unformatted sequential file (32-bit length
    markers) as a list of byte strings."""
    raw = _pathlib.Path(path).read_bytes()
    recs, pos = [], 0
    while pos < len(raw):
        n = int(_np.frombuffer(raw, "<i4", 1, pos)[0])
        if int(_np.frombuffer(raw, "<i4", 1, pos + 4 + n)[0]) != n:
            raise ValueError(f"{path}: record markers disagree")
        recs.append(raw[pos + 4:pos + 4 + n])
        pos += n + 8
    return recs


KINEMATICS_FIELDS = ("eta", "eta_x", "eta_y", "phi", "u", "v", "w", "w_z", "w_x", "w_y",
                     "u_z", "u_x", "u_y", "v_z", "v_x", "v_y")


def load_kinematics(path):
    """Read a Kinematics file as ow3d_store_kinematics (and the reference's
    StoreKinematicData) writes it: a dict with the header ('range', 'dt',
    'nz', 'geometry' as (points, 5) x y h hx hy, 'z') when present, and
    'levels', a list of dicts of the 16 fields (surface fields per slice
    point, column fields as (points, nz))."""
    recs = load_records(path)
    out, pos = {"levels": []}, 0
    if recs and len(recs[0]) == 48:
        h = recs[0]
        out["range"] = [int(v) for v in _np.frombuffer(h, "<i4", 9, 0)]
        out["dt"] = float(_np.frombuffer(h, "<f8", 1, 36)[0])
        out["nz"] = int(_np.frombuffer(h, "<i4", 1, 44)[0])
        out["geometry"] = _np.frombuffer(recs[1], "<f8").reshape(-1, 5)
        out["z"] = _np.frombuffer(recs[2], "<f8")
        pos = 3
    while pos + 16 <= len(recs):
        lv = {}
        for q, name in enumerate(KINEMATICS_FIELDS):
            a = _np.frombuffer(recs[pos + q], "<f8")
            lv[name] = a if q < 3 else a.reshape(len(_np.frombuffer(recs[pos], "<f8")), -1)
        out["levels"].append(lv)
        pos += 16
    return out


class Simulation:
    """One simulation resident on one GPU (an ow3d_handle)."""

    def __init__(self, params, h, hx=None, hxx=None, hy=None, hyy=None):
        self.params = params
        L = lib()
        self.Nxg, self.Nyg, self.Nzg = dims(params)
        self.C = self.Nxg * self.Nyg
        self.N = self.C * self.Nzg
        z = _np.zeros(self.C)
        self._geo = [_f64(h).ravel()] + [(_f64(a).ravel() if a is not None else z) for a in (hx, hxx, hy, hyy)]
        for a in self._geo:
            if a.size != self.C:
                raise ValueError(f"bathymetry arrays must have Nxg*Nyg = {self.C} entries")
        hnd = _C.c_void_p()
        _check(L.ow3d_create(_C.byref(params), *[_d(a) for a in self._geo], _C.byref(hnd)), "ow3d_create")
        self.h = hnd

    def close(self):
        if getattr(self, "h", None):
            lib().ow3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- sizes
    def device_bytes(self):
        n = _C.c_size_t()
        lib().ow3d_dims(self.h, None, None, None, _C.byref(n))
        return n.value

    # ---- the drop-in solve (iterative_solution.f90)
    def solve(self, rhs, phi0, E=None, Ex=None, Exx=None, Ey=None, Eyy=None):
        """Returns (phi, iterations, status)."""
        phi = _f64(phi0).ravel().copy()
        rhs = _f64(rhs).ravel()
        surf = [_f64(a).ravel() if a is not None else None for a in (E, Ex, Exx, Ey, Eyy)]
        it = _C.c_int()
        st = _check(lib().ow3d_solve(self.h, _d(rhs), _d(phi), *[_d(a) for a in surf], _C.byref(it)), "ow3d_solve")
        return phi, it.value, st

    def matvec(self, phi, E=None, Ex=None, Exx=None, Ey=None, Eyy=None):
        phi = _f64(phi).ravel()
        y = _np.zeros(self.N)
        surf = [_f64(a).ravel() if a is not None else None for a in (E, Ex, Exx, Ey, Eyy)]
        _check(lib().ow3d_matvec(self.h, _d(phi), _d(y), *[_d(a) for a in surf]), "ow3d_matvec")
        return y

    def precondition(self, r):
        r = _f64(r).ravel()
        u = _np.zeros(self.N)
        _check(lib().ow3d_precondition(self.h, _d(r), _d(u)), "ow3d_precondition")
        return u

    # ---- the time step (timeintegration_fsbc / Runge_Kutta_4.f90)
    def set_state(self, E, P, W=None, phi=None, t=0.0):
        arrs = [_f64(E).ravel(), _f64(P).ravel(), None if W is None else _f64(W).ravel(),
                None if phi is None else _f64(phi).ravel()]
        _check(lib().ow3d_set_state(self.h, *[_d(a) for a in arrs], float(t)), "ow3d_set_state")

    def get_state(self):
        E = _np.zeros(self.C); P = _np.zeros(self.C); W = _np.zeros(self.C); phi = _np.zeros(self.N)
        t = _C.c_double()
        _check(lib().ow3d_get_state(self.h, _d(E), _d(P), _d(W), _d(phi), _C.byref(t)), "ow3d_get_state")
        return E, P, W, phi, t.value

    def step(self, n=1):
        return _check(lib().ow3d_step(self.h, int(n)), "ow3d_step")

    def step_timed(self, n=1):
        """Advance n steps; returns (status, device milliseconds from CUDA events)."""
        ms = _C.c_double()
        st = _check(lib().ow3d_step_timed(self.h, int(n), _C.byref(ms)), "ow3d_step_timed")
        return st, ms.value

    def put_surface(self, E, P):
        _check(lib().ow3d_put_surface(self.h, _d(_f64(E).ravel()), _d(_f64(P).ravel())), "ow3d_put_surface")

    def set_relax_target(self, zone, mode, nt, dt_sample, eta, phis):
        _check(lib().ow3d_set_relax_target(self.h, zone, mode, nt, float(dt_sample), _d(_f64(eta).ravel()),
                                           _d(_f64(phis).ravel())), "ow3d_set_relax_target")

    def incident_wave_device(self, zone, nt):
        """Synthesise the deck's IncWaveType 2 incident wave for generation zone
        `zone` on the device and install it as the zone's relaxation target
        (ow3d_incident_wave_device)."""
        _check(lib().ow3d_incident_wave_device(self.h, zone, int(nt)), "ow3d_incident_wave_device")

    def relax_target(self, zone, nt):
        """The zone's relaxation target as the device holds it: (nt, box) eta, phis."""
        i0, i1, j0, j1 = self.zone_box(zone)
        box = (i1 - i0 + 1) * (j1 - j0 + 1)
        e, f = _np.zeros(nt * box), _np.zeros(nt * box)
        _check(lib().ow3d_test_relax_target(self.h, zone, _d(e), _d(f)), "ow3d_test_relax_target")
        return e.reshape(nt, box), f.reshape(nt, box)

    def set_smoother_order(self, order):
        """Row order of the multigrid smoother (ow3d_set_smoother_order):
        capi.SMOOTHER_MULTICOLOUR (default) or capi.SMOOTHER_LEXICOGRAPHIC,
        the reference's order."""
        _check(lib().ow3d_set_smoother_order(self.h, int(order)), "ow3d_set_smoother_order")

    def set_paddle_signal(self, dt, y, flux):
        """Install the flux wavemaker's signal: flux (nt, n2) at y every dt
        (ow3d_set_paddle_signal)."""
        y = _f64(y).ravel()
        flux = _np.ascontiguousarray(flux, dtype=_np.float64)
        nt, n2 = flux.shape
        _check(lib().ow3d_set_paddle_signal(self.h, nt, n2, float(dt), _d(y), _d(flux.ravel())),
               "ow3d_set_paddle_signal")

    def rollers(self):
        """The roller breaking model's rollers after the last step (ow3d_rollers):
        a dict of arrays npts, toe, x, eta, thickness, tan_phi, one entry per
        roller in the order found; empty arrays when the model is off."""
        n = _C.c_int()
        _check(lib().ow3d_rollers(self.h, 0, _C.byref(n), None, None, None, None, None, None), "ow3d_rollers")
        k = n.value
        ints = [_np.zeros(max(k, 1), dtype=_np.int32) for _ in range(2)]
        dbl = [_np.zeros(max(k, 1)) for _ in range(4)]
        I = _C.POINTER(_C.c_int)
        _check(lib().ow3d_rollers(self.h, k, _C.byref(n), *(a.ctypes.data_as(I) for a in ints), *(_d(a) for a in dbl)),
               "ow3d_rollers")
        names = ("npts", "toe", "x", "eta", "thickness", "tan_phi")
        return {nm: a[:k].copy() for nm, a in zip(names, ints + dbl)}

    def detect_breaking(self, E, update=False):
        """One call of the breaking model on the surface E (a test hook)."""
        E = _f64(E).ravel()
        _check(lib().ow3d_test_detect_breaking(self.h, _d(E), 1 if update else 0), "ow3d_test_detect_breaking")

    def accel_state(self):
        """The last step's local smoothing: (surface dw/dt, 0-based columns
        where -dw/dt reached the limit) -- a test hook."""
        Wt = _np.zeros(self.C)
        fl = _np.zeros(self.C, dtype=_np.int32)
        _check(lib().ow3d_test_accel_state(self.h, _d(Wt), fl.ctypes.data_as(_C.POINTER(_C.c_int))),
               "ow3d_test_accel_state")
        return Wt, _np.flatnonzero(fl).astype(_np.int32)

    def breaking_state(self):
        """(tan_phi, Qr_x) per column of the roller breaking model."""
        t, q = _np.zeros(self.Nxg * self.Nyg), _np.zeros(self.Nxg * self.Nyg)
        _check(lib().ow3d_test_breaking_state(self.h, _d(t), _d(q)), "ow3d_test_breaking_state")
        return t, q

    def zone_box(self, zone):
        a, b, c, d = (_C.c_int() for _ in range(4))
        _check(lib().ow3d_zone_box(self.h, zone, _C.byref(a), _C.byref(b), _C.byref(c), _C.byref(d)), "ow3d_zone_box")
        return a.value, b.value, c.value, d.value

    def write_ep(self, directory, nr, fields=0):
        _check(lib().ow3d_write_ep(self.h, _b(directory), nr, fields), "ow3d_write_ep")

    def write_ascii(self, directory, nr, fields=0):
        _check(lib().ow3d_write_ascii(self.h, _b(directory), nr, fields), "ow3d_write_ascii")

    def write_end(self, path):
        _check(lib().ow3d_write_end(self.h, _b(path)), "ow3d_write_end")

    def store_data(self, directory):
        n = _C.c_int()
        _check(lib().ow3d_store_data(self.h, _b(directory), _C.byref(n)), "ow3d_store_data")
        return n.value

    def kinematics(self):
        """u, v, w and the 9 gradient fields (9, N) of the current state."""
        u, v, w = (_np.zeros(self.N) for _ in range(3))
        g = _np.zeros(9 * self.N)
        _check(lib().ow3d_kinematics(self.h, _d(u), _d(v), _d(w), _d(g)), "ow3d_kinematics")
        return u, v, w, g.reshape(9, self.N)

    def store_kinematics(self, directory):
        n = _C.c_int()
        _check(lib().ow3d_store_kinematics(self.h, _b(directory), _C.byref(n)), "ow3d_store_kinematics")
        return n.value

    def stats(self):
        s = Stats()
        _check(lib().ow3d_get_stats(self.h, _C.byref(s)), "ow3d_get_stats")
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def reset_stats(self):
        lib().ow3d_reset_stats(self.h)

    # ---- probes (include/ow3d_test.h)
    def level_count(self):
        return lib().ow3d_level_count(self.h)

    def level_dims(self, l):
        a, b, c, d = (_C.c_int() for _ in range(4))
        _check(lib().ow3d_level_dims(self.h, l, _C.byref(a), _C.byref(b), _C.byref(c), _C.byref(d)), "level_dims")
        return a.value, b.value, c.value, d.value

    def level_size(self, l):
        nx, ny, nz, _ = self.level_dims(l)
        gy = 1 if self.params.Ny > 1 else 0
        return (nx + 2) * (ny + 2 * gy) * (nz + 1)

    def level_op(self, l, op, in1, in2=None, nu=1):
        n_out = {0: self.level_size(l), 1: self.level_size(l), 2: self.level_size(l - 1) if l > 0 else 0,
                 3: self.level_size(l), 4: self.level_size(l), 5: self.level_size(l)}[op]
        out = _np.zeros(n_out)
        a = _f64(in1).ravel(); b = None if in2 is None else _f64(in2).ravel()
        _check(lib().ow3d_test_level_op(self.h, l, op, nu, _d(a), _d(b), _d(out)), "level_op")
        return out

    def surface_derivs(self):
        """eta_x, eta_y as the device holds them (include/ow3d_test.h)."""
        Ex, Ey = _np.zeros(self.C), _np.zeros(self.C)
        _check(lib().ow3d_test_surface_derivs(self.h, _d(Ex), _d(Ey)), "surface_derivs")
        return Ex, Ey

    def stencils(self):
        SX = _np.zeros((2, self.Nxg, 7)); SY = _np.zeros((2, self.Nyg, 7 if self.params.Ny > 1 else 1))
        SZ = _np.zeros((2, self.Nzg, 7))
        _check(lib().ow3d_test_stencils(self.h, _d(SX), _d(SY), _d(SZ)), "stencils")
        return SX, SY, SZ


def version():
    return lib().ow3d_version().decode()


from . import serving  # noqa: E402,F401  (needs Simulation and OW3DError above)
