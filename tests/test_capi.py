"""CPU checks of the C ABI: the library loads, exports every symbol the
headers declare, its structs match the ctypes mirror, and the calls that need
no device behave (defaults, deck parsing, sizes, error codes)."""
import ctypes as C
import pathlib
import re
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions(headers=None):
    names = set()
    for h in headers or HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(ow3d_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_headers_declare_the_api():
    names = declared_functions()
    for core in ("ow3d_create", "ow3d_solve", "ow3d_step", "ow3d_get_state", "ow3d_destroy", "ow3d_strerror"):
        assert core in names
    assert len(names) >= 30


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True, text=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_library_exports_every_declared_symbol(ow3d):
    """The product library exports exactly the functions of include/ow3d.h;
    the testing build (the same objects) also the probes of ow3d_test.h,
    which the tests load."""
    L = ow3d.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(L, n)]
    assert not missing, missing
    api = declared_functions([ROOT / "include" / "ow3d.h"])
    probes = declared_functions([ROOT / "include" / "ow3d_test.h"])
    product = exported(ow3d.LIB_PATH.parent / "libow3d.so")
    assert api <= product and not (product & probes)
    assert {n for n in product if n.startswith("ow3d_")} == api
    assert (api | probes) <= exported(ow3d.LIB_PATH.parent / "libow3d_dev.so")


def test_struct_layouts_match(ow3d):
    L = ow3d.lib()
    assert L.ow3d_test_sizeof(0) == C.sizeof(ow3d.capi.Params)
    assert L.ow3d_test_sizeof(1) == C.sizeof(ow3d.capi.Zone)
    assert L.ow3d_test_sizeof(2) == C.sizeof(ow3d.capi.Stats)
    assert L.ow3d_test_sizeof(99) == -1


def test_fortran_binding_size(ow3d):
    """The Fortran module of the binding (include/ow3d_iface.f90) holds
    ow3d_params as an opaque byte array whose length must be the struct's
    size, and binds only names the C header declares."""
    text = (ROOT / "include" / "ow3d_iface.f90").read_text()
    sizes = [int(n) for n in re.findall(r"raw\((\d+)\)\s+! opaque to Fortran: sizeof\(ow3d_params\)", text)]
    assert sizes == [C.sizeof(ow3d.capi.Params)]
    bound = set(re.findall(r'BIND\(C, name="(ow3d_\w+)"\)', text))
    assert {"ow3d_read_deck", "ow3d_create", "ow3d_solve", "ow3d_step", "ow3d_get_state"} <= bound
    assert bound <= declared_functions()


def test_default_params_match_mirror(ow3d):
    L = ow3d.lib()
    q = ow3d.capi.Params()
    assert L.ow3d_default_params(C.byref(q)) == 0
    p = ow3d.default_params()
    for name, _ in ow3d.capi.Params._fields_:
        if name in ("zones", "sigma_filt", "Nx", "Nz", "Lx", "Ly", "Lz", "dt", "Nsteps", "g"):
            continue
        if name == "kinematics":
            assert [list(r) for r in q.kinematics] == [list(r) for r in p.kinematics] == [[0] * 9] * 20
            continue
        assert getattr(q, name) == getattr(p, name), name
    assert q.GMRESmaxiterations == 23 and q.reltol == 1e-8 and q.alpha == 3 and q.alphaprecond == 1


def test_strerror_and_version(ow3d):
    L = ow3d.lib()
    for code in (0, 1, -1, -2, -3, -4, -5, -6, -7, -8):
        s = L.ow3d_strerror(code)
        assert isinstance(s, bytes) and len(s) > 0
    assert b"sm_100a" in L.ow3d_version()


def test_estimate_bytes_grows_with_grid(ow3d):
    L = ow3d.lib()
    prev = 0
    for nx, ny, nz in ((33, 17, 9), (129, 33, 9), (257, 65, 17), (1025, 257, 17)):
        p = ow3d.default_params(Nx=nx, Ny=ny, Nz=nz)
        b = C.c_size_t()
        assert L.ow3d_estimate_bytes(C.byref(p), C.byref(b)) == 0
        n = (nx + 2) * (ny + 2) * (nz + 1)
        # at least phi, rhs and the 2 x (m+1) Krylov vectors of FP64
        assert b.value >= 8 * n * (2 * (p.GMRESmaxiterations + 1))
        assert b.value > prev
        prev = b.value
    assert prev < 8 * 2 ** 30      # the 4.8 M-unknown sea fits a B200 many times over


def test_invalid_params_rejected(ow3d):
    L = ow3d.lib()
    b = C.c_size_t()
    p = ow3d.default_params(Nx=33, Ny=17, Nz=9, alpha=2)
    assert L.ow3d_estimate_bytes(C.byref(p), C.byref(b)) == ow3d.capi.ERR_BAD_INPUT
    p = ow3d.default_params(Nx=33, Ny=17, Nz=40)
    assert L.ow3d_estimate_bytes(C.byref(p), C.byref(b)) == ow3d.capi.ERR_BAD_INPUT
    assert L.ow3d_estimate_bytes(None, C.byref(b)) == ow3d.capi.ERR_BAD_INPUT


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-device path")
def test_create_without_device_fails_loudly(ow3d):
    L = ow3d.lib()
    p = ow3d.default_params(Nx=17, Ny=9, Nz=9)
    Nxg, Nyg, _ = ow3d.dims(p)
    h = np.ones(Nxg * Nyg)
    d = h.ctypes.data_as(C.POINTER(C.c_double))
    out = C.c_void_p()
    assert L.ow3d_create(C.byref(p), d, None, None, None, None, C.byref(out)) == ow3d.capi.ERR_NO_DEVICE
    assert not out.value
    assert b"device" in L.ow3d_last_error()
    with pytest.raises(ow3d.OW3DError):
        ow3d.Simulation(p, h)


def test_null_handles_rejected(ow3d):
    L = ow3d.lib()
    assert L.ow3d_step(None, 1) == ow3d.capi.ERR_BAD_INPUT
    assert L.ow3d_set_graphs(None, 1) == ow3d.capi.ERR_BAD_INPUT
    assert L.ow3d_reset_stats(None) == ow3d.capi.ERR_BAD_INPUT
    s = ow3d.capi.Stats()
    assert L.ow3d_get_stats(None, C.byref(s)) == ow3d.capi.ERR_BAD_INPUT


def test_launch_counter_starts_without_device(ow3d):
    L = ow3d.lib()
    assert L.ow3d_launch_count() >= 0
