"""ctypes mirror of include/ow3d.h (structs, constants, signatures).

The layout of ``Params``/``Zone``/``Stats`` must match the C structs field
by field; ``tests/test_capi.py`` checks the sizes against the library's own
``sizeof`` export.
"""
import ctypes as C

OK = 0
NOT_CONVERGED = 1
ERR_BAD_INPUT = -1
ERR_CUDA = -2
ERR_OOM = -3
ERR_UNSTABLE = -4
ERR_TIMEOUT = -5
ERR_NO_DEVICE = -6
ERR_IO = -7
ERR_UNSUPPORTED = -8

PREC_FP64 = 0
PREC_MIXED = 1
KRYLOV_FGMRES = 0
KRYLOV_LGMRES = 1
SMOOTHER_MULTICOLOUR = 0
SMOOTHER_LEXICOGRAPHIC = 1
MAX_ZONES = 8
MAX_KIN_FILES = 20


class Zone(C.Structure):
    _fields_ = [
        ("x1", C.c_double), ("x2", C.c_double), ("y1", C.c_double), ("y2", C.c_double),
        ("ftype", C.c_int), ("param", C.c_double), ("XorY", C.c_char),
        ("WavegenONOFF", C.c_int), ("XorYgen", C.c_char), ("degrees", C.c_double),
        ("PhiOnOff", C.c_int),
    ]


class Params(C.Structure):
    _fields_ = [
        ("IC", C.c_int), ("IncWaveType", C.c_int),
        ("Lx", C.c_double), ("Ly", C.c_double), ("Lz", C.c_double),
        ("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
        ("GridX", C.c_int), ("GridY", C.c_int), ("GridZ", C.c_int),
        ("GhostGridX", C.c_int), ("GhostGridY", C.c_int), ("GhostGridZ", C.c_int),
        ("alpha", C.c_int), ("beta", C.c_int), ("gamma", C.c_int),
        ("alphaprecond", C.c_int), ("betaprecond", C.c_int), ("gammaprecond", C.c_int),
        ("Nsteps", C.c_int), ("dt", C.c_double), ("timemethod", C.c_int), ("CFL", C.c_double),
        ("extrapolationONOFF", C.c_int), ("time0", C.c_double),
        ("g", C.c_double),
        ("solver", C.c_int), ("Precond", C.c_int), ("MGCoarseningStrategy", C.c_int),
        ("GMRESmaxiterations", C.c_int), ("reltol", C.c_double), ("abstol", C.c_double),
        ("maxit", C.c_int), ("cyclet", C.c_char), ("nu1", C.c_int), ("nu2", C.c_int),
        ("MGmaxgrids", C.c_int),
        ("LinearONOFF", C.c_int), ("PressureTermOnOff", C.c_int),
        ("filteringONOFF", C.c_int), ("filterALPHA", C.c_int), ("filterORDER", C.c_int),
        ("sigma_filt", C.c_double * 3),
        ("relaxONOFF", C.c_int), ("relaxTransientTime", C.c_double), ("relaxNo", C.c_int),
        ("relaxXorY", C.c_char), ("relaxDegrees", C.c_double),
        ("zones", Zone * MAX_ZONES),
        ("precision", C.c_int), ("krylov", C.c_int), ("device", C.c_int),
        ("StoreDataONOFF", C.c_int), ("formattype", C.c_int),
        ("iKinematics", C.c_int), ("nOutFiles", C.c_int), ("kinematics", (C.c_int * 9) * MAX_KIN_FILES),
        ("ispec", C.c_int), ("seed", C.c_int), ("seed2", C.c_int),
        ("Tp", C.c_double), ("Hs", C.c_double), ("h0", C.c_double),
        ("kh_max", C.c_double), ("x0", C.c_double), ("y0", C.c_double),
        ("gamma_jonswap", C.c_double), ("beta0", C.c_double), ("s0", C.c_double),
        ("sf_H", C.c_double), ("sf_h", C.c_double), ("sf_L", C.c_double), ("sf_T", C.c_double),
        ("sf_uEorS", C.c_double), ("sf_wavel_or_per", C.c_int), ("sf_euler_or_stokes", C.c_int),
        ("sf_nsteps", C.c_int), ("sf_nmodes", C.c_int),
        ("bathymetry_file", C.c_char * 256),
        ("accel_tol_fact", C.c_double), ("i_breaking", C.c_int), ("PDampingONOFF", C.c_int),
        ("swenseONOFF", C.c_int), ("curvilinearONOFF", C.c_int),
        ("NDampZones", C.c_int), ("pd_type", C.c_int),
        ("pd_x0", C.c_double), ("pd_x1", C.c_double), ("pd_y0", C.c_double), ("pd_y1", C.c_double),
        ("pd_g0Phi", C.c_double), ("pd_g0Eta", C.c_double),
        ("accel_from_deck", C.c_int), ("periodic_x", C.c_int),
        ("T_half", C.c_double), ("phi_b", C.c_double), ("phi_0", C.c_double),
        ("del_fac", C.c_double), ("cel_fac", C.c_double), ("gamma_break", C.c_double),
        ("current_flag", C.c_int), ("current_Q", C.c_double),
        ("flux_ramp", C.c_double), ("flux_order", C.c_int), ("flux_file", C.c_char * 256),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("solves", C.c_int64), ("total_iterations", C.c_int64),
        ("min_iterations", C.c_int), ("max_iterations", C.c_int), ("last_iterations", C.c_int),
        ("not_converged", C.c_int64), ("last_residual", C.c_double),
        ("time", C.c_double), ("tstep", C.c_int64),
        ("last_initial_residual", C.c_double), ("last_tolerance", C.c_double),
    ]


def default_params(**kw):
    """Defaults the reference applies for omitted deck fields (mirrors
    ow3d_default_params in the C library, which is the authority on device)."""
    p = Params()
    p.IC = 0; p.IncWaveType = 0
    p.Lx = 1.0; p.Ly = 1.0; p.Lz = 1.0
    p.Nx = 17; p.Ny = 1; p.Nz = 9
    p.GridX = 0; p.GridY = 0; p.GridZ = 1
    p.GhostGridX = 1; p.GhostGridY = 1; p.GhostGridZ = 1
    p.alpha = p.beta = p.gamma = 3
    p.alphaprecond = p.betaprecond = p.gammaprecond = 1
    p.Nsteps = 1; p.dt = 0.01; p.timemethod = 1; p.CFL = 0.0
    p.extrapolationONOFF = 1; p.time0 = 0.0
    p.g = 9.81
    p.solver = 1; p.Precond = 3; p.MGCoarseningStrategy = 0
    p.GMRESmaxiterations = 23; p.reltol = 1e-8; p.abstol = 1e-6
    p.maxit = 1; p.cyclet = b"V"; p.nu1 = 1; p.nu2 = 1; p.MGmaxgrids = 0
    p.LinearONOFF = 1; p.PressureTermOnOff = 0
    p.filteringONOFF = 0; p.filterALPHA = 6; p.filterORDER = 10
    p.sigma_filt[0] = 0.08; p.sigma_filt[1] = 0.08; p.sigma_filt[2] = 0.4
    p.relaxONOFF = 0; p.relaxTransientTime = 0.0; p.relaxNo = 0
    p.relaxXorY = b"X"; p.relaxDegrees = 0.0
    p.precision = PREC_FP64; p.krylov = KRYLOV_FGMRES; p.device = 0
    p.StoreDataONOFF = 0; p.formattype = 0
    p.ispec = -1; p.gamma_jonswap = 3.3; p.s0 = 1.0
    p.sf_nsteps = 1
    p.accel_tol_fact = 1e30
    p.flux_order = 1
    for k, v in kw.items():
        if k == "zones":
            for i, z in enumerate(v):
                set_zone(p, i, **z)
            continue
        if isinstance(getattr(p, k), bytes) and isinstance(v, str):
            v = v.encode()
        setattr(p, k, v)
    return p


def set_zone(p, i, x1, x2, y1=0.0, y2=1.0, ftype=9, param=3.5, XorY="X", wavegen=0,
             XorYgen="X", degrees=0.0, phi=1):
    z = p.zones[i]
    z.x1, z.x2, z.y1, z.y2 = x1, x2, y1, y2
    z.ftype = ftype; z.param = param
    z.XorY = XorY.encode(); z.WavegenONOFF = wavegen; z.XorYgen = XorYgen.encode()
    z.degrees = degrees; z.PhiOnOff = phi


def dims(p):
    """(Nxg, Nyg, Nzg) with ghosts, as SetupCompDomain.f90 allocates them."""
    gx = p.GhostGridX if p.Nx > 1 else 0
    gy = p.GhostGridY if p.Ny > 1 else 0
    return p.Nx + 2 * gx, p.Ny + 2 * gy, p.Nz + p.GhostGridZ


_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def declare(lib):
    """Attach argtypes/restype for every exported ow3d_* symbol."""
    H = C.c_void_p
    sig = {
        "ow3d_default_params": (C.c_int, [C.POINTER(Params)]),
        "ow3d_read_deck": (C.c_int, [C.c_char_p, C.POINTER(Params)]),
        "ow3d_create": (C.c_int, [C.POINTER(Params), _D, _D, _D, _D, _D, C.POINTER(H)]),
        "ow3d_destroy": (C.c_int, [H]),
        "ow3d_dims": (C.c_int, [H, _I, _I, _I, C.POINTER(C.c_size_t)]),
        "ow3d_estimate_bytes": (C.c_int, [C.POINTER(Params), C.POINTER(C.c_size_t)]),
        "ow3d_solve": (C.c_int, [H, _D, _D, _D, _D, _D, _D, _D, _I]),
        "ow3d_solve_device": (C.c_int, [H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, _I]),
        "ow3d_matvec": (C.c_int, [H, _D, _D, _D, _D, _D, _D, _D]),
        "ow3d_precondition": (C.c_int, [H, _D, _D]),
        "ow3d_residual_device_noalloc": (C.c_int, [H] + [C.c_void_p] * 8 + [_D]),
        "ow3d_set_state": (C.c_int, [H, _D, _D, _D, _D, C.c_double]),
        "ow3d_get_state": (C.c_int, [H, _D, _D, _D, _D, _D]),
        "ow3d_put_surface": (C.c_int, [H, _D, _D]),
        "ow3d_step_timed": (C.c_int, [H, C.c_int, _D]),
        "ow3d_last_error": (C.c_char_p, []),
        "ow3d_set_relax_target": (C.c_int, [H, C.c_int, C.c_int, C.c_int, C.c_double, _D, _D]),
        "ow3d_incident_wave_device": (C.c_int, [H, C.c_int, C.c_int]),
        "ow3d_rollers": (C.c_int, [H, C.c_int, _I, _I, _I, _D, _D, _D, _D]),
        "ow3d_step": (C.c_int, [H, C.c_int]),
        "ow3d_step_batch": (C.c_int, [C.POINTER(H), C.c_int, _I, _I, _D]),
        "ow3d_get_stats": (C.c_int, [H, C.POINTER(Stats)]),
        "ow3d_reset_stats": (C.c_int, [H]),
        "ow3d_set_graphs": (C.c_int, [H, C.c_int]),
        "ow3d_set_coarse_cluster": (C.c_int, [H, C.c_int]),
        "ow3d_set_smoother_order": (C.c_int, [H, C.c_int]),
        "ow3d_read_paddle_signal": (C.c_int, [C.c_char_p, C.c_int, _D, _I, _I, _D, _D]),
        "ow3d_set_paddle_signal": (C.c_int, [H, C.c_int, C.c_int, C.c_double, _D, _D]),
        "ow3d_zone_box": (C.c_int, [H, C.c_int, _I, _I, _I, _I]),
        "ow3d_strerror": (C.c_char_p, [C.c_int]),
        "ow3d_version": (C.c_char_p, []),
        "ow3d_write_ep_file": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _D, _D, _D, _D]),
        "ow3d_write_ascii_file": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _D, _D, _D, _D]),
        "ow3d_write_end_file": (C.c_int, [C.c_char_p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, _D, _D]),
        "ow3d_read_init_file": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _D, _D, _D]),
        "ow3d_io_last_error": (C.c_char_p, []),
        "ow3d_write_ep": (C.c_int, [H, C.c_char_p, C.c_int, C.c_int]),
        "ow3d_write_ascii": (C.c_int, [H, C.c_char_p, C.c_int, C.c_int]),
        "ow3d_write_end": (C.c_int, [H, C.c_char_p]),
        "ow3d_store_data": (C.c_int, [H, C.c_char_p, _I]),
        "ow3d_kinematics": (C.c_int, [H, _D, _D, _D, _D]),
        "ow3d_incident_wave": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D, _D, _I]),
        "ow3d_stream_function_wave": (C.c_int, [C.c_void_p, C.c_int, _D, C.c_double, _D, _D, _D]),
        "ow3d_read_bathymetry": (C.c_int, [C.c_void_p, C.c_char_p, _D, _D, _D, _D, _D, _I]),
        "ow3d_initial_condition": (C.c_int, [C.c_void_p, _D, _D, _D, _D, _D, _D, _D]),
        "ow3d_store_kinematics": (C.c_int, [H, C.c_char_p, _I]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib
