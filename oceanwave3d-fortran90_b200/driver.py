"""Run an OceanWave3D input deck on the device: the reference's main program
(src/main/OceanWave3D.f90, OceanWave3DT0Setup.f90, OceanWave3DTakeATimeStep.f90)
for the parts this library builds.

    from ow3d_b200 import driver
    sim, setup, status = driver.run("OceanWave3D.inp", outdir="out")

prepare() does the host set-up (no device): the deck, the geometry and
initial state (a bathymetry file when Lz <= 0, the formula initial conditions,
a hot start from OceanWave3D.init for IC -1) and the relaxation-zone targets of
the incident wave (IncWaveType 1: the stream-function wave at every RK stage
time; 2: the reference's linear or random wave series; 3: the paddle signal
of the flux wavemaker, read from the file the deck names). A pressure-damping
zone, the current of IncWaveType 4 / 5, the breaking model and the local
smoothing need no host step: ow3d_create sets them up from the deck. run() creates the
simulation, applies the output schedule of the deck at step 0 and after every
step (EP / ASCII files, OceanWave3D.end, Kinematics files) and takes the
Nsteps - 1 steps of the reference's time loop. run() takes any backend with
the Simulation interface; files are written only by backends that write them.
"""
import pathlib

import numpy as np

from . import capi
from . import (Simulation, dims, incident_wave, initial_condition, lib, read_bathymetry, read_deck, read_init_file,
               read_paddle_signal, stream_function_wave)


def zone_box(p, zone):
    """Ghost-inclusive 1-based box (i0, i1, j0, j1) of relaxation zone `zone`,
    host-only (the box query of ow3d_incident_wave)."""
    import ctypes as C
    box = (C.c_int * 5)()
    r = lib().ow3d_incident_wave(C.byref(p), zone, 1, None, None, box)
    if r != 0:
        raise ValueError(f"zone {zone}: {lib().ow3d_last_error().decode()}")
    return tuple(box[:4])


class Setup:
    """Everything a run needs before the device is involved."""

    def __init__(self, params, geometry, E0, P0, targets, notes, paddle=None):
        self.params, self.geometry, self.E0, self.P0 = params, geometry, E0, P0
        self.targets = targets          # {zone: (mode, nt, dt_sample, eta, phis)}
        self.notes = notes              # how each part was built, for the log
        self.paddle = paddle            # flux wavemaker: (dt, y, flux) or None


def prepare(deck, deck_dir=None, steps=None):
    """Host set-up of a deck (a path or a Params). steps: the time steps the
    targets must cover (default: the deck's Nsteps)."""
    notes = []
    if isinstance(deck, capi.Params):
        p = deck
    else:
        deck = pathlib.Path(deck)
        deck_dir = deck_dir or deck.parent
        p = read_deck(deck)
    deck_dir = pathlib.Path(deck_dir or ".")
    Nxg, Nyg, _ = dims(p)
    C = Nxg * Nyg
    # the time step from the Courant number and the incident wave's speed
    # (OceanWave3DT0Setup.f90:58-90, with relaxation zones and CFL != 0)
    if p.relaxONOFF > 0 and p.CFL != 0:
        dx = p.Lx / (p.Nx - 1) if p.Nx > 1 else 0.0
        dy = p.Ly / (p.Ny - 1) if p.Ny > 1 else 0.0
        dxmin = dx if p.Nx > 1 else 2 * dy
        dymin = dy if p.Ny > 1 else 2 * dx
        if p.IncWaveType == 2:
            T, L = p.Tp, p.g * p.Tp ** 2 / (2 * np.pi)
        else:
            T, L = p.sf_T, p.sf_L
        if T > 0 and L > 0:
            p.dt = p.CFL * min(dxmin, dymin) / (L / T)
            notes.append(f"dt = {p.dt:.6g} from Courant {p.CFL} and the wave speed {L / T:.6g}")
    # geometry and initial surface (SetupInitialConditions.f90)
    if p.Lz <= 0:
        geometry, flag = read_bathymetry(p, deck_dir=deck_dir)
        E0, P0 = np.zeros(C), np.zeros(C)
        notes.append(f"bathymetry from {p.bathymetry_file.decode()} (gradient flag {flag})")
        if p.IC not in (0, -1):
            notes.append(f"IC {p.IC} with a bathymetry file: the surface starts at rest")
    elif p.IC == -1:
        geometry = {"h": np.full(C, p.Lz)}
        E0, P0 = np.zeros(C), np.zeros(C)
        notes.append("flat bottom, depth Lz")
    else:
        geometry, E0, P0 = initial_condition(p)
        notes.append(f"IC {p.IC} from its formula")
    if p.IC == -1:
        # OceanWave3D.init in the run directory (SetupInitialConditions.f90:18-27)
        Ei, Pi, t0 = read_init_file(deck_dir / "OceanWave3D.init", p.Nx, p.Ny)
        E0 = np.zeros((Nyg, Nxg)); P0 = np.zeros((Nyg, Nxg))
        gy, gx = (1 if p.Ny > 1 else 0), (1 if p.Nx > 1 else 0)
        E0[gy:Nyg - gy, gx:Nxg - gx] = Ei.reshape(p.Ny, p.Nx)
        P0[gy:Nyg - gy, gx:Nxg - gx] = Pi.reshape(p.Ny, p.Nx)
        E0, P0 = E0.ravel(), P0.ravel()
        p.time0 = t0
        notes.append(f"hot start from OceanWave3D.init at t = {t0}")
    # incident-wave targets of the generation zones
    targets = {}
    if p.relaxONOFF == 1:
        for z in range(p.relaxNo):
            zone = p.zones[z]
            if zone.WavegenONOFF != 1 or zone.XorYgen.upper() != b"X":
                continue
            if p.IncWaveType == 2:
                eta, phis, box = incident_wave(p, z)
                targets[z] = (0, eta.shape[0], p.dt, eta, phis)
                notes.append(f"zone {z}: incident wave ispec {p.ispec}, {eta.shape[0]} samples")
            elif p.IncWaveType == 1:
                i0, i1, j0, j1 = zone_box(p, z)
                x = (np.arange(Nxg) - (1 if p.Nx > 1 else 0)) * (p.Lx / max(p.Nx - 1, 1))
                xs = x[i0 - 1:i1]
                nsteps = max(p.Nsteps, 1) if steps is None else int(steps) + 1
                nt = 2 * nsteps + 2 + int(np.ceil(2 * max(p.time0, 0.0) / p.dt))
                line = [stream_function_wave(p, xs, n * 0.5 * p.dt)[:2] for n in range(nt)]
                rows = j1 - j0 + 1
                eta = np.array([np.tile(e, rows) for e, _ in line])
                phis = np.array([np.tile(f, rows) for _, f in line])
                targets[z] = (1, nt, 0.5 * p.dt, eta, phis)
                notes.append(f"zone {z}: stream-function wave at every RK stage time")
    paddle = None
    if p.IncWaveType == 3:
        # the flux wavemaker's paddle signal (setupWavePaddle.f90), named by the deck
        f = deck_dir / p.flux_file.decode()
        paddle = read_paddle_signal(f)
        notes.append(f"flux wavemaker: {f.name}, {paddle[2].shape[0]} times every {paddle[0]:g} s, "
                     f"{paddle[2].shape[1]} points in y, ramp {p.flux_ramp:g} s, order {p.flux_order}")
    if p.current_flag:
        notes.append(f"constant-flux current Q = {p.current_Q:g} m^2/s")
    if p.PDampingONOFF:
        # set up on the device by ow3d_create (PreprocessPDampingZones.f90)
        notes.append(f"pressure-damping zone x = {p.pd_x0:g} .. {p.pd_x1:g}, type {p.pd_type}, "
                     f"g0 {p.pd_g0Phi:g} (phi) {p.pd_g0Eta:g} (eta)")
    return Setup(p, geometry, E0, P0, targets, notes, paddle)


def run(deck, outdir=None, steps=None, backend=Simulation, deck_dir=None):
    """prepare() then the time loop (OceanWave3D.f90:18-28): the deck's
    output schedule at step 0 and after each of the steps (Nsteps - 1 by
    default). Returns the simulation (still open: close it when done), the
    setup and the worst step status (1: some solve reached the matvec limit,
    which the reference accepts silently)."""
    s = prepare(deck, deck_dir, steps)
    p = s.params
    sim = backend(p, **s.geometry)
    sim.set_state(s.E0, s.P0, t=p.time0)
    for z, t in s.targets.items():
        sim.set_relax_target(z, *t)
    if s.paddle is not None and hasattr(sim, "set_paddle_signal"):
        sim.set_paddle_signal(*s.paddle)
    out = None if outdir is None else str(outdir)
    writes = out is not None and hasattr(sim, "store_data")
    if out is not None:
        pathlib.Path(out).mkdir(parents=True, exist_ok=True)
    if writes:
        sim.store_data(out)
        if p.iKinematics:
            sim.store_kinematics(out)
    n = (p.Nsteps - 1) if steps is None else int(steps)
    status = 0
    for _ in range(n):
        r = sim.step(1)
        status = max(status, r)
        if writes:
            sim.store_data(out)
            if p.iKinematics:
                sim.store_kinematics(out)
    return sim, s, status
