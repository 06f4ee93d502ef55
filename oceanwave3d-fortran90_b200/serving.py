"""Continuous-batching serving loop for independent wave simulations.

Requests arrive over time (a seeded Poisson process). Each one is a whole
simulation -- its own grid, bathymetry and sea state -- that must be advanced
a given number of RK4 steps. The server keeps every admitted simulation
resident on the device (state, Krylov workspace and multigrid hierarchy live
in its handle) and advances all of them together, one step per round, through
ow3d_step_batch: one host thread keeps every simulation's next RK4 step in
flight as one CUDA graph on the simulation's own stream (the Arnoldi steps of
each solve are conditional nodes the device enables, so no host round trip
happens inside a step) and launches a simulation's next step as soon as its
previous one completes, so the simulations' kernels overlap on the GPU. In a
round, a simulation takes as many steps as fit in the longest single step of
the round (from the step times measured in the previous round), so small
simulations are not held back by large ones. Each simulation's coarse
multigrid levels run in one thread-block cluster (ow3d_set_coarse_cluster)
rather than a cooperative grid over every SM, so that the coarse cycles of
the simulations overlap too. A request is admitted as soon as it has arrived, a slot is
free and its estimated device memory (ow3d_estimate_bytes) fits in what the
running simulations leave of the memory budget; finished simulations release
their handle (and memory) at the end of the round in which they finish.

Reported: per-step latency percentiles over every step of every request (a
request's host time inside its round divided by the steps it took in the
round), request latency
(arrival to completion), and aggregate DOF-timesteps/s of the whole run.

The reference advances one simulation per process; this module has no
counterpart there. The backend object isolates the device calls so that the
scheduling logic is testable without a GPU.
"""
import ctypes as C
import dataclasses
import time

import numpy as np

from . import capi
from .workloads import G, grid_xy, linear_sea

NX_SET = (65, 129, 257, 513, 1025)          # multigrid-coarsenable sizes in [65, 1025]
NY_SET = (1, 33, 65, 129, 257)
NZ_SET = (9, 13, 17)


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float          # seconds after the stream starts
    Nx: int
    Ny: int
    Nz: int
    steps: int
    seed: int
    # filled in by the server
    admitted: float = -1.0
    finished: float = -1.0
    step_ms: list = dataclasses.field(default_factory=list)
    status: int = 0
    final_eta: np.ndarray = None

    @property
    def dof(self):
        return self.Nx * self.Ny * self.Nz


def request_stream(n=512, rate=4.0, seed=2024, nx=NX_SET, ny=NY_SET, nz=NZ_SET, steps=(100, 2000)):
    """n requests with exponential inter-arrival times (mean 1/rate seconds),
    sizes drawn uniformly from the given sets and step counts uniformly from
    [steps[0], steps[1]]."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for r in range(n):
        out.append(Request(rid=r, arrival=float(t[r]), Nx=int(rng.choice(nx)), Ny=int(rng.choice(ny)),
                           Nz=int(rng.choice(nz)), steps=int(rng.integers(steps[0], steps[1] + 1)),
                           seed=int(rng.integers(0, 2 ** 31 - 1))))
    return out


def bathymetry(p, seed):
    """Plane slope plus 3 seeded Gaussian bumps with analytic derivatives,
    depth kept within 0.3-1.0 m by construction (no clipping)."""
    rng = np.random.default_rng(seed)
    x, y = grid_xy(p)
    X, Y = np.meshgrid(x, y)
    Lx, Ly = p.Lx, max(p.Ly, 1e-9)
    h = 0.85 - 0.3 * X / Lx                     # 0.85 -> 0.55 m
    hx = np.full_like(X, -0.3 / Lx)
    hxx = np.zeros_like(X); hy = np.zeros_like(X); hyy = np.zeros_like(X)
    for _ in range(3):
        a = rng.uniform(-0.08, 0.08)
        x0 = rng.uniform(0.2, 0.8) * Lx
        y0 = rng.uniform(0.2, 0.8) * Ly if p.Ny > 1 else 0.0
        sx = rng.uniform(0.05, 0.15) * Lx
        sy = rng.uniform(0.05, 0.15) * Ly if p.Ny > 1 else 1.0
        gy = ((Y - y0) / sy) ** 2 if p.Ny > 1 else 0.0
        g = a * np.exp(-0.5 * (((X - x0) / sx) ** 2 + gy))
        h += g
        hx += -g * (X - x0) / sx ** 2
        hxx += g * (((X - x0) / sx ** 2) ** 2 - 1.0 / sx ** 2)
        if p.Ny > 1:
            hy += -g * (Y - y0) / sy ** 2
            hyy += g * (((Y - y0) / sy ** 2) ** 2 - 1.0 / sy ** 2)
    return dict(h=h.ravel(), hx=hx.ravel(), hxx=hxx.ravel(), hy=hy.ravel(), hyy=hyy.ravel())


def request_case(req, precision=capi.PREC_MIXED, dx=0.1, Hs=0.02, Tp=1.5, gamma=3.3, courant=0.5, reltol=1e-8):
    """Parameters, bathymetry and initial surface of one request."""
    p = capi.default_params(Nx=req.Nx, Ny=req.Ny, Nz=req.Nz, Lx=(req.Nx - 1) * dx,
                            Ly=(req.Ny - 1) * dx if req.Ny > 1 else 1.0, Lz=1.0, GridZ=1, reltol=reltol,
                            precision=precision)
    geo = bathymetry(p, req.seed)
    p.g = G
    p.dt = courant * dx / np.sqrt(G * float(np.max(geo["h"])))
    x, y = grid_xy(p)
    eta, phis = linear_sea(x, y, float(np.mean(geo["h"])), Hs=Hs, Tp=Tp, gamma=gamma, nfreq=16, ndir=5,
                           seed=req.seed)
    return p, geo, eta.ravel(), phis.ravel()


class DeviceBackend:
    """The device calls the server makes, through the C ABI."""

    def __init__(self, pkg, precision=capi.PREC_MIXED, coarse_cluster=False):
        """coarse_cluster: each simulation's coarse multigrid levels run in
        one thread-block cluster (ow3d_set_coarse_cluster), so that the
        coarse cycles of simulations stepped together overlap; for batched
        serving, not for one simulation at a time."""
        self.pkg = pkg
        self.lib = pkg.lib()
        self.precision = precision
        self.coarse_cluster = coarse_cluster

    def estimate_bytes(self, req):
        p = capi.default_params(Nx=req.Nx, Ny=req.Ny, Nz=req.Nz, precision=self.precision)
        b = C.c_size_t()
        st = self.lib.ow3d_estimate_bytes(C.byref(p), C.byref(b))
        if st != 0:
            raise self.pkg.OW3DError(st, f"estimate for request {req.rid}")
        return int(b.value)

    def create(self, req):
        p, geo, eta, phis = request_case(req, precision=self.precision)
        sim = self.pkg.Simulation(p, **geo)
        if self.coarse_cluster:
            st = self.lib.ow3d_set_coarse_cluster(sim.h, 1)
            if st != 0:
                raise self.pkg.OW3DError(st, "ow3d_set_coarse_cluster")
        sim.set_state(eta, phis)
        return sim

    def step_batch(self, sims, nsteps=None):
        n = len(sims)
        hs = (C.c_void_p * n)(*[s.h for s in sims])
        steps = (C.c_int * n)(*(nsteps if nsteps is not None else [1] * n))
        status = (C.c_int * n)()
        ms = (C.c_double * n)()
        self.lib.ow3d_step_batch(hs, n, steps, status, ms)
        return list(status), list(ms)

    def finish(self, sim, req):
        E, P, W, phi, t = sim.get_state()
        sim.close()
        return E


class Server:
    """Memory-gated continuous batching over a backend."""

    def __init__(self, backend, budget_bytes, max_slots=32, clock=time.perf_counter, sleep=time.sleep):
        self.backend = backend
        self.budget = int(budget_bytes)
        self.max_slots = max(1, int(max_slots))
        self.clock = clock
        self.sleep = sleep

    def run(self, requests, keep_eta=False):
        pending = sorted(requests, key=lambda r: r.arrival)
        active = []          # (req, sim, bytes, steps_done)
        used = 0
        t0 = self.clock()
        rounds = 0
        peak_slots = 0
        while pending or active:
            now = self.clock() - t0
            # admission: arrived requests in arrival order whose memory fits (later
            # smaller requests may pass a large one that does not fit yet)
            kept = []
            for req in pending:
                if req.arrival <= now and len(active) < self.max_slots:
                    need = self.backend.estimate_bytes(req)
                    if need > self.budget:
                        req.status = capi.ERR_OOM
                        req.finished = now
                        continue
                    if used + need <= self.budget:
                        sim = self.backend.create(req)
                        req.admitted = self.clock() - t0
                        active.append([req, sim, need, 0])
                        used += need
                        continue
                kept.append(req)
            pending = kept
            if not active:
                if pending:
                    wait = pending[0].arrival - (self.clock() - t0)
                    if wait > 0:
                        self.sleep(wait)
                continue
            peak_slots = max(peak_slots, len(active))
            # steps per simulation in this round: as many as fit in the
            # round's longest single step, from the last measured step times
            est = [a[0].step_ms[-1] if a[0].step_ms else None for a in active]
            known = [e for e in est if e]
            longest = max(known) if known else None
            nst = []
            for a, e in zip(active, est):
                k = 1 if (longest is None or not e) else max(1, int(longest // e))
                nst.append(min(k, a[0].steps - a[3]))
            status, ms = self.backend.step_batch([a[1] for a in active], nst)
            rounds += 1
            now = self.clock() - t0
            still = []
            for a, st, m, k in zip(active, status, ms, nst):
                req = a[0]
                req.step_ms.extend([m / k] * k)
                a[3] += k
                if st < 0 or a[3] >= req.steps:
                    req.status = st
                    req.finished = now
                    eta = self.backend.finish(a[1], req)
                    if keep_eta:
                        req.final_eta = eta
                    used -= a[2]
                else:
                    still.append(a)
            active = still
        wall = self.clock() - t0
        return summarize(requests, wall, rounds=rounds, peak_slots=peak_slots)


def run_sequential(backend, requests, keep_eta=False, clock=time.perf_counter):
    """Each request alone, one after another, ignoring arrival times: the
    baseline the batched server is compared with."""
    t0 = clock()
    for req in requests:
        sim = backend.create(req)
        req.admitted = clock() - t0
        for _ in range(req.steps):
            st, ms = backend.step_batch([sim], [1])
            req.step_ms.append(ms[0])
            if st[0] < 0:
                break
        req.status = st[0]
        req.finished = clock() - t0
        eta = backend.finish(sim, req)
        if keep_eta:
            req.final_eta = eta
    wall = clock() - t0
    return summarize(requests, wall)


def summarize(requests, wall, **extra):
    steps = np.array([m for r in requests for m in r.step_ms], dtype=np.float64)
    done = [r for r in requests if r.finished >= 0 and r.status >= 0]
    dof_steps = float(sum(r.dof * len(r.step_ms) for r in requests))
    lat = np.array([r.finished - r.arrival for r in done if r.arrival >= 0]) if done else np.zeros(0)
    out = {
        "requests": len(requests), "completed": len(done), "wall_s": wall,
        "dof_timesteps_per_s": dof_steps / wall if wall > 0 else 0.0,
        "steps": int(steps.size),
        "step_ms_p50": float(np.percentile(steps, 50)) if steps.size else None,
        "step_ms_p99": float(np.percentile(steps, 99)) if steps.size else None,
        "request_latency_s_p50": float(np.percentile(lat, 50)) if lat.size else None,
        "request_latency_s_p99": float(np.percentile(lat, 99)) if lat.size else None,
    }
    out.update(extra)
    return out
