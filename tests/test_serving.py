"""Serving loop (continuous batching, memory-gated admission): scheduling
logic on CPU with a fake backend and a fake clock; on the GPU, each
simulation's result is the same alone and in the mix."""
import numpy as np
import pytest

import cases  # noqa: F401  (puts tests/ on the path for the package loader)


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 0.0)


class FakeBackend:
    """Device stand-in: memory ~ DOF, every step costs 1 ms of fake time per
    resident simulation divided by the overlap factor."""

    def __init__(self, clock, bytes_per_dof=100, check_arrival=True):
        self.clock = clock
        self.check_arrival = check_arrival
        self.bpd = bytes_per_dof
        self.resident = {}
        self.peak = 0
        self.created = []

    def estimate_bytes(self, req):
        return req.dof * self.bpd

    def create(self, req):
        assert not self.check_arrival or req.arrival <= self.clock.t + 1e-12, "admitted before arrival"
        self.resident[req.rid] = self.estimate_bytes(req)
        self.peak = max(self.peak, sum(self.resident.values()))
        self.created.append(req.rid)
        return req

    def step_batch(self, sims, nsteps):
        # a step costs (1 + 0.1 * slots) ms; the round lasts the longest run
        c = 1.0 + 0.1 * len(sims)
        self.clock.t += 1e-3 * c * max(nsteps)
        return [0] * len(sims), [c * k for k in nsteps]

    def finish(self, sim, req):
        del self.resident[req.rid]
        return np.full(3, float(req.rid))


def small_stream(ow3d, n=40, seed=3):
    return ow3d.serving.request_stream(n=n, rate=200.0, seed=seed, nx=(65, 129), ny=(1, 33), nz=(9, 13),
                                       steps=(3, 12))


def test_request_stream_is_seeded_and_in_sets(ow3d):
    a = ow3d.serving.request_stream(n=64, seed=7)
    b = ow3d.serving.request_stream(n=64, seed=7)
    assert [(r.Nx, r.Ny, r.Nz, r.steps, r.seed, r.arrival) for r in a] == \
           [(r.Nx, r.Ny, r.Nz, r.steps, r.seed, r.arrival) for r in b]
    s = ow3d.serving
    for r in a:
        assert r.Nx in s.NX_SET and r.Ny in s.NY_SET and r.Nz in s.NZ_SET and 100 <= r.steps <= 2000
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)


def test_admission_respects_memory_budget(ow3d):
    clock = FakeClock()
    be = FakeBackend(clock)
    reqs = small_stream(ow3d)
    budget = 3 * max(r.dof for r in reqs) * be.bpd
    srv = ow3d.serving.Server(be, budget_bytes=budget, max_slots=8, clock=clock, sleep=clock.sleep)
    out = srv.run(reqs)
    assert out["completed"] == len(reqs)
    assert be.peak <= budget
    assert out["peak_slots"] <= 8
    assert all(len(r.step_ms) == r.steps for r in reqs)
    assert all(r.admitted >= r.arrival for r in reqs)
    assert out["peak_slots"] > 1            # requests overlapped


def test_oversized_request_rejected(ow3d):
    clock = FakeClock()
    be = FakeBackend(clock)
    reqs = small_stream(ow3d, n=6)
    big = max(reqs, key=lambda r: r.dof)
    srv = ow3d.serving.Server(be, budget_bytes=big.dof * be.bpd - 1, clock=clock, sleep=clock.sleep)
    srv.run(reqs)
    assert big.status == ow3d.capi.ERR_OOM and big.rid not in be.created
    assert all(r.status == 0 and len(r.step_ms) == r.steps for r in reqs if r.dof < big.dof)


def test_sequential_baseline_runs_alone(ow3d):
    clock = FakeClock()
    be = FakeBackend(clock, check_arrival=False)    # the baseline ignores arrival times
    reqs = small_stream(ow3d, n=5)
    out = ow3d.serving.run_sequential(be, reqs, clock=clock)
    assert out["completed"] == 5 and be.peak == max(r.dof for r in reqs) * be.bpd


def test_bathymetry_range_and_derivatives(ow3d):
    req = ow3d.serving.Request(rid=0, arrival=0.0, Nx=129, Ny=65, Nz=9, steps=1, seed=11)
    p, geo, eta, phis = ow3d.serving.request_case(req)
    h = geo["h"]
    assert h.min() >= 0.3 and h.max() <= 1.0
    Nxg, Nyg, _ = ow3d.dims(p)
    H = h.reshape(Nyg, Nxg)
    dx = p.Lx / (p.Nx - 1)
    fd = (H[:, 2:] - H[:, :-2]) / (2 * dx)
    assert np.max(np.abs(fd - geo["hx"].reshape(Nyg, Nxg)[:, 1:-1])) < 1e-3
    assert p.dt > 0 and eta.shape == (Nxg * Nyg,)


@pytest.mark.gpu
def test_results_same_alone_and_in_mix(ow3d):
    s = ow3d.serving
    mk = lambda: [s.Request(rid=i, arrival=0.0, Nx=65, Ny=ny, Nz=9, steps=st, seed=100 + i)
                  for i, (ny, st) in enumerate([(1, 6), (33, 4), (33, 6), (1, 3)])]
    be = s.DeviceBackend(ow3d)
    alone = mk()
    s.run_sequential(be, alone, keep_eta=True)
    mixed = mk()
    out = s.Server(be, budget_bytes=8 << 30, max_slots=4).run(mixed, keep_eta=True)
    assert out["completed"] == 4 and out["peak_slots"] == 4
    for a, m in zip(alone, mixed):
        assert a.status >= 0 and m.status >= 0
        assert np.max(np.abs(a.final_eta - m.final_eta)) <= 1e-12 * max(np.max(np.abs(a.final_eta)), 1e-30)
