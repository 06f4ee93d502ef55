"""Benchmark: DOF-timesteps/s of the RK4 free-surface step (4 Laplace solves
per step) on the 1025 x 257 x 17 irregular-sea workload, mixed precision
(FP32 multigrid, FP64 FGMRES/RK4) against the all-FP64 GPU path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU; every rank advances its own replica of the workload
(the path does not shard: replicas only) and rank 0 prints one JSON line.
The reference arm times the CPU restatement of the reference algorithm
(lexicographic Gauss-Seidel multigrid, left-preconditioned GMRES) on the
host cores, on a bounded sub-basin of the same workload.
"""
import argparse
import importlib.util
import json
import re
import os
import pathlib
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
PKG_DIR = ROOT / "oceanwave3d-fortran90_b200"
WORKLOAD = dict(Nx=1025, Ny=257, Nz=17)
METRIC = "DOF-timesteps/s (mixed FP32-MG/FP64 vs FP64, eta err <= 1e-6)"
UNIT = "DOF-timesteps/s"
CPU_SAMPLE = dict(Nx=257, Ny=65, Nz=17)      # host sample of the same sea (same dx, Nz, spectrum)


def package():
    if "ow3d_b200" in sys.modules:
        return sys.modules["ow3d_b200"]
    spec = importlib.util.spec_from_file_location("ow3d_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ow3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, gpu=0):
        self.gpu, self.rows, self.proc = gpu, [], None
        self.first = threading.Event()

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)
                self.first.set()

    def wait_first(self, timeout=3.0):
        """Block (at most `timeout` s) until nvidia-smi has produced a sample,
        so that a short timed region still falls inside the sampling."""
        if self.proc:
            self.first.wait(timeout)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dof(p):
    return p.Nx * p.Ny * p.Nz


def replica_seed(rank):
    """Each rank runs an independent replica (its own seeded sea); nothing is
    exchanged between ranks on the data path."""
    return 1234 + rank


def max_over_ranks(value, world, device):
    """Slowest rank's time: the job is done when the last replica is."""
    if world <= 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_throughput(dof_per_replica, steps, world, ms):
    """Whole-job DOF-timesteps/s: every rank advanced its replica `steps` steps."""
    return dof_per_replica * steps * world / (ms / 1e3)


def run_gpu(args, rank, world):
    import torch
    pkg = package()
    W = pkg.workloads
    lib = pkg.lib()
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    res = {}
    states = {}
    for prec in ("fp64", "mixed"):
        p, geo, E0, P0 = W.irregular_sea(**WORKLOAD, precision=(1 if prec == "mixed" else 0), seed=replica_seed(rank))
        p.device = dev
        sim = pkg.Simulation(p, **geo)
        sim.set_state(E0, P0)
        sim.step(args.warmup)
        sim.reset_stats()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        n0 = lib.ow3d_launch_count()
        with ClockSampler(dev) as clk:
            clk.wait_first()
            st, ms = sim.step_timed(args.steps)
        launches = lib.ow3d_launch_count() - n0
        ms = max_over_ranks(ms, world, "cuda")
        s = sim.stats()
        s["status"] = st
        E, P, Wv, phi, tt = sim.get_state()
        states[prec] = (E, phi)
        pb, pinfo = path_bytes_per_step(sim, s, args.steps, 8 if prec == "fp64" else 4)
        res[prec] = dict(ms=ms, stats=s, clocks=clk.summary(), params=p, bytes=sim.device_bytes(), launches=launches,
                         path_bytes=pb, path_info=pinfo)
        if prec == "mixed":
            res["sim"] = sim
        else:
            sim.close()
    # the same steps with left-preconditioned GMRES (the reference's solver
    # and stopping test: the preconditioned residual) in both precisions
    left = {}
    for prec in ("fp64", "mixed"):
        p, geo, E0, P0 = W.irregular_sea(**WORKLOAD, precision=(1 if prec == "mixed" else 0), seed=replica_seed(rank))
        p.device = dev
        p.krylov = 1
        sim2 = pkg.Simulation(p, **geo)
        sim2.set_state(E0, P0)
        sim2.step(args.warmup)
        sim2.reset_stats()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        st2, ms2 = sim2.step_timed(args.steps)
        ms2 = max_over_ranks(ms2, world, "cuda")
        s2 = sim2.stats()
        E, P, Wv, phi, tt = sim2.get_state()
        left[prec] = dict(ms=ms2, stats=s2, status=st2, state=(E, phi))
        sim2.close()
    res["left"] = left
    # e2e through the public API with host buffers: per step, push E and P from
    # pinned host memory, one RK4 step, read E, P, W back.
    sim = res.pop("sim")
    pm = res["mixed"]["params"]
    C = sim.C
    hostE = torch.empty(C, dtype=torch.float64).pin_memory().numpy()
    hostP = torch.empty(C, dtype=torch.float64).pin_memory().numpy()
    outW = torch.empty(C, dtype=torch.float64).pin_memory().numpy()
    E, P, Wv, phi, tt = sim.get_state()
    hostE[:] = E; hostP[:] = P
    sim.reset_stats()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.put_surface(hostE, hostP)
        sim.step(1)
        lib.ow3d_get_state(sim.h, pkg._d(hostE), pkg._d(hostP), pkg._d(outW), None, None)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world, "cuda")
    res["e2e_stats"] = sim.stats()
    sim.close()
    # eta / phi error of the mixed path against the FP64 path after the same steps
    Ef, phif = states["fp64"]; Em, phim = states["mixed"]
    err_eta = float(np.max(np.abs(Em - Ef)) / np.max(np.abs(Ef)))
    err_phi = float(np.max(np.abs(phim - phif)) / np.max(np.abs(phif)))
    return res, e2e_s, err_eta, err_phi, pm


def path_bytes_per_step(sim, stats, steps, s):
    """Algorithmic HBM bytes of one RK4 step of the whole path (4 Laplace
    solves and the free-surface terms), from the per-unit figures: the
    high-order operator 2*8*N + 10*8*C (the FP32 basis vector read at 4 bytes
    in mixed mode); one Gauss-Seidel sweep on level l 3*s*N_l + 5*s*C_l;
    residual + restriction 2*s*N_l + s*N_(l-1); prolongation + correction
    s*N_(l-1) + 2*s*N_l; Arnoldi step j (2j+3)*8*N plus s*N to store z_j;
    solution update (k*s + 16)*N; free surface 30*8*C. s = 8 (FP64) or 4
    (FP32 multigrid and basis). The iteration count per solve is the run's
    mean (exact when every solve took the same count)."""
    p = sim.params
    gy = 1 if p.Ny > 1 else 0
    nl = sim.level_count()
    dims = [sim.level_dims(l) for l in range(nl)]
    Cl = [(nx + 2) * (ny + 2 * gy) for nx, ny, nz, _ in dims]
    Nl = [c * (nz + 1) for c, (nx, ny, nz, _) in zip(Cl, dims)]
    N, C = Nl[-1], Cl[-1]
    vcycle = 0
    for l in range(1, nl):
        vcycle += (p.nu1 + p.nu2) * (3 * s * Nl[l] + 5 * s * Cl[l])
        vcycle += 2 * s * Nl[l] + s * Nl[l - 1] + s * Nl[l - 1] + 2 * s * Nl[l]
    solves = max(stats["solves"], 1)
    it = stats["total_iterations"] / solves            # matvecs per solve, the initial residual's included
    k = max(it - 1.0, 0.0)                              # Arnoldi steps = preconditioner applications
    per_solve = (3 * 8 * N + 10 * 8 * C + 8 * N                       # initial residual (phi, rhs -> r), its norm
                 + k * ((s + 8) * N + 10 * 8 * C)                     # operator on z_j
                 + k * vcycle                                         # V-cycles
                 + (k * k + 4 * k) * 8 * N + k * s * N                # Arnoldi steps j = 1..k, z_j stored
                 + (k * s + 16) * N)                                  # solution update
    return (stats["solves"] / steps) * per_solve + 30 * 8 * C, {
        "levels": nl, "N": N, "C": C, "sum_N_levels": int(sum(Nl)), "iterations_per_solve": it,
        "iterations_min_max": [stats["min_iterations"], stats["max_iterations"]]}


def solver_report(st, p):
    """The stopping test of the timed solves: GMRES stops at
    |r| <= reltol*|r0| + abstol (iterative_solution.f90:24,44-45), so the
    report states both terms for the last timed solve, which of them set the
    threshold, and how many solves hit the matvec limit."""
    r0, tol = st["last_initial_residual"], st["last_tolerance"]
    return {"not_converged": st["not_converged"], "reltol": p.reltol, "abstol": p.abstol,
            "last_solve": {"initial_residual": r0, "threshold": tol, "final_residual": st["last_residual"],
                           "threshold_set_by": "abstol" if p.abstol > p.reltol * r0 else "reltol"}}


def left_report(left, D, steps, world, p):
    """The timed steps with left-preconditioned GMRES, the reference's solver
    (iterative_solution.f90: SPARSKIT2 gmres, stopping on the preconditioned
    residual), in both precisions; mixed against FP64 on eta and phi."""
    out = {"note": "same workload and steps, krylov = left-preconditioned GMRES (the reference's stopping test on "
                   "the preconditioned residual); the headline uses flexible GMRES, whose test is on the true residual"}
    for prec in ("fp64", "mixed"):
        d = left[prec]
        st = d["stats"]
        out[prec] = {"value": job_throughput(D, steps, world, d["ms"]), "ms_per_step": d["ms"] / steps,
                     "avg_iterations": st["total_iterations"] / max(st["solves"], 1), **solver_report(st, p)}
    (Ef, pf), (Em, pmx) = left["fp64"]["state"], left["mixed"]["state"]
    out["mixed"]["eta_rel_err_vs_fp64"] = float(np.max(np.abs(Em - Ef)) / np.max(np.abs(Ef)))
    out["mixed"]["phi_rel_err_vs_fp64"] = float(np.max(np.abs(pmx - pf)) / np.max(np.abs(pf)))
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def kernel_roofline(pkg, p, dev):
    """Per-launch device time of the finest-level colour pass (the smoother,
    the largest kernel class of the step) and of the high-order operator,
    each timed alone with CUDA events after an L2 flush; with their
    algorithmic bytes per launch."""
    lib = pkg.lib()
    import ctypes as C
    p2 = pkg.default_params(Nx=p.Nx, Ny=p.Ny, Nz=p.Nz, Lx=p.Lx, Ly=p.Ly, Lz=p.Lz, GridZ=1, device=dev)
    Nxg, Nyg, Nzg = pkg.dims(p2)
    sim = pkg.Simulation(p2, np.ones(Nxg * Nyg))
    ncolor = sim.level_dims(sim.level_count() - 1)[3]
    reps = 20
    out = {}
    for which, name in ((2, "colour"), (0, "operator")):
        ms = C.c_double()
        if lib.ow3d_bench_kernel(sim.h, which, reps, C.byref(ms)) == 0:
            out[name] = ms.value / reps
    sim.close()
    N, Cc = Nxg * Nyg * Nzg, Nxg * Nyg
    # one Gauss-Seidel sweep of a level moves 3*s*N_l + 5*s*C_l bytes (x read
    # and written, b read, the column coefficients); a sweep is `ncolor`
    # colour passes, each covering 1/ncolor of the columns
    alg = {"colour": (3 * 8 * N + 5 * 8 * Cc) / ncolor, "operator": 2 * 8 * N + 10 * 8 * Cc}
    return {k: (v, alg[k]) for k, v in out.items()}, ncolor


def profiled_traffic(kernel):
    """DRAM bytes (read + write) per launch of `kernel` from its committed ncu
    summary (the `traffic_bytes_per_launch:` line), or None."""
    for f in sorted((ROOT / "profiles").glob(f"{kernel}_irregular_sea_*.md")):
        m = re.search(r"^traffic_bytes_per_launch:\s*(\d+)", f.read_text(), re.M)
        if m:
            return int(m.group(1))
    return None


def serving_sample(n=16, seed=2024, rate=50.0, nx=(65, 129, 257), ny=(1, 33, 65), nz=(9, 13, 17), steps=(10, 40),
                   note="sizes capped to keep the run short", slots=(None,)):
    """Bounded sample of the serving stream: n seeded requests (Poisson
    arrivals at `rate`/s, sizes drawn from nx, ny, nz, step counts from
    `steps`), served (a) one at a time with the plain FP64 path and (b) by the
    memory-gated continuous-batching server with the mixed path."""
    import torch
    pkg = package()
    S = pkg.serving
    mk = lambda: S.request_stream(n=n, rate=rate, seed=seed, nx=nx, ny=ny, nz=nz, steps=steps)
    # warm-up: one small simulation per precision (module load, first launches)
    for prec in (pkg.capi.PREC_FP64, pkg.capi.PREC_MIXED):
        be = S.DeviceBackend(pkg, precision=prec)
        w = S.Request(rid=-1, arrival=0.0, Nx=65, Ny=33, Nz=9, steps=2, seed=1)
        sim = be.create(w); be.step_batch([sim]); be.finish(sim, w)
    seq = S.run_sequential(S.DeviceBackend(pkg, precision=pkg.capi.PREC_FP64), mk())
    free, _ = torch.cuda.mem_get_info()
    keys = ("dof_timesteps_per_s", "step_ms_p50", "step_ms_p99", "request_latency_s_p50", "request_latency_s_p99",
            "wall_s", "completed", "steps")
    runs = {}
    for cap in slots:
        srv = S.Server(S.DeviceBackend(pkg, precision=pkg.capi.PREC_MIXED, coarse_cluster=True),
                       budget_bytes=int(0.5 * free), max_slots=cap or n)
        r = srv.run(mk())
        runs[cap or n] = {k: r[k] for k in keys} | {"peak_slots": r["peak_slots"],
                                                   "throughput_ratio": r["dof_timesteps_per_s"] / max(seq["dof_timesteps_per_s"], 1e-30)}
    bat = runs[slots[0] or n]
    return {
        "sample": f"{n} requests of the seeded serving stream (Poisson {rate:g}/s; Nx {min(nx)}-{max(nx)}, "
                  f"Ny {min(ny)}-{max(ny)}, Nz {min(nz)}-{max(nz)}; {steps[0]}-{steps[1]} steps each instead of "
                  f"100-2000, {note})",
        "batched_mixed": bat,
        "sequential_fp64": {k: seq[k] for k in keys},
        "throughput_ratio": bat["throughput_ratio"],
        **({"batched_mixed_by_slot_cap": runs} if len(slots) > 1 else {}),
    }


def cpu_baseline(threads, warmup=1, steps=None, budget_s=15.0, max_steps=8):
    """The reference-ordered oracle (lexicographic Gauss-Seidel multigrid,
    left-preconditioned GMRES) on `threads` host threads, on a bounded
    sample of the workload: one instance on the CPU_SAMPLE sub-basin of the
    same sea, `warmup` untimed steps, then consecutive RK4 steps timed
    together -- `steps` of them, or as many as fit in budget_s (at most
    max_steps). Returns DOF-timesteps/s, seconds, steps timed, params."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    pkg = package()
    W = pkg.workloads
    O.set_threads(threads)
    p, geo, E0, P0 = W.irregular_sea(**CPU_SAMPLE, precision=0, seed=1234)
    orc = O.Oracle(p, **geo, mode=O.MODE_REFERENCE)
    orc.set_state(E0, P0)
    if warmup > 0:
        orc.step(warmup)
    n = 0
    t0 = time.perf_counter()
    while True:
        orc.step(1)
        n += 1
        dt = time.perf_counter() - t0
        if (steps and n >= steps) or (not steps and (dt >= budget_s or n >= max_steps)):
            break
    s = orc.stats()
    return dof(p) * n / dt, dt, n, p, s["total_iterations"] / max(s["solves"], 1)


def profile_step(args):
    """One warm-up step and one step of the workload, for ncu launch lists and
    captures (prints the step time; the numbers are not bench values)."""
    pkg = package()
    kw = dict(WORKLOAD)
    if args.grid:
        kw = dict(zip(("Nx", "Ny", "Nz"), (int(v) for v in args.grid.lower().split("x"))))
    prec = 1 if args.profile == "mixed" else 0
    kr = 1 if args.krylov == "left" else 0
    def graphs_off(sim):
        if args.no_graphs:
            pkg.lib().ow3d_set_graphs(sim.h, 0)
        if args.smoother == "lexicographic":
            sim.set_smoother_order(pkg.capi.SMOOTHER_LEXICOGRAPHIC)
    if args.profile_workload == "flume":
        # the 2-D stream-function flume (257 x 9, generation and sponge zones)
        p, geo, E0, P0, targets = pkg.workloads.stream_function_2d(ppw=32, steps=4, precision=prec, krylov=kr)
        sim = pkg.Simulation(p, **geo)
        graphs_off(sim)
        sim.set_state(E0, P0)
        sim.set_relax_target(0, *targets[0])
    elif args.profile_workload == "shoal":
        # sloping bottom: multigrid levels with mixed-derivative terms, the
        # generation zone and the sponge
        sys.path.insert(0, str(ROOT / "tests"))
        import cases
        gkw = dict(zip(("Nx", "Ny", "Nz"), (int(v) for v in args.grid.lower().split("x")))) if args.grid else {}
        p, geo, target = cases.shoal_generation(pkg.workloads, 4, precision=prec, krylov=kr, **gkw)
        sim = pkg.Simulation(p, **geo)
        graphs_off(sim)
        sim.set_relax_target(0, *target(sim.zone_box(0)))
        Nxg, Nyg, _ = pkg.dims(p)
        x, y = pkg.workloads.grid_xy(p)
        E0 = np.tile(0.004 * np.cos(2 * np.pi * x / 1.56), Nyg)
        sim.set_state(E0, np.zeros_like(E0))
    else:
        p, geo, E0, P0 = pkg.workloads.irregular_sea(**kw, precision=prec)
        p.krylov = kr
        sim = pkg.Simulation(p, **geo)
        graphs_off(sim)
        sim.set_state(E0, P0)
    sim.step(1)
    # the profiled range (ncu --profile-from-start off): the second step only,
    # without the set-up's launches
    import torch
    torch.cuda.init()
    torch.cuda.cudart().cudaProfilerStart()
    st, ms = sim.step_timed(1)
    torch.cuda.cudart().cudaProfilerStop()
    s = sim.stats()
    print(f"profile {args.profile} {p.Nx}x{p.Ny}x{p.Nz}: step {ms:.2f} ms, solves {s['solves']}, "
          f"iterations {s['total_iterations']}")
    sim.close()


def largest_instance(args):
    """--config largest: one JSON line per tolerance (largest_sweep)."""
    for line in largest_sweep(args.steps, args.warmup):
        print(json.dumps(line))


def largest_sweep(steps, warmup):
    """The largest single instance, 2049 x 513 x 9 (flat 1 m, seeded JONSWAP
    sea): FP64 and mixed precision at GMRES rtol 1e-6, 1e-8 and 1e-10 with
    abstol 0 (so that the relative term alone sets each threshold), one
    record per tolerance with both precisions' DOF-timesteps/s, iterations
    per solve and the mixed path's eta error against FP64. Timed like the
    main line (device events around the steps, after warm-up steps)."""
    import torch
    pkg = package()
    W = pkg.workloads
    torch.cuda.set_device(0)
    out = []
    for rtol in (1e-6, 1e-8, 1e-10):
        res, states = {}, {}
        for prec in ("fp64", "mixed"):
            p, geo, E0, P0 = W.irregular_sea(Nx=2049, Ny=513, Nz=9, precision=(1 if prec == "mixed" else 0),
                                             reltol=rtol, abstol=0.0, seed=1234)
            sim = pkg.Simulation(p, **geo)
            sim.set_state(E0, P0)
            sim.step(warmup)
            sim.reset_stats()
            torch.cuda.synchronize()
            st, ms = sim.step_timed(steps)
            s = sim.stats()
            E, P, Wv, phi, t = sim.get_state()
            states[prec] = E
            res[prec] = dict(value=dof(p) * steps / (ms / 1e3), ms_per_step=ms / steps,
                             iterations_per_solve=s["total_iterations"] / max(s["solves"], 1),
                             **solver_report(s, p))
            sim.close()
        err = float(np.max(np.abs(states["mixed"] - states["fp64"])) / np.max(np.abs(states["fp64"])))
        out.append({"config": "largest instance 2049x513x9, flat 1 m, JONSWAP, GMRES(23) abstol 0", "rtol": rtol,
                    "unit": UNIT, "steps": steps, "warmup": warmup, "fp64": res["fp64"],
                    "mixed": res["mixed"], "speedup_mixed_vs_fp64": res["mixed"]["value"] / res["fp64"]["value"],
                    "eta_rel_err_mixed_vs_fp64": err})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop sample")
    ap.add_argument("--no-largest", action="store_true",
                    help="skip the largest-instance sweep (2049x513x9 at three tolerances, 3 timed steps each)")
    ap.add_argument("--profile", choices=["fp64", "mixed"], default=None,
                    help="profiling driver: one warm-up step then one step of the workload, no JSON line")
    ap.add_argument("--grid", default=None, help="NXxNYxNZ override for --profile (e.g. 257x65x17)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="--profile: launch every kernel directly (no CUDA graphs), for per-launch profiling")
    ap.add_argument("--profile-workload", choices=["sea", "shoal", "flume"], default="sea",
                    help="--profile workload: the irregular sea, the 257x33x9 shoal basin (sloping bottom), "
                         "or the 257x9 stream-function flume")
    ap.add_argument("--krylov", choices=["fgmres", "left"], default="fgmres",
                    help="--profile: flexible GMRES or left-preconditioned GMRES (the reference's)")
    ap.add_argument("--smoother", choices=["multicolour", "lexicographic"], default="multicolour",
                    help="--profile: smoother row order (lexicographic: the reference's)")
    ap.add_argument("--config", choices=["sea", "largest", "serving"], default="sea",
                    help="largest: the 2049x513x9 instance at three GMRES tolerances (one JSON line each); "
                         "serving: the serving stream with the configuration's size sets (one JSON line)")
    ap.add_argument("--requests", type=int, default=48, help="--config serving: number of requests")
    ap.add_argument("--slots", default=None, help="--config serving: comma-separated slot caps (default: no cap)")
    args = ap.parse_args()
    if args.profile:
        profile_step(args)
        return
    if args.config == "largest":
        largest_instance(args)
        return
    if args.config == "serving":
        # the serving stream with the configuration's size sets (Nx 65-1025,
        # Ny 1-257, Nz 9-17), step counts scaled down 10x to bound the run
        import torch
        torch.cuda.set_device(0)
        S = package().serving
        caps = tuple(int(c) for c in args.slots.split(",")) if args.slots else (None,)
        out = serving_sample(n=args.requests, seed=2024, rate=4.0, nx=S.NX_SET, ny=S.NY_SET, nz=S.NZ_SET,
                             steps=(10, 200), note="the configuration's size sets, step counts scaled down 10x",
                             slots=caps)
        print(json.dumps({"config": "serving stream", "unit": UNIT, **out}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        nthreads = os.cpu_count() or 1
        v, dt, n, p, it = cpu_baseline(nthreads, warmup=args.warmup, steps=max(args.steps, 1))
        sample = (f"{p.Nx}x{p.Ny}x{p.Nz} sub-basin of the irregular-sea workload (same dx, Nz, spectrum): "
                  f"{args.warmup} warm-up steps, then {n} consecutive RK4 steps of one instance timed together "
                  f"({dt:.1f} s, {it:.1f} matvecs per solve), reference-ordered oracle (lexicographic "
                  f"Gauss-Seidel, left GMRES), {nthreads} OpenMP threads")
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / n * 1e3, "higher_is_better": True,
            "config": {"workload": "irregular sea 1025x257x17 (sampled on host)", "sample": sample},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "dtype": "f64", "data": "synthetic (seeded JONSWAP sea)"}))
        return
    if world > 1:
        import torch
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    res, e2e_s, err_eta, err_phi, pm = run_gpu(args, rank, world)
    if rank != 0:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
        return
    pkg = package()
    D = dof(pm)
    ms_mixed, ms_fp64 = res["mixed"]["ms"], res["fp64"]["ms"]
    v_mixed = job_throughput(D, args.steps, world, ms_mixed)
    v_fp64 = job_throughput(D, args.steps, world, ms_fp64)
    peak, peak_kind = peaks()
    roof = None
    kr, ncolor = kernel_roofline(pkg, pm, int(os.environ.get("LOCAL_RANK", "0")))
    roof_op = None
    if "colour" in kr:
        kms, alg = kr["colour"]
        ach = alg / (kms / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": "k_lo_colour (one colour pass of the finest multigrid level, FP64)",
                "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "traffic": profiled_traffic("k_lo_colour"), "peak_kind": peak_kind, "alg_bytes_per_launch": alg,
                "alg_bytes_rule": f"(3*8*N + 5*8*C) / {ncolor} colours: one sweep's bytes per colour pass",
                "ms_per_launch": kms}
    if "operator" in kr:
        kms, alg = kr["operator"]
        ach = alg / (kms / 1e3) / 1e9
        roof_op = {"bound": "hbm", "kernel": "k_ho_matvec (6th-order sigma operator, FP64)", "achieved": ach,
                   "peak": peak, "unit": "GB/s", "frac": ach / peak, "traffic": profiled_traffic("k_ho_matvec"),
                   "peak_kind": peak_kind, "alg_bytes_per_launch": alg, "ms_per_launch": kms}
    path_roof = {"peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                 "per_unit": "operator 2*8*N+10*8*C; GS sweep 3sN_l+5sC_l; residual+restriction 2sN_l+sN_(l-1); "
                             "prolongation sN_(l-1)+2sN_l; Arnoldi step j (2j+3)*8N+sN; update (ks+16)N; "
                             "free surface 30*8*C",
                 **res["fp64"]["path_info"]}
    for prec in ("fp64", "mixed"):
        b = res[prec]["path_bytes"]
        ach = b / (res[prec]["ms"] / args.steps / 1e3) / 1e9
        path_roof[prec] = {"alg_bytes_per_step": b, "achieved": ach, "frac": ach / peak}
    cpu = None
    if not args.no_cpu:
        nthreads = os.cpu_count() or 1
        v, dt, n, p, it = cpu_baseline(nthreads)
        cpu = {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": f"{p.Nx}x{p.Ny}x{p.Nz} sub-basin of the same workload: 1 warm-up step, then {n} consecutive "
                         f"RK4 steps of one instance ({dt:.1f} s, {it:.1f} matvecs per solve), reference-ordered "
                         f"oracle (lexicographic Gauss-Seidel, left GMRES), {nthreads} OpenMP threads"}
        v1, dt1, n1, _, it1 = cpu_baseline(1, budget_s=15.0, max_steps=4)
        cpu["serial"] = {"value": v1, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": f"same sub-basin, 1 warm-up step, then {n1} consecutive RK4 steps on one thread "
                                   f"({dt1:.1f} s): the like-for-like figure of the serial Fortran reference"}
    serve = None
    if not args.no_serve and world == 1:
        serve = serving_sample(slots=(4, None))
    largest = None
    if not args.no_largest and world == 1:
        largest = largest_sweep(3, 3)
    C = (pm.Nx + 2) * (pm.Ny + 2)
    sm = res["mixed"]["stats"]; sf = res["fp64"]["stats"]
    out = {
        "metric": METRIC, "value": v_mixed, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (FP32 multigrid)", "data": "synthetic (seeded JONSWAP sea)",
        "config": {"workload": "irregular sea 1025x257x17, flat 1 m, JONSWAP Hs=0.05 Tp=1.5 gamma=3.3, "
                               "GMRES(23) reltol 1e-8 abstol 1e-6 (the example decks' solver line), Courant 0.5",
                   "DOF": D, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (phi 38 MB + Krylov basis ~1.8 GB per replica)"},
        "fp64": {"value": v_fp64, "ms_per_step": ms_fp64 / args.steps,
                 "avg_iterations": sf["total_iterations"] / max(sf["solves"], 1), **solver_report(sf, pm)},
        "mixed": {"value": v_mixed, "ms_per_step": ms_mixed / args.steps,
                  "avg_iterations": sm["total_iterations"] / max(sm["solves"], 1),
                  "eta_rel_err_vs_fp64": err_eta, "phi_rel_err_vs_fp64": err_phi, **solver_report(sm, pm)},
        "speedup_mixed_vs_fp64": v_mixed / v_fp64,
        "left_gmres": left_report(res["left"], D, args.steps, world, pm),
        "laplace_solves_per_s": sm["solves"] * world / (ms_mixed / 1e3),
        "e2e": {"value": job_throughput(D, args.steps, world, e2e_s * 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 2 * 8 * C, "d2h_bytes_per_step": 3 * 8 * C,
                "path": "mixed precision; per step ow3d_put_surface (E, P from pinned host memory), ow3d_step, "
                        "ow3d_get_state (E, P, W to pinned host memory); host wall clock around the steps",
                "avg_iterations": res["e2e_stats"]["total_iterations"] / max(res["e2e_stats"]["solves"], 1),
                "not_converged": res["e2e_stats"]["not_converged"]},
        "roofline": roof, "roofline_operator": roof_op, "roofline_path": path_roof, "cpu_baseline": cpu, "clocks": res["mixed"]["clocks"], "serving": serve,
        "largest_instance": largest,
        "gpu_launches": res["mixed"]["launches"],
    }
    print(json.dumps(out))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
