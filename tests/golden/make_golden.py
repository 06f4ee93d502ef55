"""Generate the golden vectors in this folder from the CPU oracle.

    python tests/golden/make_golden.py             # the fast set
    python tests/golden/make_golden.py --fullrun   # also the whole runs (run_*)

The reference has no Fortran compiler or SPARSKIT2/HSL libraries here and no
stored outputs of its own, so these vectors come from the oracle (the CPU
restatement of the reference algorithm), except host_*, which the library's
own host set-up computes (incident waves), to keep those fixed across builds. They pin the oracle and the CUDA path
against drift: test_golden.py re-runs the oracle on the same seeded inputs and
the GPU parity tests compare the device against the same files.
Each case is stored as <name>.npz; MANIFEST.txt lists their SHA-256.
"""
import hashlib
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "oracle"))


def cases_table():
    import cases
    return {
        "bump3d_17x9x9": (cases.bump_3d, dict(Nx=17, Ny=9, Nz=9)),
        "bump3d_33x17x9": (cases.bump_3d, dict(Nx=33, Ny=17, Nz=9)),
        "slope2d_33x9": (cases.slope_2d, dict(Nx=33, Nz=9)),
    }


def operator_case(oracle, case, kw, mode):
    """matvec, one preconditioner application and one solve on seeded inputs."""
    import cases
    p, geo = case(**kw)
    o = oracle.Oracle(p, **geo, mode=mode)
    surf = cases.surface(p, amp=0.03, seed=11)
    o.set_surface(*surf)
    phi = cases.field3(p, seed=1)
    r = cases.field3(p, seed=7)
    rhs = cases.fs_rhs(p, np.cos(np.linspace(0, 2 * np.pi, o.C)))
    sol, it, res, st = o.solve(rhs, np.zeros(o.N))
    return dict(surface=np.stack(surf), phi=phi, r=r, rhs=rhs, matvec=o.matvec(phi), precond=o.precond(r),
                solve=sol, iterations=np.array([it]), status=np.array([st]))


def standing_case(oracle, mode, nonlinear):
    """Ten RK4 steps of a 2-D standing wave."""
    import cases
    p, geo = cases.flat_2d(Nx=33, Nz=9, L=2.0, LinearONOFF=nonlinear, dt=0.02)
    o = oracle.Oracle(p, **geo, mode=mode)
    x = (np.arange(o.Nxg) - 1) / (p.Nx - 1) * p.Lx
    E0 = 0.02 * np.cos(np.pi * x / p.Lx)
    o.set_state(E0, np.zeros(o.Nxg))
    o.step(10)
    E, P, W, phi, t = o.get_state()
    s = o.stats()
    return dict(E0=E0, E=E, P=P, W=W, phi=phi, t=np.array([t]), iterations=np.array([s["total_iterations"]]))


def host_setup_cases():
    """Host set-up computed by the library itself (no device, no oracle): the
    stream-function wave of the first configuration (kh = 1, half the
    breaking steepness) and the first samples of a JONSWAP incident wave with
    the reference's random phases, so that these stay fixed across builds."""
    from conftest import load_package
    ow3d = load_package()
    out = {}
    p = ow3d.default_params(Nx=65, Nz=9, Lx=2 * np.pi, Ly=1.0, Lz=1.0)
    p.g = 9.81
    p.sf_H, p.sf_h, p.sf_L = 0.5 * 0.142 * np.tanh(1.0) * 2 * np.pi, 1.0, 2 * np.pi
    p.sf_wavel_or_per, p.sf_nsteps, p.sf_nmodes = 0, 6, 24
    x = np.linspace(0.0, 2 * np.pi, 33)
    eta, phis, info = ow3d.stream_function_wave(p, x, 0.25)
    out["host_stream_function_kh1"] = dict(x=x, eta=eta, phis=phis, info=np.array(info))
    q = ow3d.default_params(Nx=129, Ny=1, Nz=9, Lx=20.0, Ly=1.0, Lz=1.0, relaxONOFF=1, relaxNo=1,
                            zones=[dict(x1=0.0, x2=4.0, ftype=10, param=3.5, wavegen=1)])
    q.IncWaveType, q.ispec, q.Tp, q.Hs, q.h0, q.kh_max, q.seed, q.seed2 = 2, 1, 1.25, 0.04, 0.8, 20.0, -4, -34
    q.Nsteps, q.dt, q.g = 256, 0.02, 9.81
    e, f, box = ow3d.incident_wave(q, 0)
    out["host_jonswap_zone"] = dict(eta=e[:64, 0, ::8], phis=f[:64, 0, ::8], box=np.array(box))
    return out


def fullrun_cases():
    """Whole runs of the benchmark configurations the oracle can finish here
    in minutes (too slow to regenerate inside the test suite): the final
    state and the matvec count of every step, in the device ordering (_dev)
    and the reference ordering (_ref).

      run_shoal_257x33x9_1000   the shoal basin with its generation zone and
                                sponge, 1000 RK4 steps (reltol 1e-8, abstol 1e-6)
      run_sfwave_257x9_200      the 2-D stream-function wave (kh = 1, half the
                                breaking steepness) in the wall-bounded flume
                                with generation and sponge, 200 RK4 steps
    """
    import cases
    import oracle
    from conftest import load_package
    W = load_package().workloads
    out = {}
    for mode, tag in ((oracle.MODE_DEVICE, "dev"), (oracle.MODE_REFERENCE, "ref")):
        p, geo, target = cases.shoal_generation(W, 1000)
        o = oracle.Oracle(p, **geo, mode=mode)
        o.set_relax_target(0, *target(o.zone_box(0)))
        o.set_state(np.zeros(o.C), np.zeros(o.C))
        its = cases.run_steps(o, 1000)
        out[f"run_shoal_257x33x9_1000_{tag}"] = _final(o, its)
        p, geo, E0, P0, targets = W.stream_function_2d(ppw=32, steps=200)
        o = oracle.Oracle(p, **geo, mode=mode)
        o.set_state(E0, P0)
        o.set_relax_target(0, *targets[0])
        its = cases.run_steps(o, 200)
        out[f"run_sfwave_257x9_200_{tag}"] = _final(o, its)
    return out


def _final(o, its):
    E, P, W, phi, t = o.get_state()
    return dict(E=E, P=P, W=W, phi=phi, t=np.array([t]), step_iterations=its)


def is_fullrun(name):
    return name.startswith("run_")


def generate():
    import oracle
    out = host_setup_cases()
    for name, (case, kw) in cases_table().items():
        for mode, tag in ((oracle.MODE_REFERENCE, "ref"), (oracle.MODE_DEVICE, "dev")):
            out[f"op_{name}_{tag}"] = operator_case(oracle, case, kw, mode)
    for mode, tag in ((oracle.MODE_REFERENCE, "ref"), (oracle.MODE_DEVICE, "dev")):
        for nl in (0, 1):
            out[f"rk4_standing2d_{'nl' if nl else 'lin'}_{tag}"] = standing_case(oracle, mode, nl)
    return out


def main():
    from conftest import load_package
    load_package()
    sets = generate()
    if "--fullrun" in sys.argv:
        sets.update(fullrun_cases())
    lines = []
    # whole-run fixtures not regenerated this time keep their entries
    for f in sorted(HERE.glob("run_*.npz")):
        if f.stem not in sets:
            lines.append(f"{hashlib.sha256(f.read_bytes()).hexdigest()}  {f.name}")
    for name, arrs in sorted(sets.items()):
        f = HERE / f"{name}.npz"
        if f.exists():
            # keep a fixture whose content is unchanged up to reduction-order rounding
            with np.load(f) as old:
                same = sorted(old.files) == sorted(arrs) and all(
                    old[k].shape == np.shape(v) and np.allclose(old[k], v, rtol=1e-12, atol=1e-14 * max(1.0, np.max(np.abs(v))))
                    for k, v in arrs.items())
            if same:
                lines.append(f"{hashlib.sha256(f.read_bytes()).hexdigest()}  {f.name}")
                continue
        np.savez_compressed(f, **arrs)
        lines.append(f"{hashlib.sha256(f.read_bytes()).hexdigest()}  {f.name}")
    lines.sort(key=lambda ln: ln.split()[1])
    (HERE / "MANIFEST.txt").write_text("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
