"""Generate the golden vectors in this folder from the CPU oracle.

    python tests/golden/make_golden.py

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
    lines = []
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
    (HERE / "MANIFEST.txt").write_text("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
