"""Generate the golden vectors in this folder from the CPU oracle.

    python tests/golden/make_golden.py

The reference has no Fortran compiler or SPARSKIT2/HSL libraries here and no
stored outputs of its own, so these vectors come from the oracle (the CPU
restatement of the reference algorithm). They pin the oracle and the CUDA path
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


def generate():
    import oracle
    out = {}
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
