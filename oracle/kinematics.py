"""ORACLE -- test infrastructure only.

CPU restatement of the fluid kinematics that the reference writes to its
Kinematics files (src/IO/StoreKinematicData.f90:256-460), in numpy, from an
oracle state: the checker of ow3d_kinematics. The product path never calls it.

Every derivative is the reference's 7-point one with per-position stencils:
DiffXEven (src/functions/DiffXEven.f90:15-38), DiffYEven (the same along y)
and DiffZArbitrary (src/functions/DiffZArbitrary.f90:15-34), with windows
1..7 at the first three positions, i-3..i+3 inside and n-6..n at the last
three. The chain-rule terms use the sigma levels with the ghost level
z(1) = -z(3) (SetupCompDomain.f90:75-79) and d = h + eta at every point.
"""
import numpy as np


def _windows(n):
    """Start (0-based) of the 7-point window at each position of n."""
    i = np.arange(1, n + 1)
    s = np.where(i <= 3, 1, np.where(i <= n - 3, i - 3, n - 6))
    return s - 1


def diff(F, S, axis):
    """Order-1 7-point derivative of F (Nyg, Nxg, Nzg) along `axis` with the
    per-position stencil table S (n, 7)."""
    n = F.shape[axis]
    out = np.zeros_like(F)
    ws = _windows(n)
    Fm = np.moveaxis(F, axis, 0)
    Om = np.moveaxis(out, axis, 0)
    for pos in range(n):
        acc = np.zeros_like(Fm[0])
        for m in range(7):
            acc = acc + S[pos, m] * Fm[ws[pos] + m]
        Om[pos] = acc
    return out


def kinematics(E, Ex, Ey, phi, h, hx, hy, SX, SY, SZ, z, Nxg, Nyg, Nzg, nonlinear):
    """u, v, w and the nine gradient fields (StoreKinematicData.f90:256-460)
    as flat arrays in the device layout (k fastest, then i, then j).
    SX, SY, SZ: order-1 stencils (n, 7); E, Ex, Ey, h, hx, hy: Nxg*Nyg."""
    F = phi.reshape(Nyg, Nxg, Nzg)
    d = (h + E).reshape(Nyg, Nxg, 1)
    zz = z.reshape(1, 1, Nzg)
    three = Nyg > 1
    if nonlinear:
        sx = (1.0 - zz) / d * hx.reshape(Nyg, Nxg, 1) - zz / d * Ex.reshape(Nyg, Nxg, 1)
        sy = ((1.0 - zz) / d * hy.reshape(Nyg, Nxg, 1) - zz / d * Ey.reshape(Nyg, Nxg, 1)) if three else 0.0
    else:
        sx = sy = 0.0

    def grad(G):
        gs = diff(G, SZ, 2)
        gx = diff(G, SX, 1) + sx * gs
        gy = diff(G, SY, 0) + sy * gs if three else np.zeros_like(G)
        return gs, gx, gy

    ps, u, v = grad(F)
    if not three:
        v = np.zeros_like(F)
    w = ps / d
    out = [u, v, w]
    grads = []
    for G in (ps, u, v):
        gs, gx, gy = grad(G)
        grads += [gs / d, gx, gy]
    return [a.ravel() for a in out], np.stack([g.ravel() for g in grads])


def from_oracle(orc):
    """kinematics() of an oracle simulation's current state (the chain-rule
    terms when the deck's LinearONOFF is nonzero)."""
    E, P, W, phi, t = orc.get_state()
    Ex, Exx, Px, Ey, Eyy, Py = orc.get_derivs()
    SX, SY, SZ = orc.stencils()
    h, hx, hxx, hy, hyy = orc._keep
    return kinematics(E, Ex, Ey, phi, h, hx, hy, SX[0], SY[0], SZ[0], orc.fine_z(),
                      orc.Nxg, orc.Nyg, orc.Nzg, orc.params.LinearONOFF != 0)
