"""Shared helpers of the test suite (parity metric, case builders)."""
import numpy as np

GAMMA = 1.4


def euler_flux_scale(U, Jinv=None, gamma=GAMMA):
    """s_F = max|F| * max|metric|: the scale a residual is judged against, so
    near-freestream states (R ~ 0) are not compared against zero."""
    rho = U[..., 0]
    u = U[..., 1] / rho
    v = U[..., 2] / rho
    p = (gamma - 1.0) * (U[..., 3] - 0.5 * rho * (u * u + v * v))
    F = np.stack([U[..., 1], U[..., 1] * u + p, U[..., 1] * v, (U[..., 3] + p) * u,
                  U[..., 2], U[..., 2] * u, U[..., 2] * v + p, (U[..., 3] + p) * v])
    m = 1.0 if Jinv is None else float(np.abs(Jinv).max())
    return float(np.abs(F).max()) * m


def rel_err(R, Rref, scale):
    """Per-variable max |R - Rref| / max(max|Rref_var|, scale)."""
    out = []
    for v in range(4):
        d = float(np.abs(R[..., v] - Rref[..., v]).max())
        out.append(d / max(float(np.abs(Rref[..., v]).max()), scale))
    return max(out)


def metric_scale(mesh, P):
    """Largest metric term of a mesh at order P (through the oracle)."""
    from oracle import oracle as O
    orc = O.Oracle(mesh, P)
    return float(np.abs(orc.geometry()[1]).max())
