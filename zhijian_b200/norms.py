"""Error norms of a state or residual against a reference, per conserved
variable (rho, rho u, rho v, rho E): the figures the mixed-precision form
reports against the FP64 path and the FP64 oracle."""
from __future__ import annotations

import numpy as np

VARS = ("rho", "rhou", "rhov", "rhoE")


def state_errors(U, Uref):
    """{'l2': [...], 'linf': [...], 'l2_abs': [...], 'linf_abs': [...]} over all
    solution points: l2 = ||U - Uref||_2 / ||Uref||_2 and
    linf = max|U - Uref| / max|Uref| per variable (discrete norms over the
    points), and the same without the normalisation."""
    U = np.asarray(U, dtype=np.float64).reshape(-1, 4)
    R = np.asarray(Uref, dtype=np.float64).reshape(-1, 4)
    d = U - R
    l2a = np.sqrt(np.mean(d * d, axis=0))
    lia = np.abs(d).max(axis=0)
    l2r = np.sqrt(np.sum(d * d, axis=0)) / np.maximum(np.sqrt(np.sum(R * R, axis=0)), 1e-300)
    lir = lia / np.maximum(np.abs(R).max(axis=0), 1e-300)
    return {"l2": [float(x) for x in l2r], "linf": [float(x) for x in lir],
            "l2_abs": [float(x) for x in l2a], "linf_abs": [float(x) for x in lia]}
