"""A few SSP-RK3 steps of the benchmark's cases, for external profilers (ncu)
that capture a handful of launches:

    python profile_case.py {ns|ns32|ns_split|euler|euler32|compat|shear|shear32} [steps] [n] [P]

ns / ns32 / ns_split: Navier-Stokes (Re 5000, Pr 0.72, Roe, HU), FP64 / precision
form / split-BF16 form (tensor-core operator products at P4, P5);
euler / euler32: the inviscid physics-mode residual; compat: the reference
residual semantics.  256x256 jittered Q1 quads on [0,pi]^2 (seed 1), P3,
slip walls, dt = 2e-4 (n overrides the mesh size, P the order; above P3 dt = 3e-5).
shear / shear32: the mixed-element shear layer (n x n quads, default 384, a
seeded 30% split into triangles; Navier-Stokes Re 2000, HLLC, GA, P3) at
CFL 0.1, FP64 / precision form."""
from __future__ import annotations

import math
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from zhijian_b200 import meshgen as M  # noqa: E402
from zhijian_b200.solver import FRSolver, make_params  # noqa: E402

GAMMA, MACH = 1.4, 0.3
MODES = {
    "ns": dict(compat=False, viscous=True, riemann="Roe", flux_type="HU", Re=5000.0, Pr=0.72),
    "ns32": dict(compat=False, viscous=True, riemann="Roe", flux_type="HU", Re=5000.0, Pr=0.72,
                 precision="mixed"),
    "ns_split": dict(compat=False, viscous=True, riemann="Roe", flux_type="HU", Re=5000.0, Pr=0.72,
                     precision="split_bf16"),
    "euler": dict(compat=False, viscous=False, riemann="Roe", flux_type="HU"),
    "euler32": dict(compat=False, viscous=False, riemann="Roe", flux_type="HU", precision="mixed"),
    "compat": dict(compat=True, viscous=False, riemann="Rusanov", flux_type="HU"),
}


def shear(mode, steps, n):
    mesh = M.shear_layer_mesh(n)
    prm = make_params(poly_order=3, flux_type="GA", CFL=0.1,
                      precision="mixed" if mode == "shear32" else "fp64", **M.SHEAR_LAYER_PARAMS)
    s = FRSolver(mesh, prm)
    s.setInitialCondition(M.shear_layer)
    s.advance(s.computeTimeStep(), steps)
    s.check_state()
    print(f"{mode}: {steps} steps on {mesh.n_elem} elements, residual norm {s.computeResidual():.6e}")
    return 0 if math.isfinite(s.computeResidual()) else 1


def main(argv):
    mode = argv[1] if len(argv) > 1 else "ns"
    steps = int(argv[2]) if len(argv) > 2 else 4
    if mode in ("shear", "shear32"):
        return shear(mode, steps, int(argv[3]) if len(argv) > 3 else 384)
    n = int(argv[3]) if len(argv) > 3 else 256
    order = int(argv[4]) if len(argv) > 4 else 3
    mesh = M.tgv_mesh(n, seed=1)
    prm = make_params(poly_order=order, gamma=GAMMA, rho_inf=1.0, p_inf=1.0 / (GAMMA * MACH * MACH),
                      Mach=MACH, bcs=[(1, "slipwall")], **MODES[mode])
    s = FRSolver(mesh, prm)
    s.copyToDevice(M.taylor_green(s.solution_point_coords()))
    s.advance(2.0e-4 if order <= 3 else 3.0e-5, steps)
    s.check_state()
    print(f"{mode}: {steps} steps on {mesh.n_elem} elements, residual norm {s.computeResidual():.6e}")
    return 0 if math.isfinite(s.computeResidual()) else 1


if __name__ == "__main__":
    sys.exit(main(sys.argv))
