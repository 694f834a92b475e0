"""Times the reference's own CUDA build (oracle/_ref/ref_gpu: its kernels.cu
and fr_solver.cpp compiled for sm_100a by oracle/ref/Makefile) against this
library's compat path, which computes the same residual semantics (Rusanov,
inviscid, the reference's correction and clamps), on the benchmark mesh:

    python oracle/ref/time_reference_cuda.py [n] [steps]

256x256 jittered (seed 1) Q1 quads on [0,pi]^2, P3, slip walls, the
Taylor-Green state at M = 0.3, dt = 1e-6 (small enough that the reference
scheme, unstable at larger steps, stays smooth).  Both sides are wall-clock
times of `steps` SSP-RK3 steps after 2 warm-up steps with the device idle at
both ends: the reference's step does host work and copies each stage.  Prints
one JSON line.  Needs a GPU and the built oracle/_ref/ref_gpu (test
infrastructure: nothing here is part of the library)."""
from __future__ import annotations

import json
import math
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from zhijian_b200 import meshgen as M  # noqa: E402
from zhijian_b200.solver import FRSolver, make_params  # noqa: E402

GAMMA, MACH, DT = 1.4, 0.3, 1.0e-6


def main(argv):
    n = int(argv[1]) if len(argv) > 1 else 256
    steps = int(argv[2]) if len(argv) > 2 else 10
    mesh = M.tgv_mesh(n, seed=1)
    p_inf = 1.0 / (GAMMA * MACH * MACH)
    prm = make_params(poly_order=3, gamma=GAMMA, rho_inf=1.0, p_inf=p_inf, Mach=MACH,
                      riemann="Rusanov", flux_type="HU", compat=True, bcs=[(1, "slipwall")])
    s = FRSolver(mesh, prm)
    U = M.taylor_green(s.solution_point_coords(), GAMMA, MACH)
    dof = s.n_elem * s.n_sp

    s.copyToDevice(U)
    s.advance(DT, 2)
    t0 = time.perf_counter()
    s.advance(DT, steps)
    ours_ms = (time.perf_counter() - t0) * 1e3
    s.check_state()
    s.close()

    tmp = tempfile.mkdtemp()
    mb, ub, tb = (os.path.join(tmp, x) for x in ("m.bin", "u.bin", "t.txt"))
    O.write_mesh_bin(mb, mesh, None)
    U.tofile(ub)
    cmd = [O.REF_GPU, "time", mb, "3", repr(GAMMA), "1.0", repr(p_inf), repr(MACH), "0.0", ub,
           repr(DT), "2", str(steps), tb]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        print(r.stdout[-2000:], r.stderr[-2000:], file=sys.stderr)
        return r.returncode
    ns, ref_ms = open(tb).read().split()
    ref_ms = float(ref_ms)
    rate = lambda ms: dof * 3 * steps / (ms * 1e-3)  # noqa: E731
    out = {"workload": f"TGV {n}x{n} jittered Q1 quads, P3, reference residual semantics "
                       f"(Rusanov, inviscid), SSP-RK3, dt {DT}",
           "steps": steps, "dof_per_var": dof, "unit": "DOF-RHS/s",
           "reference_cuda": {"ms_per_step": ref_ms / steps, "value": rate(ref_ms)},
           "ours_compat": {"ms_per_step": ours_ms / steps, "value": rate(ours_ms)},
           "speedup": ref_ms / ours_ms}
    print(json.dumps(out), flush=True)
    return 0 if math.isfinite(out["speedup"]) else 1


if __name__ == "__main__":
    sys.exit(main(sys.argv))
