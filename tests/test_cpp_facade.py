"""The C++ host side: the FRSolver facade (include/zhijian_b200/fr_solver.hpp)
compiles against the C-ABI, and its driver (zhijian_b200/cpp/zj_run.cpp) runs
the reference's time loop on a GPU with the same result as the Python binding."""
import os
import subprocess

import numpy as np
import pytest

from zhijian_b200 import build

CONFIG = """gamma 1.4
rho_inf 1.225
p_inf 141855.0
Mach 0.5
AoA 0.0
poly_order 3
CFL 0.5
dt 1e-6
bc 1 farfield
"""


def test_driver_builds(zjlib):
    exe = build.build_driver()
    assert os.access(exe, os.X_OK)


@pytest.mark.gpu
def test_driver_matches_python_binding(zjlib, tmp_path):
    import math
    from zhijian_b200 import meshgen as M
    from zhijian_b200.solver import FRSolver, make_params
    exe = build.build_driver()
    cfg = tmp_path / "c.txt"
    cfg.write_text(CONFIG)
    out = subprocess.run([exe, str(cfg), "8", "8", "-5", "5", "-5", "5", "5", "vortex"],
                         capture_output=True, text=True, check=True).stdout.splitlines()
    chk = float(out[-1].split()[1])
    res_cpp = float(out[-2].split()[3])
    mesh = M.structured_quads(8, 8, -5.0, 5.0, -5.0, 5.0, 0.0, 0, (1, 1, 1, 1), {1: "farfield"})
    prm = make_params(poly_order=3, rho_inf=1.225, p_inf=141855.0, Mach=0.5, bcs=[(1, "farfield")])
    s = FRSolver(mesh, prm)
    g = 1.4
    c = math.sqrt(g * 141855.0 / 1.225)
    s.setInitialCondition(lambda xy: M.isentropic_vortex(
        xy, g, u_inf=0.5, rho_scale=1.225, p_scale=141855.0 * g))
    s.advance(1e-6, 5)
    U = s.copyToHost()
    assert abs(np.abs(U).sum() - chk) <= 1e-12 * chk
    assert abs(s.computeResidual() - res_cpp) <= 1e-9 * res_cpp


@pytest.mark.gpu
def test_driver_restart_resumes(zjlib, tmp_path):
    """20 steps in one run equal 12 steps, a restart file, and 8 more steps
    resumed from it (state, time and iteration)."""
    exe = build.build_driver()
    cfg = tmp_path / "c.txt"
    cfg.write_text(CONFIG + "restart_freq 1000\n")
    args = [exe, str(cfg), "8", "8", "-5", "5", "-5", "5"]
    full = subprocess.run(args + ["20", "vortex"], capture_output=True, text=True, check=True).stdout
    rst = tmp_path / "state.zjr"
    subprocess.run(args + ["12", "vortex", "-w", str(rst)], capture_output=True, text=True, check=True)
    resumed = subprocess.run(args + ["20", "vortex", "-r", str(rst)], capture_output=True, text=True,
                             check=True).stdout
    assert full.splitlines()[-1] == resumed.splitlines()[-1]          # bit-identical checksum
    assert full.splitlines()[-2].split()[:2] == resumed.splitlines()[-2].split()[:2]   # iteration, time


@pytest.mark.gpu
def test_driver_reads_gmsh_mesh(zjlib, tmp_path):
    """zj_run -m <file.msh>: the mesh from a Gmsh file (triangles and quads, in
    physics mode), the same steps and state as the Python binding's
    FRSolver.from_gmsh with the same parameters."""
    from zhijian_b200.solver import FRSolver, make_params
    exe = build.build_driver()
    msh = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gmsh", "triquad_v41.msh")
    cfg = tmp_path / "c.txt"
    cfg.write_text("gamma 1.4\nrho_inf 1.2\np_inf 100000.0\nMach 0.3\nAoA 5.0\npoly_order 3\n"
                   "flux_type SD\nriemann Roe\ncompat off\nviscous true\nRe 200\nPr 0.72\ndt 1e-6\n")
    out = subprocess.run([exe, str(cfg), "-m", msh, "4"], capture_output=True, text=True,
                         check=True).stdout.splitlines()
    chk = float(out[-1].split()[1])
    prm = make_params(poly_order=3, rho_inf=1.2, p_inf=1.0e5, Mach=0.3, AoA=5.0, flux_type="SD",
                      riemann="Roe", compat=False, viscous=True, Re=200.0, Pr=0.72)
    s = FRSolver.from_gmsh(msh, prm)
    s.setInitialCondition(lambda xy: _uniform(xy, 1.2, 1.0e5, 0.3, 5.0))
    s.advance(1e-6, 4)
    U = s.copyToHost()
    assert abs(np.abs(U).sum() - chk) <= 1e-12 * chk


def _uniform(xy, rho, p, mach, aoa, g=1.4):
    import math
    from zhijian_b200 import meshgen as M
    c = math.sqrt(g * p / rho)
    u, v = mach * c * math.cos(math.radians(aoa)), mach * c * math.sin(math.radians(aoa))
    shp = xy.shape[:-1]
    return M.prim_to_cons(np.full(shp, rho), np.full(shp, u), np.full(shp, v), np.full(shp, p), g)
