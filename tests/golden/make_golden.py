"""Generates the golden fixtures of tests/golden/ from the reference's own code.

    python tests/golden/make_golden.py cpu  [--out DIR]   # any host
    python tests/golden/make_golden.py gpu  [--out DIR]   # on a GPU host

"cpu" runs oracle/_ref/ref_cpu (the reference's basis.cpp, mesh.cpp and
gmsh_reader.cpp compiled from the reference sources by oracle/ref/Makefile) and
stores its operators, faces, normals, metric terms, pointwise Riemann fluxes,
ghost states and (ref_viscous.npz) the header's viscous fluxes.  "gpu" runs
oracle/_ref/ref_gpu (the reference's kernels.cu and fr_solver.cpp) and stores
the reference's own residuals and stepped states of case_defs()
(ref_gpu_residuals.npz), the 200-step trajectories of the isentropic-vortex
configuration (ref_trajectory.npz) and the reference kernel's viscous fluxes
(ref_viscous_kernel.npz); --only picks some of those three.
Inputs are seeded (SplitMix64), so every case is regenerated from its recipe.
"""
from __future__ import annotations

import argparse
import math
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from zhijian_b200 import meshgen as M  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
GAMMA = 1.4
# the dimensional twin of the vortex: every reference clamp stays inactive
RHO_S, P_S = 1.225, 101325.0 * 1.4


def mixed_mesh(n=6, seed=7):
    """Jittered n x n quads, one boundary type per side."""
    return M.structured_quads(n, n, 0.0, 1.0, 0.0, 1.0, 0.15, seed, (1, 2, 3, 4),
                              {1: "slipwall", 2: "outflow", 3: "farfield", 4: "wall"})


def mixed_tags(p_out):
    return [(1, O.BC_TYPES["slipwall"], 0.0), (2, O.BC_TYPES["outflow"], p_out),
            (3, O.BC_TYPES["farfield"], 0.0), (4, O.BC_TYPES["wall"], 0.0)]


def case_defs():
    """name -> dict(mesh, tags, P, params(rho,p,Mach,AoA), state, [dt, nsteps])."""
    cases = {}
    vm = M.vortex_mesh(20)
    # raw non-dimensional vortex (the reference clamps fire)
    cases["vortex_raw_p3"] = dict(mesh=vm, tags=None, P=3, prm=(1.0, 1.0 / GAMMA, 0.5, 0.0),
                                  state=("vortex", 1.0, 1.0), dt=0.01, nsteps=3)
    cases["vortex_dim_p3"] = dict(mesh=vm, tags=None, P=3,
                                  prm=(RHO_S, P_S / GAMMA, 0.5, 0.0),
                                  state=("vortex", RHO_S, P_S), dt=1e-6, nsteps=5)
    for P in range(1, 6):
        cases[f"mixed_p{P}"] = dict(mesh=mixed_mesh(), tags=mixed_tags(0.9e5), P=P,
                                    prm=(1.2, 1.0e5, 0.4, 10.0),
                                    state=("random", 1.2, 1.0e5, 11 + P), dt=1e-8, nsteps=3)
    cases["tgv16_p3"] = dict(mesh=M.tgv_mesh(16, seed=1), tags=None, P=3,
                             prm=(1.0, 1.0 / (GAMMA * 0.09), 0.3, 0.0), state=("tgv",),
                             dt=1e-3, nsteps=2)
    return cases


def make_state(c, coords):
    kind = c["state"][0]
    if kind == "vortex":
        return M.isentropic_vortex(coords, GAMMA, rho_scale=c["state"][1], p_scale=c["state"][2])
    if kind == "tgv":
        return M.taylor_green(coords, GAMMA, 0.3)
    _, rho0, p0, seed = c["state"]
    n_elem, nsp = coords.shape[0], coords.shape[1]
    return M.random_state(n_elem, nsp, seed, GAMMA, rho0, p0, 0.1)


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(" ".join(cmd) + "\n" + r.stdout[-2000:] + r.stderr[-2000:])
    return r


# Pointwise physics pins: state pairs covering every branch of the reference's
# Riemann solvers and ghost states (subsonic/supersonic, both wave directions,
# near-vacuum densities).
PHYS_PARAMS = dict(g=1.4, mach=0.5, aoa=10.0, rho_inf=1.2, p_inf=1.0e5, p_total=1.2e5,
                   T_total=300.0, dx=1.0, dy=0.5, p_static=0.9e5, T_wall=350.0)


def phys_samples(n=400, seed=21):
    r = M.uniform01(seed, n * 10).reshape(n, 10)
    g = PHYS_PARAMS["g"]
    out = np.empty((n, 10))
    for k in range(n):
        rho = 1.2 * (0.2 + 1.8 * r[k, :2])
        if k % 37 == 0:
            rho = rho * 1e-9
        p = 1.0e5 * (0.2 + 1.8 * r[k, 2:4])
        c = np.sqrt(g * p / rho)
        mach = 3.0 * (2.0 * r[k, 4:6] - 1.0)          # up to supersonic both ways
        ang = 2.0 * np.pi * r[k, 6:8]
        u = mach * c * np.cos(ang)
        v = mach * c * np.sin(ang)
        UL = M.prim_to_cons(rho[0], u[0], v[0], p[0], g)
        UR = M.prim_to_cons(rho[1], u[1], v[1], p[1], g)
        th = 2.0 * np.pi * r[k, 8]
        out[k] = np.concatenate([UL, UR, [np.cos(th), np.sin(th)]])
    return out


def gen_cpu(out):
    tmp = tempfile.mkdtemp()
    ops = {}
    for P in range(1, 6):
        f = os.path.join(tmp, f"ops{P}.bin")
        run([O.REF_CPU, "ops", str(P), f])
        for k, v in O.read_ops_bin(f, P).items():
            ops[f"P{P}_{k}"] = v
    np.savez_compressed(os.path.join(out, "ref_operators.npz"), **ops)
    tri = {}
    for P in range(1, 6):
        f = os.path.join(tmp, f"tri{P}.bin")
        run([O.REF_CPU, "tri", str(P), f])
        for k, v in O.read_tri_bin(f, P).items():
            tri[f"P{P}_{k}"] = v
    np.savez_compressed(os.path.join(out, "ref_triangle.npz"), **tri)
    geo = {}
    for name, mesh, tags, P in (("mixed", mixed_mesh(), mixed_tags(0.9e5), 3),
                                ("mixed", mixed_mesh(), mixed_tags(0.9e5), 5),
                                ("tgv12", M.tgv_mesh(12, seed=1), None, 3)):
        mb = os.path.join(tmp, "m.bin")
        O.write_mesh_bin(mb, mesh, tags)
        mo = os.path.join(tmp, "mo.bin")
        run([O.REF_CPU, "mesh", mb, str(P), mo])
        faces, J, Ji, sxy, area = O.read_mesh_out(mo, mesh.n_elem, (P + 1) ** 2)
        key = f"{name}_P{P}"
        for fld in faces.dtype.names:
            geo[f"{key}_face_{fld}"] = np.asarray(faces[fld])
        geo[f"{key}_J"], geo[f"{key}_Jinv"], geo[f"{key}_spxy"], geo[f"{key}_area"] = J, Ji, sxy, area
    np.savez_compressed(os.path.join(out, "ref_geometry.npz"), **geo)
    smp = phys_samples()
    fin = os.path.join(tmp, "phys_in.bin")
    with open(fin, "wb") as f:
        f.write(np.int64(smp.shape[0]).tobytes())
        f.write(smp.tobytes())
    fo = os.path.join(tmp, "phys_out.bin")
    P_ = PHYS_PARAMS
    run([O.REF_CPU, "phys", fin, fo] + [repr(P_[k]) for k in
        ("g", "mach", "aoa", "rho_inf", "p_inf", "p_total", "T_total", "dx", "dy", "p_static", "T_wall")])
    res = np.fromfile(fo, dtype=np.float64).reshape(smp.shape[0], 10, 4)
    np.savez_compressed(os.path.join(out, "ref_physics.npz"), samples=smp, out=res)
    gen_visc_header(out, tmp)
    print("cpu goldens written to", out)


# Pointwise viscous pins: a state, its conservative gradients and a right
# state with its gradients plus a normal (26 values per record), over a
# non-dimensional (T ~ 8) and a dimensional (T ~ 8e4) regime.
VISC_PARAMS = dict(g=1.4, Re=5000.0, Pr=0.72)


def visc_samples(n=256, seed=31):
    r = M.uniform01(seed, n * 26).reshape(n, 26)
    g = VISC_PARAMS["g"]
    out = np.empty((n, 26))
    for k in range(n):
        dim = k % 2 == 1
        rho0, p0 = (1.2, 1.0e5) if dim else (1.0, 1.0 / (g * 0.09))
        rows = []
        for side in range(2):
            q = r[k, 13 * side:13 * side + 13]
            rho = rho0 * (0.3 + 1.4 * q[0])
            p = p0 * (0.3 + 1.4 * q[1])
            c = np.sqrt(g * p / rho)
            u, v = c * (2.0 * q[2] - 1.0), c * (2.0 * q[3] - 1.0)
            U = M.prim_to_cons(rho, u, v, p, g)
            grad = np.abs(U) * (2.0 * q[4:12] - 1.0).reshape(2, 4) * (10.0 ** (3.0 * q[12] - 1.0))
            rows.append(np.concatenate([U, grad[0], grad[1]]))
        th = 2.0 * np.pi * r[k, 25]
        out[k] = np.concatenate([rows[0], rows[1], [np.cos(th), np.sin(th)]])
    return out


def _write_visc_in(path, smp):
    with open(path, "wb") as f:
        f.write(np.int64(smp.shape[0]).tobytes())
        f.write(smp.tobytes())


def gen_visc_header(out, tmp):
    smp = visc_samples()
    fin, fo = os.path.join(tmp, "visc_in.bin"), os.path.join(tmp, "visc_out.bin")
    _write_visc_in(fin, smp)
    V = VISC_PARAMS
    run([O.REF_CPU, "visc", fin, fo, repr(V["g"]), repr(V["Re"]), repr(V["Pr"])])
    res = np.fromfile(fo, dtype=np.float64).reshape(smp.shape[0], 3, 4)
    np.savez_compressed(os.path.join(out, "ref_viscous.npz"), samples=smp, out=res)


def gen_visc_kernel(out, tmp):
    smp = visc_samples()
    fin, fo = os.path.join(tmp, "viscsp_in.bin"), os.path.join(tmp, "viscsp_out.bin")
    _write_visc_in(fin, smp)
    V = VISC_PARAMS
    run([O.REF_GPU, "viscsp", fin, fo, repr(V["g"]), repr(V["Re"]), repr(V["Pr"])])
    n = smp.shape[0]
    a = np.fromfile(fo, dtype=np.float64)
    np.savez_compressed(os.path.join(out, "ref_viscous_kernel.npz"), samples=smp,
                        Fv=a[:4 * n].reshape(n, 4), Gv=a[4 * n:8 * n].reshape(n, 4))
    print("viscous kernel pins", n, flush=True)


# The isentropic-vortex configuration (20x20 on [-10,10]^2, P3, HU, Rusanov,
# far field) at the reference's own CFL-0.5 step for 200 steps, as the raw
# non-dimensional case (the reference's clamps fire) and its dimensional twin
# (clamps inactive at the start).  Per step: the state's per-variable sum,
# sum of squares, max and min, TRAJ_SAMPLES seeded solution points, and the
# residual norm; full states at TRAJ_FULL steps (restart points of the
# per-step comparison once the scheme's instability has amplified rounding).
TRAJ_CASES = ("vortex_raw_p3", "vortex_dim_p3")
TRAJ_STEPS = 200
TRAJ_SAMPLES = 64
TRAJ_FULL = (50, 100, 150)


def traj_sample_index(n_points, n=TRAJ_SAMPLES, seed=41):
    return np.sort((M.splitmix64(seed, n) % np.uint64(n_points)).astype(np.int64))


def traj_stats(U):
    """[4 sums, 4 sums of squares, 4 maxima, 4 minima] of a [E][n_sp][4] state."""
    X = U.reshape(-1, 4)
    return np.concatenate([X.sum(axis=0), (X * X).sum(axis=0), X.max(axis=0), X.min(axis=0)])


def gen_traj(out, tmp):
    res = {}
    defs = case_defs()
    for name in TRAJ_CASES:
        c = defs[name]
        mesh, P = c["mesh"], c["P"]
        rho, p, mach, aoa = c["prm"]
        orc = O.Oracle(mesh, P, GAMMA, rho, p, mach, aoa, tags=c["tags"])
        U = make_state(c, orc.sp_coords())
        mb, ub, tb = (os.path.join(tmp, x) for x in ("m.bin", "u.bin", "t.bin"))
        O.write_mesh_bin(mb, mesh, c["tags"])
        U.tofile(ub)
        prm = [str(P), repr(GAMMA), repr(rho), repr(p), repr(mach), repr(aoa)]
        run([O.REF_GPU, "traj", mb, *prm, ub, str(TRAJ_STEPS), tb])
        a = np.fromfile(tb, dtype=np.float64)
        dt, a = a[0], a[1:].reshape(TRAJ_STEPS, U.size + 1)
        idx = traj_sample_index(U.shape[0] * U.shape[1])
        states = a[:, :U.size].reshape((TRAJ_STEPS,) + U.shape)
        res[f"{name}_U0"] = U
        res[f"{name}_dt"] = np.array([dt])
        res[f"{name}_norm"] = a[:, U.size]
        res[f"{name}_stats"] = np.stack([traj_stats(X) for X in states])
        res[f"{name}_samples"] = states.reshape(TRAJ_STEPS, -1, 4)[:, idx, :]
        res[f"{name}_finite"] = np.array([bool(np.isfinite(X).all()) for X in states])
        for k in TRAJ_FULL:
            res[f"{name}_U{k}"] = states[k - 1]
        print(name, "dt", dt, "finite steps", int(res[f"{name}_finite"].sum()), flush=True)
    np.savez_compressed(os.path.join(out, "ref_trajectory.npz"), **res)


def gen_gpu(out, only=("residuals", "traj", "visc")):
    tmp = tempfile.mkdtemp()
    if "traj" in only:
        gen_traj(out, tmp)
    if "visc" in only:
        gen_visc_kernel(out, tmp)
    if "residuals" not in only:
        return
    res = {}
    for name, c in case_defs().items():
        mesh, P = c["mesh"], c["P"]
        rho, p, mach, aoa = c["prm"]
        orc = O.Oracle(mesh, P, GAMMA, rho, p, mach, aoa, tags=c["tags"])
        U = make_state(c, orc.sp_coords())
        mb, ub, rb = (os.path.join(tmp, x) for x in ("m.bin", "u.bin", "r.bin"))
        O.write_mesh_bin(mb, mesh, c["tags"])
        U.tofile(ub)
        prm = [str(P), repr(GAMMA), repr(rho), repr(p), repr(mach), repr(aoa)]
        run([O.REF_GPU, "rhs", mb, *prm, ub, rb])
        R = np.fromfile(rb, dtype=np.float64).reshape(U.shape)
        res[f"{name}_U"] = U
        res[f"{name}_R"] = R
        if c.get("nsteps"):
            sb = os.path.join(tmp, "s.bin")
            run([O.REF_GPU, "step", mb, *prm, ub, repr(c["dt"]), str(c["nsteps"]), sb])
            a = np.fromfile(sb, dtype=np.float64)
            n = U.size
            res[f"{name}_Ustep"] = a[:n].reshape(U.shape)
            res[f"{name}_Rstep"] = a[n:2 * n].reshape(U.shape)
            res[f"{name}_norm"] = a[2 * n:2 * n + 1]
        print(name, "max|R|", float(np.abs(R).max()), flush=True)
    np.savez_compressed(os.path.join(out, "ref_gpu_residuals.npz"), **res)
    print("gpu goldens written to", out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["cpu", "gpu"])
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default="residuals,traj,visc",
                    help="gpu: comma-separated subset of residuals, traj, visc")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.what == "cpu":
        gen_cpu(a.out)
    else:
        gen_gpu(a.out, tuple(a.only.split(",")))


if __name__ == "__main__":
    main()
