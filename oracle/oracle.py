"""TEST INFRASTRUCTURE -- ctypes wrapper of the C oracle (fr_oracle.c) and
readers for the reference harness outputs (oracle/ref/ref_harness.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference
arm use this module.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libfr_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_CPU = os.path.join(REF_DIR, "ref_cpu")
REF_GPU = os.path.join(REF_DIR, "ref_gpu")
# The reference sources the harness is compiled from; REF as in
# `make -C oracle/ref REF=...`.
REFERENCE_ROOT = os.environ.get("REF", "/root/reference")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "fr_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
               "-o", LIB + ".tmp", src, "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + r.stderr)
        os.replace(LIB + ".tmp", LIB)
    return LIB


def build_reference(gpu: bool = True) -> bool:
    """Compile the reference's own code into oracle/_ref (needs the reference
    sources; the outputs then travel with the repository snapshot)."""
    if not os.path.isdir(REFERENCE_ROOT):
        return os.path.exists(REF_CPU)
    targets = ["cpu"] + (["gpu"] if gpu else [])
    r = subprocess.run(["make", "-C", os.path.join(HERE, "ref"), *targets,
                        f"REF={REFERENCE_ROOT}"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference build failed:\n" + r.stdout + r.stderr)
    return True


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        h = C.CDLL(LIB)
        dp, ip, i64 = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int64
        h.orc_create.restype = C.c_void_p
        h.orc_create.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.c_double, i64, dp, i64, C.c_int, C.c_int,
                                 C.POINTER(C.c_int64), i64, C.POINTER(C.c_int64), C.c_int,
                                 ip, ip, dp]
        h.orc_destroy.argtypes = [C.c_void_p]
        h.orc_set_threads.argtypes = [C.c_void_p, C.c_int]
        h.orc_num_faces.restype = i64
        h.orc_num_faces.argtypes = [C.c_void_p]
        h.orc_num_sp.argtypes = [C.c_void_p]
        h.orc_faces.argtypes = [C.c_void_p, ip, ip, ip, ip, ip, ip, dp]
        h.orc_geometry.argtypes = [C.c_void_p, dp, dp]
        h.orc_operators.argtypes = [C.c_void_p, dp, dp, dp, dp, dp, dp]
        h.orc_sp_coords.argtypes = [C.c_void_p, dp]
        h.orc_rhs.argtypes = [C.c_void_p, dp, dp]
        h.orc_step.argtypes = [C.c_void_p, dp, C.c_double, C.c_int, dp]
        h.orc_compute_dt.restype = C.c_double
        h.orc_compute_dt.argtypes = [C.c_void_p, dp, C.c_double]
        h.orc_l2.restype = C.c_double
        h.orc_l2.argtypes = [dp, i64]
        h.orc_set_physics.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                      C.c_double, C.c_double]
        h.orc_set_bc_extra.argtypes = [C.c_void_p, C.c_int, ip, dp, dp, dp, dp, dp]
        h.orc_get_vcjh.argtypes = [C.c_void_p, dp, dp]
        h.orc_rhs_phys.argtypes = [C.c_void_p, dp, dp]
        h.orc_step_phys.argtypes = [C.c_void_p, dp, C.c_double, C.c_int, dp]
        h.orc_riemann_point.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, C.c_double, dp]
        h.orc_ghost_point.argtypes = [C.c_void_p, C.c_int, C.c_int, dp, C.c_double, C.c_double, dp]
        h.orc_wall_viscous_closure.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, dp]
        h.orc_viscous_flux_law.argtypes = [C.c_int, dp, dp, dp, C.c_double, C.c_double, C.c_double, dp, dp]
        h.orc_common_viscous_law.argtypes = [C.c_int, dp, dp, dp, dp, dp, dp, C.c_double, C.c_double,
                                             C.c_double, C.c_double, C.c_double, dp]
        _lib = h
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


BC_TYPES = {"interior": 0, "wall": 1, "slipwall": 2, "symmetry": 3, "farfield": 4,
            "inflow": 5, "outflow": 6, "periodic": 7}


class Oracle:
    """Compat-mode reference residual and stepper on the CPU."""

    def __init__(self, mesh, P, gamma=1.4, rho_inf=1.0, p_inf=1.0 / 1.4, Mach=0.5, AoA=0.0,
                 tags=None, threads=1):
        h = lib()
        self.P = P
        self.n1 = P + 1
        self.nsp = self.n1 ** 2
        xy = np.ascontiguousarray(mesh.xy, dtype=np.float64)
        conn = np.ascontiguousarray(mesh.conn, dtype=np.int64)
        bnd = np.ascontiguousarray(mesh.bnd, dtype=np.int64)
        nn = conn.shape[1]
        order = {4: 1, 9: 2, 25: 4}[nn]
        if tags is None:
            tags = [(t, BC_TYPES[n], 0.0) for t, n in sorted(mesh.tag_names.items())]
        tid = np.array([t[0] for t in tags] or [0], dtype=np.int32)
        tty = np.array([t[1] for t in tags] or [0], dtype=np.int32)
        tps = np.array([t[2] if len(t) > 2 else 0.0 for t in tags] or [0.0], dtype=np.float64)
        self._arrs = (xy, conn, bnd, tid, tty, tps)
        self.c = h.orc_create(P, gamma, rho_inf, p_inf, Mach, AoA, xy.shape[0], _d(xy),
                              conn.shape[0], nn, order, conn.ctypes.data_as(C.POINTER(C.c_int64)),
                              bnd.shape[0], bnd.ctypes.data_as(C.POINTER(C.c_int64)),
                              len(tags), _i(tid), _i(tty), _d(tps))
        if not self.c:
            raise ValueError("oracle rejected the mesh")
        h.orc_set_threads(self.c, threads)
        self.n_elem = conn.shape[0]
        self.shape = (self.n_elem, self.nsp, 4)

    def __del__(self):
        if getattr(self, "c", None):
            lib().orc_destroy(self.c)
            self.c = None

    def set_threads(self, n):
        lib().orc_set_threads(self.c, n)

    def rhs(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.shape)
        R = np.empty(self.shape)
        lib().orc_rhs(self.c, _d(U), _d(R))
        return R

    def step(self, U, dt, nsteps=1):
        U = np.array(U, dtype=np.float64).reshape(self.shape)
        R = np.empty(self.shape)
        lib().orc_step(self.c, _d(U), dt, nsteps, _d(R))
        return U, R

    def compute_dt(self, U, CFL):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.shape)
        return lib().orc_compute_dt(self.c, _d(U), CFL)

    def faces(self):
        nf = lib().orc_num_faces(self.c)
        a = [np.empty(nf, dtype=np.int32) for _ in range(6)]
        n = np.empty((nf, 2))
        lib().orc_faces(self.c, *[_i(x) for x in a], _d(n))
        return dict(left_elem=a[0], left_local=a[1], right_elem=a[2], right_local=a[3],
                    bc_type=a[4], bc_tag=a[5], normals=n)

    def geometry(self):
        J = np.empty((self.n_elem, self.nsp))
        Ji = np.empty((self.n_elem, self.nsp, 4))
        lib().orc_geometry(self.c, _d(J), _d(Ji))
        return J, Ji

    def operators(self):
        n1, nsp = self.n1, self.nsp
        out = dict(pts=np.empty(n1), D1=np.empty((n1, n1)), diff_xi=np.empty((nsp, nsp)),
                   diff_eta=np.empty((nsp, nsp)), interp=np.empty((4, n1, nsp)),
                   corr=np.empty((4, nsp)))
        lib().orc_operators(self.c, *[_d(out[k]) for k in
                                      ("pts", "D1", "diff_xi", "diff_eta", "interp", "corr")])
        return out

    # ---- physics mode ------------------------------------------------
    def set_physics(self, flux_type=2, riemann=0, viscous=False, Re=1000.0, Pr=0.72, T_inf=300.0):
        lib().orc_set_physics(self.c, flux_type, riemann, int(viscous), Re, Pr, T_inf)

    def set_bc_extra(self, rows):
        """rows: (tag, p_total, T_total, dir_x, dir_y, T_wall)"""
        ids = np.array([r[0] for r in rows], dtype=np.int32)
        cols = [np.array([r[k] for r in rows], dtype=np.float64) for k in range(1, 6)]
        self._extra = (ids, cols)
        lib().orc_set_bc_extra(self.c, len(rows), _i(ids), *[_d(x) for x in cols])

    def vcjh(self):
        gL, gR = np.empty(self.n1), np.empty(self.n1)
        lib().orc_get_vcjh(self.c, _d(gL), _d(gR))
        return gL, gR

    def rhs_phys(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.shape)
        R = np.empty(self.shape)
        lib().orc_rhs_phys(self.c, _d(U), _d(R))
        return R

    def step_phys(self, U, dt, nsteps=1):
        U = np.array(U, dtype=np.float64).reshape(self.shape)
        R = np.empty(self.shape)
        lib().orc_step_phys(self.c, _d(U), dt, nsteps, _d(R))
        return U, R

    def ghost(self, bc_type, tag, Ui, nx, ny):
        Ui = np.ascontiguousarray(Ui, dtype=np.float64)
        out = np.empty(4)
        lib().orc_ghost_point(self.c, bc_type, tag, _d(Ui), nx, ny, _d(out))
        return out

    def wall_closure(self, bc_type, tag, nx, ny, Fvn):
        """The walls' Neumann data applied to a boundary face's common normal
        viscous flux (orc_wall_viscous_closure)."""
        out = np.array(Fvn, dtype=np.float64)
        lib().orc_wall_viscous_closure(self.c, bc_type, tag, nx, ny, _d(out))
        return out

    def sp_coords(self):
        xy = np.empty((self.n_elem, self.nsp, 2))
        lib().orc_sp_coords(self.c, _d(xy))
        return xy


# ------------------------------------------------ reference harness files --

def write_mesh_bin(path, mesh, tags=None):
    """Mesh file read by ref_harness.cpp load_mesh()."""
    xy = np.ascontiguousarray(mesh.xy, dtype=np.float64)
    conn = np.ascontiguousarray(mesh.conn, dtype=np.int64)
    bnd = np.ascontiguousarray(mesh.bnd, dtype=np.int64)
    nn = conn.shape[1]
    if tags is None:
        tags = [(t, BC_TYPES[n], 0.0) for t, n in sorted(mesh.tag_names.items())]
    with open(path, "wb") as f:
        f.write(struct.pack("<q", xy.shape[0]))
        f.write(xy.tobytes())
        f.write(struct.pack("<qii", conn.shape[0], nn, {4: 1, 9: 2, 25: 4}[nn]))
        f.write(conn.tobytes())
        f.write(struct.pack("<q", bnd.shape[0]))
        f.write(bnd.tobytes())
        f.write(struct.pack("<i", len(tags)))
        for t in tags:
            f.write(struct.pack("<iid", int(t[0]), int(t[1]), float(t[2]) if len(t) > 2 else 0.0))


def read_ops_bin(path, P):
    n1 = P + 1
    nsp = n1 * n1
    a = np.fromfile(path, dtype=np.float64)
    o, out = 0, {}
    for k, shp in (("pts", (n1,)), ("D1", (n1, n1)), ("diff_xi", (nsp, nsp)),
                   ("diff_eta", (nsp, nsp)), ("interp", (4, n1, nsp)), ("corr", (4, nsp))):
        n = int(np.prod(shp))
        out[k] = a[o:o + n].reshape(shp)
        o += n
    return out


def read_tri_bin(path, P):
    """The reference's triangle FROperators as written by ref_cpu "tri"."""
    n1, nt = P + 1, (P + 1) * (P + 2) // 2
    a = np.fromfile(path, dtype=np.float64)
    o, out = 0, {}
    for k, shp in (("xi", (nt,)), ("eta", (nt,)), ("fp_loc", (3, n1)), ("interp", (3, n1, nt)),
                   ("diff_xi", (nt, nt)), ("diff_eta", (nt, nt)), ("corr", (3, nt)), ("weights", (nt,))):
        n = int(np.prod(shp))
        out[k] = a[o:o + n].reshape(shp)
        o += n
    assert o == a.size
    return out


def read_mesh_out(path, n_elem, nsp):
    with open(path, "rb") as f:
        raw = f.read()
    nf = struct.unpack_from("<q", raw, 0)[0]
    rec = np.dtype([("le", "<i4"), ("ll", "<i4"), ("re", "<i4"), ("rl", "<i4"),
                    ("bct", "<i4"), ("tag", "<i4"), ("nx", "<f8"), ("ny", "<f8")])
    faces = np.frombuffer(raw, dtype=rec, count=nf, offset=8)
    o = 8 + nf * rec.itemsize
    rest = np.frombuffer(raw, dtype=np.float64, offset=o)
    J = rest[:n_elem * nsp].reshape(n_elem, nsp)
    Ji = rest[n_elem * nsp:n_elem * nsp * 5].reshape(n_elem, nsp, 4)
    sxy = rest[n_elem * nsp * 5:n_elem * nsp * 7].reshape(n_elem, nsp, 2)
    area = rest[n_elem * nsp * 7:n_elem * nsp * 7 + n_elem]
    return faces, J, Ji, sxy, area


def riemann_point(which, UL, UR, nx, ny, g):
    UL = np.ascontiguousarray(UL, dtype=np.float64)
    UR = np.ascontiguousarray(UR, dtype=np.float64)
    out = np.empty(4)
    lib().orc_riemann_point(which, _d(UL), _d(UR), nx, ny, g, _d(out))
    return out


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def viscous_point(law, U, dx, dy, g, Re, Pr):
    """(Fv, Gv) at one state with conservative gradients: law 0 the kernel's
    mu = T^0.7/Re (the residual's), law 1 the header's Sutherland law."""
    U, dx, dy = _c(U), _c(dx), _c(dy)
    F, G = np.empty(4), np.empty(4)
    lib().orc_viscous_flux_law(law, _d(U), _d(dx), _d(dy), g, Re, Pr, _d(F), _d(G))
    return F, G


def common_viscous_point(law, UL, UR, dxL, dyL, dxR, dyR, nx, ny, g, Re, Pr):
    """Common normal viscous flux of one face point (BR2Scheme::commonFlux)."""
    a = [_c(x) for x in (UL, UR, dxL, dyL, dxR, dyR)]
    out = np.empty(4)
    lib().orc_common_viscous_law(law, *[_d(x) for x in a], nx, ny, g, Re, Pr, _d(out))
    return out
