"""Python view of the C-ABI with the reference's FRSolver method names
(include/solver/fr_solver.hpp:77-180): initialize, setInitialCondition,
advance, computeTimeStep, computeResidual, copyToHost, copyToDevice.

Everything runs in libzj_fr.so; this module only marshals arguments.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .meshgen import QuadMesh


def make_params(poly_order=3, gamma=1.4, rho_inf=1.0, p_inf=1.0 / 1.4, Mach=0.5, AoA=0.0,
                flux_type="HU", riemann="Rusanov", CFL=0.5, viscous=False, Re=1000.0,
                Pr=0.72, compat=True, precision="fp64", bcs=(), config_text=None, T_inf=300.0):
    """A zj_params with the reference defaults, then the given values.
    bcs: iterable of (tag, type name[, p_static]).  config_text is parsed
    with the reference grammar after the keyword values."""
    p = L.Params()
    lib = L.lib()
    lib.zj_params_default(C.byref(p))
    p.poly_order = poly_order
    p.gamma = gamma
    p.rho_inf = rho_inf
    p.p_inf = p_inf
    p.Mach = Mach
    p.AoA = AoA
    p.flux_type = L.FLUX_TYPES[flux_type] if isinstance(flux_type, str) else int(flux_type)
    p.riemann = L.RIEMANN[riemann] if isinstance(riemann, str) else int(riemann)
    p.CFL = CFL
    p.viscous = int(bool(viscous))
    p.Re = Re
    p.Pr = Pr
    p.T_inf = T_inf
    p.compat = int(bool(compat))
    p.precision = {"fp64": L.FP64, "mixed": L.MIXED, "split_bf16": L.SPLIT_BF16}[precision]
    p.n_bc = 0
    for b in bcs:
        # (tag, type[, p_static]) or a dict with keys tag, type, p_static,
        # p_total, T_total, T_wall, dir_x, dir_y
        d = dict(b) if isinstance(b, dict) else dict(tag=b[0], type=b[1],
                                                    p_static=b[2] if len(b) > 2 else 0.0)
        s = p.bc[p.n_bc]
        s.tag = int(d["tag"])
        s.type = L.BC_TYPES[d["type"]] if isinstance(d["type"], str) else int(d["type"])
        s.p_static = float(d.get("p_static", 0.0))
        s.p_total = float(d.get("p_total", 0.0))
        s.T_total = float(d.get("T_total", 0.0))
        s.T_wall = float(d.get("T_wall", 0.0))
        s.dir_x, s.dir_y = float(d.get("dir_x", 1.0)), float(d.get("dir_y", 0.0))
        p.n_bc += 1
    if config_text is not None:
        L.check(lib.zj_params_parse_string(config_text.encode(), C.byref(p)))
    return p


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def mesh_desc(mesh):
    """The zj_mesh_desc of a QuadMesh or MixedMesh, with the arrays it points
    into (keep them alive while the descriptor is used)."""
    xy = np.ascontiguousarray(mesh.xy, dtype=np.float64)
    if hasattr(mesh, "offsets"):          # MixedMesh: quads and triangles
        conn = np.ascontiguousarray(mesh.conn, dtype=np.int64)
        et = np.ascontiguousarray(mesh.etype, dtype=np.int32)
        ne = et.shape[0]
        eo = np.ones(ne, dtype=np.int32)
        off = np.ascontiguousarray(mesh.offsets, dtype=np.int64)
    else:
        conn = np.ascontiguousarray(mesh.conn, dtype=np.int64)
        ne, nn = conn.shape
        et = np.ones(ne, dtype=np.int32)
        eo = np.full(ne, {4: 1, 9: 2, 25: 4}[nn], dtype=np.int32)
        off = (np.arange(ne + 1, dtype=np.int64) * nn)
    bnd = np.ascontiguousarray(mesh.bnd, dtype=np.int64)
    d = L.MeshDesc()
    d.n_nodes = xy.shape[0]
    d.xy = _dptr(xy)
    d.n_elem = ne
    d.elem_type = et.ctypes.data_as(C.POINTER(C.c_int32))
    d.elem_order = eo.ctypes.data_as(C.POINTER(C.c_int32))
    d.conn_offsets = off.ctypes.data_as(C.POINTER(C.c_int64))
    d.conn = conn.ctypes.data_as(C.POINTER(C.c_int64))
    d.n_bnd_edges = bnd.shape[0]
    d.bnd_edges = bnd.ctypes.data_as(C.POINTER(C.c_int64))
    return d, [xy, conn, et, eo, off, bnd]


class FRSolver:
    """One zj_solver handle."""

    def __init__(self, mesh: QuadMesh, params: L.Params):
        lib = L.lib()
        d, self._keep = mesh_desc(mesh)
        h = C.c_void_p()
        L.check(lib.zj_solver_create(C.byref(d), C.byref(params), C.byref(h)))
        self._attach(h, params)

    @classmethod
    def from_handle(cls, h, params: L.Params, keep=()) -> "FRSolver":
        """Wrap a handle the library created (a part of a partition)."""
        s = cls.__new__(cls)
        s._keep = list(keep)
        s._attach(h, params)
        return s

    @classmethod
    def from_gmsh(cls, path: str, params: L.Params) -> "FRSolver":
        """A solver on an ASCII Gmsh mesh (zj_solver_create_from_gmsh)."""
        h = C.c_void_p()
        L.check(L.lib().zj_solver_create_from_gmsh(str(path).encode(), C.byref(params), C.byref(h)))
        self = cls.__new__(cls)
        self._keep = []
        self._attach(h, params)
        return self

    def _attach(self, h, params):
        lib = L.lib()
        self.h = h
        self.params = params
        self.n_elem = lib.zj_num_elements(h)
        self.n_sp = lib.zj_num_solution_points(h)
        self.n_faces = lib.zj_num_faces(h)
        self.shape = (self.n_elem, self.n_sp, 4)
        self._host = np.zeros(self.shape)

    def close(self):
        if getattr(self, "h", None):
            L.lib().zj_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, code):
        L.check(code, self.h)

    # -- reference method names ------------------------------------------
    def solution_point_coords(self) -> np.ndarray:
        xy = np.zeros((self.n_elem, self.n_sp, 2))
        self._ck(L.lib().zj_solution_point_coords(self.h, _dptr(xy)))
        return xy

    def setInitialCondition(self, ic):
        """ic maps an [..., 2] coordinate array to an [..., 4] state array."""
        self.copyToDevice(np.asarray(ic(self.solution_point_coords()), dtype=np.float64))

    def copyToDevice(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.shape)
        self._ck(L.lib().zj_set_state(self.h, _dptr(U)))

    def copyToHost(self, out: np.ndarray = None) -> np.ndarray:
        """The current state; into ``out`` (C-contiguous float64) when given."""
        if out is None:
            out = np.empty(self.shape)
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == np.prod(self.shape)
        self._ck(L.lib().zj_get_state(self.h, _dptr(out)))
        return out

    solution = copyToHost

    def copyToDeviceAsync(self, U: np.ndarray):
        """Queue the host-to-device copy of U (C-contiguous float64 of the
        state's shape) on the handle's stream and return.  U must stay alive
        and unchanged until synchronize(); page-locked memory lets the copy
        overlap other streams' work."""
        assert U.dtype == np.float64 and U.flags.c_contiguous and U.size == np.prod(self.shape)
        self._ck(L.lib().zj_set_state_async(self.h, C.c_void_p(U.ctypes.data)))

    def copyToHostAsync(self, out: np.ndarray):
        """Queue the device-to-host copy of the state into out on the handle's
        stream and return; out holds it after synchronize()."""
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == np.prod(self.shape)
        self._ck(L.lib().zj_get_state_async(self.h, C.c_void_p(out.ctypes.data)))

    def advance(self, dt: float, nsteps: int = 1, sync: bool = True):
        self._ck(L.lib().zj_step(self.h, float(dt), int(nsteps)))
        if sync:
            self.synchronize()

    def set_step_graphs(self, enable: bool):
        """Replay blocks of six steps from captured CUDA graphs (default on)."""
        self._ck(L.lib().zj_set_step_graphs(self.h, int(bool(enable))))

    def synchronize(self):
        self._ck(L.lib().zj_synchronize(self.h))

    def computeTimeStep(self) -> float:
        v = C.c_double()
        self._ck(L.lib().zj_compute_dt(self.h, C.byref(v)))
        return v.value

    def computeResidual(self) -> float:
        v = C.c_double()
        self._ck(L.lib().zj_residual_norm(self.h, C.byref(v)))
        return v.value

    def check_state(self):
        self._ck(L.lib().zj_check_state(self.h))

    # -- residual entry points ------------------------------------------
    def rhs(self, U: np.ndarray) -> np.ndarray:
        """R(U) through host buffers."""
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.shape)
        R = np.empty(self.shape)
        self._ck(L.lib().zj_rhs_host(self.h, _dptr(U), _dptr(R)))
        return R

    def rhs_device(self, U_ptr: int, R_ptr: int):
        """R(U) on device pointers (e.g. torch tensors' data_ptr())."""
        self._ck(L.lib().zj_rhs(self.h, C.c_void_p(U_ptr), C.c_void_p(R_ptr)))

    def set_stream(self, stream_ptr: int):
        self._ck(L.lib().zj_set_stream(self.h, C.c_void_p(stream_ptr)))

    def element_kinds(self) -> np.ndarray:
        """[E] 0 triangle, 1 quadrilateral."""
        k = np.zeros(self.n_elem, dtype=np.int32)
        self._ck(L.lib().zj_element_kinds(self.h, k.ctypes.data_as(C.POINTER(C.c_int32))))
        return k

    def slot_mask(self) -> np.ndarray:
        """[E][n_sp] True for the state slots an element uses (a triangle
        uses its first (P+1)(P+2)/2)."""
        k = self.element_kinds()
        nt = L.lib().zj_num_triangle_points(self.h)
        m = np.ones((self.n_elem, self.n_sp), dtype=bool)
        m[k == 0, nt:] = False
        return m

    # -- restart files ----------------------------------------------------
    def write_restart(self, path: str):
        """State, time and iteration into a restart file (zj_restart_write)."""
        self._ck(L.lib().zj_restart_write(self.h, str(path).encode()))

    def read_restart(self, path: str):
        """Load a restart file and resume its time and iteration."""
        self._ck(L.lib().zj_restart_read(self.h, str(path).encode()))

    # -- differentiation (physics mode, FP64; device pointers) ------------
    def rhs_jvp(self, U_ptr: int, V_ptr: int, JV_ptr: int, R_ptr: int = 0, dRe: float = 0.0):
        """JV = dR/dU . V + dR/dRe dRe (and R(U) into R_ptr if given)."""
        self._ck(L.lib().zj_rhs_jvp(self.h, C.c_void_p(U_ptr), C.c_void_p(V_ptr), dRe,
                                    C.c_void_p(R_ptr or None), C.c_void_p(JV_ptr)))

    def rhs_vjp(self, U_ptr: int, L_ptr: int, W_ptr: int, with_re: bool = False):
        """W = (dR/dU)^T L; returns L . dR/dRe when with_re."""
        v = C.c_double()
        self._ck(L.lib().zj_rhs_vjp(self.h, C.c_void_p(U_ptr), C.c_void_p(L_ptr), C.c_void_p(W_ptr),
                                    C.byref(v) if with_re else None))
        return v.value if with_re else None

    def step_vjp(self, U_ptr: int, dt: float, B_ptr: int, A_ptr: int, with_re: bool = False):
        """A = dJ/dU(n) from B = dJ/dU(n+1) for one SSP-RK3 step from U;
        returns that step's dJ/dRe contribution when with_re."""
        v = C.c_double(0.0)
        self._ck(L.lib().zj_step_vjp(self.h, C.c_void_p(U_ptr), dt, C.c_void_p(B_ptr), C.c_void_p(A_ptr),
                                     C.byref(v) if with_re else None))
        return v.value if with_re else None

    def adjoint_run(self, dt: float, nsteps: int, k_ckpt: int, G_ptr: int):
        """Checkpointed discrete adjoint of nsteps steps from the current
        state: G holds dJ/dU(final) in, dJ/dU(initial) out.  Returns
        {dRe, bytes, ms_forward, ms_adjoint}."""
        dre, fw, bw = C.c_double(), C.c_double(), C.c_double()
        nb = C.c_int64()
        self._ck(L.lib().zj_adjoint_run(self.h, dt, nsteps, k_ckpt, C.c_void_p(G_ptr), C.byref(dre),
                                        C.byref(nb), C.byref(fw), C.byref(bw)))
        return {"dRe": dre.value, "bytes": nb.value, "ms_forward": fw.value, "ms_adjoint": bw.value}

    @property
    def time(self) -> float:
        return L.lib().zj_time(self.h)

    @property
    def iteration(self) -> int:
        return L.lib().zj_iteration(self.h)
