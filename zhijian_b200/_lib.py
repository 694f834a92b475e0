"""ctypes binding of the C-ABI in include/zj_fr.h (libzj_fr.so, in-tree).

Loading fails loudly when the library is missing: there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzj_fr.so")

OK, ERR_ARG, ERR_CUDA, ERR_NAN, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_IO = range(7)
STATUS_NAMES = {0: "ZJ_OK", 1: "ZJ_ERR_ARG", 2: "ZJ_ERR_CUDA", 3: "ZJ_ERR_NAN",
                4: "ZJ_ERR_TIMEOUT", 5: "ZJ_ERR_UNSUPPORTED", 6: "ZJ_ERR_IO"}

BC_TYPES = {"interior": 0, "wall": 1, "slipwall": 2, "symmetry": 3, "farfield": 4,
            "inflow": 5, "outflow": 6, "periodic": 7}
FLUX_TYPES = {"DG": 0, "SD": 1, "HU": 2, "GA": 3}
RIEMANN = {"Rusanov": 0, "Roe": 1, "HLLC": 2}
FP64, MIXED, SPLIT_BF16 = 0, 1, 2
MAX_BC = 32


class BCSpec(C.Structure):
    _fields_ = [("tag", C.c_int), ("type", C.c_int), ("p_static", C.c_double),
                ("p_total", C.c_double), ("T_total", C.c_double), ("T_wall", C.c_double),
                ("dir_x", C.c_double), ("dir_y", C.c_double)]


class Params(C.Structure):
    _fields_ = [("gamma", C.c_double), ("Pr", C.c_double), ("Re", C.c_double),
                ("Mach", C.c_double), ("T_inf", C.c_double), ("p_inf", C.c_double),
                ("rho_inf", C.c_double), ("AoA", C.c_double),
                ("poly_order", C.c_int), ("flux_type", C.c_int), ("riemann", C.c_int),
                ("CFL", C.c_double), ("dt", C.c_double), ("t_final", C.c_double),
                ("max_iter", C.c_int), ("viscous", C.c_int),
                ("output_freq", C.c_int), ("restart_freq", C.c_int),
                ("case_name", C.c_char * 64),
                ("compat", C.c_int), ("precision", C.c_int),
                ("n_bc", C.c_int), ("bc", BCSpec * MAX_BC)]


# int exchange(void* user, int kind, int row_bytes, const void* send_dev,
#              void* recv_dev, void* stream): the transport of zj_part_step
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)
XCHG_TRACES, XCHG_GRADIENTS = 1, 2


class MeshDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("xy", C.POINTER(C.c_double)),
                ("n_elem", C.c_int64), ("elem_type", C.POINTER(C.c_int32)),
                ("elem_order", C.POINTER(C.c_int32)),
                ("conn_offsets", C.POINTER(C.c_int64)), ("conn", C.POINTER(C.c_int64)),
                ("n_bnd_edges", C.c_int64), ("bnd_edges", C.POINTER(C.c_int64))]


_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run zhijian_b200/build.py "
                           "(the CUDA path has no fallback)")
    h = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
    sig = {
        "zj_abi_version": (ip, []),
        "zj_params_default": (None, [C.POINTER(Params)]),
        "zj_params_parse_file": (ip, [C.c_char_p, C.POINTER(Params)]),
        "zj_params_parse_string": (ip, [C.c_char_p, C.POINTER(Params)]),
        "zj_solver_create": (ip, [C.POINTER(MeshDesc), C.POINTER(Params), C.POINTER(vp)]),
        "zj_solver_create_from_gmsh": (ip, [C.c_char_p, C.POINTER(Params), C.POINTER(vp)]),
        "zj_solver_destroy": (None, [vp]),
        "zj_last_error": (C.c_char_p, [vp]),
        "zj_num_elements": (C.c_int64, [vp]),
        "zj_num_solution_points": (ip, [vp]),
        "zj_num_faces": (C.c_int64, [vp]),
        "zj_state_size": (C.c_int64, [vp]),
        "zj_solution_point_coords": (ip, [vp, dp]),
        "zj_set_state": (ip, [vp, dp]),
        "zj_get_state": (ip, [vp, dp]),
        "zj_set_state_async": (ip, [vp, vp]),
        "zj_set_step_graphs": (ip, [vp, ip]),
        "zj_get_state_async": (ip, [vp, vp]),
        "zj_set_state_device": (ip, [vp, vp]),
        "zj_get_state_device": (ip, [vp, vp]),
        "zj_step": (ip, [vp, C.c_double, ip]),
        "zj_synchronize": (ip, [vp]),
        "zj_rhs": (ip, [vp, vp, vp]),
        "zj_rhs_host": (ip, [vp, dp, dp]),
        "zj_rhs_noalloc": (ip, [vp, vp, vp]),
        "zj_residual_norm": (ip, [vp, dp]),
        "zj_compute_dt": (ip, [vp, dp]),
        "zj_check_state": (ip, [vp]),
        "zj_time": (C.c_double, [vp]),
        "zj_iteration": (ip, [vp]),
        "zj_set_stream": (ip, [vp, vp]),
        "zj_get_stream": (vp, [vp]),
        "zj_element_kinds": (ip, [vp, C.POINTER(C.c_int32)]),
        "zj_num_triangle_points": (ip, [vp]),
        "zj_restart_write": (ip, [vp, C.c_char_p]),
        "zj_restart_read": (ip, [vp, C.c_char_p]),
        "zj_gmsh_read": (ip, [C.c_char_p, C.POINTER(vp)]),
        "zj_gmsh_free": (None, [vp]),
        "zj_gmsh_desc": (C.POINTER(MeshDesc), [vp]),
        "zj_gmsh_num_groups": (ip, [vp]),
        "zj_gmsh_group": (ip, [vp, ip, C.POINTER(ip), C.POINTER(ip), C.POINTER(C.c_char_p)]),
        "zj_rhs_jvp": (ip, [vp, vp, vp, C.c_double, vp, vp]),
        "zj_rhs_vjp": (ip, [vp, vp, vp, vp, dp]),
        "zj_step_vjp": (ip, [vp, vp, C.c_double, vp, vp, dp]),
        "zj_adjoint_run": (ip, [vp, C.c_double, ip, ip, vp, dp, C.POINTER(C.c_int64), dp, dp]),
        "zj_partition": (ip, [C.POINTER(MeshDesc), ip, C.POINTER(C.c_int32)]),
        "zj_halo_plan_size": (ip, [C.POINTER(MeshDesc), C.POINTER(C.c_int32), ip, ip, C.POINTER(ip),
                                   C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "zj_halo_plan": (ip, [C.POINTER(MeshDesc), C.POINTER(C.c_int32), ip, ip, C.POINTER(C.c_int32),
                              C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                              C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "zj_solver_create_part": (ip, [C.POINTER(MeshDesc), C.POINTER(Params), C.POINTER(C.c_int32), ip, ip,
                                       C.POINTER(vp)]),
        "zj_part_elements": (ip, [vp, C.POINTER(C.c_int64)]),
        "zj_parts_step": (ip, [C.POINTER(vp), ip, C.c_double, ip]),
        "zj_parts_rhs": (ip, [C.POINTER(vp), ip, C.POINTER(vp), C.POINTER(vp)]),
        "zj_parts_synchronize": (ip, [C.POINTER(vp), ip]),
        "zj_parts_residual_norm": (ip, [C.POINTER(vp), ip, dp]),
        "zj_part_step": (ip, [vp, C.c_double, ip, EXCHANGE_FN, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(h, name)
        f.restype = res
        f.argtypes = args
    _lib = h
    return h


class ZJError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def check(code: int, handle=None):
    if code != OK:
        m = lib().zj_last_error(handle)
        raise ZJError(code, m.decode() if m else "")
