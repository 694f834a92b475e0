"""Python view of the library's Gmsh reader (zj_gmsh_read): ASCII MSH v2.2 /
v4.1 meshes as arrays, with the boundary groups and their inferred types."""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib as L
from .meshgen import MixedMesh, QuadMesh

BC_NAMES = {v: k for k, v in L.BC_TYPES.items()}


@dataclasses.dataclass
class GmshData:
    xy: np.ndarray            # [n_nodes][2]
    elem_type: np.ndarray     # [n_elem] 0 triangle, 1 quadrilateral
    elem_order: np.ndarray    # [n_elem]
    offsets: np.ndarray       # [n_elem + 1]
    conn: np.ndarray          # flat node ids
    bnd: np.ndarray           # [n_bnd][3] (v0, v1, physical tag)
    groups: list              # [(tag, zj_bc_type, name)]

    def element(self, e: int) -> np.ndarray:
        return self.conn[self.offsets[e]:self.offsets[e + 1]]

    def to_quad_mesh(self) -> QuadMesh:
        """The mesh as a QuadMesh (all elements quadrilaterals of one order)."""
        if np.any(self.elem_type != 1) or len(set(self.elem_order.tolist())) != 1:
            raise ValueError("not a single-order quadrilateral mesh")
        nn = int(self.offsets[1] - self.offsets[0])
        return QuadMesh(self.xy.copy(), self.conn.reshape(-1, nn).copy(), self.bnd.copy(),
                        {t: BC_NAMES[ty] for t, ty, _ in self.groups})


    def to_mixed_mesh(self) -> MixedMesh:
        """The mesh as a MixedMesh (straight-sided triangles and quadrilaterals,
        their first three / four nodes)."""
        if np.any(self.elem_order != 1):
            raise ValueError("not a straight-sided (order 1) mesh")
        conn, off = [], [0]
        for e in range(len(self.elem_type)):
            nv = 3 if self.elem_type[e] == 0 else 4
            conn.extend(self.element(e)[:nv].tolist())
            off.append(len(conn))
        return MixedMesh(self.xy.copy(), self.elem_type.astype(np.int32), np.array(off, dtype=np.int64),
                         np.array(conn, dtype=np.int64), self.bnd.copy(),
                         {t: BC_NAMES[ty] for t, ty, _ in self.groups})


def read_gmsh(path: str) -> GmshData:
    lib = L.lib()
    h = C.c_void_p()
    L.check(lib.zj_gmsh_read(str(path).encode(), C.byref(h)))
    try:
        d = lib.zj_gmsh_desc(h).contents
        nn, ne, nb = d.n_nodes, d.n_elem, d.n_bnd_edges
        xy = np.ctypeslib.as_array(d.xy, shape=(nn * 2,)).reshape(nn, 2).copy()
        et = np.ctypeslib.as_array(d.elem_type, shape=(ne,)).copy()
        eo = np.ctypeslib.as_array(d.elem_order, shape=(ne,)).copy()
        off = np.ctypeslib.as_array(d.conn_offsets, shape=(ne + 1,)).copy()
        conn = np.ctypeslib.as_array(d.conn, shape=(int(off[-1]),)).copy()
        bnd = (np.ctypeslib.as_array(d.bnd_edges, shape=(nb * 3,)).reshape(nb, 3).copy()
               if nb else np.zeros((0, 3), dtype=np.int64))
        groups = []
        for i in range(lib.zj_gmsh_num_groups(h)):
            tag, ty, name = C.c_int(), C.c_int(), C.c_char_p()
            L.check(lib.zj_gmsh_group(h, i, C.byref(tag), C.byref(ty), C.byref(name)))
            groups.append((tag.value, ty.value, name.value.decode()))
        return GmshData(xy, et, eo, off, conn, bnd, groups)
    finally:
        lib.zj_gmsh_free(h)
