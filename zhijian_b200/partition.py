"""Partitioned meshes: the parts of a mesh as one handle each, driven
together (zj_partition, zj_solver_create_part, zj_parts_*; the C-ABI's
partition section), and the halo plan that orders the trace rows crossing
each cut.

The reference partitions with METIS (src/mesh/partitioner.cpp:10-93) and
exchanges element data over MPI (src/parallel/mpi_comm.cpp:68-171); here the
partition is a recursive coordinate bisection and what crosses a cut is the
face traces (the only coupling of the FR residual between elements)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .solver import FRSolver, mesh_desc


def partition(mesh, nparts: int) -> np.ndarray:
    """Part of every element (recursive coordinate bisection, balanced)."""
    d, keep = mesh_desc(mesh)
    part = np.empty(mesh.n_elem, dtype=np.int32)
    L.check(L.lib().zj_partition(C.byref(d), nparts, part.ctypes.data_as(C.POINTER(C.c_int32))))
    return part


def halo_plan(mesh, part: np.ndarray, rank: int) -> dict:
    """Part `rank`'s view: its elements (global ids, ascending) and its
    interfaces grouped by neighbouring part, each group in the global face
    order -- per interface the global face, this part's side and the other
    side as global element*4 + local edge."""
    d, keep = mesh_desc(mesh)
    part = np.ascontiguousarray(part, dtype=np.int32)
    nparts = int(part.max()) + 1
    pp = part.ctypes.data_as(C.POINTER(C.c_int32))
    n_nbr, n_if, n_el = C.c_int(), C.c_int64(), C.c_int64()
    lib = L.lib()
    L.check(lib.zj_halo_plan_size(C.byref(d), pp, nparts, rank, C.byref(n_nbr), C.byref(n_if), C.byref(n_el)))
    nbr = np.empty(max(n_nbr.value, 1), dtype=np.int32)
    off = np.empty(n_nbr.value + 1, dtype=np.int64)
    face, mine, remote = (np.empty(max(n_if.value, 1), dtype=np.int64) for _ in range(3))
    elems = np.empty(n_el.value, dtype=np.int64)
    i64 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))
    L.check(lib.zj_halo_plan(C.byref(d), pp, nparts, rank, nbr.ctypes.data_as(C.POINTER(C.c_int32)), i64(off),
                             i64(face), i64(mine), i64(remote), i64(elems)))
    n = n_if.value
    return {"nbr": nbr[:n_nbr.value], "off": off, "face": face[:n], "mine": mine[:n], "remote": remote[:n],
            "elems": elems}


class PartitionedSolver:
    """The parts of a mesh as handles (one per part, each on devices[rank]
    or the current device), stepped together from this process; the state
    crosses the interface as the parts' slices of the whole mesh's
    [E][n_sp][4] array."""

    def __init__(self, mesh, params: L.Params, nparts: int = 2, part=None, devices=None):
        import torch
        lib = L.lib()
        self.part = partition(mesh, nparts) if part is None else np.ascontiguousarray(part, dtype=np.int32)
        self.nparts = nparts
        d, keep = mesh_desc(mesh)
        self.parts, self.elems = [], []
        prev = torch.cuda.current_device()
        for r in range(nparts):
            if devices is not None:
                torch.cuda.set_device(devices[r])
            h = C.c_void_p()
            L.check(lib.zj_solver_create_part(C.byref(d), C.byref(params),
                                              self.part.ctypes.data_as(C.POINTER(C.c_int32)), nparts, r,
                                              C.byref(h)))
            s = FRSolver.from_handle(h, params)
            ids = np.empty(s.n_elem, dtype=np.int64)
            L.check(lib.zj_part_elements(h, ids.ctypes.data_as(C.POINTER(C.c_int64))), h)
            self.parts.append(s)
            self.elems.append(ids)
        torch.cuda.set_device(prev)
        self.n_elem = mesh.n_elem
        self.n_sp = self.parts[0].n_sp
        self._arr = (C.c_void_p * nparts)(*[s.h for s in self.parts])

    def _ck(self, code):
        L.check(code, self.parts[0].h)

    def solution_point_coords(self) -> np.ndarray:
        out = np.empty((self.n_elem, self.n_sp, 2))
        for s, ids in zip(self.parts, self.elems):
            out[ids] = s.solution_point_coords()
        return out

    def copyToDevice(self, U: np.ndarray):
        for s, ids in zip(self.parts, self.elems):
            s.copyToDevice(np.ascontiguousarray(U[ids]))

    def copyToHost(self) -> np.ndarray:
        self.synchronize()
        out = np.empty((self.n_elem, self.n_sp, 4))
        for s, ids in zip(self.parts, self.elems):
            out[ids] = s.copyToHost()
        return out

    def advance(self, dt: float, nsteps: int = 1, sync: bool = True):
        self._ck(L.lib().zj_parts_step(self._arr, self.nparts, dt, nsteps))
        if sync:
            self.synchronize()

    def synchronize(self):
        self._ck(L.lib().zj_parts_synchronize(self._arr, self.nparts))

    def rhs(self, U: np.ndarray) -> np.ndarray:
        import torch
        Ud = [torch.from_numpy(np.ascontiguousarray(U[ids])).cuda() for ids in self.elems]
        Rd = [torch.empty_like(u) for u in Ud]
        torch.cuda.synchronize()
        ua = (C.c_void_p * self.nparts)(*[u.data_ptr() for u in Ud])
        ra = (C.c_void_p * self.nparts)(*[r.data_ptr() for r in Rd])
        self._ck(L.lib().zj_parts_rhs(self._arr, self.nparts, ua, ra))
        self.synchronize()
        out = np.empty((self.n_elem, self.n_sp, 4))
        for r, ids in zip(Rd, self.elems):
            out[ids] = r.cpu().numpy()
        return out

    def computeResidual(self) -> float:
        v = C.c_double()
        self._ck(L.lib().zj_parts_residual_norm(self._arr, self.nparts, C.byref(v)))
        return v.value

    def computeTimeStep(self) -> float:
        return min(s.computeTimeStep() for s in self.parts)

    def close(self):
        for s in self.parts:
            s.close()
        self.parts = []
