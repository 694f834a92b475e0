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


# ---------------------------------------------------------------------------
# One process per GPU: a part stepped alone (zj_part_step); the caller's
# transport moves its cut-face rows at each exchange.

class _DeviceBytes:
    """A device byte range as an object torch can view without copying
    (the CUDA array interface)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 2}


def device_bytes(ptr: int, nbytes: int):
    """torch uint8 view of nbytes of device memory at ptr."""
    import torch
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device="cuda")


class PartProcess:
    """Part `rank` of a partition as this process's handle (the reference's
    rank with its MeshPartitioner slice and MPICommunicator halo).
    `advance(dt, nsteps, exchange)` steps it; at each exchange the library
    calls exchange(kind, row_bytes, send_ptr, recv_ptr, stream_ptr) with the
    part's rows for every neighbour in send (rows [off[i], off[i+1]) of
    `plan` for neighbour plan["nbr"][i]); it must fill recv with the
    neighbours' rows for this part in the same layout (see nccl_exchange and
    LocalExchange)."""

    def __init__(self, mesh, params: L.Params, part: np.ndarray, rank: int):
        lib = L.lib()
        self.part = np.ascontiguousarray(part, dtype=np.int32)
        self.nparts = int(self.part.max()) + 1
        self.rank = rank
        d, keep = mesh_desc(mesh)
        h = C.c_void_p()
        L.check(lib.zj_solver_create_part(C.byref(d), C.byref(params),
                                          self.part.ctypes.data_as(C.POINTER(C.c_int32)), self.nparts, rank,
                                          C.byref(h)))
        self.solver = FRSolver.from_handle(h, params)
        self.plan = halo_plan(mesh, self.part, rank)
        self.elems = self.plan["elems"]
        self._err = None

    def advance(self, dt: float, nsteps: int, exchange):
        def cb(user, kind, row_bytes, send, recv, stream):
            try:
                return int(exchange(kind, row_bytes, send or 0, recv or 0, stream or 0) or 0)
            except Exception as e:   # reported after the step returns
                self._err = e
                return 1
        fn = L.EXCHANGE_FN(cb)
        code = L.lib().zj_part_step(self.solver.h, dt, nsteps, fn, None)
        if self._err is not None:
            err, self._err = self._err, None
            raise err
        L.check(code, self.solver.h)

    def copyToDevice(self, U_global: np.ndarray):
        self.solver.copyToDevice(np.ascontiguousarray(U_global[self.elems]))

    def copyToHost(self) -> np.ndarray:
        return self.solver.copyToHost()

    def close(self):
        self.solver.close()


def nccl_exchange(plan: dict, group=None):
    """exchange for PartProcess.advance over torch.distributed (NCCL, one
    process per GPU): per neighbour a send of this part's block and a receive
    of the neighbour's, batched, ordered on the part's stream."""
    import torch
    import torch.distributed as dist
    nbr, off = [int(q) for q in plan["nbr"]], [int(o) for o in plan["off"]]

    def fn(kind, row_bytes, send_ptr, recv_ptr, stream_ptr):
        n = off[-1] * row_bytes if off else 0
        if n == 0:
            return 0
        send, recv = device_bytes(send_ptr, n), device_bytes(recv_ptr, n)
        with torch.cuda.stream(torch.cuda.ExternalStream(stream_ptr)):
            ops = []
            for i, q in enumerate(nbr):
                a, b = off[i] * row_bytes, off[i + 1] * row_bytes
                ops.append(dist.P2POp(dist.isend, send[a:b], q, group))
                ops.append(dist.P2POp(dist.irecv, recv[a:b], q, group))
            for w in dist.batch_isend_irecv(ops):
                w.wait()   # the part's stream waits for the transfers
        return 0
    return fn


class LocalExchange:
    """The transport for parts stepped by threads of one process (all on
    one device): each thread's exchange publishes its send block, waits for
    the others, copies its neighbours' blocks for it into its receive buffer
    and waits again before returning (the senders' buffers are reused by
    their next exchange).  A failed or missing part breaks the barrier after
    `timeout` seconds and the steps end with ZJ_ERR_IO."""

    def __init__(self, plans: list, timeout: float = 60.0):
        import threading
        self.plans = plans
        self.sent = {}
        self.barrier = threading.Barrier(len(plans), timeout=timeout)

    def for_rank(self, rank: int):
        import torch
        plan = self.plans[rank]

        def fn(kind, row_bytes, send_ptr, recv_ptr, stream_ptr):
            torch.cuda.ExternalStream(stream_ptr).synchronize()   # the send block is written
            self.sent[rank] = send_ptr
            self.barrier.wait()
            for i, q in enumerate(plan["nbr"]):
                pq = self.plans[int(q)]
                j = int(np.nonzero(pq["nbr"] == rank)[0][0])
                cnt = int(plan["off"][i + 1] - plan["off"][i])
                assert cnt == int(pq["off"][j + 1] - pq["off"][j])
                src = device_bytes(self.sent[int(q)] + int(pq["off"][j]) * row_bytes, cnt * row_bytes)
                dst = device_bytes(recv_ptr + int(plan["off"][i]) * row_bytes, cnt * row_bytes)
                dst.copy_(src)
            torch.cuda.synchronize()
            self.barrier.wait()
            return 0
        return fn
