"""One mesh spread over several GPUs by blocks.

The reference runs a mesh's blocks on several MPI ranks under Parthenon: every
rank steps its own blocks, ghost cells between ranks are filled from the
neighbour's interior at send time (the exchange at ideal_grmhd.cc:78), and
EstimateTimestepMesh reduces dt over all blocks
(initialization/timestep_estimation.cc:13-102). Here every rank is one process
with one GPU and one shard engine (``pangu_shard_create``). A stage is three
engine calls; between the first and the last the halo messages move with
torch.distributed point-to-point calls (NCCL between GPUs, gloo on CPU) while
the middle part (source, Recovery, heating) runs on the GPU. dt is reduced with
an all-reduce(min), the one collective of a cycle besides the halo transfer.

The result is bit-identical to the same mesh stepped by one engine: the
exchange copies the same values in the same order, and the minimum over
blocks does not depend on how the blocks are grouped.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .engine import RK2_BETA, Engine, EngineError, _check, _torch, lib
from .params import (ParameterInput, engine_precision, mesh_struct, params_struct,
                     process_packages)


def block_ranks(mesh: abi.Mesh, nranks: int) -> np.ndarray:
    """Contiguous split of the block lattice (x1 fastest) into nranks runs of
    nearly equal length: block b goes to rank b * nranks // NB."""
    nb = mesh.nbx1 * mesh.nbx2 * mesh.nbx3
    if not 1 <= nranks <= nb:
        raise ValueError(f"{nranks} ranks for {nb} blocks: every rank needs a block")
    return (np.arange(nb) * nranks // nb).astype(np.int32)


def shard_plan(params: abi.Params, mesh: abi.Mesh, block_rank, rank: int):
    """The halo plan of one rank, computed on the host (no GPU needed).

    Returns (send_counts, recv_counts, send_cells, recv_cells): entries per
    peer and the cells in message order, as offsets b * ncell + cell of the
    whole mesh's block b."""
    L = lib()
    br = np.ascontiguousarray(block_rank, dtype=np.int32)
    nranks = int(br.max()) + 1
    snd, rcv = np.zeros(nranks, np.int64), np.zeros(nranks, np.int64)
    i32 = br.ctypes.data_as(C.POINTER(C.c_int32))
    i64 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))  # noqa: E731
    _check(L.pangu_shard_plan(C.byref(params), C.byref(mesh), i32, nranks, rank, i64(snd),
                              i64(rcv), None, None), "pangu_shard_plan")
    sc, rc = np.zeros(int(snd.sum()), np.int64), np.zeros(int(rcv.sum()), np.int64)
    _check(L.pangu_shard_plan(C.byref(params), C.byref(mesh), i32, nranks, rank, i64(snd),
                              i64(rcv), i64(sc), i64(rc)), "pangu_shard_plan")
    return snd, rcv, sc, rc


def message_offsets(counts, width: int) -> np.ndarray:
    """Start of each peer's message in a buffer of `width` values per entry
    (peers in rank order), plus the end."""
    return np.concatenate([[0], np.cumsum(np.asarray(counts, np.int64) * width)])


def exchange_halos(send, recv, send_counts, recv_counts, width: int, group=None):
    """Posts every peer's halo message: send[...] of peer q goes to rank q,
    recv[...] of peer q comes from rank q. Returns the requests; the caller
    waits on them (on a GPU, waiting orders the current stream after the
    transfer, so work queued meanwhile overlaps it)."""
    import torch.distributed as dist
    so, ro = message_offsets(send_counts, width), message_offsets(recv_counts, width)
    ops = []
    for q in range(len(send_counts)):
        if send_counts[q]:
            ops.append(dist.P2POp(dist.isend, send[so[q]:so[q + 1]], q, group))
    for q in range(len(recv_counts)):
        if recv_counts[q]:
            ops.append(dist.P2POp(dist.irecv, recv[ro[q]:ro[q + 1]], q, group))
    return dist.batch_isend_irecv(ops) if ops else []


class Shard:
    """Rank `rank`'s blocks of a mesh: a shard engine, its two stage
    containers, halo buffers and the dt policy of the job.

    Local block q is the q-th block of the lattice that block_rank assigns
    to this rank."""

    def __init__(self, pin: ParameterInput, nranks: int, rank: int, device=0, block_rank=None):
        torch = _torch()
        self.pin = pin
        self.packages = process_packages(pin)
        self.params = params_struct(self.packages)
        self.params.precision = engine_precision(pin)
        self.mesh = mesh_struct(pin)
        self.nranks, self.rank = nranks, rank
        self.block_rank = (block_ranks(self.mesh, nranks) if block_rank is None
                           else np.asarray(block_rank, np.int32))
        self.blocks = np.flatnonzero(self.block_rank == rank)
        self.engine = Engine(self.params, self.mesh, device,
                             shard=(self.block_rank, nranks, rank))
        self.base, self.one = self.engine.new_containers()
        dev = self.engine.device
        self.width = self.engine.nf + 1
        self.send_counts, self.recv_counts = self.engine.halo_counts(nranks)
        self.send = torch.zeros(sum(self.send_counts) * self.width, dtype=torch.float64,
                                device=dev)
        self.recv = torch.zeros(sum(self.recv_counts) * self.width, dtype=torch.float64,
                                device=dev)
        self.dt_init = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
        self.dt_factor = pin.get_or_add_real("parthenon/time", "dt_factor", 2.0)
        self.dt = torch.full((1,), self.dt_init, dtype=torch.float64, device=dev)
        self.dt_est = torch.zeros(1, dtype=torch.float64, device=dev)
        self.cycle = 0

    def message(self, buf, counts, peer):
        """The slice of a send or receive buffer that holds peer's message."""
        o = message_offsets(counts, self.width)
        return buf[o[peer]:o[peer + 1]]

    def load(self, prim):
        """This rank's blocks of the whole mesh's initial primitives
        ([block][var][k][j][i]); ghosts are filled by start()."""
        torch = _torch()
        local = np.ascontiguousarray(np.asarray(prim)[self.blocks])
        self.base.prim.copy_(torch.as_tensor(local, device=self.engine.device)
                             .to(self.base.prim.dtype))

    def pack_initial(self):
        self.engine.halo_pack(self.base, self.send)

    def start(self):
        """After the initial halo cells are unpacked: local exchange, physical
        BCs and container "1" = "base"."""
        self.engine.halo_unpack(self.base, self.recv)
        self.engine.job_start(0, self.base, self.one)

    def begin(self, st):
        self.engine.stage_begin(st, self.base, self.one, RK2_BETA[st % 2], self.dt, self.send)

    def middle(self, st):
        self.engine.stage_middle(st, self.base, self.one, RK2_BETA[st % 2], self.dt)

    def end(self, st):
        self.engine.stage_end(st, self.base, self.one, self.recv,
                              self.dt_est if st == 2 else None)

    def update_dt(self):
        self.engine.update_dt(self.dt, self.dt_est, self.dt_factor)

    def primitives(self) -> np.ndarray:
        """This rank's blocks, FP64 [local block][var][k][j][i]."""
        return self.base.prim.double().cpu().numpy()

    def counters(self) -> np.ndarray:
        return self.engine.counters()


class ShardedSimulation(Shard):
    """A Shard stepped over torch.distributed, one process per GPU (rank r of
    the group drives GPU `device`, by default its local rank)."""

    def __init__(self, pin: ParameterInput, group=None, device=None, block_rank=None):
        import os

        import torch.distributed as dist
        if not dist.is_initialized():
            raise EngineError("ShardedSimulation needs an initialised process group")
        self.group = group
        rank, nranks = dist.get_rank(group), dist.get_world_size(group)
        if device is None:
            device = int(os.environ.get("LOCAL_RANK", rank))
        super().__init__(pin, nranks, rank, device, block_rank)

    def _transfer(self):
        return exchange_halos(self.send, self.recv, self.send_counts, self.recv_counts,
                              self.width, self.group)

    def set_primitives(self, prim):
        """Initial primitives of the whole mesh (every rank passes the same
        array); the ghost fill crosses ranks like a stage's exchange."""
        self.load(prim)
        self.pack_initial()
        for w in self._transfer():
            w.wait()
        self.start()

    def step(self, fixed_dt: bool = False):
        """One rk2 cycle of the whole mesh; afterwards every rank holds
        dt = min(dt_factor * dt, min over all blocks of the estimate)."""
        import torch.distributed as dist
        for st in (1, 2):
            self.begin(st)
            works = self._transfer()
            self.middle(st)
            for w in works:
                w.wait()
            self.end(st)
        if not fixed_dt:
            dist.all_reduce(self.dt_est, op=dist.ReduceOp.MIN, group=self.group)
            self.update_dt()
        self.cycle += 1

    def total_counters(self) -> np.ndarray:
        """The counters summed over all ranks."""
        import torch
        import torch.distributed as dist
        t = torch.as_tensor(self.counters().astype(np.int64), device=self.engine.device)
        dist.all_reduce(t, group=self.group)
        return t.cpu().numpy().astype(np.uint64)
