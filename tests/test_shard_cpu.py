"""Block sharding on CPU: the halo plan and the message transfer.

The plan comes from the engine library's host code (pangu_shard_plan, no GPU).
The oracle's ghost exchange is the checker: the cells that cross ranks, moved
as halo messages in plan order, must receive exactly what one engine's
exchange gives them. The transfer itself runs over gloo between two and three
processes, with the same message layout as the device pack/unpack kernels
([entry][Nf primitives, flag]) and the dt all-reduce(min).
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from parity_util import Case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MESHES = ["ot_blocks", "torus3d_blocks", "cks_excise"]


def _plans(case, block_rank):
    from pangu_b200.shard import shard_plan
    n = int(block_rank.max()) + 1
    return [shard_plan(case.params, case.mesh, block_rank, r) for r in range(n)]


def _random_state(case, seed):
    rng = np.random.default_rng(seed)
    shape = case.oracle.new_containers()[0].prim.shape
    prim = rng.standard_normal(shape)
    flag = rng.integers(0, 2, size=(shape[0],) + shape[2:]).astype(np.float64)
    return prim, flag


def _oracle_exchange(case, prim, flag):
    base, _ = case.oracle.new_containers()
    base.prim[...] = prim
    base.flag[...] = flag
    case.oracle.exchange_ghosts(base)
    return np.array(base.prim), np.array(base.flag)


def pack(prim, flag, cells):
    """[entry][Nf primitives, flag] of the given whole-mesh cell offsets."""
    nb, nf = prim.shape[:2]
    pf, ff = prim.reshape(nb, nf, -1), flag.reshape(nb, -1)
    ncell = pf.shape[2]
    b, c = cells // ncell, cells % ncell
    buf = np.empty((len(cells), nf + 1))
    buf[:, :nf] = pf[b, :, c]
    buf[:, nf] = ff[b, c]
    return buf.ravel()


def unpack(prim, flag, cells, buf):
    nb, nf = prim.shape[:2]
    pf, ff = prim.reshape(nb, nf, -1), flag.reshape(nb, -1)
    ncell = pf.shape[2]
    b, c = cells // ncell, cells % ncell
    m = buf.reshape(len(cells), nf + 1)
    pf[b, :, c] = m[:, :nf]
    ff[b, c] = m[:, nf]


def _split(a, counts):
    o = np.concatenate([[0], np.cumsum(counts)])
    return [a[o[q]:o[q + 1]] for q in range(len(counts))]


@pytest.mark.parametrize("name", MESHES)
@pytest.mark.parametrize("nranks", [2, 3])
def test_plans_pair_up(name, nranks):
    case = Case(name)
    from pangu_b200.shard import block_ranks
    for br in (block_ranks(case.mesh, nranks),
               (np.arange(case.oracle.nb) % nranks).astype(np.int32)):
        plans = _plans(case, br)
        for r in range(nranks):
            assert plans[r][0][r] == plans[r][1][r] == 0  # nothing to itself
            for q in range(nranks):
                assert plans[r][0][q] == plans[q][1][r]
            # a rank sends only its own interior cells and fills only its own ghosts
            ncell = case.oracle.new_containers()[0].flag[0].size
            assert np.all(br[plans[r][2] // ncell] == r)
            assert np.all(br[plans[r][3] // ncell] == r)


@pytest.mark.parametrize("name", MESHES)
def test_every_block_its_own_rank_reproduces_the_exchange(name):
    """With one block per rank every exchange entry crosses ranks (no mesh
    here wraps a block onto itself), so the messages alone must give the
    whole ghost fill of the oracle's exchange."""
    case = Case(name)
    nb = case.oracle.nb
    br = np.arange(nb, dtype=np.int32)
    plans = _plans(case, br)
    prim, flag = _random_state(case, 7)
    ref_prim, ref_flag = _oracle_exchange(case, prim, flag)
    got_prim, got_flag = prim.copy(), flag.copy()
    for r in range(nb):
        recv_cells = _split(plans[r][3], plans[r][1])
        for q in range(nb):
            if plans[r][1][q]:
                send_cells = _split(plans[q][2], plans[q][0])[r]
                unpack(got_prim, got_flag, recv_cells[q], pack(prim, flag, send_cells))
    np.testing.assert_array_equal(got_prim, ref_prim)
    np.testing.assert_array_equal(got_flag, ref_flag)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, name, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    from parity_util import Case as C_
    from pangu_b200.shard import block_ranks, exchange_halos, shard_plan
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    case = C_(name)
    br = block_ranks(case.mesh, world)
    snd, rcv, sc, rc = shard_plan(case.params, case.mesh, br, rank)
    prim, flag = _random_state(case, 11)  # the same state on every rank
    width = prim.shape[1] + 1
    send = torch.from_numpy(pack(prim, flag, sc))
    recv = torch.full((int(rcv.sum()) * width,), np.nan, dtype=torch.float64)
    for w in exchange_halos(send, recv, snd.tolist(), rcv.tolist(), width):
        w.wait()
    got_prim, got_flag = np.full_like(prim, np.nan), np.full_like(flag, np.nan)
    unpack(got_prim, got_flag, rc, recv.numpy())
    np.savez(os.path.join(out, f"rank{rank}.npz"), prim=got_prim, flag=got_flag, cells=rc)
    local_dt = torch.tensor([1.0e-3 * (3 - rank)], dtype=torch.float64)
    dist.all_reduce(local_dt, op=dist.ReduceOp.MIN)
    with open(os.path.join(out, f"dt{rank}.txt"), "w") as f:
        f.write(repr(local_dt.item()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("ot_blocks", 2), ("torus3d_blocks", 3)])
def test_halo_transfer_over_gloo(tmp_path, name, world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, world, port, name, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    case = Case(name)
    prim, flag = _random_state(case, 11)
    ref_prim, ref_flag = _oracle_exchange(case, prim, flag)
    nb, nf = prim.shape[:2]
    total = 0
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        cells = d["cells"]
        total += len(cells)
        ncell = prim[0, 0].size
        b, c = cells // ncell, cells % ncell
        np.testing.assert_array_equal(d["prim"].reshape(nb, nf, -1)[b, :, c],
                                      ref_prim.reshape(nb, nf, -1)[b, :, c])
        np.testing.assert_array_equal(d["flag"].reshape(nb, -1)[b, c],
                                      ref_flag.reshape(nb, -1)[b, c])
        assert float(open(tmp_path / f"dt{r}.txt").read()) == 1.0e-3 * (3 - (world - 1))
    assert total > 0


def test_plan_rejects_bad_assignments():
    """pangu_shard_plan validates its arguments before any work (no GPU)."""
    import ctypes as C
    from pangu_b200 import abi
    from pangu_b200.engine import lib
    case = Case("ot_blocks")
    L = lib()
    nb = case.oracle.nb
    counts = (C.c_int64 * 4)()
    def plan(br, nranks, rank):
        a = np.ascontiguousarray(br, dtype=np.int32)
        return L.pangu_shard_plan(C.byref(case.params), C.byref(case.mesh),
                                  a.ctypes.data_as(C.POINTER(C.c_int32)), nranks, rank,
                                  counts, counts, None, None)
    ok = (np.arange(nb) % 2).astype(np.int32)
    assert plan(ok, 2, 0) == abi.PANGU_OK
    assert plan(ok, 2, 2) == abi.PANGU_EINVAL           # rank out of range
    assert plan(ok + 5, 2, 0) == abi.PANGU_EINVAL       # block on a rank that does not exist
    assert plan(ok, 0, 0) == abi.PANGU_EINVAL           # no ranks
    assert L.pangu_shard_plan(C.byref(case.params), C.byref(case.mesh), None, 2, 0, counts,
                              counts, None, None) == abi.PANGU_EINVAL
