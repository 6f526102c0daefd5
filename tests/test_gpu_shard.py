"""Block sharding of one mesh over several engines, on one GPU.

Every rank's shard engine runs in this process on cuda:0 and the halo
messages are plain device copies between the shards' buffers, so no kernel
waits on another. The sharded mesh must equal the same mesh stepped by one
engine bit for bit: primitives, conserved variables, flags, dt and the summed
counters, for contiguous and interleaved block assignments, 2D and 3D, FP64
and the mixed form.
"""
import numpy as np
import pytest

from parity_util import Case

pytestmark = pytest.mark.gpu


def _transfer(shards):
    for r, dst in enumerate(shards):
        for q, src in enumerate(shards):
            n = dst.recv_counts[q]
            assert src.send_counts[r] == n
            if n:
                dst.message(dst.recv, dst.recv_counts, q).copy_(
                    src.message(src.send, src.send_counts, r))


def _run_sharded(pin, prim0, nranks, steps, block_rank=None):
    import torch
    from pangu_b200.shard import Shard
    shards = [Shard(pin, nranks, r, block_rank=block_rank) for r in range(nranks)]
    for sh in shards:
        sh.load(prim0)
        sh.pack_initial()
    _transfer(shards)
    for sh in shards:
        sh.start()
    for _ in range(steps):
        for st in (1, 2):
            for sh in shards:
                sh.begin(st)
            _transfer(shards)
            for sh in shards:
                sh.middle(st)
            for sh in shards:
                sh.end(st)
        est = min(sh.dt_est.item() for sh in shards)
        for sh in shards:
            sh.dt_est.fill_(est)
            sh.update_dt()
    torch.cuda.synchronize()
    return shards


def _run_single(pin, prim0, steps):
    import torch
    from pangu_b200.engine import Simulation
    sim = Simulation(pin)
    sim.set_primitives(prim0)
    for _ in range(steps):
        sim.step()
    torch.cuda.synchronize()
    return sim


def _assemble(shards, name, nb):
    parts = [getattr(sh.base, name).double().cpu().numpy() for sh in shards]
    out = np.empty((nb,) + parts[0].shape[1:])
    for sh, a in zip(shards, parts):
        out[sh.blocks] = a
    return out


def _check_equal(sim, shards):
    nb = sim.engine.nb
    for name in ("prim", "cons", "flag"):
        np.testing.assert_array_equal(_assemble(shards, name, nb),
                                      getattr(sim.base, name).double().cpu().numpy(), err_msg=name)
    assert all(sh.dt.item() == sim.dt.item() for sh in shards)
    total = sum(sh.counters().astype(np.int64) for sh in shards)
    np.testing.assert_array_equal(total, sim.engine.counters().astype(np.int64))


@pytest.mark.parametrize("name,nranks,assign", [
    ("ot_blocks", 2, "contiguous"), ("ot_blocks", 3, "contiguous"),
    ("ot_blocks", 4, "interleaved"), ("torus3d_blocks", 3, "contiguous"),
    ("torus3d_blocks", 2, "interleaved"), ("cks_excise", 2, "contiguous")])
def test_sharded_mesh_matches_one_engine(name, nranks, assign):
    case = Case(name)
    nb = case.mesh.nbx1 * case.mesh.nbx2 * case.mesh.nbx3
    br = None if assign == "contiguous" else (np.arange(nb) % nranks).astype(np.int32)
    steps = 3
    sim = _run_single(case.pin, case.prim0, steps)
    shards = _run_sharded(case.pin, case.prim0, nranks, steps, br)
    assert sum(sum(sh.recv_counts) for sh in shards) > 0
    _check_equal(sim, shards)


def test_sharded_torus_2d_and_mixed():
    from pangu_b200 import params as prm
    from pangu_b200 import problems
    for precision in ("fp64", "mixed"):
        pin, gen = problems.make_problem("torus", nx1=64, nx2=32, bx=(16, 16, 1), seed=3)
        pin.set("b200", "precision", precision)
        mesh = prm.mesh_struct(pin)
        prim0 = gen(problems.Geometry(mesh), prm.process_packages(pin), pin)
        sim = _run_single(pin, prim0, 3)
        shards = _run_sharded(pin, prim0, 3, 3)
        _check_equal(sim, shards)


def test_shard_refuses_the_one_call_stage():
    import torch
    from pangu_b200.engine import EngineError
    from pangu_b200.shard import Shard
    case = Case("ot_blocks")
    sh = Shard(case.pin, 2, 0)
    with pytest.raises(EngineError):
        sh.engine.stage(1, sh.base, sh.one, 0.5, sh.dt)
    with pytest.raises(EngineError):  # a shard with halo entries needs its buffers
        sh.engine.stage_begin(1, sh.base, sh.one, 0.5, sh.dt, None)
    torch.cuda.synchronize()
