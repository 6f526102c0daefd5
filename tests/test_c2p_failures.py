"""Failure handling of the C2P chain and FixRecovery on crafted states
(the oracle; tests/test_gpu_failures.py checks the engine against it).

A state whose conserved energy or momentum is corrupted defeats Scheme2D and
is recovered by Scheme1Dvsq, the next link of the chain (invertor.cc:185-197).
A negative conserved density defeats the whole chain: the cell's flag drops
to 0 and FixRecovery (recovery_fixer.cc:52-115) replaces its primitives by the
mean of its four edge neighbours, or of its four diagonal neighbours when an
edge neighbour failed too, sets its velocity to zero and its flag to 1."""
import numpy as np

from pangu_b200 import abi
from parity_util import Case

RHO, ENY = 0, 1
CNT = {n: k for k, n in enumerate(abi.COUNTER_NAMES)}


def crafted(cells, var, value):
    """OT 32x32 (Minkowski, chainer) with the conserved variable var of the
    given interior cells (j, i offsets) set to value."""
    case = Case("ot_mc_laxf")
    base, _ = case.oracle_containers()
    case.oracle.calculate_conservative(base)
    s = case.geo.interior()
    idx = [(s[1].start + dj, s[2].start + di) for dj, di in cells]
    for j, i in idx:
        base.cons[0, var, 0, j, i] = value
    return case, base, idx


def test_chain_falls_back_to_1dvsq():
    case, base, idx = crafted([(5, 7)], ENY, 10.0)
    O = case.oracle
    O.reset_counters()
    O.recovery(base)
    c = O.counters()
    n = case.mesh.nx1 * case.mesh.nx2
    assert c[CNT["c2p_1dvsq"]] == 1 and c[CNT["c2p_2d"]] == n - 1 and c[CNT["c2p_fail"]] == 0
    assert base.flag[0, 0][idx[0]] == 1.0


def test_failed_cell_repaired_from_edge_neighbours():
    case, base, idx = crafted([(5, 7)], RHO, -1.0)
    O = case.oracle
    O.reset_counters()
    O.recovery(base)
    (j, i), = idx
    assert O.counters()[CNT["c2p_fail"]] == 1
    flags = base.flag[0, 0]
    assert flags[j, i] == 0.0 and (flags[case.geo.interior()[1:]] == 0).sum() == 1
    before = base.prim[0, :, 0].copy()
    O.fix_recovery(base)
    want = 0.25 * (before[:, j + 1, i] + before[:, j - 1, i] + before[:, j, i - 1] +
                   before[:, j, i + 1])
    want[2:5] = 0.0  # velocity reset
    np.testing.assert_array_equal(base.prim[0, :, 0, j, i], want)
    assert base.flag[0, 0, j, i] == 1.0 and O.counters()[CNT["fix_recovery"]] == 1


def test_adjacent_failures_use_diagonal_neighbours():
    case, base, idx = crafted([(5, 7), (5, 8)], RHO, -1.0)
    O = case.oracle
    O.reset_counters()
    O.recovery(base)
    assert O.counters()[CNT["c2p_fail"]] == 2
    before = base.prim[0, :, 0].copy()
    O.fix_recovery(base)
    for j, i in idx:  # each has a failed edge neighbour: diagonal mean
        want = 0.25 * (before[:, j + 1, i + 1] + before[:, j + 1, i - 1] +
                       before[:, j - 1, i + 1] + before[:, j - 1, i - 1])
        want[2:5] = 0.0
        np.testing.assert_array_equal(base.prim[0, :, 0, j, i], want)
    assert O.counters()[CNT["fix_recovery"]] == 2
