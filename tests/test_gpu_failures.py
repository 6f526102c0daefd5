"""The engine's C2P chain and FixRecovery on the crafted failing states of
tests/test_c2p_failures.py: flags, repaired primitives and counters equal
the oracle's bit for bit."""
import numpy as np
import pytest

from parity_util import field, to_device
from test_c2p_failures import ENY, RHO, crafted

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cells,var,value", [([(5, 7)], ENY, 10.0), ([(5, 7)], RHO, -1.0),
                                             ([(5, 7), (5, 8)], RHO, -1.0),
                                             ([(0, 0), (9, 3), (10, 3)], RHO, -1.0)])
def test_engine_failure_handling_matches_oracle(cells, var, value):
    import torch
    from pangu_b200.engine import Engine
    case, base, idx = crafted(cells, var, value)
    eng = Engine(case.params, case.mesh)
    dbase, _ = eng.new_containers()
    to_device(base, dbase)
    eng.reset_counters()
    case.oracle.reset_counters()
    case.oracle.recovery(base)
    eng.recovery(dbase)
    case.oracle.fix_recovery(base)
    eng.fix_recovery(dbase)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(field(dbase, "prim"), base.prim)
    np.testing.assert_array_equal(field(dbase, "flag"), base.flag)
    np.testing.assert_array_equal(eng.counters(), case.oracle.counters())
