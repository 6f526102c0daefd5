"""The oracle's per-cell restatement against golden vectors produced by the
reference's own per-cell code (tests/golden/make_golden.py). Both are built
with g++ -O2 -ffp-contract=off, so the comparison is bit-exact -- except for
outputs that pass through pow/exp/log: the reference's host build calls the
C library's (which misrounds a few per cent of results by one ulp), the
oracle and the engine the correctly rounded double-double routines of
pangu_b200/csrc/pgmath.h. Those outputs are held to two ulp."""
import os

import numpy as np
import pytest

import pyoracle as po

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "cell_golden.npz"))
O = po.CellAPI(po.lib(), "or_")


def eq(a, b):
    np.testing.assert_array_equal(np.asarray(a), np.asarray(b))


def ulp2(a, b):
    np.testing.assert_allclose(np.asarray(a), np.asarray(b), rtol=2 * 2.0 ** -52, atol=0)


def test_metric_and_christoffel():
    for n, (mt, x, ah) in enumerate(zip(G["m_type"], G["m_x"], G["m_ah"])):
        gcov, gcon, gdet = O.metric(int(mt), x, *ah)
        eq(gcov, G["m_gcov"][n]); eq(gcon, G["m_gcon"][n]); eq(gdet, G["m_gdet"][n])
        eq(O.christoffel(int(mt), x, *ah), G["m_conn"][n])


def test_flux_and_fast_speed():
    for n in range(len(G["f_P"])):
        m = G["f_idx"][n]
        d = int(G["f_dir"][n])
        args = (G["f_gam"][n], G["f_P"][n], G["m_gcov"][m], G["m_gcon"][m])
        eq(O.flux(*args, G["m_gdet"][m], d), G["f_flux"][n])
        eq(O.fast_speed(*args, max(d, 1)), G["f_speed"][n])


def test_reconstruction():
    for n, q in enumerate(G["r_q"]):
        eq(O.recon(1, q), G["r_mc"][n])
        eq(O.recon(0, q), G["r_ppm4"][n])


@pytest.mark.parametrize("scheme", [0, 1, 2, 3], ids=["2d", "1dvsq", "1d", "kastaun"])
def test_c2p_schemes(scheme):
    sel = np.nonzero(G["c_scheme_status"][:, 0] == scheme)[0]
    assert len(sel) > 100
    for n in sel:
        m = G["c_midx"][n]
        st, pr = O.invert(scheme, G["c_U"][n], G["c_Pin"][n], G["c_gam"][n],
                          G["m_gcov"][m], G["m_gcon"][m])
        assert st == G["c_scheme_status"][n, 1]
        ulp2(pr, G["c_Pout"][n])


def test_heating_and_clamp():
    for n in range(len(G["h_out"])):
        ulp2(O.heating(G["h_params"][n], G["h_flags"][n], G["h_cell"][n]), G["h_out"][n])
    for n, (t, e) in enumerate(G["k_in"]):
        eq(O.clamp(1e-3, 1e3, t, e), G["k_out"][n])
