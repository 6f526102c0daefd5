"""Generates tests/golden/cell_golden.npz from the REFERENCE's own code.

The reference's per-cell headers (pangu/src/metric, physics, interpolation,
recovery/scheme_*.h) are compiled from where they lie by oracle/build.py
(through the stand-in headers of oracle/refshim) into
oracle/_ref/libpangu_refcell.so. This script feeds that library seeded
inputs and stores inputs and outputs. The fixture pins the oracle's per-cell
restatement (tests/test_oracle_golden.py) on machines without the reference
sources. Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402

SEED = 20261203
A_SPIN, H_MKS = 0.9375, 0.7


def metric_points(rng, n):
    """(mtype, x[4]) samples away from coordinate singularities."""
    pts = []
    for _ in range(n):
        mt = int(rng.integers(0, 4))
        if mt in (1, 3):  # BL / MKS: r = exp(x1) in [1.65, 33] (outside BL horizon)
            x = [0.0, rng.uniform(0.5, 3.5), rng.uniform(-0.98, 0.98), rng.uniform(-np.pi, np.pi)]
        elif mt == 2:  # CKS: r in [1.5, 20]
            while True:
                x = [0.0, *rng.uniform(-20, 20, 3)]
                if np.linalg.norm(x[1:]) > 1.5:
                    break
        else:
            x = [0.0, *rng.uniform(-3, 3, 3)]
        pts.append((mt, np.array(x)))
    return pts


def random_prims(rng, hard=False):
    P = np.zeros(10)
    P[0] = 10 ** rng.uniform(-6, 1)
    P[1] = P[0] * 10 ** rng.uniform(-6 if not hard else -9, 1)
    P[2:5] = rng.normal(size=3) * 10 ** rng.uniform(-2, 0.8 if hard else 0.3)
    P[5:8] = rng.normal(size=3) * 10 ** rng.uniform(-3, 1.0 if hard else 0.3) * np.sqrt(P[0])
    P[8] = 10 ** rng.uniform(-3, 1)
    P[9] = P[8] * rng.uniform(0.001, 0.9)
    return P


def main():
    rng = np.random.default_rng(SEED)
    R = po.CellAPI(po.reflib(), "ref_")
    out = {}

    # --- metric + Christoffel ------------------------------------------------
    pts = metric_points(rng, 240)
    ab = [(A_SPIN, H_MKS) if i % 3 else (0.0, 0.0) for i in range(len(pts))]
    out["m_type"] = np.array([p[0] for p in pts], dtype=np.int32)
    out["m_x"] = np.array([p[1] for p in pts])
    out["m_ah"] = np.array(ab)
    gcov, gcon, gdet, conn = [], [], [], []
    for (mt, x), (a, h) in zip(pts, ab):
        g1, g2, d = R.metric(mt, x, a, h)
        gcov.append(g1); gcon.append(g2); gdet.append(d)
        conn.append(R.christoffel(mt, x, a, h))
    out["m_gcov"], out["m_gcon"] = np.array(gcov), np.array(gcon)
    out["m_gdet"], out["m_conn"] = np.array(gdet), np.array(conn)

    # --- fluxes and fast speeds at those metric points ------------------------
    gams = [5.0 / 3.0, 4.0 / 3.0, 2.0]
    fP, fdir, fgam, fidx, fout, sout = [], [], [], [], [], []
    for n in range(len(pts)):
        for d in range(4):
            P = random_prims(rng, hard=(n % 5 == 0))
            gam = gams[(n + d) % 3]
            fP.append(P); fdir.append(d); fgam.append(gam); fidx.append(n)
            fout.append(R.flux(gam, P, gcov[n], gcon[n], gdet[n], d))
            sout.append(R.fast_speed(gam, P, gcov[n], gcon[n], max(d, 1)))
    out["f_P"], out["f_dir"] = np.array(fP), np.array(fdir, dtype=np.int32)
    out["f_gam"], out["f_idx"] = np.array(fgam), np.array(fidx, dtype=np.int32)
    out["f_flux"], out["f_speed"] = np.array(fout), np.array(sout)

    # --- reconstruction -------------------------------------------------------
    qs = []
    for n in range(400):
        kind = n % 4
        if kind == 0:
            q = rng.normal(size=5)
        elif kind == 1:
            q = np.sort(rng.normal(size=5)) * (1 if n % 8 < 4 else -1)
        elif kind == 2:
            q = np.full(5, rng.normal())
            q[rng.integers(0, 5)] += rng.normal() * 1e-3
        else:
            q = np.array([0, 1, 3, 1, 0], float) * rng.uniform(0.1, 10)
        qs.append(q)
    out["r_q"] = np.array(qs)
    out["r_mc"] = np.array([R.recon(1, q) for q in qs])
    out["r_ppm4"] = np.array([R.recon(0, q) for q in qs])

    # --- conservative-to-primitive: all four schemes --------------------------
    iU, iG, iS, iPin, iPout, imt = [], [], [], [], [], []
    for n in range(len(pts)):
        mt, x = pts[n]
        if mt == 2 and np.linalg.norm(x[1:]) < 2.5:
            continue
        if not (-gcon[n][0] > 0):  # no lapse (inside an ergoregion of the map)
            continue
        for rep in range(2):
            P = random_prims(rng, hard=(rep == 1))
            gam = gams[(n + rep) % 3]
            P[8] = (gam - 1.0) * P[1] * P[0] ** (-gam)  # consistent entropy
            C = R.flux(gam, P, gcov[n], gcon[n], gdet[n], 0)
            sg = np.sqrt(abs(gdet[n]))
            alpha = 1.0 / np.sqrt(-gcon[n][0])
            ag = alpha * (1.0 / sg)
            U = np.zeros(9)
            U[0] = ag * C[0]
            U[1] = ag * (C[1] - C[0])
            U[2:5] = ag * C[2:5]
            U[5:8] = ag * C[5:8]
            U[8] = ag * C[8]
            guess = np.zeros(9)
            pert = 1.0 + 0.05 * rng.normal(size=5) * (0 if rep == 0 and n % 2 else 1)
            guess[0:5] = P[0:5] * pert
            guess[5:8] = alpha * C[5:8] * (1.0 / sg)
            guess[8] = P[8] * (1.0 + 0.02 * rng.normal())
            for sch in range(4):
                st, pr = R.invert(sch, U, guess, gam, gcov[n], gcon[n])
                iU.append(U); iG.append(gam); iS.append((sch, st)); iPin.append(guess)
                iPout.append(pr); imt.append(n)
    out["c_U"], out["c_gam"] = np.array(iU), np.array(iG)
    out["c_scheme_status"] = np.array(iS, dtype=np.int32)
    out["c_Pin"], out["c_Pout"] = np.array(iPin), np.array(iPout)
    out["c_midx"] = np.array(imt, dtype=np.int32)

    # --- electron heating and the entropy clamp -------------------------------
    hp_l, hf_l, hc_l, ho_l = [], [], [], []
    for n in range(600):
        model = n % 6
        hp = [rng.choice([5 / 3, 4 / 3]), 5 / 3, 4 / 3, 0.1, 1e-3, 1e3]
        flags = [model, int(rng.integers(0, 2)), int(rng.integers(0, 2)), int(rng.integers(0, 2))]
        rho = 10 ** rng.uniform(-5, 0)
        cell = [rho, rho * 10 ** rng.uniform(-4, 0), rho * 10 ** rng.uniform(-3, 1),
                10 ** rng.uniform(-3, 0), 10 ** rng.uniform(-3, 0), 10 ** rng.uniform(-4, -1)]
        hp_l.append(hp); hf_l.append(flags); hc_l.append(cell)
        ho_l.append(R.heating(hp, flags, cell))
    out["h_params"], out["h_flags"] = np.array(hp_l), np.array(hf_l, dtype=np.int32)
    out["h_cell"], out["h_out"] = np.array(hc_l), np.array(ho_l)
    cl_in = rng.uniform(-1, 2, size=(200, 2)) * np.array([1.0, 1.0])
    out["k_in"] = cl_in
    out["k_out"] = np.array([R.clamp(1e-3, 1e3, t, e) for t, e in cl_in])

    path = os.path.join(HERE, "cell_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
