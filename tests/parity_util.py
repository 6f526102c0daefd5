"""Shared helpers of the parity tests: cases, containers on both sides,
relative L1 norms. Test infrastructure."""
from __future__ import annotations

import numpy as np

from pangu_b200 import params as prm
from pangu_b200 import problems

import pyoracle as po


CASES = {
    # name: (problem, kwargs, param overrides)
    "ot_mc_laxf": ("ot", dict(n=32), {}),
    "ot_ppm4_hll_heat": ("ot", dict(n=32), {("core", "limiter"): "ppm4",
                                            ("core", "riemann_solver"): "hll",
                                            ("core", "enable_heating"): True,
                                            ("parthenon/mesh", "nghost"): 3}),
    "ot_blocks": ("ot", dict(n=32, nblock=16), {}),
    "bw_hll": ("bw", dict(n=128), {}),
    "torus_ppm4_laxf": ("torus", dict(nx1=64, nx2=32), {}),
    "torus_mc_hll": ("torus", dict(nx1=64, nx2=32, limiter="mc", riemann="hll"), {}),
    "torus_robuster": ("torus", dict(nx1=48, nx2=24), {("core", "recovery"): "robuster"}),
    "torus_kawazura": ("torus", dict(nx1=48, nx2=24), {("electron", "model"): "kawazura"}),
    "torus3d_blocks": ("torus", dict(nx1=32, nx2=16, nx3=8, bx=(16, 8, 4)), {}),
    "torus3d_hll": ("torus", dict(nx1=32, nx2=16, nx3=8, bx=(16, 8, 8), riemann="hll"), {}),
    "torus_bl": ("torus", dict(nx1=48, nx2=24), {("metric", "type"): "bl"}),
    "cks_excise": ("cks", dict(n=16, nblock=8), {}),
}


class Case:
    def __init__(self, name, extra=None):
        """extra: more (block, key) -> value settings of the input, applied
        after the case's own (e.g. mesh extents)."""
        problem, kw, over = CASES[name]
        pin, gen = problems.make_problem(problem, **kw)
        for (blk, key), v in {**over, **(extra or {})}.items():
            pin.set(blk, key, v)
        self.name = name
        self.pin = pin
        self.packages = prm.process_packages(pin)
        self.params = prm.params_struct(self.packages)
        self.mesh = prm.mesh_struct(pin)
        self.geo = problems.Geometry(self.mesh)
        if (("metric", "type") in over) and over[("metric", "type")] == "bl":
            # the BL map has its horizon at r ~ 1.35: start the grid outside
            self.mesh.x1min = 0.7
            self.geo = problems.Geometry(self.mesh)
        self.prim0 = gen(self.geo, self.packages, pin)
        self.oracle = po.Oracle(self.params, self.mesh)

    def oracle_containers(self):
        base, one = self.oracle.new_containers()
        base.prim[...] = self.prim0
        self.oracle.exchange_ghosts(base)
        self.oracle.apply_boundary_conditions(base)
        one.prim[...] = base.prim
        one.cons[...] = base.cons
        return base, one


def to_device(host, dev):
    """Copies every field of a host container into a device container."""
    import torch
    for f in ("prim", "cons", "flux1", "flux2", "flux3", "alfven", "efield", "flag"):
        getattr(dev, f).copy_(torch.from_numpy(np.ascontiguousarray(getattr(host, f))))


def field(dev, name):
    return getattr(dev, name).cpu().numpy()


def interior(geo, a):
    """Interior view of a [NB][NF][k][j][i] (or [NB][k][j][i]) array."""
    s = geo.interior()
    if a.ndim == 5:
        return a[:, :, s[0], s[1], s[2]]
    return a[:, s[0], s[1], s[2]]


def rel_l1(a, b, axis_field=1, vectors=((2, 5), (5, 8))):
    """Per-field relative L1 norm sum|a-b| / sum|b| (fields along axis 1).

    A component of a vector field (momentum/velocity: fields 2-4, magnetic
    field: 5-7 when present) is normalised by the L1 norm of the whole
    vector: a component that vanishes analytically (B^3 of an axisymmetric
    torus, u^3 of a planar flow) holds only rounding noise, which has no
    meaningful relative size of its own."""
    nf = a.shape[axis_field]
    a = np.moveaxis(a, axis_field, 0).reshape(nf, -1)
    b = np.moveaxis(b, axis_field, 0).reshape(nf, -1)
    num = np.abs(a - b).sum(axis=1)
    den = np.abs(b).sum(axis=1)
    if nf >= 9:
        for lo, hi in vectors:
            den[lo:hi] = np.maximum(den[lo:hi], den[lo:hi].sum())
    elif nf >= 5:
        den[2:5] = np.maximum(den[2:5], den[2:5].sum())
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def div_b_corner(geo, cons, nf_bx=5):
    """Corner-centred divergence of the conserved field (2D, x1-x2), the
    quantity flux-CT keeps at roundoff. Returns an array over interior
    corners."""
    s = geo.interior()
    B1 = cons[:, nf_bx + 0, 0]
    B2 = cons[:, nf_bx + 1, 0]
    js, je = s[1].start, s[1].stop
    is_, ie = s[2].start, s[2].stop
    dx1, dx2 = geo.dx[0], geo.dx[1]
    b1 = B1[:, js - 1:je, is_ - 1:ie]
    b2 = B2[:, js - 1:je, is_ - 1:ie]
    div = ((b1[:, 1:, 1:] + b1[:, :-1, 1:]) - (b1[:, 1:, :-1] + b1[:, :-1, :-1])) / (2 * dx1) + \
          ((b2[:, 1:, 1:] + b2[:, 1:, :-1]) - (b2[:, :-1, 1:] + b2[:, :-1, :-1])) / (2 * dx2)
    return div[:, 1:, 1:]
