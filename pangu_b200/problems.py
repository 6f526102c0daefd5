"""Initial conditions of the benchmark problems (host side, numpy).

Each generator fills the interior primitives of every meshblock; ghost cells
are then filled by the engine's initial boundary fill (exchange + physical
BCs), as Parthenon does after ``ProblemGenerator``. Both the engine and the
CPU oracle step from the same arrays.

* ``orszag_tang``: the classical Orszag-Tang vortex on [0,1]^2 with
  rho = 25/(36 pi), p = 5/(12 pi), v = 0.5 (-sin 2 pi y, sin 2 pi x),
  B = (-sin 2 pi y, sin 4 pi x)/sqrt(4 pi), weighted velocity W v.
* ``brio_wu``: relativistic Brio-Wu shock tube on [-0.5, 0.5], gamma = 2,
  (rho, p) = (1, 1) | (0.125, 0.1), Bx = 0.5, By = +1 | -1.
* ``fm_torus``: Fishbone-Moncrief torus in MKS coordinates, restating
  pangu/problem/fm_torus_mks/problem_generator.cpp:103-558 (ProblemGenerator
  and MeshPostInitialization) with a seeded counter-based generator in place of
  Kokkos::Random_XorShift64_Pool (whose draw order is not reproducible).
"""
from __future__ import annotations

import math

import numpy as np

from . import abi
from .params import ParameterInput, num_components


# ---------------------------------------------------------------------------
# mesh geometry shared with the engine (same rounding as the engine's tables)
# ---------------------------------------------------------------------------
class Geometry:
    """Index ranges and cell-centre coordinates of every meshblock."""

    def __init__(self, mesh: abi.Mesh):
        self.mesh = mesh
        self.nx = [mesh.nx1, mesh.nx2, mesh.nx3]
        self.nbx = [mesh.nbx1, mesh.nbx2, mesh.nbx3]
        self.act = [n > 1 for n in self.nx]
        self.ng = mesh.ng
        self.N = [self.nx[d] + 2 * self.ng * self.act[d] for d in range(3)]
        self.start = [self.ng * self.act[d] for d in range(3)]
        self.nb = self.nbx[0] * self.nbx[1] * self.nbx[2]
        mins = [mesh.x1min, mesh.x2min, mesh.x3min]
        maxs = [mesh.x1max, mesh.x2max, mesh.x3max]
        self.dx = [(maxs[d] - mins[d]) / float(self.nbx[d] * self.nx[d]) for d in range(3)]
        self.mins = mins
        self.shape = (self.N[2], self.N[1], self.N[0])

    def block_lattice(self, b):
        return (b % self.nbx[0], (b // self.nbx[0]) % self.nbx[1],
                b // (self.nbx[0] * self.nbx[1]))

    def origin(self, b, d):
        bl = self.block_lattice(b)[d]
        bxmin = self.mins[d] + float(bl * self.nx[d]) * self.dx[d]
        return bxmin - float(self.ng * self.act[d]) * self.dx[d]

    def xc(self, b, d):
        """Cell-centre coordinates along direction d over the entire range."""
        idx = np.arange(self.N[d], dtype=np.float64)
        return self.origin(b, d) + (idx + 0.5) * self.dx[d]

    def interior(self):
        s, n = self.start, self.nx
        return (slice(s[2], s[2] + n[2]), slice(s[1], s[1] + n[1]), slice(s[0], s[0] + n[0]))


def _nf(enable_B, enable_heating):
    return num_components(enable_B, enable_heating)


def _slots(enable_B, enable_heating):
    s = {"rho": 0, "u": 1, "u1": 2, "u2": 3, "u3": 4}
    n = 5
    if enable_B:
        s.update(b1=5, b2=6, b3=7)
        n = 8
    s["ent"] = n
    if enable_heating:
        s["kel"] = n + 1
    return s


def _alloc(geo, nf):
    return np.zeros((geo.nb, nf) + geo.shape)


# ---------------------------------------------------------------------------
# Orszag-Tang
# ---------------------------------------------------------------------------
def orszag_tang_input(n: int = 256, nblock: int | None = None) -> ParameterInput:
    nb = nblock or n
    pin = ParameterInput()
    for k, v in dict(nx1=n, x1min=0.0, x1max=1.0, ix1_bc="periodic", ox1_bc="periodic",
                     nx2=n, x2min=0.0, x2max=1.0, ix2_bc="periodic", ox2_bc="periodic",
                     nx3=1, x3min=-0.5, x3max=0.5, ix3_bc="periodic", ox3_bc="periodic",
                     nghost=2).items():
        pin.set("parthenon/mesh", k, v)
    for k, v in dict(nx1=nb, nx2=nb, nx3=1).items():
        pin.set("parthenon/meshblock", k, v)
    for k, v in dict(cfl_number=0.4, adiabatic_index=5.0 / 3.0, riemann_solver="laxf",
                     limiter="mc", recovery="chainer", enable_B=True,
                     enable_heating=False).items():
        pin.set("core", k, v)
    pin.set("metric", "type", "minkowski")
    for k, v in dict(integrator="rk2", dt_init=1e-5, dt_factor=1.3, nlim=100).items():
        pin.set("parthenon/time", k, v)
    return pin


def orszag_tang(geo: Geometry, packages) -> np.ndarray:
    c = packages["core"].params
    gam = c["adiabatic_index"]
    eB, eH = c["enable_B"], c["enable_heating"]
    S = _slots(eB, eH)
    P = _alloc(geo, _nf(eB, eH))
    rho0 = 25.0 / (36.0 * math.pi)
    p0 = 5.0 / (12.0 * math.pi)
    for b in range(geo.nb):
        x = geo.xc(b, 0)[None, :]
        y = geo.xc(b, 1)[:, None]
        vx = -0.5 * np.sin(2 * math.pi * y) + 0 * x
        vy = 0.5 * np.sin(2 * math.pi * x) + 0 * y
        W = 1.0 / np.sqrt(1.0 - vx * vx - vy * vy)
        P[b, S["rho"]] = rho0
        P[b, S["u"]] = p0 / (gam - 1.0)
        P[b, S["u1"]] = W * vx
        P[b, S["u2"]] = W * vy
        if eB:
            P[b, S["b1"]] = -np.sin(2 * math.pi * y) / math.sqrt(4 * math.pi) + 0 * x
            P[b, S["b2"]] = np.sin(4 * math.pi * x) / math.sqrt(4 * math.pi) + 0 * y
        P[b, S["ent"]] = (gam - 1.0) * P[b, S["u"]] * P[b, S["rho"]] ** (-gam)
        if eH:
            P[b, S["kel"]] = c["fel_0"] * P[b, S["ent"]]
    return P


# ---------------------------------------------------------------------------
# Brio-Wu
# ---------------------------------------------------------------------------
def brio_wu_input(n: int = 1024, nblock: int | None = None) -> ParameterInput:
    pin = ParameterInput()
    for k, v in dict(nx1=n, x1min=-0.5, x1max=0.5, ix1_bc="outflow", ox1_bc="outflow",
                     nx2=1, x2min=-0.5, x2max=0.5, ix2_bc="periodic", ox2_bc="periodic",
                     nx3=1, x3min=-0.5, x3max=0.5, ix3_bc="periodic", ox3_bc="periodic",
                     nghost=2).items():
        pin.set("parthenon/mesh", k, v)
    for k, v in dict(nx1=nblock or n, nx2=1, nx3=1).items():
        pin.set("parthenon/meshblock", k, v)
    for k, v in dict(cfl_number=0.4, adiabatic_index=2.0, riemann_solver="hll",
                     limiter="mc", recovery="chainer", enable_B=True,
                     enable_heating=True).items():
        pin.set("core", k, v)
    pin.set("metric", "type", "minkowski")
    for k, v in dict(integrator="rk2", dt_init=1e-5, dt_factor=1.3).items():
        pin.set("parthenon/time", k, v)
    return pin


def brio_wu(geo: Geometry, packages) -> np.ndarray:
    c = packages["core"].params
    gam = c["adiabatic_index"]
    eB, eH = c["enable_B"], c["enable_heating"]
    S = _slots(eB, eH)
    P = _alloc(geo, _nf(eB, eH))
    for b in range(geo.nb):
        x = geo.xc(b, 0)[None, None, :] + np.zeros(geo.shape)
        left = x < 0
        P[b, S["rho"]] = np.where(left, 1.0, 0.125)
        P[b, S["u"]] = np.where(left, 1.0, 0.1) / (gam - 1.0)
        if eB:
            P[b, S["b1"]] = 0.5
            P[b, S["b2"]] = np.where(left, 1.0, -1.0)
        P[b, S["ent"]] = (gam - 1.0) * P[b, S["u"]] * P[b, S["rho"]] ** (-gam)
        if eH:
            P[b, S["kel"]] = c["fel_0"] * P[b, S["ent"]]
    return P


# ---------------------------------------------------------------------------
# Fishbone-Moncrief torus (MKS)
# ---------------------------------------------------------------------------
def fm_torus_input(nx1=512, nx2=256, nx3=1, bx=None, *, gamma=5.0 / 3.0,
                   limiter="ppm4", riemann="laxf", a=0.9375, h=0.7, rin=6.0,
                   rmax=12.0, kappa=1e-3, beta=100.0, seed=0) -> ParameterInput:
    bx = bx or (nx1, nx2, nx3)
    pin = ParameterInput()
    mesh = dict(nx1=nx1, x1min=0.2, x1max=6.0, ix1_bc="outflow", ox1_bc="outflow",
                nx2=nx2, x2min=-1.0, x2max=1.0, ix2_bc="reflecting", ox2_bc="reflecting",
                nx3=nx3, x3min=-3.1415926535897, x3max=3.1415926535897,
                ix3_bc="periodic", ox3_bc="periodic",
                nghost=3 if limiter == "ppm4" else 2)
    for k, v in mesh.items():
        pin.set("parthenon/mesh", k, v)
    for k, v in zip(("nx1", "nx2", "nx3"), bx):
        pin.set("parthenon/meshblock", k, v)
    core = dict(cfl_number=0.3, adiabatic_index=gamma, recovery="chainer",
                density_floor=1e-5, energy_floor=4.64e-9, density_floor_pow=-1.5,
                energy_floor_pow=-2.5, riemann_solver=riemann, limiter=limiter,
                enable_heating=True, enable_B=True)
    for k, v in core.items():
        pin.set("core", k, v)
    for k, v in dict(type="mks", h=h, a=a).items():
        pin.set("metric", k, v)
    for k, v in dict(rin=rin, rmax=rmax, kappa=kappa, perturbation=4e-2, beta=beta,
                     aphi_rho_cut=0.2, magnetic_field="sane", seed=seed).items():
        pin.set("fm_torus", k, v)
    for k, v in dict(integrator="rk2", dt_init=1e-5, dt_factor=1.3).items():
        pin.set("parthenon/time", k, v)
    return pin


def _lfish_calc(r, a):  # problem_generator.cpp:22-35
    sr = math.sqrt(r)
    return (((a ** 2 - 2.0 * a * sr + r ** 2) *
             ((-2.0 * a * r * (a ** 2 - 2.0 * a * sr + r ** 2)) /
              math.sqrt(2.0 * a * sr + (-3.0 + r) * r) +
              ((a + (-2.0 + r) * sr) * (r ** 3 + a ** 2 * (2.0 + r))) /
              math.sqrt(1 + (2.0 * a) / r ** 1.5 - 3.0 / r))) /
            (r ** 3 * math.sqrt(2.0 * a * sr + (-3.0 + r) * r) * (a ** 2 + (-2.0 + r) * r)))


def _theta_map(x2, h):  # MKS.h:15-23
    return 0.5 * math.pi * (x2 + 1.0) + 0.5 * h * np.sin(math.pi * (x2 + 1.0))


def _jac(f, x, delta=1e-5):
    xh, xl = x + delta, x - delta
    return (f(xh) - f(xl)) / (xh - xl)


def _ks_code_metric(x1, x2, a, h):
    """MKS.h:25-107 on arrays: returns gcov[..., 4, 4]."""
    r = np.exp(x1)
    th = _theta_map(x2, h)
    J1 = _jac(np.exp, x1)
    J2 = _jac(lambda z: _theta_map(z, h), x2)
    cth, sth = np.cos(th), np.sin(th)
    S = r * r + a * a * cth * cth
    g = np.zeros(np.broadcast(r, th).shape + (4, 4))
    g[..., 0, 0] = -1.0 + 2.0 * r / S
    g[..., 0, 1] = g[..., 1, 0] = 2.0 * r / S
    g[..., 0, 3] = g[..., 3, 0] = -2.0 * a * r * sth * sth / S
    g[..., 1, 1] = 1.0 + 2.0 * r / S
    g[..., 1, 3] = g[..., 3, 1] = -a * (1.0 + 2.0 * r / S) * sth * sth
    g[..., 2, 2] = S
    g[..., 3, 3] = sth * sth * (S + a * a * sth * sth * (1.0 + 2.0 * r / S))
    J = np.stack([np.ones_like(J1 * J2), J1 + 0 * J2, J2 + 0 * J1, np.ones_like(J1 * J2)], -1)
    return g * J[..., :, None] * J[..., None, :]


def _bl_code_metric(x1, x2, a, h):
    """BL.h:25-107 on arrays."""
    r = np.exp(x1)
    th = _theta_map(x2, h)
    J1 = _jac(np.exp, x1)
    J2 = _jac(lambda z: _theta_map(z, h), x2)
    cth, sth = np.cos(th), np.sin(th)
    sth2, r2, a2 = sth * sth, r * r, a * a
    mu = 1.0 + a2 * cth * cth / r2
    de = 1.0 - 2.0 / r + a2 / r2
    irm = 1.0 / (r * mu)
    g = np.zeros(np.broadcast(r, th).shape + (4, 4))
    g[..., 0, 0] = -1.0 + 2.0 * irm
    g[..., 0, 3] = g[..., 3, 0] = -2.0 * a * sth2 * irm
    g[..., 1, 1] = mu / de
    g[..., 2, 2] = r2 / mu
    g[..., 3, 3] = r2 * sth2 * (1.0 + a2 / r2 + 2.0 * a2 * sth2 / (r * r2 * mu))
    J = np.stack([np.ones_like(J1 * J2), J1 + 0 * J2, J2 + 0 * J1, np.ones_like(J1 * J2)], -1)
    return g * J[..., :, None] * J[..., None, :], J1, J2


def _state_bsq(P, S, gcov, gcon):
    """bsq of CalculateState (state_calculation.h:19-69) on arrays."""
    alpha = 1.0 / np.sqrt(-gcon[..., 0, 0])
    ut = np.stack([P[S["u1"]], P[S["u2"]], P[S["u3"]]], -1)
    gij = gcov[..., 1:, 1:]
    lor = np.sqrt(1.0 + np.einsum("...i,...ij,...j->...", ut, gij, ut))
    ucon = np.zeros(ut.shape[:-1] + (4,))
    ucon[..., 0] = lor / alpha
    for d in range(3):
        ucon[..., d + 1] = ut[..., d] - ucon[..., 0] * gcon[..., 0, d + 1] * alpha * alpha
    ucov = np.einsum("...ij,...j->...i", gcov, ucon)
    B = np.stack([P[S["b1"]], P[S["b2"]], P[S["b3"]]], -1)
    bcon = np.zeros_like(ucon)
    bcon[..., 0] = np.einsum("...i,...i->...", B, ucov[..., 1:])
    for d in range(3):
        bcon[..., d + 1] = (B[..., d] + bcon[..., 0] * ucon[..., d + 1]) / ucon[..., 0]
    bcov = np.einsum("...ij,...j->...i", gcov, bcon)
    return np.einsum("...i,...i->...", bcon, bcov)


def hash_uniform(seed: int, b: int, shape) -> np.ndarray:
    """Counter-based uniform numbers in [-1, 1) for the cells of block b:
    SplitMix64 (Steele, Lea and Flood 2014) of seed * golden + cell index,
    top 53 bits. The device generator (kernels.cuh) computes the same values,
    so both give the same perturbation for the same seed."""
    n = int(np.prod(shape))
    gold = np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) * gold + (np.uint64(b) * np.uint64(n) + np.arange(n, dtype=np.uint64))
        z = z + gold
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    return (2.0 * u - 1.0).reshape(shape)


def fm_torus(geo: Geometry, packages, pin: ParameterInput) -> np.ndarray:
    c = packages["core"].params
    m = packages["metric"].params
    gam = c["adiabatic_index"]
    eB, eH = c["enable_B"], c["enable_heating"]
    S = _slots(eB, eH)
    a, h = m["a"], m["h"]
    rin = pin.get_or_add_real("fm_torus", "rin", 6.0)
    rmax = pin.get_or_add_real("fm_torus", "rmax", 12.0)
    kappa = pin.get_or_add_real("fm_torus", "kappa", 1.0e-3)
    pert = pin.get_or_add_real("fm_torus", "perturbation", 4.0e-2)
    beta_target = pin.get_or_add_real("fm_torus", "beta", 100.0)
    cut = pin.get_or_add_real("fm_torus", "aphi_rho_cut", 0.2)
    seed = pin.get_or_add_integer("fm_torus", "seed", 0)
    a2 = a * a
    l = _lfish_calc(rmax, a)
    sthin, cthin = math.sin(math.pi / 2), math.cos(math.pi / 2)
    DDin = rin * rin - 2.0 * rin + a2
    AAin = (rin * rin + a2) ** 2 - DDin * a2 * sthin * sthin
    SSin = rin * rin + a2 * cthin * cthin
    lnh_in = (0.5 * math.log((1.0 + math.sqrt(1.0 + 4.0 * (l * l * SSin * SSin) * DDin /
                                              (AAin * AAin * sthin * sthin))) / (SSin * DDin / AAin))
              - 0.5 * math.sqrt(1.0 + 4.0 * (l * l * SSin * SSin) * DDin / (AAin * AAin * sthin * sthin))
              - 2.0 * a * rin * l / AAin)

    P = _alloc(geo, _nf(eB, eH))
    for b in range(geo.nb):
        x1 = geo.xc(b, 0)[None, None, :]
        x2 = geo.xc(b, 1)[None, :, None]
        r = np.exp(x1) + 0 * x2
        th = _theta_map(x2, h) + 0 * x1
        sth, cth = np.sin(th), np.cos(th)
        gcov = _ks_code_metric(x1, x2, a, h)
        gcon = np.linalg.inv(gcov)
        gbl, J1, J2 = _bl_code_metric(x1, x2, a, h)
        alpha = 1.0 / np.sqrt(-gcon[..., 0, 0])
        betas = [gcon[..., 0, d] * alpha * alpha for d in (1, 2, 3)]
        DD = r * r - 2.0 * r + a2
        AA = (r * r + a2) ** 2 - DD * a2 * sth * sth
        SS = r * r + a2 * cth * cth
        with np.errstate(all="ignore"):
            lnh = (0.5 * np.log((1.0 + np.sqrt(1.0 + 4.0 * (l * l * SS * SS) * DD /
                                               (AA * sth * AA * sth))) / (SS * DD / AA))
                   - 0.5 * np.sqrt(1.0 + 4.0 * (l * l * SS * SS) * DD / (AA * AA * sth * sth))
                   - 2.0 * a * r * l / AA - lnh_in)
            lnh = np.where(r >= rin, lnh, 1.0)
            inside = (lnh >= 0.0) & (r >= rin)
            hm1 = np.exp(lnh) - 1.0
            inside &= hm1 > 0.0
            rho = np.where(inside, (hm1 * (gam - 1.0) / (kappa * gam)) ** (1.0 / (gam - 1.0)), 0.0)
        rnd = hash_uniform(seed, b, geo.shape)
        eint = np.where(inside, kappa * rho ** gam / (gam - 1.0), 0.0) * (1.0 + pert * rnd)
        eint = np.where(inside, eint, 0.0)
        with np.errstate(all="ignore"):
            ent = np.where(inside, (gam - 1.0) * eint * rho ** (-gam), 0.0)
            expm2chi = SS * SS * DD / (AA * AA * sth * sth)
            up1 = np.sqrt((-1.0 + np.sqrt(1.0 + 4.0 * l * l * expm2chi)) / 2.0)
            up_bl = (2.0 * a * r * np.sqrt(1.0 + up1 * up1) / np.sqrt(AA * SS * DD)
                     + np.sqrt(SS / AA) * up1 / sth)
            AAq = gbl[..., 0, 0]
            BBq = 2.0 * gbl[..., 0, 3] * up_bl
            CCq = 1.0 + gbl[..., 3, 3] * up_bl * up_bl
            u0 = (-BBq - np.sqrt(BBq * BBq - 4.0 * AAq * CCq)) / (2.0 * AAq)
        # BL -> KS -> code (problem_generator.cpp:50-101): u^r_BL = 0, so the
        # KS transformation leaves (u0, 0, 0, up) and the diagonal code
        # Jacobian leaves it unchanged.
        wv = [betas[0] * u0, betas[1] * u0, up_bl + betas[2] * u0]
        P[b, S["rho"]] = rho
        P[b, S["u"]] = eint
        for d in range(3):
            P[b, S[f"u{d+1}"]] = np.where(inside, wv[d], 0.0)
        P[b, S["ent"]] = ent
        if eH:
            P[b, S["kel"]] = c["fel_0"] * ent

    # MeshPostInitialization (problem_generator.cpp:291-558)
    rhomax = float(P[:, S["rho"]].max())
    umax = float(P[:, S["u"]].max())
    if not rhomax > 0.0:
        # the enthalpy never exceeds its inner-edge value: these (a, rin,
        # rmax) admit no bound torus and the normalisation is undefined
        raise ValueError(f"no bound torus for a={a}, rin={rin}, rmax={rmax}")
    P[:, S["rho"]] /= rhomax
    P[:, S["u"]] /= rhomax
    if not eB:
        return P
    inter = geo.interior()
    bsq_max = 0.0
    for b in range(geo.nb):
        rho = P[b, S["rho"]]
        A = np.zeros(geo.shape)
        avg = 0.25 * (rho[:, 1:, 1:] + rho[:, 1:, :-1] + rho[:, :-1, 1:] + rho[:, :-1, :-1])
        A[:, 1:, 1:] = np.maximum(avg - cut, 0.0)
        x1 = geo.xc(b, 0)[None, None, :]
        x2 = geo.xc(b, 1)[None, :, None]
        gcov = _ks_code_metric(x1, x2, a, h)
        gdet = np.linalg.det(gcov)
        sg = np.sqrt(np.abs(gdet))
        a00 = np.roll(np.roll(A, 1, axis=1), 1, axis=2)
        a01 = np.roll(A, 1, axis=2)
        a10 = np.roll(A, 1, axis=1)
        a11 = A
        b1 = -(a00 - a01 + a10 - a11) / (2.0 * geo.dx[1] * sg)
        b2 = (a00 + a01 - a10 - a11) / (2.0 * geo.dx[0] * sg)
        P[b, S["b1"]][inter] = b1[inter]
        P[b, S["b2"]][inter] = b2[inter]
        gcon = np.linalg.inv(gcov)
        bsq = _state_bsq(P[b], S, gcov, gcon)
        bsq_max = max(bsq_max, float(bsq[inter].max()))
    beta_min = 2.0 * (gam - 1.0) * (umax / rhomax) / (bsq_max + 1.0e-30)
    norm = math.sqrt(beta_min / beta_target)
    for b in range(geo.nb):
        for key in ("b1", "b2", "b3"):
            P[b, S[key]][inter] *= norm
    return P


def problem_struct(name: str, pin: ParameterInput) -> abi.Problem:
    """The device generator's description of a named problem (pangu_generate):
    kind plus the <fm_torus> parameters of a torus."""
    pb = abi.Problem()
    pb.kind = abi.PROBLEM[name]
    if pb.kind == abi.PROBLEM["torus"]:
        g = lambda k, v: pin.get_or_add_real("fm_torus", k, v)  # noqa: E731
        pb.rin, pb.rmax, pb.kappa = g("rin", 6.0), g("rmax", 12.0), g("kappa", 1.0e-3)
        pb.perturbation, pb.beta = g("perturbation", 4.0e-2), g("beta", 100.0)
        pb.aphi_rho_cut = g("aphi_rho_cut", 0.2)
        pb.seed = pin.get_or_add_integer("fm_torus", "seed", 0)
    return pb


# ---------------------------------------------------------------------------
# Atmosphere around a spinning hole in Cartesian Kerr-Schild coordinates
# ---------------------------------------------------------------------------
def cks_atmosphere_input(n: int = 16, nblock: int | None = None, a: float = 0.5,
                         r_excise: float = 1.5) -> ParameterInput:
    """A box around the hole with outflow faces. The box is offset so that no
    cell centre or face lies on z = 0, where the ring singularity (r = 0 for
    x^2 + y^2 <= a^2) sits; the hole is excised within r_excise."""
    pin = ParameterInput()
    for d in (1, 2, 3):
        for k, v in {f"nx{d}": n, f"x{d}min": -3.9, f"x{d}max": 4.1,
                     f"ix{d}_bc": "outflow", f"ox{d}_bc": "outflow"}.items():
            pin.set("parthenon/mesh", k, v)
        pin.set("parthenon/meshblock", f"nx{d}", nblock or n)
    pin.set("parthenon/mesh", "nghost", 2)
    for k, v in dict(cfl_number=0.3, adiabatic_index=5.0 / 3.0, riemann_solver="laxf",
                     limiter="mc", recovery="chainer", enable_B=True, enable_heating=False,
                     density_floor=1e-6, energy_floor=1e-8).items():
        pin.set("core", k, v)
    for k, v in dict(type="cks", a=a, excise=True, r_excise=r_excise).items():
        pin.set("metric", k, v)
    for k, v in dict(integrator="rk2", dt_init=1e-5, dt_factor=1.3).items():
        pin.set("parthenon/time", k, v)
    return pin


def cks_atmosphere(geo: Geometry, packages) -> np.ndarray:
    """rho = 1e-2 r^-1.5, u = 1e-4 r^-2.5 (r the spherical radius of the
    cell centre, at least 1), zero weighted velocity, uniform B^z = 0.05."""
    c = packages["core"].params
    gam = c["adiabatic_index"]
    S = _slots(c["enable_B"], c["enable_heating"])
    P = _alloc(geo, _nf(c["enable_B"], c["enable_heating"]))
    for b in range(geo.nb):
        x = geo.xc(b, 0)[None, None, :]
        y = geo.xc(b, 1)[None, :, None]
        z = geo.xc(b, 2)[:, None, None]
        r = np.maximum(np.sqrt(x * x + y * y + z * z), 1.0)
        P[b, S["rho"]] = 1e-2 * r ** -1.5
        P[b, S["u"]] = 1e-4 * r ** -2.5
        if c["enable_B"]:
            P[b, S["b3"]] = 0.05
        P[b, S["ent"]] = (gam - 1.0) * P[b, S["u"]] * P[b, S["rho"]] ** (-gam)
        if c["enable_heating"]:
            P[b, S["kel"]] = c["fel_0"] * P[b, S["ent"]]
    return P


def make_problem(name: str, **kw):
    """Returns (ParameterInput, generator) for a named benchmark problem."""
    if name in ("orszag_tang", "ot"):
        return orszag_tang_input(**kw), lambda geo, pk, pin: orszag_tang(geo, pk)
    if name in ("brio_wu", "bw"):
        return brio_wu_input(**kw), lambda geo, pk, pin: brio_wu(geo, pk)
    if name in ("fm_torus", "torus"):
        return fm_torus_input(**kw), fm_torus
    if name in ("cks_atmosphere", "cks"):
        return cks_atmosphere_input(**kw), lambda geo, pk, pin: cks_atmosphere(geo, pk)
    raise ValueError(f"unknown problem {name!r}")
