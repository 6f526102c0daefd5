"""ctypes mirrors of the POD structs and constants of include/pangu_b200.h."""
from __future__ import annotations

import ctypes as C

PANGU_OK = 0
PANGU_EINVAL = -1
PANGU_ECUDA = -2
PANGU_ENOMEM = -3
PANGU_ENGHOST = -4
PANGU_ETOOBIG = -5
PANGU_EFULL = -6

RIEMANN = {"laxf": 0, "hll": 1}
PRECISION = {"fp64": 0, "mixed": 1}
LIMITER = {"ppm4": 0, "mc": 1}
RECOVERY = {"chainer": 0, "robuster": 1}
METRIC = {"minkowski": 0, "bl": 1, "cks": 2, "mks": 3}
HEATING_MODEL = {"constant": 0, "howes": 1, "kawazura": 2, "werner": 3,
                 "rowan": 4, "sharma": 5}
BC = {"periodic": 0, "outflow": 1, "reflecting": 2}

CNT_RHO_FLOOR = 0
CNT_ENG_FLOOR = 1
CNT_LORENTZ_CAP = 2
CNT_C2P_2D = 3
CNT_C2P_1DVSQ = 4
CNT_C2P_1D = 5
CNT_C2P_FAIL = 6
CNT_FIXRECOVERY = 7
CNT_KASTAUN_FAIL = 8
CNT_EXCISED = 9
NCOUNTERS = 16
COUNTER_NAMES = ["rho_floor", "eng_floor", "lorentz_cap", "c2p_2d",
                 "c2p_1dvsq", "c2p_1d", "c2p_fail", "fix_recovery",
                 "kastaun_fail", "excised"]


class Params(C.Structure):
    _fields_ = [
        ("cfl_number", C.c_double),
        ("adiabatic_index", C.c_double),
        ("riemann_solver", C.c_int32),
        ("limiter", C.c_int32),
        ("density_floor", C.c_double),
        ("energy_floor", C.c_double),
        ("density_floor_pow", C.c_double),
        ("energy_floor_pow", C.c_double),
        ("enable_B", C.c_int32),
        ("recovery", C.c_int32),
        ("enable_heating", C.c_int32),
        ("precision", C.c_int32),
        ("sigma_max", C.c_double),
        ("lorentz_max", C.c_double),
        ("model", C.c_int32),
        ("limit_kel", C.c_int32),
        ("suppress_highb_heat", C.c_int32),
        ("enforce_positive_dissipation", C.c_int32),
        ("fel_constant", C.c_double),
        ("gamma_e", C.c_double),
        ("gamma_p", C.c_double),
        ("ratio_min", C.c_double),
        ("ratio_max", C.c_double),
        ("fel_0", C.c_double),
        ("metric_type", C.c_int32),
        ("excise", C.c_int32),
        ("a", C.c_double),
        ("h", C.c_double),
        ("r_excise", C.c_double),
        ("dexcise", C.c_double),
        ("pexcise", C.c_double),
    ]


class Mesh(C.Structure):
    _fields_ = [
        ("nx1", C.c_int32), ("nx2", C.c_int32), ("nx3", C.c_int32),
        ("nbx1", C.c_int32), ("nbx2", C.c_int32), ("nbx3", C.c_int32),
        ("ng", C.c_int32), ("reserved0", C.c_int32),
        ("x1min", C.c_double), ("x1max", C.c_double),
        ("x2min", C.c_double), ("x2max", C.c_double),
        ("x3min", C.c_double), ("x3max", C.c_double),
        ("bc", C.c_int32 * 6),
    ]


class Pack(C.Structure):
    _fields_ = [
        ("prim", C.c_void_p), ("cons", C.c_void_p),
        ("flux1", C.c_void_p), ("flux2", C.c_void_p), ("flux3", C.c_void_p),
        ("alfven", C.c_void_p), ("efield", C.c_void_p), ("flag", C.c_void_p),
        # per-(block, component) pointer tables (device arrays), NULL: contiguous
        ("prim_vars", C.c_void_p), ("cons_vars", C.c_void_p),
        ("flux1_vars", C.c_void_p), ("flux2_vars", C.c_void_p), ("flux3_vars", C.c_void_p),
        ("alfven_vars", C.c_void_p), ("efield_vars", C.c_void_p), ("flag_vars", C.c_void_p),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("jobs", C.c_int64), ("ticks", C.c_int64),
        ("wall_s", C.c_double), ("zone_cycles", C.c_double),
        ("zone_cycles_per_s", C.c_double), ("p50_s", C.c_double), ("p99_s", C.c_double),
        ("hbm_bytes", C.c_uint64), ("hbm_peak_bytes", C.c_uint64),
        ("memory_waits", C.c_int64),
    ]


PROBLEM = {"ot": 0, "orszag_tang": 0, "bw": 1, "brio_wu": 1, "torus": 2, "fm_torus": 2}


class Problem(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("seed", C.c_int32),
        ("rin", C.c_double), ("rmax", C.c_double), ("kappa", C.c_double),
        ("perturbation", C.c_double), ("beta", C.c_double), ("aphi_rho_cut", C.c_double),
    ]
