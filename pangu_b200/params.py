"""Inputfile parsing and package registration, mirroring PANGU's surface.

``ParameterInput`` reads Parthenon-style inputfiles (``<block>`` headers and
``key = value`` lines). ``core_initialize`` and ``metric_initialize`` register
the same keys, defaults and validation as ``core::Initialize`` and
``metric::Initialize`` (pangu/src/initialization/package_registration.cc:16-177),
and ``primitive_field_names`` reproduces the field list and order of
package_registration.cc:84-96.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

from . import abi


def _parse_bool(v: str) -> bool:
    s = v.strip().lower()
    if s in ("true", "1", "yes", "on"):
        return True
    if s in ("false", "0", "no", "off"):
        return False
    raise ValueError(f"not a boolean: {v!r}")


class ParameterInput:
    """Parthenon ParameterInput: blocks of key = value pairs."""

    def __init__(self, text: str = ""):
        self.blocks: dict[str, dict[str, str]] = {}
        block = None
        for raw in text.splitlines():
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            m = re.match(r"^<\s*([^>]+?)\s*>$", line)
            if m:
                block = m.group(1)
                self.blocks.setdefault(block, {})
                continue
            if "=" in line and block is not None:
                k, v = line.split("=", 1)
                self.blocks[block][k.strip()] = v.strip()

    @classmethod
    def from_file(cls, path: str) -> "ParameterInput":
        with open(path) as f:
            return cls(f.read())

    def set(self, block: str, key: str, value) -> None:
        if isinstance(value, bool):
            value = "true" if value else "false"
        self.blocks.setdefault(block, {})[key] = str(value)

    def has(self, block: str, key: str) -> bool:
        return key in self.blocks.get(block, {})

    def _get_or_add(self, block, key, default, conv):
        b = self.blocks.setdefault(block, {})
        if key not in b:
            b[key] = ("true" if default else "false") if isinstance(default, bool) else str(default)
            return default
        return conv(b[key])

    def get_or_add_real(self, block, key, default: float) -> float:
        return self._get_or_add(block, key, float(default), float)

    def get_or_add_integer(self, block, key, default: int) -> int:
        return self._get_or_add(block, key, int(default), lambda s: int(float(s)))

    def get_or_add_string(self, block, key, default: str) -> str:
        return self._get_or_add(block, key, default, lambda s: s)

    def get_or_add_boolean(self, block, key, default: bool) -> bool:
        return self._get_or_add(block, key, bool(default), _parse_bool)

    def dump(self) -> str:
        """The parameters as inputfile text (blocks and key = value lines);
        ParameterInput(p.dump()) gives the same parameters back."""
        out = []
        for block, kv in self.blocks.items():
            out.append(f"<{block}>")
            out += [f"{k} = {v}" for k, v in kv.items()]
            out.append("")
        return "\n".join(out)

    def check_required(self, block, key) -> None:
        if not self.has(block, key):
            raise ValueError(f"<{block}>/{key} is required")


@dataclass
class StateDescriptor:
    """The params and field names a package registers."""
    name: str
    params: dict = field(default_factory=dict)
    fields: list = field(default_factory=list)

    def param(self, key):
        return self.params[key]


MODELS = tuple(abi.HEATING_MODEL)


def core_initialize(pin: ParameterInput) -> StateDescriptor:
    """core::Initialize (package_registration.cc:16-149)."""
    pkg = StateDescriptor("core")
    P = pkg.params
    P["cfl_number"] = pin.get_or_add_real("core", "cfl_number", 0.8)
    P["adiabatic_index"] = pin.get_or_add_real("core", "adiabatic_index", 5.0 / 3.0)
    P["riemann_solver"] = pin.get_or_add_string("core", "riemann_solver", "laxf")
    P["limiter"] = pin.get_or_add_string("core", "limiter", "ppm4")
    P["density_floor"] = pin.get_or_add_real("core", "density_floor", 1.0e-6)
    P["energy_floor"] = pin.get_or_add_real("core", "energy_floor", 1.0e-8)
    P["density_floor_pow"] = pin.get_or_add_real("core", "density_floor_pow", -1.5)
    P["energy_floor_pow"] = pin.get_or_add_real("core", "energy_floor_pow", -2.5)
    P["enable_B"] = pin.get_or_add_boolean("core", "enable_B", False)
    P["recovery"] = pin.get_or_add_string("core", "recovery", "chainer")
    if P["recovery"] not in ("chainer", "robuster"):  # package_registration.cc:38-40
        raise ValueError("<core>/recovery must be 'chainer' or 'robuster', got: "
                         + P["recovery"])
    P["enable_heating"] = pin.get_or_add_boolean("core", "enable_heating", False)
    P["sigma_max"] = pin.get_or_add_real("core", "sigma_max", 50)
    P["lorentz_max"] = pin.get_or_add_real("core", "lorentz_max", 50)
    model = pin.get_or_add_string("electron", "model", "constant")
    if model not in MODELS:  # heating_model.h:111-121 (parseModel)
        raise ValueError("Invalid electrons/model. Allowed values: constant, "
                         "howes, kawazura, werner, rowan, sharma.")
    P["model_name"] = model
    P["fel_constant"] = pin.get_or_add_real("electron", "fel_constant", 0.1)
    P["gamma_e"] = pin.get_or_add_real("electron", "gamma_e", 4.0 / 3.0)
    P["gamma_p"] = pin.get_or_add_real("electron", "gamma_p", 5.0 / 3.0)
    P["limit_kel"] = pin.get_or_add_boolean("electron", "limit_kel", True)
    P["suppress_highb_heat"] = pin.get_or_add_boolean("electron", "suppress_highb_heat", False)
    P["enforce_positive_dissipation"] = pin.get_or_add_boolean(
        "electron", "enforce_positive_dissipation", False)
    P["ratio_min"] = pin.get_or_add_real("electron", "ratio_min", 0.001)
    P["ratio_max"] = pin.get_or_add_real("electron", "ratio_max", 1000.0)
    P["fel_0"] = pin.get_or_add_real("electron", "fel_0", 0.1)
    P["primitive_field_names"] = primitive_field_names(P["enable_B"], P["enable_heating"])
    # Field registration (package_registration.cc:98-145).
    pkg.fields = ["density", "energy", "entropy"]
    if P["enable_heating"]:
        pkg.fields.append("electron_entropy")
    pkg.fields += ["weighted_velocity", "alfven"]
    if P["enable_B"]:
        pkg.fields += ["magnetic_field", "electric_field"]
    pkg.fields.append("conservative")
    if P["recovery"] == "chainer":
        pkg.fields.append("flag")
    return pkg


def metric_initialize(pin: ParameterInput) -> StateDescriptor:
    """metric::Initialize (package_registration.cc:152-177)."""
    pkg = StateDescriptor("metric")
    P = pkg.params
    P["metric_type"] = pin.get_or_add_string("metric", "type", "minkowski")
    P["a"] = pin.get_or_add_real("metric", "a", 0.0)
    P["h"] = pin.get_or_add_real("metric", "h", 0.0)
    P["excise"] = pin.get_or_add_boolean("metric", "excise", False)
    P["r_excise"] = pin.get_or_add_real("metric", "r_excise", 1.0)
    P["dexcise"] = pin.get_or_add_real("metric", "dexcise", 1.0e-8)
    P["pexcise"] = pin.get_or_add_real("metric", "pexcise", 0.333e-12)
    return pkg


def primitive_field_names(enable_B: bool, enable_heating: bool) -> list[str]:
    """package_registration.cc:84-90."""
    names = ["density", "energy", "weighted_velocity"]
    if enable_B:
        names.append("magnetic_field")
    names.append("entropy")
    if enable_heating:
        names.append("electron_entropy")
    return names


def num_components(enable_B: bool, enable_heating: bool) -> int:
    """package_registration.cc:92-96."""
    return 6 + (3 if enable_B else 0) + (1 if enable_heating else 0)


def process_packages(pin: ParameterInput) -> dict[str, StateDescriptor]:
    """ProcessPackages (ideal_grmhd.cc:122-131)."""
    return {"core": core_initialize(pin), "metric": metric_initialize(pin)}


def params_struct(packages: dict[str, StateDescriptor]) -> abi.Params:
    """Packs the registered params into the C-ABI struct."""
    c = packages["core"].params
    m = packages["metric"].params
    if c["riemann_solver"] not in abi.RIEMANN:  # riemann_solver.cc:25
        raise ValueError("Unknown Riemann solver: " + c["riemann_solver"])
    if c["limiter"] not in abi.LIMITER:
        raise ValueError("Unknown limiter: " + c["limiter"])
    p = abi.Params()
    p.cfl_number = c["cfl_number"]
    p.adiabatic_index = c["adiabatic_index"]
    p.riemann_solver = abi.RIEMANN[c["riemann_solver"]]
    p.limiter = abi.LIMITER[c["limiter"]]
    p.density_floor = c["density_floor"]
    p.energy_floor = c["energy_floor"]
    p.density_floor_pow = c["density_floor_pow"]
    p.energy_floor_pow = c["energy_floor_pow"]
    p.enable_B = int(c["enable_B"])
    p.recovery = abi.RECOVERY[c["recovery"]]
    p.enable_heating = int(c["enable_heating"])
    p.sigma_max = c["sigma_max"]
    p.lorentz_max = c["lorentz_max"]
    p.model = abi.HEATING_MODEL[c["model_name"]]
    p.limit_kel = int(c["limit_kel"])
    p.suppress_highb_heat = int(c["suppress_highb_heat"])
    p.enforce_positive_dissipation = int(c["enforce_positive_dissipation"])
    p.fel_constant = c["fel_constant"]
    p.gamma_e = c["gamma_e"]
    p.gamma_p = c["gamma_p"]
    p.ratio_min = c["ratio_min"]
    p.ratio_max = c["ratio_max"]
    p.fel_0 = c["fel_0"]
    # Unknown metric strings fall back to Minkowski (e.g. laxf.cc:58-61).
    p.metric_type = abi.METRIC.get(m["metric_type"], 0)
    p.excise = int(m["excise"])
    p.a = m["a"]
    p.h = m["h"]
    p.r_excise = m["r_excise"]
    p.dexcise = m["dexcise"]
    p.pexcise = m["pexcise"]
    return p


def engine_precision(pin: ParameterInput) -> int:
    """<b200>/precision = fp64 (default) | mixed: the engine's arithmetic. Not a
    reference key; the reference is FP64 throughout."""
    name = pin.get_or_add_string("b200", "precision", "fp64")
    if name not in abi.PRECISION:
        raise ValueError("Unknown precision: " + name)
    return abi.PRECISION[name]


def mesh_struct(pin: ParameterInput) -> abi.Mesh:
    """<parthenon/mesh> + <parthenon/meshblock> into the C-ABI mesh struct.

    ``nghost`` defaults to 2 as in Parthenon; PPM4 needs 3 (the engine
    refuses a smaller value, the reference silently reads out of bounds).
    """
    for key in ("ix1_bc", "ox1_bc", "ix2_bc", "ox2_bc"):  # ideal_grmhd.cc:14-17
        pin.check_required("parthenon/mesh", key)
    m = abi.Mesh()
    nx = [pin.get_or_add_integer("parthenon/mesh", f"nx{d}", 1) for d in (1, 2, 3)]
    bx = [pin.get_or_add_integer("parthenon/meshblock", f"nx{d}", nx[d - 1]) for d in (1, 2, 3)]
    for d in range(3):
        if nx[d] % bx[d]:
            raise ValueError(f"mesh nx{d+1}={nx[d]} is not a multiple of meshblock nx{d+1}={bx[d]}")
    m.nx1, m.nx2, m.nx3 = bx
    m.nbx1, m.nbx2, m.nbx3 = (nx[d] // bx[d] for d in range(3))
    m.ng = pin.get_or_add_integer("parthenon/mesh", "nghost", 2)
    for d, (lo, hi) in enumerate(((-0.5, 0.5),) * 3, start=1):
        setattr(m, f"x{d}min", pin.get_or_add_real("parthenon/mesh", f"x{d}min", lo))
        setattr(m, f"x{d}max", pin.get_or_add_real("parthenon/mesh", f"x{d}max", hi))
    bcs = []
    for d in (1, 2, 3):
        for side in ("i", "o"):
            name = pin.get_or_add_string("parthenon/mesh", f"{side}x{d}_bc", "periodic")
            if name not in abi.BC:
                raise ValueError(f"unsupported boundary condition {name!r}")
            bcs.append(abi.BC[name])
    m.bc[:] = bcs
    return m
