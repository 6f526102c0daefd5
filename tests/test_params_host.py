"""Host-side parameter handling: inputfile parsing, the registered defaults
and validation of core::Initialize / metric::Initialize
(package_registration.cc:16-177), the engine precision key and the mesh
struct built from <parthenon/mesh>."""
import pytest

from pangu_b200 import abi
from pangu_b200 import params as prm

INPUT = """
<parthenon/mesh>
nx1 = 64      # cells
x1min = 0.2
x1max = 6.0
ix1_bc = outflow
ox1_bc = outflow
nx2 = 32
x2min = -1.0
x2max = 1.0
ix2_bc = reflecting
ox2_bc = reflecting
nghost = 3

<parthenon/meshblock>
nx1 = 32
nx2 = 16

<core>
enable_B = true
limiter = ppm4

<metric>
type = mks
a = 0.9375
h = 0.7
"""


def test_inputfile_parsing_and_mesh():
    pin = prm.ParameterInput(INPUT)
    m = prm.mesh_struct(pin)
    assert (m.nx1, m.nx2, m.nx3) == (32, 16, 1)
    assert (m.nbx1, m.nbx2, m.nbx3) == (2, 2, 1)
    assert m.ng == 3 and m.x1min == 0.2 and m.x2max == 1.0
    assert list(m.bc) == [abi.BC["outflow"]] * 2 + [abi.BC["reflecting"]] * 2 + \
        [abi.BC["periodic"]] * 2


def test_registered_defaults():
    pin = prm.ParameterInput(INPUT)
    p = prm.params_struct(prm.process_packages(pin))
    assert p.cfl_number == 0.8 and p.adiabatic_index == 5.0 / 3.0
    assert p.riemann_solver == abi.RIEMANN["laxf"] and p.limiter == abi.LIMITER["ppm4"]
    assert p.density_floor == 1e-6 and p.energy_floor == 1e-8
    assert p.density_floor_pow == -1.5 and p.energy_floor_pow == -2.5
    assert p.enable_B == 1 and p.enable_heating == 0
    assert p.recovery == abi.RECOVERY["chainer"]
    assert p.sigma_max == 50 and p.lorentz_max == 50
    assert p.model == abi.HEATING_MODEL["constant"] and p.limit_kel == 1
    assert p.gamma_e == 4.0 / 3.0 and p.gamma_p == 5.0 / 3.0
    assert p.ratio_min == 1e-3 and p.ratio_max == 1e3
    assert p.metric_type == abi.METRIC["mks"] and p.a == 0.9375 and p.h == 0.7
    assert p.r_excise == 1.0 and p.dexcise == 1e-8 and p.pexcise == 0.333e-12
    assert p.precision == 0


def test_field_registration():
    pk = prm.core_initialize(prm.ParameterInput(INPUT))
    assert pk.params["primitive_field_names"] == ["density", "energy", "weighted_velocity",
                                                  "magnetic_field", "entropy"]
    assert "flag" in pk.fields and "electric_field" in pk.fields
    assert prm.num_components(True, False) == 9


@pytest.mark.parametrize("block,key,value", [("core", "recovery", "newton"),
                                             ("electron", "model", "bogus")])
def test_invalid_options_raise(block, key, value):
    pin = prm.ParameterInput(INPUT)
    pin.set(block, key, value)
    with pytest.raises(ValueError):
        prm.process_packages(pin)


def test_unknown_riemann_solver_raises():
    pin = prm.ParameterInput(INPUT)
    pin.set("core", "riemann_solver", "roe")
    with pytest.raises(ValueError):
        prm.params_struct(prm.process_packages(pin))


def test_precision_key():
    pin = prm.ParameterInput(INPUT)
    assert prm.engine_precision(pin) == 0
    pin.set("b200", "precision", "mixed")
    assert prm.engine_precision(pin) == 1
    pin.set("b200", "precision", "fp16")
    with pytest.raises(ValueError):
        prm.engine_precision(pin)


def test_mesh_errors():
    pin = prm.ParameterInput(INPUT)
    pin.set("parthenon/meshblock", "nx1", 24)  # 64 is not a multiple of 24
    with pytest.raises(ValueError):
        prm.mesh_struct(pin)
    pin = prm.ParameterInput(INPUT.replace("ix1_bc = outflow", ""))
    with pytest.raises(ValueError):
        prm.mesh_struct(pin)


def test_inputfile_dump_round_trip():
    pin = prm.ParameterInput(INPUT)
    pin.set("b200", "precision", "mixed")
    again = prm.ParameterInput(pin.dump())
    assert again.blocks == pin.blocks
    p1 = prm.params_struct(prm.process_packages(pin))
    p2 = prm.params_struct(prm.process_packages(again))
    assert bytes(p1) == bytes(p2)
