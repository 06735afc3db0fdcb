"""Configuration files of the reference read into Parameter (ConfigurationFile::load,
basics/config/ConfigurationFile.cpp:60-100; Parameter::readConfigData, Parameter.cpp:80-300): the
parse rules (comments, trimming, skipped lines, last line wins, 'true' as the only true) and the keys
of the hot path with the reference's defaults."""
import pytest

from virtualfluids_b200 import Parameter, VfbError
from virtualfluids_b200.simulation import config_bool, load_configuration_file

TEXT = """# DrivenCavity-like configuration
Path = ./output   # comment after a value
Viscosity_LB=0.0032
\tVelocity_LB =  0.05\t
QuadricLimiterP = 0.02
ForcingX = 1e-6
MainKernelName = K17CompressibleNavierStokes
WriteGrid = True
UseInitNeq = true
EmptyValue =
= no key
no equals sign
Viscosity_LB = 0.004
"""


def test_parse_rules(tmp_path):
    f = tmp_path / "config.txt"
    f.write_text(TEXT)
    cfg = load_configuration_file(f)
    assert cfg["Path"] == "./output"
    assert cfg["Velocity_LB"] == "0.05"
    assert cfg["Viscosity_LB"] == "0.004"            # the later line wins
    assert "EmptyValue" not in cfg and "" not in cfg
    assert not config_bool(cfg["WriteGrid"]) and config_bool(cfg["UseInitNeq"])
    with pytest.raises(FileNotFoundError):
        load_configuration_file(tmp_path / "missing.txt")


def test_parameter_from_configuration_file(tmp_path):
    f = tmp_path / "config.txt"
    f.write_text(TEXT)
    p = Parameter.from_configuration_file(f)
    assert p.viscosity_lb == 0.004 and p.velocity_lb == 0.05
    assert p.forcing == (1e-6, 0.0, 0.0)
    assert p.quadric_limiters == (0.02, 0.01, 0.01)
    assert p.main_kernel == "K17CompressibleNavierStokes"
    assert p.omega == 1.0 / (3.0 * 0.004 + 0.5)
    bad = tmp_path / "bad.txt"
    bad.write_text("MainKernelName = K15CompressibleNavierStokes\n")
    with pytest.raises(VfbError):
        Parameter.from_configuration_file(bad)
