"""The K17 parameter checks of Parameter (Parameter::checkParameterValidityCumulantK17,
Parameter.cpp:424-445), restating the reference's unit tests
(tests/unit-tests/gpu/core/Parameter/ParameterTest.cpp:273-330): a warning above a velocity of
0.1 and above a viscosity of 1/42 (at the finest level), none below and none for another main
kernel. This build's registry knows only K17, so "another main kernel" is a Parameter whose main
kernel is not configured (configure_main_kernel rejects unknown names at once)."""
import warnings

import pytest

from virtualfluids_b200 import K17ParameterWarning, Parameter


def _k17(velocity=None, viscosity=None):
    p = Parameter()
    if velocity is not None:
        p.set_velocity_lb(velocity)
    if viscosity is not None:
        p.set_viscosity_lb(viscosity)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    return p


@pytest.mark.parametrize("velocity, viscosity, warned", [
    (0.11, None, True), (0.09, None, False), (None, 0.024, True), (None, 0.023, False)])
def test_cumulant_k17_thresholds(velocity, viscosity, warned):
    p = _k17(velocity, viscosity)
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        out = p.check_parameter_validity_cumulant_k17()
    assert bool(out) == warned
    assert any(issubclass(w.category, K17ParameterWarning) for w in caught) == warned


def test_other_main_kernel_gives_no_warning():
    p = Parameter()
    p.set_velocity_lb(42.0)
    p.set_viscosity_lb(10.0)
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        assert p.check_parameter_validity_cumulant_k17() == []
    assert not caught


def test_viscosity_of_the_finest_level_counts():
    """0.01 is fine on one level, but 0.04 on the second of two (nu 2^level, Parameter.cpp:404)."""
    p = _k17(viscosity=0.01)
    with warnings.catch_warnings(record=True):
        warnings.simplefilter("always")
        assert p.check_parameter_validity_cumulant_k17(0) == []
        assert len(p.check_parameter_validity_cumulant_k17(2)) == 1
