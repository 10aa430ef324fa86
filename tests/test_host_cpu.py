"""Host-side option handling (no GPU): engine option overrides and their types."""
import pytest


def test_engine_option_overrides_are_typed_like_the_defaults():
    from amaterasu_b200.scf_benchmark import parse_engine_options
    opts = parse_engine_options(["c64_tolerance_floor=5e-7", "refine_max_iterations=2", "tc_subspace=false",
                                 "autotune=1", "tc_min_npw=2048"])
    assert opts == {"c64_tolerance_floor": 5e-7, "refine_max_iterations": 2, "tc_subspace": False,
                    "autotune": True, "tc_min_npw": 2048}
    assert isinstance(opts["refine_max_iterations"], int)
    with pytest.raises(ValueError):
        parse_engine_options(["no_such_option=1"])


def test_scf_benchmark_config_applies_overrides():
    from amaterasu_b200.scf_benchmark import _config
    c = _config("si215_gamma", "mixed", {"refine_max_iterations": 3})
    assert c.engine.precision == "mixed" and c.engine.refine_max_iterations == 3
    assert c.occupations.scheme == "gaussian" and c.scf.tol_energy == 1e-5
