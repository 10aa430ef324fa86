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


def test_device_timeout_is_raised_not_ignored(monkeypatch):
    """A timed-out device wait (device error word != 0) must stop the SCF step: the check
    reads the tensor-core and eigensolver status words and raises; with every word clear
    it returns quietly."""
    import ctypes as ct

    from amaterasu_b200 import engine as E

    words = {"ama_tc_status": 0, "ama_subspace_tc_status": 0, "ama_solver_status": 0}

    def fake_call(name, *args):
        out = args[-1]  # ctypes byref(c_int32)
        ct.cast(out, ct.POINTER(ct.c_int32))[0] = words[name]

    monkeypatch.setattr(E, "call", fake_call)

    class FakeEngine:
        handle = ct.c_void_p(1)

    E.check_device_status(FakeEngine())
    words["ama_subspace_tc_status"] = 3
    with pytest.raises(E.DeviceTimeout, match="subspace tensor-core"):
        E.check_device_status(FakeEngine())
    words.update(ama_subspace_tc_status=0, ama_tc_status=2)
    with pytest.raises(E.DeviceTimeout, match="nonlocal"):
        E.check_device_status(FakeEngine())
    words.update(ama_tc_status=0, ama_solver_status=1)
    with pytest.raises(E.DeviceTimeout, match="eigensolver"):
        E.check_device_status(FakeEngine())
