import os
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


def golden(name: str):
    path = GOLDEN / name
    if not path.exists():
        pytest.skip(f"golden fixture {name} not generated")
    return np.load(path, allow_pickle=False)


@pytest.fixture(scope="session")
def si_pseudo(tmp_path_factory):
    from amaterasu_b200.pseudo import read_upf, write_synthetic_upf
    path = write_synthetic_upf(tmp_path_factory.mktemp("pp") / "Si.synthetic.upf")
    return read_upf(path)


@pytest.fixture(scope="session")
def mini_system(si_pseudo):
    """Si2 fcc, ecut 8 Ha, two explicit k-points, 6 bands (the mini.npz system)."""
    from amaterasu_b200 import kpoints as kp
    from amaterasu_b200.cells import si2_primitive
    from amaterasu_b200.system import build_system
    ks = kp.explicit([[0.0, 0.0, 0.0], [0.125, -0.25, 0.375]])
    return build_system(si2_primitive(), {"Si": si_pseudo}, 8.0, 32.0, kpoints=ks, nbands=6)


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
