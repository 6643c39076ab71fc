"""Shared test set-up: the `gpu` marker, import paths, and problem builders used by several tests."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# Material and cohesive constants of the benchmark RVEs: matrix E = 3.5 GPa, nu = 0.35; fiber
# E = 72 GPa, nu = 0.22 (in MPa); bilinear interface sigma_c = 50 MPa, delta_c2 = 5e-3 * L and
# an initial stiffness sigma_c / delta_c1 with delta_c1 = delta_c2 / 1e4.
E_M, NU_M, E_F, NU_F = 3.5e3, 0.35, 72e3, 0.22
LAW_PARAMS = {
    1: (50.0, 5e-7, 5e-3, 0.0),       # BL: sigma_c, delta_c1, delta_c2
    2: (50.0, 5e-7, 5e-3, 0.0),       # BLNU
    3: (50.0, 2e-4, 3e-4, 1.0),       # XN: sigma_c, delta_cn, delta_ct, q
    4: (50.0, 2e-4, 3e-4, 1.0),       # XNNU
    5: (50.0, 2e-4, 1.0, 0.0),        # OP: sigma_c, delta_c, beta
    6: (50.0, 2e-4, 1.0, 0.0),        # OPNU
    7: (50.0, 2e-4, 1.0, 0.0),        # OPAUG
    8: (50.0, 2e-4, 1.0, 0.0),        # OPNUAUG
}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def random_dof_field(n_free: int, n_const: int, seed: int, scale: float = 1e-3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(-scale, scale, n_free + n_const)


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle library (oracle/_ref) not built")
    return ref
