import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

# per-pose energy tolerance: 1e-5 relative or 1e-4 kcal/mol absolute
REL_TOL = 1e-5
ABS_TOL_KJ = 1e-4 * 4.184


def energy_close(a, b, scale=None):
    """|a - b| <= max(1e-5 * scale, 1e-4 kcal/mol); scale defaults to |b|.

    The engine sums FP32 pair terms, so its error is bounded relative to the
    condition of the sum: the tests pass scale = sum over pairs of |LJ| +
    |Coulomb| from the FP64 oracle (for a translate/rotate dE = E_new - E_old,
    the sum over both energies' pairs)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    sc = np.abs(b) if scale is None else np.asarray(scale, dtype=np.float64)
    return np.abs(a - b) <= np.maximum(REL_TOL * sc, ABS_TOL_KJ)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def native_lib():
    from pygcmc_b200 import build
    build.build()
    from pygcmc_b200._native import lib
    return lib()


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def protein_small(native_lib):
    from pygcmc_b200 import system as S
    return S.protein_system(seed=3, n_atoms=3000, box=48.0, radius=18.0, mcsteps=400, conf_bias=256)


@pytest.fixture(scope="session")
def water_small(native_lib):
    from pygcmc_b200 import system as S
    return S.water_box(n_water=400, box=26.0, seed=2, mcsteps=200, conf_bias=128)
