import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "ed-lgt_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libedgpu.so")


@pytest.fixture(scope="session")
def golden_small():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "small_cases.npz"))


@pytest.fixture(scope="session")
def golden_generic():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "generic_su2_cases.npz"))


@pytest.fixture(scope="session")
def golden_string():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "string_cases.npz"))


@pytest.fixture(scope="session")
def golden_pins():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "validation_pins.npz"))


@pytest.fixture(scope="session")
def golden_big():
    import numpy as np

    path = os.path.join(GOLDEN, "big_cases.npz")
    if not os.path.exists(path):
        pytest.skip("big_cases.npz not generated")
    return np.load(path)


@pytest.fixture(scope="session")
def golden_dyn():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "dynamics_cases.npz"))


@pytest.fixture(scope="session")
def golden_twobody():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "twobody_cases.npz"))


@pytest.fixture(scope="session")
def golden_entropy():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "entropy_cases.npz"))


@pytest.fixture(scope="session")
def golden_momentum():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "momentum_cases.npz"))


@pytest.fixture(scope="session")
def golden_full():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "full_spectrum_cases.npz"))


@pytest.fixture(scope="session")
def golden_nbody():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "nbody_cases.npz"))


@pytest.fixture(scope="session")
def golden_overlap():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "overlap_cases.npz"))


@pytest.fixture(scope="session")
def golden_state():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "state_cases.npz"))


@pytest.fixture(scope="session")
def golden_local():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "local_hamiltonian_cases.npz"))


@pytest.fixture(scope="session")
def golden_integrated():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "integrated_cases.npz"))


@pytest.fixture(scope="session")
def golden_wide():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "wide_cases.npz"))


@pytest.fixture(scope="session")
def golden_thermal():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "thermal_cases.npz"))
