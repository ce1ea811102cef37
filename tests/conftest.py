import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libpmgpu.so")


_SYSTEMS = {}


def cached_system(name):
    """Seeded systems are deterministic; generate each once per session."""
    from protomol_b200 import systems
    if name not in _SYSTEMS:
        _SYSTEMS[name] = getattr(systems, name)()
    return _SYSTEMS[name]


@pytest.fixture(scope="session")
def water216():
    return cached_system("water_box_216")


@pytest.fixture(scope="session")
def chain14281():
    return cached_system("chain_in_water_14281")


@pytest.fixture(scope="session")
def small_chain():
    from protomol_b200 import systems
    return systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
