import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libyamc_b200.so")


def _write(spec, tmp_path_factory, name, seed=1):
    from yamc_b200 import systems
    d = str(tmp_path_factory.mktemp(name))
    return systems.write_system(spec, d, seed=seed)


@pytest.fixture(scope="session")
def tiny_files(tmp_path_factory):
    from yamc_b200 import systems
    return _write(systems.small_spec(), tmp_path_factory, "tiny")


@pytest.fixture(scope="session")
def tiny_biased_files(tmp_path_factory):
    from yamc_b200 import systems
    return _write(systems.small_spec(name="tinyb", xlambda=0.1), tmp_path_factory, "tinyb", seed=2)


@pytest.fixture(scope="session")
def spce_files(tmp_path_factory):
    from yamc_b200 import systems
    return _write(systems.WORKLOADS["spce256"], tmp_path_factory, "spce256")


@pytest.fixture(scope="session")
def nacl_files(tmp_path_factory):
    from yamc_b200 import systems
    return _write(systems.WORKLOADS["nacl1m"], tmp_path_factory, "nacl1m", seed=3)


@pytest.fixture(scope="session")
def nacl4k_files(tmp_path_factory):
    from yamc_b200 import systems
    return _write(systems.WORKLOADS["nacl4k"], tmp_path_factory, "nacl4k", seed=5)


@pytest.fixture(scope="session")
def nacl16k_files(tmp_path_factory):
    from yamc_b200 import systems
    return _write(systems.WORKLOADS["nacl16k"], tmp_path_factory, "nacl16k", seed=6)
