"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on any machine: the oracle against the reference's
known-answer tests, the host logic, and the C ABI's exports. `-m gpu` runs
the CUDA path against the oracle on a B200.
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for path in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 and the built CUDA library")


@pytest.fixture(scope="session")
def cuda_lib():
    """The built library; a GPU test fails (does not skip) when it is absent."""
    from tangle_b200.build import build
    from tangle_b200.device import load_library

    build()
    return load_library()
