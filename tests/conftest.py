"""Shared test setup.

Markers: `gpu` tests need a CUDA device (run on the B200 box); everything
else runs on the CPU.  The CUDA library and the CLIs are loaded from the
package directory; GPU tests fail (not skip) when they are missing.
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.dirname(__file__))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def load_gb():
    spec = importlib.util.spec_from_file_location(
        "goldbach_gpu_b200", os.path.join(ROOT, "goldbach-gpu_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["goldbach_gpu_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def gbmod():
    return load_gb()


@pytest.fixture(scope="session")
def ctx(gbmod):
    c = gbmod.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib
    return oracle_lib.Oracle()
