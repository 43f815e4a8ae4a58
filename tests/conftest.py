"""Shared test set-up: the `gpu` marker, and loaders for the library binding and the oracle."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "gpu-n-queens_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def load_nqb():
    """Imports the package directory gpu-n-queens_b200/ as module `gpu_n_queens_b200`."""
    name = "gpu_n_queens_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_nqo():
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import nqo
    return nqo


def load_nqsf():
    load_nqo()
    import nqsf
    return nqsf


@pytest.fixture(scope="session")
def nqsf():
    return load_nqsf()


@pytest.fixture(scope="session")
def nqb():
    return load_nqb()


@pytest.fixture(scope="session")
def nqo():
    return load_nqo()
