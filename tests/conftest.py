"""Shared fixtures of the test suite.

Libraries:
  product  gaseous-gusty-ball_b200/libggb_cuda.so        (the CUDA implementation)
  oracle   oracle/_build/liboracle*_{32,64}.so           (CPU restatement; checker only)
  ref      oracle/_ref/libggbref{32,64}.so               (upstream sources compiled
                                                          unmodified; present where they
                                                          were built)
GPU tests are marked ``gpu``; everything else runs on a CPU-only machine.
"""
import ctypes
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gaseous-gusty-ball_b200")
ORACLE_BUILD = os.path.join(ROOT, "oracle", "_build")
REF_BUILD = os.path.join(ROOT, "oracle", "_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, PKG)

import ggb_api  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAVE_GPU = _have_gpu()


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA GPU on this machine")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def _lib(path, real):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.relpath(path, ROOT)} is not built")
    return ggb_api.Api(path, real)


@pytest.fixture(scope="session")
def orc32():
    return _lib(os.path.join(ORACLE_BUILD, "liboracle_drv32.so"), ctypes.c_float)


@pytest.fixture(scope="session")
def orc64():
    return _lib(os.path.join(ORACLE_BUILD, "liboracle_drv64.so"), ctypes.c_double)


@pytest.fixture(scope="session")
def ref32():
    a = _lib(os.path.join(REF_BUILD, "libggbref32.so"), ctypes.c_float)
    a.lib.drv_set_threads(1)  # reductions in index order, like the serial restatement
    return a


@pytest.fixture(scope="session")
def ref64():
    a = _lib(os.path.join(REF_BUILD, "libggbref64.so"), ctypes.c_double)
    a.lib.drv_set_threads(1)
    return a


@pytest.fixture(scope="session")
def gpu():
    if not HAVE_GPU:
        pytest.skip("no CUDA GPU")
    path = ggb_api.PRODUCT_LIB
    if not os.path.exists(path):
        raise RuntimeError("libggb_cuda.so is missing: run __graft_entry__.build() first")
    return ggb_api.Api(path, ctypes.c_float)
