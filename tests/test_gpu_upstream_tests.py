"""The upstream test programs (tests/test_*.c of gaseous-gusty-ball), compiled
unchanged against the upstream headers and linked against libggb_cuda.so
(oracle/Makefile builds them into oracle/_ref/test_*_cuda), must pass."""
import os
import subprocess

import pytest

from conftest import REF_BUILD


def _run(name):
    exe = os.path.join(REF_BUILD, f"test_{name}_cuda")
    if not os.path.exists(exe):
        pytest.skip(f"{exe} was not built (needs the upstream sources at build time)")
    p = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0 and f"test_{name}: OK" in p.stdout, p.stdout + p.stderr
    return p.stdout


def test_upstream_noise_test_on_product_library():
    """noise.h is host code in the product, so this one runs without a GPU."""
    _run("noise")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cubesphere", "poisson", "flow"])
def test_upstream_test_on_product_library(name):
    print(_run(name))
