"""ggb_remove_mean_noalloc — the mean removal for callers that cannot allocate
device memory (a process whose device memory is all reserved by another
allocator, or a steady-state loop that must not call cudaMalloc / cudaFree,
which synchronise the device).  Its output must equal fluid_remove_mean's on
the same input, on two calls in a row (the second call runs on scratch that
still holds the first call's partial sums).  This file is collected last so
that a run stopping at the first failure has run every other test first."""
import ctypes as C

import numpy as np
import pytest

import ggb_api as G
import ggb_cases as K

pytestmark = pytest.mark.gpu


def _bind(gpu):
    gpu.lib.ggb_remove_mean_noalloc.restype = C.c_int
    gpu.lib.ggb_remove_mean_noalloc.argtypes = [C.POINTER(gpu.T["CubeSphere"]), C.POINTER(C.c_float)]


# N=64: 24,576 cells, exactly six 4096-cell blocks; N=50: 15,000 cells, whose
# last block is partial (its cell range is clamped to the grid)
@pytest.mark.parametrize("N", [64, 50])
def test_noalloc_mean_removal_matches_fluid_remove_mean(gpu, N):
    _bind(gpu)
    g = gpu.grid(N)
    fs = G.FluidSim(gpu, g)  # two device-resident (managed) buffers of ncells floats
    a, b = fs.field("omega"), fs.field("psi")
    pos = g.arrays()["pos"].astype(np.float64)
    rng = np.random.default_rng(5)
    for call, field in enumerate((K.psi_exact(pos) + 3.0, rng.normal(2.0, 1.0, size=g.n))):
        a[:] = field.astype(np.float32)
        b[:] = field.astype(np.float32)
        gpu.lib.fluid_remove_mean(C.byref(g.cs), fs.F.omega)
        rc = gpu.lib.ggb_remove_mean_noalloc(C.byref(g.cs), fs.F.psi)
        assert rc == 0, f"call {call}"
        # same mean to FP32 rounding: both reduce the same FP64 sum in another order
        assert np.max(np.abs(a.astype(np.float64) - b)) <= 1e-6 * np.max(np.abs(field)), f"call {call}"
        assert abs(float(np.sum(g.arrays()["area"].astype(np.float64) * b))) < 1e-5
    fs.free()
    g.free()


def test_noalloc_rejects_host_buffers(gpu):
    """A pageable host array would need a staging allocation: the entry point
    refuses it with -1 and leaves it untouched."""
    _bind(gpu)
    g = gpu.grid(16)
    f = np.linspace(1.0, 2.0, g.n).astype(np.float32)
    keep = f.copy()
    rc = gpu.lib.ggb_remove_mean_noalloc(C.byref(g.cs), f.ctypes.data_as(C.POINTER(C.c_float)))
    assert rc == -1
    assert np.array_equal(f, keep)
    g.free()
