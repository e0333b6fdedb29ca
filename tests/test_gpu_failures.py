"""Failure detection, exercised without faulting the GPU.

  * a grid barrier whose wait runs out: one block of a cooperative launch
    never arrives, the others give up after a short limit and return, and the
    device stays usable;
  * a NaN written into omega: the solve ends as upstream's would (no
    iterations, relres NaN) and records why in its status bits;
  * a solve stopped by cg_maxit records it;
  * corrupted public grid arrays are reported by the validator;
  * allocation failure, injected on the host: cs_init, particles_init and
    render_init return -1 (upstream's convention for them) and the library
    keeps working afterwards.
"""
import ctypes as C
import math

import numpy as np
import pytest

import ggb_api as G
import ggb_cases as K

pytestmark = pytest.mark.gpu

SOLVE_TIMEOUT, SOLVE_NONFINITE, SOLVE_BREAKDOWN, SOLVE_MAXIT = 1, 2, 4, 8


def _bind(gpu):
    L = gpu.lib
    L.ggb_barrier_timeout_probe.restype = C.c_int
    L.ggb_barrier_timeout_probe.argtypes = [C.c_double, C.POINTER(C.c_double)]
    L.ggb_barrier_bench.restype = C.c_double
    L.ggb_barrier_bench.argtypes = [C.c_int]
    L.ggb_solve_flags.restype = C.c_int
    L.ggb_solve_flags.argtypes = [C.POINTER(gpu.T["Fluid"])]
    L.ggb_grid_validate.restype = C.c_long
    L.ggb_grid_validate.argtypes = [C.POINTER(gpu.T["CubeSphere"])]
    L.ggb_inject_alloc_failure.restype = None
    L.ggb_inject_alloc_failure.argtypes = [C.c_long]


def _poisson_flags(gpu, N, omega_fn, tol=1e-6, maxit=500):
    g = gpu.grid(N)
    fs = G.FluidSim(gpu, g, cg_tol=tol, cg_maxit=maxit)
    pos = g.arrays()["pos"].astype(np.float64)
    fs.field("omega")[:] = omega_fn(pos).astype(np.float32)
    it = gpu.lib.fluid_solve_psi(C.byref(fs.F))
    out = dict(it=it, relres=fs.F.cg_relres, flags=gpu.lib.ggb_solve_flags(C.byref(fs.F)),
               psi=fs.field("psi").copy())
    fs.free()
    g.free()
    return out


def test_barrier_wait_runs_out_and_returns(gpu):
    _bind(gpu)
    ms = C.c_double()
    assert gpu.lib.ggb_barrier_timeout_probe(5.0, C.byref(ms)) == 1
    # the waiting blocks gave up after about the limit, not the 2 s default
    assert 4.0 <= ms.value < 500.0, ms.value
    # the context is intact: complete barriers and a solve still work
    assert gpu.lib.ggb_barrier_bench(100) > 0
    ok = _poisson_flags(gpu, 16, lambda p: K.lap_exact(p))
    assert ok["flags"] == 0 and ok["relres"] <= 1e-6


def test_nan_in_omega_is_reported(gpu):
    _bind(gpu)

    def om(p):
        w = K.lap_exact(p)
        w[123] = np.nan
        return w

    r = _poisson_flags(gpu, 16, om)
    assert r["flags"] & SOLVE_NONFINITE
    assert r["it"] == 0 and math.isnan(r["relres"])
    # a clean solve afterwards has no flags
    assert _poisson_flags(gpu, 16, lambda p: K.lap_exact(p))["flags"] == 0


def test_maxit_is_reported(gpu):
    _bind(gpu)
    r = _poisson_flags(gpu, 32, lambda p: K.lap_exact(p), tol=1e-12, maxit=2)
    assert r["it"] == 2 and r["flags"] == SOLVE_MAXIT and r["relres"] > 1e-12


def test_grid_validate_detects_corruption(gpu):
    _bind(gpu)
    g = gpu.grid(16)
    assert gpu.lib.ggb_grid_validate(C.byref(g.cs)) == 0
    a = g.arrays()
    keep_w, keep_nb, keep_area = a["w"][3, 0], a["nbr"][7, 1], a["area"][11]
    a["w"][3, 0] = np.nan
    a["nbr"][7, 1] = -5
    a["area"][11] = 0.0
    assert gpu.lib.ggb_grid_validate(C.byref(g.cs)) == 3
    a["w"][3, 0], a["nbr"][7, 1], a["area"][11] = keep_w, keep_nb, keep_area
    assert gpu.lib.ggb_grid_validate(C.byref(g.cs)) == 0
    g.free()


@pytest.mark.parametrize("after", [0, 3, 12])
def test_injected_allocation_failure(gpu, after):
    _bind(gpu)
    T = gpu.T
    cs = T["CubeSphere"]()
    P = T["Particles"]()
    r = T["Render"]()
    gpu.lib.ggb_inject_alloc_failure(after)
    try:
        rc_cs = gpu.lib.cs_init(C.byref(cs), 32)
        gpu.lib.ggb_inject_alloc_failure(min(after, 2))
        rc_p = gpu.lib.particles_init(C.byref(P), 1000)
        gpu.lib.ggb_inject_alloc_failure(0)
        rc_r = gpu.lib.render_init(C.byref(r), 64, C.c_float(1.0), C.c_float(0.35))
    finally:
        gpu.lib.ggb_inject_alloc_failure(-1)
    assert rc_cs == -1 and rc_p == -1 and rc_r == -1
    assert not cs.pos and not P.pos and not r.buf
    # allocation works again afterwards and the library is intact
    out = K.poisson(gpu, 16)
    assert float(out["relres"]) <= 1e-6
