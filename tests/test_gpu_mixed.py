"""The mixed-precision Poisson solve (ggb_fluid_set_precision(F, 1)): FP16
V-cycle vectors and coarse slot weights with FP32 accumulation inside a
flexible FP32 CG; FP64 dots, residual norm and mean projections.

Its error is stated against the FP64 oracle (the CPU restatement built with
FP64 storage, solved to 1e-10 or below) on the same grid tables as the GPU
(the upstream FP64 build computes its own, slightly different grid, whose
cell areas differ by up to 0.2 %; ggb_cases.load_tables):
  * psi relative L2 error <= 1e-5 of a solve at tolerance 1e-6 (N=64 and the
    N=512 grid of the large workload; a forced, rotating flow at N=128);
  * velocity <= 5e-5: u is a difference of neighbouring FP32 psi values, so
    FP32 storage of psi alone limits it to about 1e-5;
  * the iteration count stays within two of the plain solve's;
  * a multi-step run with forcing and rotation follows the FP32 restatement
    to 1e-4 relative L2, as the plain path does.
"""
import ctypes as C

import numpy as np
import pytest

import ggb_cases as K

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("N", [64, 512])
def test_mixed_poisson_vs_fp64_oracle(gpu, orc64, N):
    ref = K.poisson(orc64, N, tol=1e-10, tables=K.tables_of(gpu, N))
    mixed = K.poisson(gpu, N, tol=1e-6, mixed=True)
    plain = K.poisson(gpu, N, tol=1e-6)
    e_psi, e_vel = rel_l2(mixed["psi"], ref["psi"]), rel_l2(mixed["vel"], ref["vel"])
    print(f"N={N}: mixed psi rel {e_psi:.2e}, vel rel {e_vel:.2e}, its {int(mixed['iters'])} "
          f"(plain {int(plain['iters'])}, plain psi rel {rel_l2(plain['psi'], ref['psi']):.2e})")
    assert float(mixed["relres"]) <= 1e-6
    assert e_psi <= 1e-5 and e_vel <= 5e-5
    assert abs(int(mixed["iters"]) - int(plain["iters"])) <= 2


def test_mixed_short_run(gpu, orc32):
    g = orc32.grid(32)
    vel0, vband = K.initial_velocity(orc32, g, seed=3)
    g.free()
    a = K.run(gpu, 32, 3000, 96, 5, vel0, vband, forcing=0.5, rotation=3.0, mixed=True)
    b = K.run(orc32, 32, 3000, 96, 5, vel0, vband, forcing=0.5, rotation=3.0)
    assert np.max(np.abs(a["cg"] - b["cg"])) <= 2
    for k in ("omega", "psi", "vel"):
        assert rel_l2(a[k], b[k]) < 1e-4, (k, rel_l2(a[k], b[k]))


def test_mixed_solve_of_a_running_flow(gpu, orc64):
    """psi of the mixed solve after 10 steps of a forced, rotating flow at
    N=128, against the FP64 solve of the same omega on the same tables
    (tolerance 1e-12)."""
    go = orc64.grid(128)
    v64, b64 = K.initial_velocity(orc64, go, seed=4)
    go.free()
    a = K.run(gpu, 128, 20000, 128, 10, v64.astype(np.float32), b64.astype(np.float32), forcing=0.5,
              rotation=10.0, tol=1e-6, mixed=True)
    ref = K.solve_fp64(orc64, 128, K.tables_of(gpu, 128), a["omega"])
    e_psi, e_vel = rel_l2(a["psi"], ref["psi"]), rel_l2(a["vel"], ref["vel"])
    print(f"running flow N=128: mixed psi rel {e_psi:.2e}, vel rel {e_vel:.2e}, its {a['cg'].tolist()}")
    assert e_psi <= 1e-5 and e_vel <= 5e-5
