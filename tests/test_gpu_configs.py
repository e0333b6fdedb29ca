"""Parity of the CUDA path at the sizes of the measured workloads, through the
C ABI, against the CPU restatement on identical inputs (the restatement's own
initial velocity, strip colours and Fibonacci particles).

  * small workload, in full: N=64, 100,000 particles, 256^2 faces, upstream's
    default PCG tolerance 1e-4, 200 steps, compared every 50 steps;
  * default workload for 20 steps: N=256, 1,000,000 particles, 1024^2 faces:
    - at PCG tolerance 1e-4 against the FP32 restatement (at the workload's own
      tolerance 1e-6 the FP32 upstream solve diverges, so it has no FP32
      counterpart);
    - at tolerance 1e-6, plain and mixed precision, against the FP64 oracle on
      the same grid tables with the oracle's time steps: the trajectory, and
      the last solve against an FP64 solve of the same omega (1e-12).

The flow is chaotic, so differences of rounding size grow with the steps:
particles are compared by the median and 99th percentile of the angle between
their positions (the maximum is not a stable measure), and face images by the
mean absolute texel difference and the fraction of texel channels that differ
by more than 1e-2.  Every bound below is stated with the measured value it
covers (a B200 run of this build): a factor of a few above it.
"""
import numpy as np
import pytest

import ggb_cases as K
import ggb_inputs

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def angles(a, b):
    return K.angle_between(a, b)


def compare(a, b):
    ang = angles(a["pos"], b["pos"])
    d = np.abs(np.asarray(a["faces"], np.float64) - b["faces"])
    return dict(omega=rel_l2(a["omega"], b["omega"]), psi=rel_l2(a["psi"], b["psi"]), vel=rel_l2(a["vel"], b["vel"]),
                ang_med=float(np.median(ang)), ang_p99=float(np.percentile(ang, 99)), face_mean=float(d.mean()),
                face_frac=float((d > 1e-2).mean()))


def test_small_workload_full_run(gpu, orc32):
    """N=64, 100k particles, 256^2 faces, tolerance 1e-4, 200 steps."""
    S = ggb_inputs.SMALL
    g = orc32.grid(S["N"])
    vel0, vband = K.initial_velocity(orc32, g, seed=S["seed"], bands=S["bands"])
    g.free()
    snaps = (50, 100, 150, 200)
    kw = dict(forcing=S["forcing"], rotation=S["rotation"], tol=S["cg_tol"], snaps=snaps)
    a = K.run(gpu, S["N"], S["particles"], S["R"], S["steps"], vel0, vband, **kw)
    b = K.run(orc32, S["N"], S["particles"], S["R"], S["steps"], vel0, vband, **kw)
    assert np.max(np.abs(a["cg"] - b["cg"])) <= 1
    assert np.max(np.abs(a["dts"] - b["dts"]) / b["dts"]) < 1e-4
    for s in snaps:
        e = compare(a["snap"][s], b["snap"][s])
        print(f"small workload, step {s}: {e}")
        # measured at step 50: fields <= 4.5e-6, angles 2.7e-7 / 2.1e-6, face mean 3.2e-6
        # measured at step 200: fields <= 6.5e-5, angles 4.7e-6 / 1.3e-4, face mean 2.0e-4, frac 0.12 %
        f_tol, med_tol, p99_tol, mean_tol, frac_tol = (
            (3e-5, 2e-6, 2e-5, 3e-5, 1e-4) if s <= 50 else (3e-4, 3e-5, 1e-3, 1e-3, 1e-2))
        assert max(e["omega"], e["psi"], e["vel"]) < f_tol, (s, e)
        assert e["ang_med"] < med_tol and e["ang_p99"] < p99_tol, (s, e)
        assert e["face_mean"] < mean_tol and e["face_frac"] < frac_tol, (s, e)


def test_default_workload_fp32_tolerance_1e4(gpu, orc32):
    """N=256, 1M particles, 1024^2 faces, 20 steps at upstream's default
    tolerance against the FP32 restatement."""
    D = ggb_inputs.DEFAULT
    g = orc32.grid(D["N"])
    vel0, vband = K.initial_velocity(orc32, g, seed=D["seed"], bands=D["bands"])
    g.free()
    snaps = (5, 20)
    kw = dict(forcing=D["forcing"], rotation=D["rotation"], tol=1e-4, snaps=snaps)
    b = K.run(orc32, D["N"], D["particles"], D["R"], 20, vel0, vband, **kw)
    a = K.run(gpu, D["N"], D["particles"], D["R"], 20, vel0, vband, **kw)
    assert np.max(np.abs(a["cg"] - b["cg"])) <= 1
    for s in snaps:
        e = compare(a["snap"][s], b["snap"][s])
        print(f"default workload, tolerance 1e-4, step {s}: {e}")
        # measured at step 20: fields <= 1.8e-5, angles 5.6e-8 / 3.8e-7, face mean 4.0e-6, frac 1.2e-5
        assert max(e["omega"], e["psi"], e["vel"]) < 1e-4, (s, e)
        assert e["ang_med"] < 1e-6 and e["ang_p99"] < 5e-6, (s, e)
        assert e["face_mean"] < 5e-5 and e["face_frac"] < 1e-3, (s, e)


def test_default_workload_vs_fp64_oracle(gpu, orc64):
    """N=256, 1M particles, 1024^2 faces at the workload's tolerance 1e-6,
    plain and mixed precision, 20 steps against the FP64 oracle (tolerance
    1e-10) on the same grid tables and with the oracle's time steps."""
    D = ggb_inputs.DEFAULT
    N, n_p, R = D["N"], D["particles"], D["R"]
    g = orc64.grid(N)
    v64, b64 = K.initial_velocity(orc64, g, seed=D["seed"], bands=D["bands"])
    g.free()
    tab = K.tables_of(gpu, N)
    snaps = (5, 20)
    ref = K.run(orc64, N, n_p, R, 20, v64, b64, forcing=D["forcing"], rotation=D["rotation"], tol=1e-10, snaps=snaps,
                tables=tab)
    for mixed in (False, True):
        a = K.run(gpu, N, n_p, R, 20, v64.astype(np.float32), b64.astype(np.float32), forcing=D["forcing"],
                  rotation=D["rotation"], tol=D["cg_tol"], snaps=snaps, dts_in=ref["dts"], mixed=mixed)
        name = "mixed" if mixed else "plain"
        for s in snaps:
            e = compare(a["snap"][s], ref["snap"][s])
            print(f"default workload vs FP64 oracle, {name}, step {s}: {e}")
            assert e["psi"] < 1e-4 and e["vel"] < 1e-4 and e["omega"] < 1e-4, (name, s, e)
            assert e["ang_med"] < 1e-6 and e["ang_p99"] < 1e-5, (name, s, e)
        # the last solve against the FP64 solve of the same omega
        last = K.solve_fp64(orc64, N, tab, a["omega"])
        e_psi, e_vel = rel_l2(a["psi"], last["psi"]), rel_l2(a["vel"], last["vel"])
        print(f"default workload, {name}: last solve vs FP64 solve of the same omega: psi {e_psi:.2e}, u {e_vel:.2e}, "
              f"CG iterations {a['cg'].tolist()}")
        assert e_psi <= 1e-5 and e_vel <= 5e-5
