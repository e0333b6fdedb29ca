"""Generates the golden fixtures of tests/golden/ from the upstream build.

The upstream sources are compiled unmodified by oracle/Makefile into
oracle/_ref/libggbref32.so (as shipped) and oracle/_ref/libggbref64.so
(-Dfloat=double); this script runs the parity cases of tests/ggb_cases.py on
them with one OpenMP thread and stores the results.  Run from the repository
root:  python tests/golden/make_golden.py
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "gaseous-gusty-ball_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import ggb_api  # noqa: E402
import ggb_cases as K  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def save(name, d):
    np.savez_compressed(os.path.join(OUT, name), **{k: np.asarray(v) for k, v in d.items()})
    print("wrote", name, os.path.getsize(os.path.join(OUT, name + ".npz")), "bytes")


def main():
    r32 = ggb_api.Api(os.path.join(ROOT, "oracle", "_ref", "libggbref32.so"), ctypes.c_float)
    r64 = ggb_api.Api(os.path.join(ROOT, "oracle", "_ref", "libggbref64.so"), ctypes.c_double)
    r32.lib.drv_set_threads(1)
    for N in (8, 16):
        save(f"grid_N{N}", K.grid_tables(r32, N))
    # point location of the 100k test directions at N=64
    g = r32.grid(64)
    dirs = K.lcg_dirs()
    cells = np.array([g.cell_of(d) for d in dirs], np.int32)
    centres = np.array([g.cell_of(p) for p in g.arrays()["pos"].astype(np.float64)], np.int32)
    g.free()
    save("cellof_N64", dict(cells=cells, centres=centres))
    save("ops_N16", K.operators(r32, 16))
    save("poisson_N16", K.poisson(r32, 16))
    # a short full run (initial state from the upstream build's driver)
    g = r32.grid(16)
    vel0, vband = K.initial_velocity(r32, g)
    g.free()
    run = K.run(r32, 16, 600, 40, 4, vel0, vband)
    run.update(vel_init=vel0, vband=vband)
    save("run_N16", run)
    g = r64.grid(16)
    v64, b64 = K.initial_velocity(r64, g)
    g.free()
    run64 = K.run(r64, 16, 600, 40, 4, v64, b64)
    run64.update(vel_init=v64, vband=b64)
    save("run64_N16", run64)
    prev, pos, col = K.random_arcs(800, seed=7, max_angle=0.08)
    dep = K.deposit(r32, 48, prev, pos, col, fade_steps=3)
    dep.update(prev=prev, pos=pos, col=col)
    save("deposit_R48", dep)


if __name__ == "__main__":
    main()
