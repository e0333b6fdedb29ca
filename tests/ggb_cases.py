"""Parity cases that run on any library exporting the gaseous-gusty-ball API.

Each case takes an ``ggb_api.Api`` and returns a dict of numpy arrays.  The
same case run on the CUDA product, on the CPU restatement and on the upstream
build gives the arrays that the tests compare; tests/golden/make_golden.py
stores the upstream build's results as fixtures.
"""
import ctypes as C

import numpy as np

import ggb_api as G
import ggb_inputs


def lcg_dirs(count=100_000, seed=12345):
    """The 100k directions of upstream tests/test_cubesphere.c:31-34
    (LCG s = s*1664525 + 1013904223, frand = (s >> 8) / 2^24)."""
    s = np.uint64(seed)
    out = np.empty((count, 3), np.float64)
    vals = np.empty(3 * count, np.float64)
    m = np.uint64(0xFFFFFFFF)
    for k in range(3 * count):
        s = (s * np.uint64(1664525) + np.uint64(1013904223)) & m
        vals[k] = float(int(s) >> 8) / 16777216.0
    v = vals.reshape(count, 3) * 2 - 1
    out[:] = v / np.linalg.norm(v, axis=1, keepdims=True)
    return out


def grid_tables(api, N):
    g = api.grid(N)
    a = g.arrays()
    out = {k: v.copy() for k, v in a.items()}
    out["total_area"] = np.array(g.cs.total_area)
    out["asym_count"] = np.array(g.cs.asym_count)
    out["open_cells"] = np.array(g.cs.open_cells)
    g.free()
    return out


def sorted_links(t):
    """Per-cell links sorted by neighbour index: (nbr, w, elen, gc) with -1 / 0 padding."""
    n = t["nnb"].shape[0]
    nb = np.full((n, 8), -1, np.int64)
    w = np.zeros((n, 8), np.float64)
    el = np.zeros((n, 8), np.float64)
    gc = np.zeros((n, 8, 3), np.float64)
    for c in range(n):
        m = int(t["nnb"][c])
        order = np.argsort(t["nbr"][c, :m], kind="stable")
        nb[c, :m] = t["nbr"][c, :m][order]
        w[c, :m] = t["w"][c, :m][order]
        el[c, :m] = t["elen"][c, :m][order]
        gc[c, :m] = t["gc"][c, :m][order]
    return nb, w, el, gc


def psi_exact(p):
    """psi = x*y + z/2 (l = 2 and l = 1 harmonics); upstream tests/test_poisson.c:10-13."""
    return p[:, 0] * p[:, 1] + 0.5 * p[:, 2]


def lap_exact(p):
    return -6 * p[:, 0] * p[:, 1] - 1.0 * p[:, 2]


def operators(api, N):
    """Laplacian of psi_exact, curl / divergence of a smooth tangent field, mean removal."""
    g = api.grid(N)
    n, nr = g.n, api.np_real
    pos = g.arrays()["pos"].astype(np.float64)
    x = psi_exact(pos).astype(nr)
    y = np.zeros(n, nr)
    api.lib.fluid_laplacian(C.byref(g.cs), api.ptr(x), api.ptr(y))
    # tangent field: rotation about a tilted axis plus a gradient-like part
    ax = np.array([0.3, 0.9, 0.2])
    vel = np.cross(ax, pos) + 0.5 * (np.array([0, 0, 1.0]) - pos * pos[:, 2:3])
    vel = np.ascontiguousarray(vel.reshape(-1), nr)
    curl = np.zeros(n, nr)
    div = np.zeros(n, nr)
    api.lib.fluid_curl(C.byref(g.cs), api.ptr(vel), api.ptr(curl))
    api.lib.fluid_divergence(C.byref(g.cs), api.ptr(vel), api.ptr(div))
    f = (pos[:, 0] + 2.0).astype(nr)
    api.lib.fluid_remove_mean(C.byref(g.cs), api.ptr(f))
    g.free()
    return dict(lap=y, curl=curl, div=div, mean_removed=f)


TABLE_KEYS = ("pos", "area", "nnb", "nbr", "w", "elen", "gc")


def tables_of(api, N):
    """The public grid tables of `api`'s cs_init(N) (copies) and its total area."""
    g = api.grid(N)
    out = {k: v.copy() for k, v in g.arrays().items()}
    out["total_area"] = float(g.cs.total_area)
    g.free()
    return out


def load_tables(api, g, tables):
    """Overwrites the public tables of grid g (before any fluid_init on it)
    with `tables`, so that a library built with FP64 storage solves exactly
    the discrete problem whose FP32 tables another library built: its
    operators read these arrays.  (The upstream FP32 and FP64 builds compute
    different grids: the FP64 build keeps cell positions in double, and its
    cell areas differ from the FP32 build's by up to 0.2 %.)"""
    a = g.arrays()
    for k in TABLE_KEYS:
        a[k][...] = tables[k].astype(a[k].dtype)
    g.cs.total_area = tables["total_area"]


def poisson(api, N, tol=1e-6, maxit=5000, mixed=False, tables=None):
    """upstream tests/test_poisson.c:51-72: solve Laplacian(psi) = lap_exact."""
    g = api.grid(N)
    if tables is not None:
        load_tables(api, g, tables)
    fs = G.FluidSim(api, g, cg_tol=tol, cg_maxit=maxit, mixed=mixed)
    pos = g.arrays()["pos"].astype(np.float64)
    om = fs.field("omega")
    om[:] = lap_exact(pos).astype(api.np_real)
    api.lib.fluid_remove_mean(C.byref(g.cs), fs.F.omega)
    it = api.lib.fluid_solve_psi(C.byref(fs.F))
    api.lib.fluid_compute_velocity(C.byref(fs.F))
    out = dict(psi=fs.field("psi").copy(), vel=fs.field("vel", 3).copy(), iters=np.array(it),
               relres=np.array(fs.F.cg_relres))
    fs.free()
    g.free()
    return out


def initial_velocity(api, g, seed=1, bands=8):
    """Initial velocity of the application driver, computed by `api`'s driver
    (drv_initial_velocity) or its GPU kernel (ggb_initial_velocity)."""
    n = g.n
    ip = G.InitParams(bands, 1.0, 0.5, 3.0, 2.0, 0.5, 4, seed)
    vel = np.zeros(3 * n, api.np_real)
    vb = np.zeros(3 * n, api.np_real)
    fn = api.lib.drv_initial_velocity if api.has("drv_initial_velocity") else api.lib.ggb_initial_velocity
    fn(C.byref(g.cs), C.byref(ip), api.ptr(vel), api.ptr(vb))
    return vel, vb


def run(api, N, particles, R, steps, vel0, vband, forcing=0.5, rotation=3.0, tol=1e-6, fixed_dt=0.0,
        cfl=1.0, fade=0.02, strip_seed=1, bfecc=1, snaps=(), dts_in=None, maxit=500, mixed=False, tables=None):
    """The application driver's step loop (upstream src/main.c:421-438):
    dt from CFL, particles_advect, fluid_step, render_fade, render_deposit.
    snaps: steps after which the state is recorded in out["snap"][step];
    dts_in: the time step of every step (instead of the CFL step);
    tables: grid tables to load into the grid first (load_tables)."""
    g = api.grid(N)
    if tables is not None:
        load_tables(api, g, tables)
    fs = G.FluidSim(api, g, forcing=forcing, rotation=rotation, cg_tol=tol, bfecc=bfecc, cg_maxit=maxit, mixed=mixed)
    nr = api.np_real
    fs.set_state(np.asarray(vel0, nr), None if vband is None else np.asarray(vband, nr))
    out = dict(omega0=fs.field("omega").copy(), psi0=fs.field("psi").copy(), vel0=fs.field("vel", 3).copy(),
               it0=np.array(fs.F.cg_iters))
    ps = G.ParticleSet(api, particles)
    ps.colour(ggb_inputs.strip(strip_seed))
    out["col"] = ps.array("col", 4).copy()
    sp = G.Splat(api, R)
    dts, cgs = [], []
    if snaps:
        out["snap"] = {}
    for s in range(steps):
        dt = fixed_dt
        if dts_in is not None:
            dt = float(dts_in[s])
        elif dt <= 0:
            vmax = fs.max_speed()
            dt = cfl * g.cs.h / (vmax if vmax > 1e-6 else 1e-6)
        ps.advect(g, fs.F.vel, dt)
        fs.step(dt)
        sp.fade(fade)
        sp.deposit(ps)
        dts.append(dt)
        cgs.append(fs.F.cg_iters)
        if s + 1 in snaps:
            out["snap"][s + 1] = dict(omega=fs.field("omega").copy(), psi=fs.field("psi").copy(),
                                      vel=fs.field("vel", 3).copy(), pos=ps.array("pos", 3).copy(),
                                      faces=sp.faces())
    out.update(omega=fs.field("omega").copy(), psi=fs.field("psi").copy(), vel=fs.field("vel", 3).copy(),
               pos=ps.array("pos", 3).copy(), prev=ps.array("prev", 3).copy(), faces=sp.faces(),
               dts=np.array(dts), cg=np.array(cgs), g=np.array(sp.r.g))
    sp.free()
    ps.free()
    fs.free()
    g.free()
    return out


def deposit(api, R, prev, pos, col, fade_steps=0, fade=0.02, radius=1.0, alpha=0.35):
    """One render_deposit of given particle arcs (after `fade_steps` fades).
    With the GPU library, out["windowed"] is the number of tiles composited in
    several key-range windows (ggb_render_stats)."""
    ps = G.ParticleSet(api, prev.shape[0])
    nr = api.np_real
    ps.array("prev", 3)[:] = prev.astype(nr)
    ps.array("pos", 3)[:] = pos.astype(nr)
    ps.array("col", 4)[:] = col.astype(nr)
    sp = G.Splat(api, R, radius, alpha)
    for _ in range(fade_steps):
        sp.fade(fade)
    sp.deposit(ps)
    out = dict(faces=sp.faces(), g=np.array(sp.r.g))
    if api.has("ggb_render_stats"):
        nt, nw, ne = C.c_uint(), C.c_uint(), C.c_uint()
        api.lib.ggb_render_stats(C.byref(sp.r), C.byref(nt), C.byref(nw), C.byref(ne))
        out["windowed"] = nw.value
    sp.free()
    ps.free()
    return out


def random_arcs(n, seed, max_angle):
    """n random unit-vector arcs (prev, pos) of angle <= max_angle, and colours."""
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, 3))
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    t = rng.normal(size=(n, 3))
    t -= a * np.sum(t * a, axis=1, keepdims=True)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    th = rng.uniform(0, max_angle, size=(n, 1))
    b = a * np.cos(th) + t * np.sin(th)
    col = rng.uniform(0.05, 1.0, size=(n, 4))
    return a.astype(np.float32), b.astype(np.float32), col.astype(np.float32)


def solve_fp64(orc64, N, tables, omega, tol=1e-12):
    """psi and u of the FP64 oracle solving omega on the given grid tables
    (remove_mean, fluid_solve_psi, fluid_compute_velocity)."""
    g = orc64.grid(N)
    load_tables(orc64, g, tables)
    fs = G.FluidSim(orc64, g, cg_tol=tol, cg_maxit=20000)
    fs.field("omega")[:] = np.asarray(omega, np.float64)
    orc64.lib.fluid_remove_mean(C.byref(g.cs), fs.F.omega)
    orc64.lib.fluid_solve_psi(C.byref(fs.F))
    orc64.lib.fluid_compute_velocity(C.byref(fs.F))
    out = dict(psi=fs.field("psi").copy(), vel=fs.field("vel", 3).copy())
    fs.free()
    g.free()
    return out


def angle_between(a, b):
    """Angle (rad) between corresponding rows of two arrays of 3-vectors, in
    FP64 as atan2(|a x b|, a . b): accurate for small angles, where the
    arccos of a normalised dot product loses half the digits (FP32 norms of
    unit vectors alone would read as angles of some 1e-4)."""
    a = np.asarray(a, np.float64).reshape(-1, 3)
    b = np.asarray(b, np.float64).reshape(-1, 3)
    return np.arctan2(np.linalg.norm(np.cross(a, b), axis=1), np.sum(a * b, 1))
