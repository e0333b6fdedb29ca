"""ctypes binding of the gaseous-gusty-ball C API.

The API is the one of the upstream headers src/cubesphere.h, src/fluid.h,
src/particles.h, src/render.h and src/noise.h (same struct layouts, same
symbols), as exported by this package's ``libggb_cuda.so`` (and by any other
library that implements the same API with the same layouts).  ``real`` is the
element type of the stored arrays: ``ctypes.c_float`` for the API as declared,
``ctypes.c_double`` for a build compiled with ``-Dfloat=double``.

Python here is plumbing for tests and benchmarks; the computation happens in
the loaded library.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIB = os.path.join(HERE, "libggb_cuda.so")


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


def _types(real):
    P = C.POINTER

    class CubeSphere(C.Structure):
        _fields_ = [("N", C.c_int), ("ncells", C.c_int), ("h", C.c_double), ("pos", P(real)),
                    ("area", P(real)), ("nnb", P(C.c_ubyte)), ("nbr", P(C.c_int)), ("w", P(real)),
                    ("elen", P(real)), ("gc", P(real)), ("total_area", C.c_double),
                    ("asym_count", C.c_int), ("open_cells", C.c_int)]

    class FluidParams(C.Structure):
        _fields_ = [("forcing", C.c_double), ("rotation", C.c_double), ("bfecc", C.c_int),
                    ("cg_tol", C.c_double), ("cg_maxit", C.c_int), ("multigrid", C.c_int)]

    class MGLevel(C.Structure):
        _fields_ = [("cs", CubeSphere), ("x", P(real)), ("b", P(real)), ("r", P(real)),
                    ("dinv", P(real)), ("ptap", P(C.c_int)), ("pw", P(real)), ("rstart", P(C.c_int)),
                    ("ridx", P(C.c_int)), ("rw", P(real))]

    class Fluid(C.Structure):
        _fields_ = [("cs", P(CubeSphere)), ("prm", FluidParams), ("nlev", C.c_int), ("lev", P(MGLevel))] + \
                   [(nm, P(real)) for nm in ("omega", "omega_band", "psi", "vel", "q0", "q1", "q2", "dep_b",
                                             "dep_f", "r", "p", "Ap", "z", "dinv")] + \
                   [("cg_iters", C.c_int), ("cg_relres", C.c_double)]

    class Particles(C.Structure):
        _fields_ = [("n", C.c_int), ("pos", P(real)), ("prev", P(real)), ("col", P(real))]

    class SplatRec(C.Structure):
        _fields_ = [("px", real), ("py", real), ("pidx", C.c_uint32), ("bin", C.c_uint32)]

    class ThreadRecs(C.Structure):
        _fields_ = [("v", P(SplatRec)), ("n", C.c_size_t), ("cap", C.c_size_t), ("hist", P(C.c_size_t)),
                    ("cursor", P(C.c_size_t))]

    class Render(C.Structure):
        _fields_ = [("R", C.c_int), ("buf", P(real)), ("g", C.c_double), ("radius", real), ("alpha", real),
                    ("strip_h", C.c_int), ("nstrips", C.c_int), ("nbins", C.c_int), ("maxthreads", C.c_int),
                    ("tr", P(ThreadRecs)), ("sorted", P(SplatRec)), ("sorted_cap", C.c_size_t),
                    ("bin_start", P(C.c_size_t))]

    class Noise(C.Structure):
        _fields_ = [("perm", C.c_ubyte * 512)]

    class CurlParams(C.Structure):
        _fields_ = [("scale", C.c_double), ("lacunarity", C.c_double), ("gain", C.c_double), ("octaves", C.c_int)]

    return dict(CubeSphere=CubeSphere, FluidParams=FluidParams, MGLevel=MGLevel, Fluid=Fluid,
                Particles=Particles, Render=Render, Noise=Noise, CurlParams=CurlParams)


class InitParams(C.Structure):
    """Initial-condition parameters (bands, noise) of the application driver."""
    _fields_ = [("bands", C.c_int), ("band_amp", C.c_double), ("noise_amp", C.c_double),
                ("noise_scale", C.c_double), ("noise_lacunarity", C.c_double), ("noise_gain", C.c_double),
                ("noise_octaves", C.c_int), ("seed", C.c_uint)]


def _view(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).view(dtype)


class Api:
    """The C API of one library.  ``real`` is c_float or c_double."""

    def __init__(self, path, real=C.c_float, mode=None):
        self.path = path
        self.real = real
        self.np_real = np.float32 if real is C.c_float else np.float64
        self.lib = C.CDLL(path, mode=mode if mode is not None else C.RTLD_LOCAL)
        self.T = _types(real)
        T, L, P = self.T, self.lib, C.POINTER
        R = P(real)
        sig = {
            "cs_init": (C.c_int, [P(T["CubeSphere"]), C.c_int]),
            "cs_free": (None, [P(T["CubeSphere"])]),
            "cs_face_of": (C.c_int, [Vec3]),
            "cs_face_ab_to_dir": (Vec3, [C.c_int, C.c_double, C.c_double]),
            "cs_locate": (None, [P(T["CubeSphere"]), Vec3, P(C.c_int), P(C.c_double), P(C.c_double)]),
            "cs_cell_of": (C.c_int, [P(T["CubeSphere"]), Vec3]),
            "cs_taps": (None, [P(T["CubeSphere"]), Vec3, P(C.c_int), P(C.c_double)]),
            "cs_sample_scalar": (C.c_double, [P(T["CubeSphere"]), R, Vec3]),
            "cs_sample_vec": (Vec3, [P(T["CubeSphere"]), R, Vec3]),
            "fluid_init": (C.c_int, [P(T["Fluid"]), P(T["CubeSphere"]), P(T["FluidParams"])]),
            "fluid_free": (None, [P(T["Fluid"])]),
            "fluid_curl": (None, [P(T["CubeSphere"]), R, R]),
            "fluid_divergence": (None, [P(T["CubeSphere"]), R, R]),
            "fluid_laplacian": (None, [P(T["CubeSphere"]), R, R]),
            "fluid_remove_mean": (None, [P(T["CubeSphere"]), R]),
            "fluid_set_state": (None, [P(T["Fluid"]), R, R]),
            "fluid_solve_psi": (C.c_int, [P(T["Fluid"])]),
            "fluid_compute_velocity": (None, [P(T["Fluid"])]),
            "fluid_step": (None, [P(T["Fluid"]), C.c_double]),
            "fluid_max_speed": (C.c_double, [P(T["Fluid"])]),
            "particles_init": (C.c_int, [P(T["Particles"]), C.c_int]),
            "particles_free": (None, [P(T["Particles"])]),
            "particles_color_from_image": (None, [P(T["Particles"]), R, C.c_int, C.c_int]),
            "particles_advect": (None, [P(T["Particles"]), P(T["CubeSphere"]), R, C.c_double]),
            "render_init": (C.c_int, [P(T["Render"]), C.c_int, real, real]),
            "render_free": (None, [P(T["Render"])]),
            "render_fade": (None, [P(T["Render"]), C.c_double]),
            "render_deposit": (None, [P(T["Render"]), P(T["Particles"])]),
            "render_texel": (None, [P(T["Render"]), C.c_int, C.c_int, C.c_int, R]),
            "render_sample_dir": (None, [P(T["Render"]), C.c_double, C.c_double, C.c_double, R]),
            "render_pixel8": (None, [R, R, P(C.c_ubyte)]),
            "noise_init": (None, [P(T["Noise"]), C.c_uint]),
            "simplex3": (C.c_double, [P(T["Noise"]), Vec3, P(Vec3)]),
            "curl_noise": (Vec3, [P(T["Noise"]), Vec3, P(T["CurlParams"])]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        self.sig = sig
        # optional extras
        for name, res, args in [
            ("ggb_launch_count", C.c_long, []),
            ("ggb_render_read", None, [P(T["Render"]), R]),
            ("ggb_render_stats", None, [P(T["Render"]), P(C.c_uint), P(C.c_uint), P(C.c_uint)]),
            ("ggb_render_repeats", C.c_ulong, [P(T["Render"])]),
            ("ggb_render_repeats_grown", C.c_ulong, [P(T["Render"])]),
            ("ggb_encode_faces", C.c_int, [P(T["Render"]), P(C.c_float), P(C.c_int), P(C.c_ubyte)]),
            ("ggb_encode_net", C.c_int, [P(T["Render"]), P(C.c_float), P(C.c_ubyte)]),
            ("ggb_checkpoint_save", C.c_int, [C.c_char_p, P(T["Fluid"]), P(T["Particles"]), P(T["Render"])]),
            ("ggb_batch_create", C.c_void_p, [C.c_int, P(P(T["Fluid"])), P(P(T["Particles"])), P(P(T["Render"])),
                                              P(C.c_double), P(C.c_double)]),
            ("ggb_batch_step", C.c_int, [C.c_void_p, C.c_int]),
            ("ggb_batch_solve_blocks", C.c_int, [C.c_void_p, C.c_int]),
            ("ggb_batch_blocks", None, [C.c_void_p, P(C.c_int)]),
            ("ggb_batch_solve_ms", C.c_double, [C.c_void_p]),
            ("ggb_batch_cost", C.c_double, [C.c_int, C.c_int]),
            ("ggb_batch_dt", None, [C.c_void_p, P(C.c_double)]),
            ("ggb_batch_free", None, [C.c_void_p]),
            ("ggb_batch_host_ms", C.c_double, [C.c_void_p, P(C.c_double), P(C.c_double)]),
            ("ggb_checkpoint_load", C.c_int, [C.c_char_p, P(T["Fluid"]), P(T["Particles"]), P(T["Render"])]),
            ("ggb_encode_preview", C.c_int, [P(T["Render"]), P(C.c_float), P(C.c_ubyte)]),
            ("ggb_initial_velocity", None, [P(T["CubeSphere"]), P(InitParams), R, R]),
            ("drv_initial_velocity", None, [P(T["CubeSphere"]), P(InitParams), R, R]),
            ("drv_run", C.c_long, [P(T["CubeSphere"]), P(T["Fluid"]), P(T["Particles"]), P(T["Render"]),
                                   C.c_int, C.c_double, C.c_double, C.c_double, P(C.c_double), P(C.c_int),
                                   P(C.c_double)]),
            ("ggb_fluid_set_precision", C.c_int, [P(T["Fluid"]), C.c_int]),
            ("ggb_solve_flags", C.c_int, [P(T["Fluid"])]),
            ("drv_max_threads", C.c_int, []),
            ("drv_set_threads", None, [C.c_int]),
        ]:
            if hasattr(L, name):
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args

    def has(self, name):
        return hasattr(self.lib, name)

    def ptr(self, arr):
        """Pointer to a contiguous numpy array of the stored element type."""
        assert arr.dtype == self.np_real and arr.flags["C_CONTIGUOUS"]
        return arr.ctypes.data_as(C.POINTER(self.real))

    # ------------------------------------------------------------ objects
    def grid(self, N):
        return Grid(self, N)


class Grid:
    def __init__(self, api, N):
        self.api = api
        self.cs = api.T["CubeSphere"]()
        rc = api.lib.cs_init(C.byref(self.cs), N)
        if rc != 0:
            raise RuntimeError(f"cs_init({N}) failed in {api.path}")

    @property
    def n(self):
        return self.cs.ncells

    def arrays(self):
        a, cs, n, nr = self.api, self.cs, self.cs.ncells, self.api.np_real
        return dict(pos=_view(cs.pos, 3 * n, nr).reshape(n, 3), area=_view(cs.area, n, nr),
                    nnb=_view(cs.nnb, n, np.uint8), nbr=_view(cs.nbr, 8 * n, np.int32).reshape(n, 8),
                    w=_view(cs.w, 8 * n, nr).reshape(n, 8), elen=_view(cs.elen, 8 * n, nr).reshape(n, 8),
                    gc=_view(cs.gc, 24 * n, nr).reshape(n, 8, 3))

    def free(self):
        if self.cs.pos:
            self.api.lib.cs_free(C.byref(self.cs))

    def cell_of(self, d):
        return self.api.lib.cs_cell_of(C.byref(self.cs), Vec3(*map(float, d)))

    def locate(self, d):
        f, x, y = C.c_int(), C.c_double(), C.c_double()
        self.api.lib.cs_locate(C.byref(self.cs), Vec3(*map(float, d)), C.byref(f), C.byref(x), C.byref(y))
        return f.value, x.value, y.value


class FluidSim:
    """Fluid + optional particles / render for one grid."""

    def __init__(self, api, grid, forcing=0.0, rotation=0.0, bfecc=1, cg_tol=1e-4, cg_maxit=500, multigrid=1,
                 mixed=False):
        self.api, self.grid = api, grid
        T = api.T
        self.prm = T["FluidParams"](forcing, rotation, bfecc, cg_tol, cg_maxit, multigrid)
        self.F = T["Fluid"]()
        if api.lib.fluid_init(C.byref(self.F), C.byref(grid.cs), C.byref(self.prm)) != 0:
            raise RuntimeError("fluid_init failed")
        if mixed:
            # the mixed-precision solve exists only in the CUDA library
            if not api.has("ggb_fluid_set_precision"):
                raise RuntimeError(f"{api.path} has no mixed-precision solve")
            if api.lib.ggb_fluid_set_precision(C.byref(self.F), 1) != 0:
                raise RuntimeError("ggb_fluid_set_precision failed")

    def field(self, name, comps=1):
        n = self.grid.n
        return _view(getattr(self.F, name), comps * n, self.api.np_real)

    def set_state(self, vel, vband=None):
        a = self.api
        vel = np.ascontiguousarray(vel, a.np_real)
        vb = None if vband is None else a.ptr(np.ascontiguousarray(vband, a.np_real))
        a.lib.fluid_set_state(C.byref(self.F), a.ptr(vel), vb)

    def step(self, dt):
        self.api.lib.fluid_step(C.byref(self.F), float(dt))

    def solve(self):
        return self.api.lib.fluid_solve_psi(C.byref(self.F))

    def max_speed(self):
        return self.api.lib.fluid_max_speed(C.byref(self.F))

    def free(self):
        if self.F.omega:
            self.api.lib.fluid_free(C.byref(self.F))


class ParticleSet:
    def __init__(self, api, n):
        self.api = api
        self.P = api.T["Particles"]()
        if api.lib.particles_init(C.byref(self.P), int(n)) != 0:
            raise RuntimeError("particles_init failed")

    def array(self, name, comps):
        return _view(getattr(self.P, name), comps * self.P.n, self.api.np_real).reshape(self.P.n, comps)

    def colour(self, img):
        a = self.api
        img = np.ascontiguousarray(img, a.np_real)
        h, w = img.shape[:2]
        a.lib.particles_color_from_image(C.byref(self.P), a.ptr(img), w, h)

    def advect(self, grid, vel_ptr, dt):
        self.api.lib.particles_advect(C.byref(self.P), C.byref(grid.cs), vel_ptr, float(dt))

    def free(self):
        if self.P.pos:
            self.api.lib.particles_free(C.byref(self.P))


class Splat:
    def __init__(self, api, R, radius=1.0, alpha=0.35):
        self.api = api
        self.r = api.T["Render"]()
        if api.lib.render_init(C.byref(self.r), int(R), radius, alpha) != 0:
            raise RuntimeError("render_init failed")

    def fade(self, f):
        self.api.lib.render_fade(C.byref(self.r), float(f))

    def deposit(self, ps):
        self.api.lib.render_deposit(C.byref(self.r), C.byref(ps.P))

    def faces(self):
        """All texels (premultiplied RGBA) as [6, R, R, 4]."""
        a, R = self.api, self.r.R
        out = np.empty((6, R, R, 4), a.np_real)
        if a.has("ggb_render_read"):
            a.lib.ggb_render_read(C.byref(self.r), a.ptr(out))
        else:
            buf = _view(self.r.buf, 6 * R * R * 4, a.np_real).reshape(6, R, R, 4)
            out[...] = buf * a.np_real(self.r.g)
        return out

    def free(self):
        if self.r.buf:
            self.api.lib.render_free(C.byref(self.r))


IMAGE_IO_LIB = os.path.join(HERE, "libggb_image_io.so")


class ImageIO:
    """PNG files through libggb_image_io.so (the upstream src/image_io.h API:
    ``png_load_rgba``, ``png_save``)."""

    def __init__(self, path=IMAGE_IO_LIB):
        self.lib = C.CDLL(path)
        self.lib.png_load_rgba.restype = C.POINTER(C.c_float)
        self.lib.png_load_rgba.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        self.lib.png_save.restype = C.c_int
        self.lib.png_save.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        self._free = C.CDLL(None).free
        self._free.argtypes = [C.c_void_p]

    def load(self, path):
        """float32 array (h, w, 4) in [0, 1], or None when the file is rejected."""
        w, h = C.c_int(0), C.c_int(0)
        p = self.lib.png_load_rgba(os.fsencode(path), C.byref(w), C.byref(h))
        if not p:
            return None
        try:
            return np.ctypeslib.as_array(p, shape=(h.value * w.value * 4,)).copy().reshape(h.value, w.value, 4)
        finally:
            self._free(p)

    def save(self, path, img):
        """img: uint8 array (h, w, 3 or 4).  Returns png_save's status (0 or -1)."""
        img = np.ascontiguousarray(img, dtype=np.uint8)
        h, w, ch = img.shape
        return self.lib.png_save(os.fsencode(path), w, h, ch, img.ctypes.data)
