"""The C-ABI boundary, checked without a GPU: libggb_cuda.so loads and exports
every function and data symbol that include/*.h declares (image_io.h's PNG
functions: libggb_image_io.so), and the struct
layouts of include/*.h equal those of the upstream headers (so callers built
against either header share one ABI)."""
import ctypes
import os
import re
import subprocess

import pytest

import ggb_api
from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")


def _upstream_src():
    """The upstream header directory: $GGB_UPSTREAM_SRC, else the one that
    oracle/Makefile recorded when it built the upstream sources (None when
    neither exists, e.g. on a machine without the upstream sources)."""
    p = os.environ.get("GGB_UPSTREAM_SRC")
    if not p:
        rec = os.path.join(ROOT, "oracle", "_ref", "upstream_src.path")
        if os.path.exists(rec):
            p = open(rec).read().strip()
    return p if p and os.path.isdir(p) else None


UPSTREAM_SRC = _upstream_src()


def _strip_bodies(text):
    """Drop everything inside braces that follow a ')' (inline function bodies)."""
    out, depth, i = [], 0, 0
    while i < len(text):
        ch = text[i]
        if ch == "{" and (depth or text[:i].rstrip().endswith(")")):
            depth += 1
        elif ch == "}" and depth:
            depth -= 1
            if depth == 0:
                out.append(";")
        elif not depth:
            out.append(ch)
        i += 1
    return "".join(out)


# header -> the library that exports its functions (all others: libggb_cuda.so)
OTHER_LIBS = {"image_io.h": ggb_api.IMAGE_IO_LIB}


def declared_symbols(headers=None):
    """Function names declared (not defined inline) in include/*.h (or in the
    given header names), plus extern data."""
    funcs, data = set(), set()
    for fn in sorted(os.listdir(INCLUDE)):
        if not fn.endswith(".h") or (headers is not None and fn not in headers):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = _strip_bodies(text)
        for m in re.finditer(r"^\s*(?!static|typedef|#|return)[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text,
                             flags=re.M):
            funcs.add(m.group(1))
        for m in re.finditer(r"^\s*extern\s+const\s+\w+\s+(\w+)\s*\[", text, flags=re.M):
            data.add(m.group(1))
    return funcs, data


def test_headers_declare_the_upstream_api():
    funcs, data = declared_symbols()
    expected = {"cs_init", "cs_free", "cs_face_of", "cs_face_ab_to_dir", "cs_locate", "cs_cell_of", "cs_taps",
                "cs_sample_scalar", "cs_sample_vec", "fluid_init", "fluid_free", "fluid_curl", "fluid_divergence",
                "fluid_laplacian", "fluid_remove_mean", "fluid_set_state", "fluid_solve_psi",
                "fluid_compute_velocity", "fluid_step", "fluid_max_speed", "particles_init", "particles_free",
                "particles_color_from_image", "particles_advect", "render_init", "render_free", "render_fade",
                "render_deposit", "render_texel", "render_sample_dir", "render_pixel8", "noise_init", "simplex3",
                "curl_noise"}
    assert expected <= funcs, expected - funcs
    assert data == {"cs_face_center", "cs_face_right", "cs_face_up"}


def test_product_library_exports_every_declared_symbol():
    assert os.path.exists(ggb_api.PRODUCT_LIB), "build the library first (__graft_entry__.build())"
    lib = ctypes.CDLL(ggb_api.PRODUCT_LIB)
    mine = [h for h in os.listdir(INCLUDE) if h.endswith(".h") and h not in OTHER_LIBS]
    funcs, data = declared_symbols(mine)
    missing = [s for s in sorted(funcs | data) if not hasattr(lib, s)]
    assert not missing, missing
    for header, path in OTHER_LIBS.items():
        other = ctypes.CDLL(path)
        funcs, _ = declared_symbols([header])
        assert funcs and not [s for s in funcs if not hasattr(other, s)], (header, funcs)


def test_product_library_has_no_cpu_fallback_symbols():
    """The product never links the checker: none of the oracle / driver symbols."""
    out = subprocess.run(["nm", "-D", "--defined-only", ggb_api.PRODUCT_LIB], capture_output=True, text=True).stdout
    assert "drv_run" not in out and "drv_initial_velocity" not in out
    needed = subprocess.run(["readelf", "-d", ggb_api.PRODUCT_LIB], capture_output=True, text=True).stdout
    assert "oracle" not in needed


LAYOUT_PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "cubesphere.h"
#include "fluid.h"
#include "particles.h"
#include "render.h"
#include "noise.h"
#define P(T, f) printf(#T "." #f " %zu\n", offsetof(T, f))
int main(void) {
  printf("CubeSphere %zu\nFluidParams %zu\nMGLevel %zu\nFluid %zu\nParticles %zu\nRender %zu\nNoise %zu\nCurlParams %zu\n",
         sizeof(CubeSphere), sizeof(FluidParams), sizeof(MGLevel), sizeof(Fluid), sizeof(Particles), sizeof(Render),
         sizeof(Noise), sizeof(CurlParams));
  P(CubeSphere, h); P(CubeSphere, gc); P(CubeSphere, total_area); P(CubeSphere, open_cells);
  P(Fluid, prm); P(Fluid, lev); P(Fluid, omega); P(Fluid, vel); P(Fluid, dinv); P(Fluid, cg_iters); P(Fluid, cg_relres);
  P(Particles, col); P(Render, g); P(Render, radius); P(Render, tr); P(Render, bin_start);
  return 0;
}
"""


def _layout(tmp_path, incdir, tag):
    src = tmp_path / f"probe_{tag}.c"
    src.write_text(LAYOUT_PROBE)
    exe = tmp_path / f"probe_{tag}"
    subprocess.run(["/usr/bin/gcc", "-std=gnu11", f"-I{incdir}", "-o", str(exe), str(src), "-lm"], check=True)
    return subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout


def test_struct_layouts_match_ctypes(tmp_path):
    lines = dict(l.rsplit(" ", 1) for l in _layout(tmp_path, INCLUDE, "inc").strip().splitlines())
    T = ggb_api._types(ctypes.c_float)
    for name in ("CubeSphere", "FluidParams", "MGLevel", "Fluid", "Particles", "Render", "Noise", "CurlParams"):
        assert int(lines[name]) == ctypes.sizeof(T[name]), name
    assert int(lines["Fluid.cg_relres"]) == T["Fluid"].cg_relres.offset


@pytest.mark.skipif(UPSTREAM_SRC is None, reason="upstream headers not present on this machine "
                                                 "(set GGB_UPSTREAM_SRC or build oracle/_ref)")
def test_struct_layouts_match_upstream_headers(tmp_path):
    assert _layout(tmp_path, INCLUDE, "inc") == _layout(tmp_path, UPSTREAM_SRC, "up")
