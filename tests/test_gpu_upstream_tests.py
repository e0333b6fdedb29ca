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


# ------------------------------------------------ the upstream application driver

# Small run of the driver: the settings of the short-run parity case (N=32,
# 3000 particles, 96^2 faces, 5 steps, forcing and rotation), all outputs.
DRIVER_ARGS = ["--grid", "32", "--particles", "3000", "--res", "96", "--steps", "5", "--every", "5", "--net",
               "--preview", "--seed", "3", "--forcing", "0.5", "--rotation", "3"]


def _driver(kind, tmp_path, extra=(), tag=""):
    """Run upstream src/main.c (unchanged) built by oracle/Makefile: `ref` on the
    upstream library, `cuda` on libggb_cuda.so; both write PNG files through
    libggb_image_io's zlib writer.  Returns {file name: decoded image}."""
    import numpy as np

    import ggb_inputs
    import pngfile
    exe = os.path.join(REF_BUILD, f"gaseous-gusty-ball_{kind}")
    if not os.path.exists(exe):
        pytest.skip(f"{exe} was not built (needs the upstream sources at build time)")
    src = tmp_path / "strip.png"
    if not src.exists():   # the seeded benchmark strip, written by the independent encoder
        src.write_bytes(pngfile.encode(np.round(ggb_inputs.strip() * 255).astype(np.int64), 6, 8))
    out = tmp_path / f"out_{kind}{tag}"
    p = subprocess.run([exe, "-i", str(src), "-o", str(out)] + DRIVER_ARGS + list(extra), capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "step 5/5" in p.stderr, p.stderr
    return {f: pngfile.decode((out / f).read_bytes())[0] for f in sorted(os.listdir(out))}


def test_upstream_driver_on_upstream_library_writes_png_files(tmp_path):
    """The driver links with the zlib PNG files in place of src/image_io.c and
    reads the strip / writes its outputs: faces, net, preview, GL names."""
    import numpy as np
    imgs = _driver("ref", tmp_path)
    assert sorted(imgs) == sorted([f"gg{k}.png" for k in range(6)] + ["gg-net.png", "gg-preview.png"])
    R = 96
    for k in range(6):
        assert imgs[f"gg{k}.png"].shape == (R, R, 4)
    assert imgs["gg-net.png"].shape == (3 * R, 4 * R, 4) and imgs["gg-preview.png"].shape == (R, 2 * R, 4)
    cell = {0: (1, 0), 1: (1, 1), 2: (1, 2), 3: (1, 3), 4: (0, 0), 5: (2, 0)}   # face -> (row, col) in the net
    for k, (cy, cx) in cell.items():
        np.testing.assert_array_equal(imgs["gg-net.png"][cy * R:(cy + 1) * R, cx * R:(cx + 1) * R], imgs[f"gg{k}.png"])
    assert imgs["gg0.png"][..., 3].max() > 0            # trails were drawn
    gl = _driver("ref", tmp_path, ["--layout", "gl", "--sequence", "--bg", "204060"], tag="gl")
    names = [f"gg-00005-{n}.png" for n in ("posx", "negx", "posy", "negy", "posz", "negz")]
    assert set(names) <= set(gl) and all(gl[n].shape == (R, R, 3) for n in names)


@pytest.mark.gpu
def test_upstream_driver_on_product_library_matches_upstream(tmp_path):
    """src/main.c linked against libggb_cuda.so runs the same job as on the
    upstream library, and its 8-bit outputs agree: opaque composites within one
    level in all but a few texels, the transparent alpha within one level."""
    import numpy as np
    for extra, tag in ((["--bg", "204060"], "bg"), ([], "")):
        a = _driver("cuda", tmp_path, extra, tag)
        b = _driver("ref", tmp_path, extra, tag)
        assert sorted(a) == sorted(b)
        for f in a:
            x, y = a[f].astype(np.int64), b[f].astype(np.int64)
            assert x.shape == y.shape, f
            if tag == "bg":
                d = np.abs(x - y)
                assert np.mean(d > 1) < 1e-3 and d.max() <= 8, (f, np.mean(d > 1), d.max())
                assert np.mean(d) < 0.05, (f, np.mean(d))
            else:
                assert np.abs(x[..., 3] - y[..., 3]).max() <= 1, f
