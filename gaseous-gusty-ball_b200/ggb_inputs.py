"""Seeded synthetic inputs of the benchmark workloads.

The strip is a 64 x 1024 (width x height) RGBA8 image of 16 equal horizontal
bands, each a seeded uniform-random RGB colour, with per-pixel uniform +-8
noise and alpha 255, returned as floats in [0, 1] (row 0 = north), which is
what the application driver's PNG loader hands to particles_color_from_image.
"""
import numpy as np


def strip(seed=1, width=64, height=1024, bands=16, noise=8):
    rng = np.random.default_rng(seed)
    cols = rng.integers(0, 256, size=(bands, 3))
    rows = np.minimum(np.arange(height) * bands // height, bands - 1)
    img = np.empty((height, width, 4), np.int32)
    img[..., :3] = cols[rows][:, None, :]
    img[..., :3] += rng.integers(-noise, noise + 1, size=(height, width, 3))
    img[..., 3] = 255
    return (np.clip(img, 0, 255).astype(np.float32) / 255.0)


# Workloads (sizes and physical settings of the configurations this
# implementation is measured and tested on).
SMALL = dict(N=64, particles=100_000, R=256, forcing=0.0, rotation=0.0, cg_tol=1e-4, cg_maxit=500,
             bands=8, band_amp=1.0, noise_amp=0.5, noise_scale=3.0, noise_lacunarity=2.0, noise_gain=0.5,
             noise_octaves=4, seed=1, cfl=1.0, fade=0.02, alpha=0.35, radius=1.0, steps=200, every=50)
DEFAULT = dict(SMALL, N=256, particles=1_000_000, R=1024, cg_tol=1e-6, steps=1000, every=100)


if __name__ == "__main__":
    # python ggb_inputs.py OUT.png [seed]: the strip as the application driver's
    # input image (8-bit RGBA, written through libggb_image_io.so)
    import os
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import ggb_api

    seed = int(sys.argv[2]) if len(sys.argv) > 2 else 1
    img = np.round(strip(seed) * 255).astype(np.uint8)
    if ggb_api.ImageIO().save(sys.argv[1], img) != 0:
        sys.exit(1)
