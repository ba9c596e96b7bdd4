"""Test infrastructure (the checker, never the product): a numpy restatement
of layercom_cig's stitching of depth-window ADCIG volumes
(src/layercom_cig.cpp).  Pinned bit for bit to the reference tool's outputs
in tests/golden/golden_stitch.npz (tests/test_stitch_oracle.py).

Volumes are [n3][n2][n1] float32 (depth n1 fastest), as the RSF files."""
from __future__ import annotations

import math

import numpy as np


def blend_weights(count: int) -> np.ndarray:
    """src/layercom_cig.cpp:522-528: w = 0.5 (1 - cos(pi u)), u = bi / (count - 1)
    (u = 1 for a single row), in double, rounded once to float."""
    u = [bi / (count - 1) if count > 1 else 1.0 for bi in range(count)]
    return np.array([0.5 * (1.0 - math.cos(3.14159265358979323846 * x)) for x in u], np.float32)


def lateral_scale(n2: int, aper: int, scale: float) -> np.ndarray:
    """src/layercom_cig.cpp:455-466: a linear taper from `scale` at the two
    lateral edges to 1 over `aper` columns (double, rounded once)."""
    out = np.ones(n2, np.float32)
    if aper > 0:
        for i2 in range(n2):
            edge = min(i2, n2 - 1 - i2)
            if edge < aper:
                taper = 1.0 if aper == 1 else 1.0 - edge / (aper - 1)
                out[i2] = np.float32(1.0 + (scale - 1.0) * taper)
    return out


def stitch(n1: int, windows, volumes, scales=None, stitch_blend: int = 15, scalex_aper: int = 0,
           scalex_scale: float = 1.0) -> np.ndarray:
    """src/layercom_cig.cpp:470-535.  windows: [(start, end)] depth rows;
    volumes: [n3][n2][end-start+1] float32 each.  Raises ValueError naming
    the window (1-based) whose scaled samples are not all finite."""
    n3, n2 = volumes[0].shape[0], volumes[0].shape[1]
    scales = [1.0] * len(windows) if scales is None else scales
    lat = lateral_scale(n2, scalex_aper, scalex_scale)
    out = np.zeros((n3, n2, n1), np.float32)
    previous_end = -1
    for k, ((start, end), vol) in enumerate(zip(windows, volumes)):
        vol = np.asarray(vol, np.float32)
        assert vol.shape == (n3, n2, end - start + 1)
        sx = lat if k > 0 else np.ones(n2, np.float32)
        scale = (np.float32(scales[k]) * sx).astype(np.float32)          # [n2]
        with np.errstate(over="ignore", invalid="ignore"):
            v = (vol * scale[None, :, None]).astype(np.float32)
        bad = ~np.isfinite(v)
        if bad.any():
            raise ValueError("window %d contains non-finite samples after scaling" % (k + 1))
        overlap = previous_end - start + 1 if k > 0 else 0
        blend = min(stitch_blend, overlap) if (overlap > 0 and stitch_blend >= 0) else overlap
        keep = overlap - blend
        # rows below the window above: written
        out[:, :, start + overlap:end + 1] = v[:, :, overlap:]
        # shared rows: the first `keep` keep the upper value, the rest blend
        if overlap > 0 and blend > 0:
            w = blend_weights(blend)[None, None, :]
            rows = slice(start + keep, start + overlap)
            o = out[:, :, rows]
            out[:, :, rows] = (o * (np.float32(1.0) - w)).astype(np.float32) + \
                (v[:, :, keep:overlap] * w).astype(np.float32)
        previous_end = end
    return out
