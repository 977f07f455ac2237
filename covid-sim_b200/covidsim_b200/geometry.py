"""Distances used by the host side (set-up only), restating src/Dist.cpp."""
import math

import numpy as np

EARTH_RADIUS = (40003200 / 3.1415926535) / 2  # src/Constants.h:10-58


def dist2_utm(p, x1, y1, x2, y2):
    """dist2UTM (src/Dist.cpp:23-48) on scalars, with the cs_params tables."""
    x = abs(x1 - x2) / 2
    y = abs(y1 - y2) / 2
    xi, yi = math.floor(x), math.floor(y)
    x -= xi
    y -= yi
    x = (1 - x) * p.sinx[int(xi)] + x * p.sinx[int(xi) + 1]
    y = (1 - y) * p.sinx[int(yi)] + y * p.sinx[int(yi) + 1]
    yt = abs(y1 + p.bbox_bottom_left_y)
    yi = math.floor(yt)
    cy1 = yt - yi
    cy1 = (1 - cy1) * p.cosx[int(yi)] + cy1 * p.cosx[int(yi) + 1]
    yt = abs(y2 + p.bbox_bottom_left_y)
    yi = math.floor(yt)
    cy2 = yt - yi
    cy2 = (1 - cy2) * p.cosx[int(yi)] + cy2 * p.cosx[int(yi) + 1]
    x = abs(1000 * (y * y + x * x * cy1 * cy2))
    xi = math.floor(x)
    x -= xi
    y = (1 - x) * p.asin2sqx[int(xi)] + x * p.asin2sqx[int(xi) + 1]
    return 4 * EARTH_RADIUS * EARTH_RADIUS * y


def dist2_raw(p, ax, ay, bx, by):
    """dist2_raw (src/Dist.cpp:162-169)."""
    if p.DoUTM_coords:
        return dist2_utm(p, ax, ay, bx, by)
    x, y = abs(ax - bx), abs(ay - by)
    if p.DoPeriodicBoundaries:
        if x > p.width_deg * 0.5:
            x = p.width_deg - x
        if y > p.height_deg * 0.5:
            y = p.height_deg - y
    return x * x + y * y


def km_per_degree(lat_deg):
    """Approximate metres per degree of longitude and latitude at a latitude."""
    return 111195.0 * math.cos(math.radians(lat_deg)), 111195.0


def morton2(ix, iy, bits=16):
    """Interleave the low `bits` bits of two integer arrays (Z-order curve)."""
    ix = np.asarray(ix, dtype=np.uint64)
    iy = np.asarray(iy, dtype=np.uint64)

    def spread(v):
        v = v & np.uint64(0xFFFFFFFF)
        v = (v | (v << np.uint64(16))) & np.uint64(0x0000FFFF0000FFFF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x3333333333333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x5555555555555555)
        return v

    return spread(ix) | (spread(iy) << np.uint64(1))
