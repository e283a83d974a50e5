"""Seeded synthetic still images for the intra-search workloads (no public dataset is named for them).

Luma is the sum of piecewise-constant random Voronoi cells (levels 16-235), random-orientation linear gradients,
random-orientation sinusoids with periods of 4-64 pixels and Gaussian noise (sigma 3); the 12 MP workload adds
oriented step edges (2-40 per 256x256 area).  Chroma planes use the same recipe at their own resolution, centred at
the mid level.  10-bit planes are the 8-bit recipe mapped with round(v * 1023 / 255) (the reference's 8->10-bit
mapping, encoder/src/k_misc.cu:351-372).  Deterministic for a seed (numpy PCG64).
"""
import numpy as np


def _plane(rng, w, h, centre, spread, edges, cell=48):
    """One plane: float64 array h x w, before noise and clipping."""
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    # Voronoi cells on a jittered grid: nearest of the seeds in the 3x3 neighbouring grid cells
    gw, gh = (w + cell - 1) // cell + 2, (h + cell - 1) // cell + 2
    sx = (np.arange(gw)[None, :] - 1 + rng.random((gh, gw))) * cell
    sy = (np.arange(gh)[:, None] - 1 + rng.random((gh, gw))) * cell
    lv = rng.uniform(centre - spread, centre + spread, (gh, gw))
    cx = (xx // cell).astype(np.int64) + 1
    cy = (yy // cell).astype(np.int64) + 1
    best = np.full((h, w), np.inf)
    val = np.zeros((h, w))
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            gx, gy = np.clip(cx + dx, 0, gw - 1), np.clip(cy + dy, 0, gh - 1)
            d = (xx - sx[gy, gx]) ** 2 + (yy - sy[gy, gx]) ** 2
            m = d < best
            best[m] = d[m]
            val[m] = lv[gy, gx][m]
    out = val
    diag = float(np.hypot(w, h))
    for _ in range(2):   # linear gradients
        th = rng.uniform(0, np.pi)
        a = rng.uniform(10, 40) * (spread / 110.0)
        out = out + a * ((xx - w / 2) * np.cos(th) + (yy - h / 2) * np.sin(th)) / (diag / 2)
    for _ in range(3):   # sinusoids, period 4-64 px
        th = rng.uniform(0, np.pi)
        per = rng.uniform(4, 64)
        a = rng.uniform(3, 12) * (spread / 110.0)
        ph = rng.uniform(0, 2 * np.pi)
        out = out + a * np.sin(2 * np.pi * (xx * np.cos(th) + yy * np.sin(th)) / per + ph)
    if edges:            # oriented step edges, 2-40 per 256x256 area, each over a disc of radius 24-96
        for ay in range(0, h, 256):
            for ax in range(0, w, 256):
                n = int(rng.integers(2, 41))
                for _ in range(n):
                    ex, ey = ax + rng.uniform(0, 256), ay + rng.uniform(0, 256)
                    th = rng.uniform(0, np.pi)
                    r = rng.uniform(24, 96)
                    amp = rng.choice([-1, 1]) * rng.uniform(10, 40) * (spread / 110.0)
                    x0, x1 = int(max(0, ex - r)), int(min(w, ex + r + 1))
                    y0, y1 = int(max(0, ey - r)), int(min(h, ey + r + 1))
                    if x0 >= x1 or y0 >= y1:
                        continue
                    px, py = xx[y0:y1, x0:x1] - ex, yy[y0:y1, x0:x1] - ey
                    m = (px * px + py * py < r * r) & (px * np.cos(th) + py * np.sin(th) > 0)
                    out[y0:y1, x0:x1] += amp * m
    return out


def make_image(width, height, seed, edges=False, bit_depth=8, chroma_444=False):
    """(Y, U, V) numpy planes (uint8 for 8-bit, uint16 for 10-bit), 4:2:0 chroma of ((w+1)//2, (h+1)//2)."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    cw, ch = (width, height) if chroma_444 else ((width + 1) // 2, (height + 1) // 2)
    planes = []
    for p, (w, h) in enumerate(((width, height), (cw, ch), (cw, ch))):
        if p == 0:
            f = _plane(rng, w, h, 125.5, 109.5, edges)
        else:
            f = _plane(rng, w, h, 128.0, 48.0, edges, cell=48 if chroma_444 else 24)
        f = f + rng.normal(0.0, 3.0, f.shape)
        v = np.clip(np.rint(f), 0, 255).astype(np.uint8)
        if bit_depth == 10:
            v = np.rint(v.astype(np.float64) * 1023.0 / 255.0).astype(np.uint16)
        planes.append(np.ascontiguousarray(v))
    return tuple(planes)


def make_smooth_image(width, height, seed, bit_depth=8, chroma_444=False):
    """A smooth image (low-amplitude gradients and long-period waves, no noise) on which the search keeps large blocks:
    the 64-sample-side blocks whose 4:4:4 chroma is coded in several tx blocks.  Same plane layout as make_image."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    cw, ch = (width, height) if chroma_444 else ((width + 1) // 2, (height + 1) // 2)
    planes = []
    for p, (w, h) in enumerate(((width, height), (cw, ch), (cw, ch))):
        yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
        f = np.full((h, w), 128.0 if p else rng.uniform(60, 180))
        for _ in range(2):
            th = rng.uniform(0, np.pi)
            f += rng.uniform(5, 25) * ((xx - w / 2) * np.cos(th) + (yy - h / 2) * np.sin(th)) / max(w, h)
        th, per = rng.uniform(0, np.pi), rng.uniform(60, 200)
        f += rng.uniform(2, 8) * np.sin(2 * np.pi * (xx * np.cos(th) + yy * np.sin(th)) / per)
        v = np.clip(np.rint(f), 0, 255).astype(np.uint8)
        if bit_depth == 10:
            v = np.rint(v.astype(np.float64) * 1023.0 / 255.0).astype(np.uint16)
        planes.append(np.ascontiguousarray(v))
    return tuple(planes)
