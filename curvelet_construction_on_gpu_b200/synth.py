"""Seeded synthetic third-order edge maps for the benchmark workloads.

The reference ships no benchmark data; these generators stand in for it with
the shapes, sizes and value distributions of the five workloads:

* ``plain_small``  480x320, 40 arcs + 10 segments, 10% clutter      (~6k edges)
* ``plain_hd``     1920x1080, 1,500 curves, 20% clutter             (~250k edges)
* ``mixed64``      64 maps, sizes from {640x480 .. 3840x2160}, density x U_log[0.25, 4]
* ``dense_4k``     3840x2160, 6,000 curves (half short high-curvature arcs), 40% clutter

Edges are rows ``x y theta strength`` (the column layout of the reference's
edge files, cpu_curvelet/data_io.hpp:22-79) with theta wrapped to (-pi, pi].
Curves are sampled every 1.0 px, with N(0, 0.1 px) position noise along the
normal and N(0, 0.03 rad) orientation noise; strength is U[2, 20] on curves and
U[1, 5] on clutter. Samples that fall outside the image are dropped.
Every map is a pure function of its seed (numpy PCG64).
"""
from __future__ import annotations

import math

import numpy as np

IMAGE_SIZES = [(640, 480), (1280, 720), (1920, 1080), (3840, 2160)]


def _wrap_pi(a: np.ndarray) -> np.ndarray:
    """Wraps to (-pi, pi]."""
    w = np.remainder(a + math.pi, 2.0 * math.pi) - math.pi
    w[w <= -math.pi] += 2.0 * math.pi
    return w


def _arcs(rng, n, W, H, radius, length):
    """n circular arcs: centre uniform in the image, random start angle and sense."""
    out = []
    cx = rng.uniform(0, W, n)
    cy = rng.uniform(0, H, n)
    phi0 = rng.uniform(0, 2 * math.pi, n)
    sense = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    length = np.minimum(length, 2 * math.pi * radius)
    for i in range(n):
        m = max(int(length[i]), 2)
        s = np.arange(m, dtype=np.float64)  # arc-length samples, 1.0 px apart
        phi = phi0[i] + sense[i] * s / radius[i]
        nx, ny = np.cos(phi), np.sin(phi)  # outward normal
        r = radius[i] + rng.normal(0.0, 0.1, m)
        x = cx[i] + r * nx
        y = cy[i] + r * ny
        tang = phi + sense[i] * (math.pi / 2)
        out.append((x, y, tang + rng.normal(0.0, 0.03, m)))
    return out


def _segments(rng, n, W, H, length):
    out = []
    x0 = rng.uniform(0, W, n)
    y0 = rng.uniform(0, H, n)
    ang = rng.uniform(0, 2 * math.pi, n)
    for i in range(n):
        m = max(int(length[i]), 2)
        s = np.arange(m, dtype=np.float64)
        dx, dy = math.cos(ang[i]), math.sin(ang[i])
        off = rng.normal(0.0, 0.1, m)
        x = x0[i] + s * dx - off * dy
        y = y0[i] + s * dy + off * dx
        out.append((x, y, ang[i] + rng.normal(0.0, 0.03, m)))
    return out


def _assemble(rng, curves, W, H, clutter_frac):
    if curves:
        x = np.concatenate([c[0] for c in curves])
        y = np.concatenate([c[1] for c in curves])
        t = np.concatenate([c[2] for c in curves])
    else:
        x = y = t = np.zeros(0)
    s = rng.uniform(2.0, 20.0, x.shape[0])
    nc = int(round(clutter_frac * x.shape[0]))
    xc = rng.uniform(0, W, nc)
    yc = rng.uniform(0, H, nc)
    tc = rng.uniform(-math.pi, math.pi, nc)
    sc = rng.uniform(1.0, 5.0, nc)
    x = np.concatenate([x, xc])
    y = np.concatenate([y, yc])
    t = np.concatenate([t, tc])
    s = np.concatenate([s, sc])
    keep = (x >= 0) & (x < W) & (y >= 0) & (y < H)
    e = np.stack([x[keep], y[keep], _wrap_pi(t[keep]), s[keep]], axis=1)
    return np.ascontiguousarray(e, dtype=np.float64)


def _hd_curves(rng, n, W, H):
    """The 1920x1080 curve mix: 80% arcs (radius log-U[4, 400], length U[20, 400]),
    20% segments (length U[20, 300])."""
    n_arc = int(round(0.8 * n))
    n_seg = n - n_arc
    radius = np.exp(rng.uniform(math.log(4.0), math.log(400.0), n_arc))
    alen = rng.uniform(20.0, 400.0, n_arc)
    slen = rng.uniform(20.0, 300.0, n_seg)
    return _arcs(rng, n_arc, W, H, radius, alen) + _segments(rng, n_seg, W, H, slen)


def plain_small(seed: int = 0, W: int = 480, H: int = 320) -> np.ndarray:
    """480x320 (or W x H): 40 arcs (radius U[8, 200], length U[20, 300]), 10
    segments (length U[20, 200]), 10% clutter; ~6k edges."""
    rng = np.random.Generator(np.random.PCG64(seed))
    radius = rng.uniform(8.0, 200.0, 40)
    alen = rng.uniform(20.0, 300.0, 40)
    slen = rng.uniform(20.0, 200.0, 10)
    curves = _arcs(rng, 40, W, H, radius, alen) + _segments(rng, 10, W, H, slen)
    return _assemble(rng, curves, W, H, 0.10)


def plain_hd(seed: int = 1000) -> np.ndarray:
    """1920x1080: 1,500 curves of the HD mix, 20% clutter; ~250k edges."""
    rng = np.random.Generator(np.random.PCG64(seed))
    W, H = 1920, 1080
    return _assemble(rng, _hd_curves(rng, 1500, W, H), W, H, 0.20)


def mixed_map(seed: int) -> np.ndarray:
    """One map of the ragged mix: image size uniform from IMAGE_SIZES, curves =
    0.7 per 1,000 px^2 x density log-U[0.25, 4], HD curve mix, 20% clutter."""
    rng = np.random.Generator(np.random.PCG64(seed))
    W, H = IMAGE_SIZES[int(rng.integers(0, len(IMAGE_SIZES)))]
    density = math.exp(rng.uniform(math.log(0.25), math.log(4.0)))
    n = max(1, int(round(0.7e-3 * W * H * density)))
    return _assemble(rng, _hd_curves(rng, n, W, H), W, H, 0.20)


def mixed_map_image(seed: int) -> tuple[int, int]:
    """The image size (W, H) that mixed_map(seed) draws."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return IMAGE_SIZES[int(rng.integers(0, len(IMAGE_SIZES)))]


def mixed64(base_seed: int = 2000, n_maps: int = 64) -> list[np.ndarray]:
    return [mixed_map(base_seed + i) for i in range(n_maps)]


def dense_4k(seed: int = 4000) -> np.ndarray:
    """3840x2160: 6,000 curves, half short high-curvature arcs (radius U[3, 15],
    length U[10, 60]) and half of the HD mix, 40% clutter; ~2M edges."""
    rng = np.random.Generator(np.random.PCG64(seed))
    W, H = 3840, 2160
    radius = rng.uniform(3.0, 15.0, 3000)
    alen = rng.uniform(10.0, 60.0, 3000)
    curves = _arcs(rng, 3000, W, H, radius, alen) + _hd_curves(rng, 3000, W, H)
    return _assemble(rng, curves, W, H, 0.40)


def stress_mix(base_seed: int = 5000, n_dense: int = 16, n_small: int = 1024) -> tuple[list[np.ndarray], list[str]]:
    """The stress stream's maps: n_dense dense 3840x2160 maps (dense_4k) and
    n_small config-0 maps at 640x480, interleaved in a seeded random order.
    Returns (maps, kinds) with kinds "dense" / "small"."""
    maps = [(dense_4k(base_seed + i), "dense") for i in range(n_dense)]
    maps += [(plain_small(base_seed + 100 + i, 640, 480), "small") for i in range(n_small)]
    order = np.random.Generator(np.random.PCG64(base_seed)).permutation(len(maps))
    return [maps[i][0] for i in order], [maps[i][1] for i in order]


def write_edge_file(path: str, edges: np.ndarray) -> None:
    """Writes rows in the reference edge-file format with round-trip precision."""
    np.savetxt(path, edges, fmt="%.17g", delimiter="\t")


# ---- curvelet sets for the link-graph / contour stage -----------------------------
def contour_fuzz(seed: int = 0, n_edges: int = 3000, width: int = 5, size: float = 120.0,
                 max_per_anchor: int = 4) -> tuple[np.ndarray, np.ndarray]:
    """Edges on random polylines (about 1 px apart, some 2-3 px gaps) and random
    curvelet chains over them: for each anchor in ascending order, up to
    max_per_anchor rows [anchor + 1, anchor + 1, then a random walk through
    nearby edges], width - 1 edges at most, zero-padded. The walks cross each
    other and run both ways, so the link graph has junctions, reversed links,
    gaps and cycles. Returns (edges [n, 4], chains [C, width] uint32)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = []
    while sum(len(p) for p in pts) < n_edges:
        k = int(rng.integers(5, 60))
        step = rng.choice([0.9, 1.0, 1.2, 2.6], size=k, p=[0.4, 0.35, 0.2, 0.05])
        ang = rng.uniform(0, 2 * np.pi) + np.cumsum(rng.normal(0, 0.25, k))
        xy = rng.uniform(0, size, 2) + np.cumsum(np.column_stack([np.cos(ang), np.sin(ang)]) * step[:, None], 0)
        pts.append(xy)
    xy = np.concatenate(pts)[:n_edges]
    order = rng.permutation(n_edges)  # ids are not in curve order
    xy = xy[order]
    edges = np.column_stack([xy, rng.uniform(-np.pi, np.pi, n_edges), rng.uniform(1, 10, n_edges)])
    # neighbours within 3 px through a coarse grid
    cell = np.floor(xy / 3.0).astype(np.int64)
    key = cell[:, 0] * 100003 + cell[:, 1]
    buckets: dict = {}
    for i, k in enumerate(key.tolist()):
        buckets.setdefault(k, []).append(i)

    def near(i):
        cx, cy = cell[i]
        out = []
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                out += buckets.get(int((cx + dx) * 100003 + cy + dy), [])
        return [j for j in out if j != i and np.hypot(*(xy[j] - xy[i])) < 3.0]

    rows = []
    for a in range(n_edges):
        for _ in range(int(rng.integers(0, max_per_anchor + 1))):
            L = int(rng.integers(2, width))
            chain = [a]
            while len(chain) < L:
                cand = [j for j in near(chain[-1]) if j not in chain]
                if not cand:
                    break
                chain.append(int(rng.choice(cand)))
            if len(chain) < 2:
                continue
            row = np.zeros(width, np.uint32)
            row[0] = a + 1
            row[1:1 + len(chain)] = np.asarray(chain) + 1
            rows.append(row)
    chains = np.asarray(rows, np.uint32).reshape(-1, width)
    return edges, chains


def contour_rings(seed: int = 0, n_rings: int = 6, width: int = 5) -> tuple[np.ndarray, np.ndarray]:
    """Closed contours: rings of 8 to 200 edges about 1 px apart, ids shuffled
    across rings, each edge the anchor of one chain running along its ring (so
    every link points the same way round and each ring is a cycle); one ring
    has a 3 px gap and one runs the other way. Returns (edges, chains)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ring_pts, ring_ids = [], []
    base = 0
    for r in range(n_rings):
        k = int(rng.integers(8, 200)) if r else 8
        rad = k / (2 * np.pi)
        t = np.arange(k) * 2 * np.pi / k
        if r == 1:  # a gap: the last step is about 3 px
            t = np.arange(k) * (2 * np.pi - 3.0 / rad) / (k - 1)
        c = rng.uniform(0, 400, 2)
        ring_pts.append(c + rad * np.column_stack([np.cos(t), np.sin(t)]))
        seq = list(range(base, base + k))
        if r == 2:
            seq = seq[::-1]
        ring_ids.append(seq)
        base += k
    n = base
    perm = rng.permutation(n)  # position in ring order -> edge id
    xy = np.zeros((n, 2))
    for pts, seq in zip(ring_pts, ring_ids):
        for p, s in zip(pts, seq):
            xy[perm[s]] = p
    edges = np.column_stack([xy, rng.uniform(-np.pi, np.pi, n), rng.uniform(1, 10, n)])
    rows = []
    for seq in ring_ids:
        k = len(seq)
        for i in range(k):
            chain = [perm[seq[(i + j) % k]] for j in range(width - 1)]
            row = np.zeros(width, np.uint32)
            row[0] = chain[0] + 1
            row[1:] = np.asarray(chain) + 1
            rows.append(row)
    chains = np.asarray(rows, np.uint32)
    chains = chains[np.argsort(chains[:, 0], kind="stable")]
    return edges, chains
