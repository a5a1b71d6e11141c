"""CPU restatement of pieces of the reference painter, for testing.

Test infrastructure only (tests import it; the accelerated library never
does).  Each function restates one algorithm of the reference in plain
Python / numpy, cites the reference file it follows, and is itself pinned
against the reference: by the known-answer vectors of the reference's own
tests (tests/golden/reference_kat.json) and by the compiled reference
(oracle/_ref/libnbpt_oracle.so, see oracle/oracle.py).

The complete path tracer is not restated here: its oracle is the reference
painter itself, compiled from its own sources (oracle/Makefile).
"""

from __future__ import annotations

import math

import numpy as np

MASK32 = 0xFFFFFFFF
MASK64 = 0xFFFFFFFFFFFFFFFF

# ---------------------------------------------------------------------------
# random numbers


def seed_seq(words, count: int = 4) -> list[int]:
    """std::seed_seq::generate (the algorithm of [rand.util.seedseq])."""
    n = count
    s = len(words)
    t = 11 if n >= 623 else 7 if n >= 68 else 5 if n >= 39 else 3 if n >= 7 else (n - 1) // 2
    p = (n - t) // 2
    q = p + t
    b = [0x8B8B8B8B] * n
    m = max(s + 1, n)

    def tw(x):
        return (x ^ (x >> 27)) & MASK32

    for k in range(m):
        r1 = (1664525 * tw(b[k % n] ^ b[(k + p) % n] ^ b[(k - 1) % n])) & MASK32
        if k == 0:
            r2 = (r1 + s) & MASK32
        elif k <= s:
            r2 = (r1 + k % n + words[k - 1]) & MASK32
        else:
            r2 = (r1 + k % n) & MASK32
        b[(k + p) % n] = (b[(k + p) % n] + r1) & MASK32
        b[(k + q) % n] = (b[(k + q) % n] + r2) & MASK32
        b[k % n] = r2
    for k in range(m, m + n):
        r3 = (1566083941 * tw((b[k % n] + b[(k + p) % n] + b[(k - 1) % n]) & MASK32)) & MASK32
        r4 = (r3 - k % n) & MASK32
        b[(k + p) % n] ^= r3
        b[(k + q) % n] ^= r4
        b[k % n] = r4
    return b


class Pcg:
    """PCG-XSH-RR 64/32 seeded from four seed_seq words
    (src/com/random/pcg.h:53-62, pcg.cpp:57-92)."""

    MULTIPLIER = 6364136223846793005

    def __init__(self, words):
        d = seed_seq(list(words), 4)
        self.state = d[0] | (d[1] << 32)
        self.increment = d[2] | (d[3] << 32) | 1

    def __call__(self) -> int:
        x = self.state
        self.state = (x * self.MULTIPLIER + self.increment) & MASK64
        s = (((x >> 18) ^ x) >> 27) & MASK32
        r = x >> 59
        return ((s >> r) | (s << ((32 - r) & 31))) & MASK32

    def canonical(self, double: bool = True) -> float:
        """std::generate_canonical: two draws for double, one for float."""
        if double:
            x0 = self()
            x1 = self()
            total = np.float64(x0) + np.float64(x1) * np.float64(4294967296.0)
            r = total / np.float64(18446744073709551616.0)
            return float(np.nextafter(np.float64(1), np.float64(0))) if r >= 1 else float(r)
        r = np.float32(self()) / np.float32(4294967296.0)
        return float(np.nextafter(np.float32(1), np.float32(0))) if r >= 1 else float(r)

    def uniform(self, a, b, double: bool = True) -> float:
        """std::uniform_real_distribution: canonical * (b - a) + a."""
        if double:
            return float(np.float64(self.canonical(True)) * (np.float64(b) - np.float64(a)) + np.float64(a))
        return float(np.float32(self.canonical(False)) * (np.float32(b) - np.float32(a)) + np.float32(a))


def sj_strata(dimension: int, spp: int) -> int:
    """Strata per dimension (src/sampling/sj_sampler.h:51-73)."""
    v = spp ** (1.0 / dimension)
    f = math.floor(v)
    if f ** dimension >= spp:
        return f
    return math.ceil(v)


def sj_points(dimension: int, spp: int, words, double: bool = True) -> np.ndarray:
    """Stratified jittered points of one pixel (sj_sampler.h:75-205); the
    first dimension varies fastest and each coordinate is drawn with rejection
    of the upper bound (src/com/random/uniform.h:24-34)."""
    k = sj_strata(dimension, spp)
    ft = np.float64 if double else np.float32
    size = ft(1) / ft(k)
    offsets = [ft(0)] + [ft(0) + ft(i) * size for i in range(1, k)] + [ft(1)]
    g = Pcg(words)
    out = np.zeros((k ** dimension, dimension))
    for s in range(k ** dimension):
        rest = s
        for d in range(dimension):
            idx = rest % k
            rest //= k
            a, b = offsets[idx], offsets[idx + 1]
            while True:
                v = ft(g.uniform(a, b, double))
                if v < b:
                    break
            out[s, d] = v
    return out


# ---------------------------------------------------------------------------
# painting driver


def paintbrush_pixels(size, paint_height: int) -> list[tuple[int, ...]]:
    """Pixel order of the painter's paintbrush
    (src/painter/painting/paintbrush.h:162-205): the screen is walked in
    bands of `paint_height` along the reversed axis order, then every pixel's
    coordinates are reversed back and its second coordinate flipped."""
    size = list(size)
    n = len(size)
    brush = [min(size[i], paint_height) for i in range(n - 1)] + [1]
    rsize = size[::-1]
    pixels: list[list[int]] = []

    # blocks of `brush` over the reversed screen, dimension 0 outermost
    def blocks(dim, prefix_min, prefix_max):
        if dim == n:
            yield list(prefix_min), list(prefix_max)
            return
        for lo in range(0, rsize[dim], brush[dim]):
            hi = min(lo + brush[dim], rsize[dim])
            yield from blocks(dim + 1, prefix_min + [lo], prefix_max + [hi])

    def inner(dim, lo, hi, prefix):
        if dim == n:
            yield list(prefix)
            return
        for v in range(lo[dim], hi[dim]):
            yield from inner(dim + 1, lo, hi, prefix + [v])

    for lo, hi in blocks(0, [], []):
        pixels.extend(inner(0, lo, hi, []))
    out = []
    for p in pixels:
        q = p[::-1]
        q[1] = size[1] - 1 - q[1]
        out.append(tuple(q))
    return out


# ---------------------------------------------------------------------------
# pixel estimator


def gaussian_filter_weight(x: np.ndarray, radius: float = 1.5) -> np.ndarray:
    """Truncated Gaussian pixel filter (src/painter/pixels/pixel_filter.h:43-69,
    gaussian.h:38-78): prod_i max(0, exp(alpha x_i^2) - exp(alpha r^2)),
    width = r / 2.5, alpha = -1 / (2 width^2).  x: [..., dimension]."""
    width = radius / 2.5
    alpha = -1 / (2 * width * width)
    e = math.exp(alpha * radius * radius)
    w = np.maximum(0.0, np.exp(alpha * x[..., 0] * x[..., 0]) - e)
    for i in range(1, x.shape[-1]):
        w = w * np.maximum(0.0, np.exp(alpha * x[..., i] * x[..., i]) - e)
    return w


def create_samples(keys, count: int):
    """Held-out extremes of one group of samples
    (src/painter/pixels/samples/create.cpp:147-197, com/sort.h:26-46,
    com/create.h:28-55): with more than `count` samples the count/2 lowest
    and count/2 highest keys are kept aside and the rest summed; otherwise
    all are kept, sorted.  Returns (kept indices in order, summed indices,
    full)."""
    order = sorted(range(len(keys)), key=lambda i: keys[i])
    if len(keys) <= count:
        return order, [], False
    half = count // 2
    return order[:half] + order[-half:], order[half:-half], True


def luminance_rgb(rgb) -> float:
    """linear_float_to_linear_luminance (src/color/conversion.h:255-260)."""
    r, g, b = (max(np.float32(0), np.float32(c)) for c in rgb)
    return float(np.float32(0.2126) * r + np.float32(0.7152) * g + np.float32(0.0722) * b)


# ---------------------------------------------------------------------------
# geometry


def orthogonal_complement(v: np.ndarray) -> np.ndarray:
    """Cofactor orthogonal complement of N-1 row vectors in N-space
    (src/numerical/complement.h:45-101), vectorised over leading axes."""
    n = v.shape[-1]
    out = np.zeros(v.shape[:-2] + (n,))
    for i in range(n):
        cols = [c for c in range(n) if c != i]
        m = v[..., :, cols]
        d = np.linalg.det(m)
        out[..., i] = -d if (i & 1) else d
    return out


def simplex_planes(vertices: np.ndarray) -> np.ndarray:
    """Hyperplane and barycentric hyperplanes of (n-1)-simplices
    (src/geometry/spatial/hyperplane_simplex.h:82-111).  vertices: [F, N, N];
    returns [F, N, N+1] (n, d) rows.  numpy determinants: equal to the
    reference's to rounding, not bit for bit."""
    f, n, _ = vertices.shape
    vec = vertices[:, : n - 1, :] - vertices[:, n - 1 : n, :]
    normal = orthogonal_complement(vec)
    normal /= np.linalg.norm(normal, axis=1, keepdims=True)
    out = np.zeros((f, n, n + 1))
    out[:, 0, :n] = normal
    out[:, 0, n] = np.einsum("fi,fi->f", normal, vertices[:, n - 1])
    for i in range(n - 1):
        vv = vec.copy()
        vv[:, i, :] = normal
        pn = orthogonal_complement(vv)
        pd = np.einsum("fi,fi->f", vertices[:, n - 1], pn)
        dist = np.einsum("fi,fi->f", pn, vertices[:, i]) - pd
        out[:, i + 1, :n] = pn / dist[:, None]
        out[:, i + 1, n] = pd / dist
    return out


def simplex_intersect(planes: np.ndarray, org: np.ndarray, dir: np.ndarray) -> np.ndarray:
    """Ray / simplex distances (hyperplane_simplex.h:177-207) for every ray
    against every facet: [R, F], 0 where there is no hit."""
    n = org.shape[1]
    pn = planes[:, 0, :n]
    pd = planes[:, 0, n]
    t = (pd[None, :] - org @ pn.T) / (dir @ pn.T)
    ok = t > 0
    point = org[:, None, :] + dir[:, None, :] * t[:, :, None]
    total = np.zeros_like(t)
    for i in range(n - 1):
        bc = np.einsum("rfi,fi->rf", point, planes[:, i + 1, :n]) - planes[None, :, i + 1, n]
        ok &= (bc > 0) & (bc < 1)
        total += bc
    ok &= total < 1
    return np.where(ok, t, 0.0)
