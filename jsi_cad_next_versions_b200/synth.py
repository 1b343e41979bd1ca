"""Seeded synthetic NURBS surfaces in the EGADS layout used by VERSION5.

A surface is an ``ivec`` of 7 ints and a float32 ``data`` array, the layout of
``NurbsFace`` (JSI_CAD_NEXT_VERSION5/include/nurbs_data.hpp:1-10) and of
``BuildEvalContext`` (JSI_CAD_NEXT_VERSION5/src/evaluation/evaluation.cu:239-257):

    ivec = [flags, degU, nCPu, nKu, degV, nCPv, nKv]   flags bit 1 (value 2) = rational
    data = [U knots (nKu)] [V knots (nKv)] [CP xyz, u fastest (3*nCPu*nCPv)] [w (nCPu*nCPv) if rational]

The reference's own distance inputs (``dist_case*.cu``) are not in its
checkout, so the query workloads are built here from a documented generator:
splitmix64 for the bit stream, 53-bit uniforms, Box-Muller normals.  Geometry
is built in float64 and rounded once to float32; every engine (reference,
oracle, GPU) reads the same float32 values.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_MASK64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea & Flood 2014) with 53-bit uniform doubles."""

    def __init__(self, seed: int):
        self.state = seed & _MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK64
        return z ^ (z >> 31)

    def uniform(self, n: int | None = None, lo: float = 0.0, hi: float = 1.0):
        if n is None:
            return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))
        out = np.empty(n, dtype=np.float64)
        for q in range(n):
            out[q] = (self.next_u64() >> 11) * (1.0 / (1 << 53))
        return lo + (hi - lo) * out

    def normal(self, n: int, sigma: float = 1.0):
        """Box-Muller pairs; the cosine branch first, then the sine branch."""
        out = np.empty(n, dtype=np.float64)
        q = 0
        while q < n:
            u1 = self.uniform()
            u2 = self.uniform()
            r = math.sqrt(-2.0 * math.log(1.0 - u1))
            out[q] = r * math.cos(2.0 * math.pi * u2)
            if q + 1 < n:
                out[q + 1] = r * math.sin(2.0 * math.pi * u2)
            q += 2
        return sigma * out

    def randint(self, lo: int, hi: int) -> int:
        """Uniform integer in [lo, hi]."""
        return lo + int(self.uniform() * (hi - lo + 1)) if hi > lo else lo


@dataclass
class Surface:
    """One NURBS surface in EGADS layout."""

    ivec: np.ndarray          # int32[7]
    data: np.ndarray          # float32[ndata]
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def ndata(self) -> int:
        return int(self.data.shape[0])

    @property
    def rational(self) -> bool:
        return bool(int(self.ivec[0]) & 2)

    def rect(self):
        """Full parameter domain (ustart, vstart, ustop, vstop) as float32,
        as ``NurbsFace::get_ubegin/get_uend/...`` return them."""
        nku = int(self.ivec[3])
        nkv = int(self.ivec[6])
        d = self.data
        return (np.float32(d[0]), np.float32(d[nku]), np.float32(d[nku - 1]), np.float32(d[nku + nkv - 1]))

    def control_net(self):
        """(ncpv, ncpu, 3) float32 view of the control points and (ncpv, ncpu) weights or None."""
        nku, ncpu, ncpv, nkv = int(self.ivec[3]), int(self.ivec[2]), int(self.ivec[5]), int(self.ivec[6])
        off = nku + nkv
        cp = self.data[off:off + 3 * ncpu * ncpv].reshape(ncpv, ncpu, 3)
        w = None
        if self.rational:
            w = self.data[off + 3 * ncpu * ncpv: off + 4 * ncpu * ncpv].reshape(ncpv, ncpu)
        return cp, w


def clamped_uniform_knots(n: int, p: int) -> np.ndarray:
    """p+1 zeros, interior i/(n-p) for i = 1..n-p-1, p+1 ones (n control points)."""
    interior = [i / (n - p) for i in range(1, n - p)]
    return np.array([0.0] * (p + 1) + interior + [1.0] * (p + 1), dtype=np.float64)


def make_surface(cp_xyz: np.ndarray, degu: int, degv: int, weights: np.ndarray | None = None,
                 uknots: np.ndarray | None = None, vknots: np.ndarray | None = None, name: str = "") -> Surface:
    """Pack a (ncpv, ncpu, 3) float64 control net into EGADS layout."""
    ncpv, ncpu, _ = cp_xyz.shape
    if ncpu < degu + 1 or ncpv < degv + 1:
        raise ValueError("control net smaller than degree + 1")
    U = clamped_uniform_knots(ncpu, degu) if uknots is None else np.asarray(uknots, np.float64)
    V = clamped_uniform_knots(ncpv, degv) if vknots is None else np.asarray(vknots, np.float64)
    flags = 2 if weights is not None else 0
    ivec = np.array([flags, degu, ncpu, U.size, degv, ncpv, V.size], dtype=np.int32)
    parts = [U, V, cp_xyz.reshape(-1)]
    if weights is not None:
        parts.append(np.asarray(weights, np.float64).reshape(-1))
    data = np.concatenate(parts).astype(np.float32)
    return Surface(ivec=ivec, data=data, name=name)


def _grid(n_u: int, n_v: int, lo: float = 0.0, hi: float = 1.0):
    x = lo + (hi - lo) * (np.arange(n_u, dtype=np.float64) / (n_u - 1))
    y = lo + (hi - lo) * (np.arange(n_v, dtype=np.float64) / (n_v - 1))
    X, Y = np.meshgrid(x, y)  # (n_v, n_u): u fastest
    return X, Y


# ---------------------------------------------------------------------------
# Query workloads.  Each returns (surface A, surface B, query parameters).
# ---------------------------------------------------------------------------

def distance_pair_sine(seed_a: int = 1, seed_b: int = 2, n: int = 16, deg: int = 3):
    """Two bicubic 16x16 patches: z = 0.2 sin(3 pi x) sin(3 pi y) + U(+-0.01);
    B is built the same way from another seed, rotated 30 degrees about z and
    lifted by 0.5.  First round nuv=64, three refinement rounds at nuv=16,
    top-k 64, final Newton step."""
    def one(seed):
        rng = SplitMix64(seed)
        X, Y = _grid(n, n)
        Z = 0.2 * np.sin(3 * np.pi * X) * np.sin(3 * np.pi * Y) + rng.uniform(n * n, -0.01, 0.01).reshape(n, n)
        return np.stack([X, Y, Z], axis=-1)
    a = one(seed_a)
    b = one(seed_b)
    c, s = math.cos(math.radians(30.0)), math.sin(math.radians(30.0))
    bx = c * b[..., 0] - s * b[..., 1]
    by = s * b[..., 0] + c * b[..., 1]
    b = np.stack([bx, by, b[..., 2] + 0.5], axis=-1)
    A = make_surface(a, deg, deg, name=f"sine16_seed{seed_a}")
    B = make_surface(b, deg, deg, name=f"sine16_seed{seed_b}_rot30_z+0.5")
    return A, B, dict(nuv0=64, nuv_refine=16, k=64, rounds=4)


def distance_pair_hard_wave(seed_a: int = 3, seed_b: int = 4, n: int = 64, deg: int = 3, scale: float = 1.0):
    """Hard-wave pair: bicubic 64x64, A z = 0.05 sin(20 pi x) cos(20 pi y) + N(0, 1e-3);
    B is the same field phase-shifted by pi and lifted by 0.1 (own noise seed).
    ``scale`` multiplies every control point coordinate (the 4x copy uses 4
    with nuv0=2048)."""
    def one(seed, phase, lift):
        rng = SplitMix64(seed)
        X, Y = _grid(n, n)
        Z = 0.05 * np.sin(20 * np.pi * X + phase) * np.cos(20 * np.pi * Y) + lift + rng.normal(n * n, 1e-3).reshape(n, n)
        return np.stack([X, Y, Z], axis=-1) * scale
    A = make_surface(one(seed_a, 0.0, 0.0), deg, deg, name=f"hardwave64_seed{seed_a}_x{scale:g}")
    B = make_surface(one(seed_b, math.pi, 0.1), deg, deg, name=f"hardwave64_seed{seed_b}_pi_z+0.1_x{scale:g}")
    nuv0 = 512 if scale == 1.0 else 2048
    return A, B, dict(nuv0=nuv0, nuv_refine=16, k=8, rounds=4)


def intersection_pair_saddle_plane(seed_a: int = 5, seed_b: int = 6, n: int = 32, deg: int = 3):
    """Rational bicubic 32x32 pair on [-1,1]^2 with weights U[0.5, 2]:
    A is the saddle z = x^2 - y^2, B the plane z = 0.3 x + 0.1 plus
    0.05 sin(8 pi x) sin(8 pi y).  nuv0=256, padding on and off."""
    def one(seed, fz):
        rng = SplitMix64(seed)
        X, Y = _grid(n, n, -1.0, 1.0)
        W = rng.uniform(n * n, 0.5, 2.0).reshape(n, n)
        return np.stack([X, Y, fz(X, Y)], axis=-1), W
    a, wa = one(seed_a, lambda X, Y: X * X - Y * Y)
    b, wb = one(seed_b, lambda X, Y: 0.3 * X + 0.1 + 0.05 * np.sin(8 * np.pi * X) * np.sin(8 * np.pi * Y))
    A = make_surface(a, deg, deg, weights=wa, name=f"saddle32_rat_seed{seed_a}")
    B = make_surface(b, deg, deg, weights=wb, name=f"plane32_rat_seed{seed_b}")
    return A, B, dict(nuv0=256, nuv_refine=16, rounds=6, use_k=1)


def random_surface(rng: SplitMix64, name: str = "") -> Surface:
    """One surface of the mixed batch: degrees uniform in {2..5} per
    direction, net sizes log-uniform in [4, 64] per direction (at least
    degree+1), 30% rational with w ~ U[0.5, 2], random-phase sinusoidal height
    field of amplitude U[0.01, 0.2]."""
    degu = rng.randint(2, 5)
    degv = rng.randint(2, 5)
    ncpu = max(degu + 1, int(round(math.exp(rng.uniform(None, math.log(4), math.log(64))))))
    ncpv = max(degv + 1, int(round(math.exp(rng.uniform(None, math.log(4), math.log(64))))))
    amp = rng.uniform(None, 0.01, 0.2)
    fx = rng.uniform(None, 1.0, 6.0)
    fy = rng.uniform(None, 1.0, 6.0)
    px = rng.uniform(None, 0.0, 2 * math.pi)
    py = rng.uniform(None, 0.0, 2 * math.pi)
    X, Y = _grid(ncpu, ncpv)
    Z = amp * np.sin(2 * np.pi * fx * X + px) * np.cos(2 * np.pi * fy * Y + py)
    rational = rng.uniform() < 0.3
    W = rng.uniform(ncpu * ncpv, 0.5, 2.0).reshape(ncpv, ncpu) if rational else None
    return make_surface(np.stack([X, Y, Z], axis=-1), degu, degv, weights=W, name=name)


def mixed_batch(n_pairs: int = 4096, seed: int = 7):
    """The mixed query batch: n_pairs surface pairs, half distance, half
    intersection, nuv0 uniform in [64, 512] per pair.  The second surface of
    each pair is lifted by U[-0.1, 0.1] so that both near-miss and crossing
    pairs occur."""
    rng = SplitMix64(seed)
    out = []
    for q in range(n_pairs):
        a = random_surface(rng, name=f"batch{q}a")
        b = random_surface(rng, name=f"batch{q}b")
        lift = rng.uniform(None, -0.1, 0.1)
        ncpu, ncpv = int(b.ivec[2]), int(b.ivec[5])
        off = int(b.ivec[3] + b.ivec[6])
        xyz = b.data[off:off + 3 * ncpu * ncpv].reshape(-1, 3).astype(np.float64)
        xyz[:, 2] += lift
        b.data[off:off + 3 * ncpu * ncpv] = xyz.reshape(-1).astype(np.float32)
        kind = "distance" if (q % 2 == 0) else "intersection"
        nuv0 = rng.randint(64, 512)
        out.append((a, b, dict(kind=kind, nuv0=nuv0)))
    return out
