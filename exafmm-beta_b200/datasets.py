"""Seeded body generators for the benchmark workloads, plus the reference's own.

The reference's generators (include/dataset.h) draw with drand48 from fixed
shapes ([-pi, pi]^3 cube, radius-pi sphere, octant, Plummer scaled by
3*pi/16, [-1, 1]^3 lattice); `reference_bodies` reproduces them bit for bit
(`drand48` is the POSIX stream).  The workloads this engine is measured on use
different shapes, so they are generated here with numpy's PCG64 from an
explicit seed and handed, as the same (n, 4) array, to both the GPU engine and
the CPU checkers.

Every generator returns float64 (n, 4): x, y, z, charge.
"""
from __future__ import annotations

import numpy as np


def _zero_mean(q: np.ndarray) -> np.ndarray:
    return q - q.mean()


def cube(n: int, seed: int = 1, charge: str = "uniform") -> np.ndarray:
    """Uniform in [-1, 1]^3; charges U[-1, 1] shifted to zero net charge."""
    rng = np.random.default_rng(seed)
    x = np.empty((n, 4))
    x[:, :3] = rng.uniform(-1.0, 1.0, (n, 3))
    x[:, 3] = _zero_mean(rng.uniform(-1.0, 1.0, n)) if n else 0.0
    return x


def sphere(n: int, seed: int = 1) -> np.ndarray:
    """Uniform on the unit sphere surface (normalized Gaussians); charges U[-1, 1]."""
    rng = np.random.default_rng(seed)
    g = rng.normal(size=(n, 3))
    x = np.empty((n, 4))
    x[:, :3] = g / np.linalg.norm(g, axis=1)[:, None]
    x[:, 3] = rng.uniform(-1.0, 1.0, n)
    return x


def plummer(n: int, seed: int = 2, rmax: float = 20.0, scale: float = 1.0) -> np.ndarray:
    """Plummer sphere: radius by the inverse CDF (U^(-2/3) - 1)^(-1/2) (the form of
    include/dataset.h:121), rejected beyond rmax, isotropic directions; equal
    charges 1/n."""
    rng = np.random.default_rng(seed)
    out = np.empty((0, 3))
    while len(out) < n:
        m = int((n - len(out)) * 1.05) + 16
        u = rng.uniform(size=m)
        with np.errstate(divide="ignore"):
            r = scale / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        r = r[np.isfinite(r) & (r <= rmax * scale)]
        g = rng.normal(size=(len(r), 3))
        out = np.vstack([out, g / np.linalg.norm(g, axis=1)[:, None] * r[:, None]])
    x = np.empty((n, 4))
    x[:, :3] = out[:n]
    x[:, 3] = 1.0 / n
    return x


def water_box(n_waters: int, seed: int = 5, density: float = 0.0334):
    """Rigid 3-site waters (O -0.834, H +0.417, O-H 0.9572 A, H-O-H 104.52 deg) at
    random positions and orientations in a cubic box of edge L = (n/density)^(1/3),
    mapped to [-L/2, L/2]^3.  Returns (xyzq, L)."""
    rng = np.random.default_rng(seed)
    L = (n_waters / density) ** (1.0 / 3.0)
    O = rng.uniform(-L / 2, L / 2, (n_waters, 3))
    # random rotation per molecule from normalized quaternions
    q = rng.normal(size=(n_waters, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    w, a, b, c = q.T
    R = np.stack([
        np.stack([1 - 2 * (b * b + c * c), 2 * (a * b - c * w), 2 * (a * c + b * w)], -1),
        np.stack([2 * (a * b + c * w), 1 - 2 * (a * a + c * c), 2 * (b * c - a * w)], -1),
        np.stack([2 * (a * c - b * w), 2 * (b * c + a * w), 1 - 2 * (a * a + b * b)], -1),
    ], 1)
    d, half = 0.9572, np.deg2rad(104.52) / 2
    h1 = np.array([d * np.sin(half), 0.0, d * np.cos(half)])
    h2 = np.array([-d * np.sin(half), 0.0, d * np.cos(half)])
    H1 = O + R @ h1
    H2 = O + R @ h2
    pos = np.stack([O, H1, H2], 1).reshape(-1, 3)
    pos = (pos + L / 2) % L - L / 2  # wrap into the box
    chg = np.tile([-0.834, 0.417, 0.417], n_waters)
    return np.c_[pos, chg], L


def log_uniform_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)


def strided_sample(n: int, k: int) -> np.ndarray:
    """Dataset::sampleBodies (include/dataset.h:290-298): every (n // k)-th body."""
    if k >= n:
        return np.arange(n)
    return np.arange(k) * (n // k)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """Verify::getDif*/getNrm* (include/verify.h:42-107): sqrt(sum|a-b|^2 / sum|b|^2),
    b being the reference argument."""
    num = float(np.sum((np.asarray(a) - np.asarray(b)) ** 2))
    den = float(np.sum(np.asarray(b) ** 2))
    return float(np.sqrt(num / den)) if den > 0 else float(np.sqrt(num))


# ---------------------------------------------------------------------------
# The reference's own generators, Dataset::initBodies (include/dataset.h:29-257),
# bit for bit: the same drand48 streams, the same IEEE arithmetic in the same
# order, pow / sin / cos from the C math library (Python's math module).

_DRAND_A = 0x5DEECE66D
_DRAND_C = 0xB
_MASK48 = (1 << 48) - 1
_LO24 = (1 << 24) - 1


def _mulmod48(x, y):
    """x * y mod 2^48 for uint64 values below 2^48 (24-bit halves, no overflow)."""
    xl, xh = x & _LO24, x >> np.uint64(24)
    yl, yh = y & _LO24, y >> np.uint64(24)
    return (xl * yl + (((xh * yl + xl * yh) & _LO24) << np.uint64(24))) & _MASK48


def drand48(seed: int, count: int) -> np.ndarray:
    """The first `count` values of drand48() after srand48(seed) (POSIX: the
    48-bit congruence X <- (0x5DEECE66D X + 11) mod 2^48 from X = seed << 16 |
    0x330E, the low 32 bits of seed; each value is the new X / 2^48).  Computed
    in blocks: a block of B values is the previous one advanced by a^B, c_B."""
    x = (((int(seed) & 0xFFFFFFFF) << 16) | 0x330E) & _MASK48
    if count <= 0:
        return np.zeros(0)
    B = min(count, 4096)
    first = np.empty(B, np.uint64)
    for i in range(B):
        x = (_DRAND_A * x + _DRAND_C) & _MASK48
        first[i] = x
    aB, cB = 1, 0
    for _ in range(B):  # X_{k+B} = aB X_k + cB
        aB, cB = (_DRAND_A * aB) & _MASK48, (_DRAND_A * cB + _DRAND_C) & _MASK48
    out = np.empty(count, np.uint64)
    out[:B] = first
    a, c = np.uint64(aB), np.uint64(cB)
    for k in range(B, count, B):
        m = min(B, count - k)
        out[k:k + m] = (_mulmod48(out[k - B:k - B + m], a) + c) & _MASK48
    return out.astype(np.float64) * 2.0 ** -48


def _split_range(begin: int, end: int, i: int, num_split: int):
    """Dataset::splitRange (include/dataset.h:18-26)."""
    size = end - begin
    inc, rem = size // num_split, size % num_split
    begin += i * inc + min(i, rem)
    end = begin + inc + (1 if rem > i else 0)
    return begin, end


def _ref_lattice(n: int, mpirank: int, mpisize: int) -> np.ndarray:
    import math
    nx = int(math.pow(n * mpisize, 1.0 / 3))
    b, e = _split_range(0, nx, mpirank, mpisize)
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(nx), np.arange(b, e), indexing="ij")
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.stack([(g.reshape(-1) / float(nx - 1)) * 2 - 1 for g in (ix, iy, iz)], axis=1)


def _ref_positions(kind: str, n: int, seed: int, num_split: int) -> np.ndarray:
    import math
    X = np.zeros((n, 3))
    for s in range(num_split):
        b, e = _split_range(0, n, s, num_split)
        m = e - b
        if kind == "c":  # cube (dataset.h:52-66)
            X[b:e] = (drand48(seed + s, 3 * m).reshape(m, 3) * 2) * math.pi - math.pi
        elif kind == "s":  # sphere (dataset.h:68-86)
            Y = drand48(seed + s, 3 * m).reshape(m, 3) * 2 - 1
            r = np.sqrt((Y[:, 0] * Y[:, 0] + Y[:, 1] * Y[:, 1]) + Y[:, 2] * Y[:, 2])
            X[b:e] = Y * (math.pi / r)[:, None]
        elif kind == "o":  # octant (dataset.h:88-103)
            d = drand48(seed + s, 2 * m).reshape(m, 2)
            th = (d[:, 0] * math.pi) * 0.5
            ph = (d[:, 1] * math.pi) * 0.5
            st = np.array([math.sin(v) for v in th])
            ct = np.array([math.cos(v) for v in th])
            sp = np.array([math.sin(v) for v in ph])
            cp = np.array([math.cos(v) for v in ph])
            X[b:e, 0] = ((2 * math.pi) * st) * cp - math.pi
            X[b:e, 1] = ((2 * math.pi) * st) * sp - math.pi
            X[b:e, 2] = (2 * math.pi) * ct - math.pi
        elif kind == "p":  # plummer (dataset.h:105-137): triples until R < 100
            scale = 3.0 * math.pi / 16.0
            tries = m + m // 500 + 16
            while True:
                d = drand48(seed + s, 3 * tries).reshape(tries, 3)
                R = np.array([1.0 / math.sqrt(math.pow(v, -2.0 / 3.0) - 1.0) for v in d[:, 0]])
                keep = np.nonzero(R < 100.0)[0]
                if len(keep) >= m:
                    break
                tries *= 2
            keep = keep[:m]
            R, X2, X3 = R[keep], d[keep, 1], d[keep, 2]
            Z = (1.0 - 2.0 * X2) * R
            w = np.sqrt(R * R - Z * Z)
            ang = (2.0 * math.pi) * X3
            X[b:e, 0] = (w * np.array([math.cos(v) for v in ang])) * scale
            X[b:e, 1] = (w * np.array([math.sin(v) for v in ang])) * scale
            X[b:e, 2] = Z * scale
    return X


def _ref_charges(n: int, seed: int, num_split: int) -> np.ndarray:
    """Dataset::initSource for Laplace (dataset.h:141-154): drand48() - 0.5 per
    split, minus the split's average summed in body order."""
    q = np.zeros(n)
    for s in range(num_split):
        b, e = _split_range(0, n, s, num_split)
        v = drand48(seed + s, e - b) - 0.5
        avg = 0.0
        for x in v.tolist():
            avg += x
        avg /= (e - b)
        q[b:e] = v - avg
    return q


def reference_bodies(n: int, distribution: str, mpirank: int = 0, mpisize: int = 1,
                     num_split: int = 1) -> np.ndarray:
    """Dataset::initBodies(numBodies, distribution, mpirank, mpisize, numSplit)
    (include/dataset.h:229-257) as float64 (m, 4): x, y, z, charge.  The
    distribution is chosen by its first letter as there: lattice (m = the
    largest whole cube root of n * mpisize, cubed, this rank's slab of it),
    cube, sphere, octant or plummer, seeded with mpirank (+ the split index);
    the charges restart the same drand48 stream (initSource).  Targets start at
    zero (initTarget) in this engine's results."""
    kind = distribution[:1]
    if kind == "l":
        X = _ref_lattice(n, mpirank, mpisize)
    elif kind in ("c", "s", "o", "p"):
        X = _ref_positions(kind, n, mpirank, num_split)
    else:
        raise ValueError(f"Unknown data distribution {distribution}")
    q = _ref_charges(len(X), mpirank, num_split)
    return np.column_stack([X, q])


# Dataset's text files (include/dataset.h:162-204, 259-287): one value a line in
# the C++ stream's default format (%g, 6 significant digits); sources are x, y,
# z, q per body, targets the four target values.  Reads go on from a byte
# position and return the position after the last value read (the reference
# keeps it in the Dataset object, one position for both files).

def _write_values(fname: str, a: np.ndarray) -> str:
    with open(fname, "w") as f:
        f.write("".join(f"{v:g}\n" for v in np.asarray(a, dtype=np.float64).reshape(-1).tolist()))
    return fname


def _read_values(fname: str, count: int, position: int):
    import re
    with open(fname, "rb") as f:
        f.seek(position)
        data = f.read()
    vals, end = [], 0
    for m in re.finditer(rb"\S+", data):
        if len(vals) == count:
            break
        vals.append(float(m.group()))
        end = m.end()
    if len(vals) < count:
        raise ValueError(f"{fname}: {len(vals)} values from byte {position}, {count} wanted")
    return np.array(vals), position + end


def write_sources(xyzq: np.ndarray, rank: int = 0, path: str = "./") -> str:
    """Dataset::writeSources: path + 'source%04d.dat' (rank)."""
    return _write_values(f"{path}source{rank:04d}.dat", np.asarray(xyzq)[:, :4])


def read_sources(n: int, rank: int = 0, path: str = "./", position: int = 0):
    """Dataset::readSources of n bodies from byte `position`: ((n, 4) x, y, z, q; next position)."""
    v, pos = _read_values(f"{path}source{rank:04d}.dat", 4 * n, position)
    return v.reshape(n, 4), pos


def write_targets(trg: np.ndarray, rank: int = 0, path: str = "./") -> str:
    """Dataset::writeTargets: path + 'target%04d.dat' (rank)."""
    return _write_values(f"{path}target{rank:04d}.dat", np.asarray(trg)[:, :4])


def read_targets(n: int, rank: int = 0, path: str = "./", position: int = 0):
    """Dataset::readTargets of n bodies from byte `position`: ((n, 4) targets; next position)."""
    v, pos = _read_values(f"{path}target{rank:04d}.dat", 4 * n, position)
    return v.reshape(n, 4), pos
