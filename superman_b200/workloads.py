"""Seeded synthetic inputs for the benchmark configurations.

One generator family (SplitMix64, counter-indexed) so C, C++ and Python
callers can reproduce the same matrices:  output i of stream `seed` is
mix(seed + (i + 1) * 0x9E3779B97F4A7C15) with the SplitMix64 finaliser, and a
uniform double in [0, 1) is its top 53 bits times 2^-53.

Workloads (all row-major, float64 / complex128):
  dense_uniform(n, seed)        a_ij ~ U[0, 1)
  binary_bernoulli(n, seed, p)  Bernoulli(p) with the identity OR-ed in
  sparse_perm_plus(n, seed, k)  random permutation + k extra nonzeros per row at
                                uniform columns, values U[0.5, 1.5)
  haar_unitary(N, seed)         QR of a complex Gaussian, R diagonal made
                                positive (Haar measure)
  haar_block(n, seed, N=256)    top-left n x n block of haar_unitary(N, seed)
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """Outputs offset .. offset+count-1 of the SplitMix64 stream of `seed`."""
    with np.errstate(over="ignore"):
        i = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """U[0, 1) doubles: top 53 bits of each SplitMix64 output times 2^-53."""
    return (splitmix64(seed, count, offset) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def dense_uniform(n: int, seed: int) -> np.ndarray:
    return uniform(seed, n * n).reshape(n, n)


def binary_bernoulli(n: int, seed: int, p: float = 0.5) -> np.ndarray:
    a = (uniform(seed, n * n).reshape(n, n) < p).astype(np.uint8)
    a |= np.eye(n, dtype=np.uint8)
    return a


def sparse_perm_plus(n: int, seed: int, extra: int = 3) -> np.ndarray:
    """Random permutation matrix plus `extra` nonzeros per row at uniform
    columns (collisions merge), values U[0.5, 1.5)."""
    u = uniform(seed, n + n * extra + n * (extra + 1))
    perm = np.arange(n)
    for i in range(n - 1, 0, -1):  # Fisher-Yates driven by the stream
        j = int(u[i] * (i + 1))
        perm[i], perm[j] = perm[j], perm[i]
    a = np.zeros((n, n))
    cols = (u[n:n + n * extra] * n).astype(np.int64).reshape(n, extra)
    vals = 0.5 + u[n + n * extra:].reshape(n, extra + 1)
    for i in range(n):
        a[i, perm[i]] = vals[i, 0]
        for k in range(extra):
            a[i, cols[i, k]] = vals[i, k + 1]
    return a


def complex_gaussian(seed: int, shape) -> np.ndarray:
    count = int(np.prod(shape))
    u = uniform(seed, 2 * count)
    u1, u2 = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log1p(-u1))
    th = 2.0 * np.pi * u2
    return ((r * np.cos(th)) + 1j * (r * np.sin(th))).reshape(shape) / np.sqrt(2.0)


def haar_unitary(N: int, seed: int) -> np.ndarray:
    g = complex_gaussian(seed, (N, N))
    q, r = np.linalg.qr(g)
    d = np.diagonal(r)
    return q * (d / np.abs(d))


def haar_block(n: int, seed: int, N: int = 256) -> np.ndarray:
    return np.ascontiguousarray(haar_unitary(N, seed)[:n, :n])


# ------------------------------------------------------------ serving stream --
# Request i of the seeded serving stream: n uniform in [n_lo, n_hi]; with
# probability 1/2 a real U[0, 1) matrix (dense_uniform(n, seed * 1000003 + i)),
# else an n x n block, at seeded row/column offsets, of Haar unitary i % 4
# (haar_unitary(256, seed + i % 4)).  One numpy Generator(seed) drives n, the
# kind and the offsets, in that order per request.

def serve_stream_meta(n_lo: int, n_hi: int, count: int, seed: int = 2026):
    """[(n, is_complex, r0, c0)] per request, without building the matrices."""
    rng = np.random.default_rng(seed)
    meta = []
    for _ in range(count):
        n = int(rng.integers(n_lo, n_hi + 1))
        if rng.random() < 0.5:
            meta.append((n, False, 0, 0))
        else:
            r0, c0 = rng.integers(0, 256 - n + 1, size=2)
            meta.append((n, True, int(r0), int(c0)))
    return meta


class ServeStream:
    """Builds the matrices of the seeded serving stream on demand."""

    def __init__(self, n_lo: int, n_hi: int, count: int, seed: int = 2026):
        self.seed = seed
        self.meta = serve_stream_meta(n_lo, n_hi, count, seed)
        self._unitaries = {}

    def __len__(self):
        return len(self.meta)

    def matrix(self, i: int) -> np.ndarray:
        n, cplx, r0, c0 = self.meta[i]
        if not cplx:
            return dense_uniform(n, self.seed * 1000003 + i)
        k = i % 4
        if k not in self._unitaries:
            self._unitaries[k] = haar_unitary(256, self.seed + k)
        return np.ascontiguousarray(self._unitaries[k][r0:r0 + n, c0:c0 + n])

    def matrices(self):
        return [self.matrix(i) for i in range(len(self.meta))]

    def first_index(self, n: int, cplx: bool) -> int:
        """Index of the first request of size n and the given kind (-1 if none)."""
        for i, (m, c, _, _) in enumerate(self.meta):
            if m == n and c == cplx:
                return i
        return -1


def matrix_sha256(a: np.ndarray) -> str:
    """Digest of a matrix's float64 bytes (complex: interleaved re/im), row-major."""
    import hashlib
    a = np.ascontiguousarray(a)
    b = a.view(np.float64) if np.iscomplexobj(a) else a.astype(np.float64, copy=False)
    return hashlib.sha256(np.ascontiguousarray(b).tobytes()).hexdigest()
