"""Julia's ``MersenneTwister(seed)`` and ``rand(rng, n, n)``, restated in NumPy.

TEST INFRASTRUCTURE ONLY.  This module belongs to the oracle: the tests, the
smoke check and the CPU-baseline leg of the benchmark may use it; the product
path never imports it (the library carries its own, independent restatement in
C, ``csrc/esc_rng.cpp``, which the tests compare with this one bit for bit).

The reference draws the initial noise with
``rand(MersenneTwister(seed), n, n)`` (``core_shell.jl:32``; ``checks.jl:4``
through ``initial_fields``).  Both pieces live outside the reference, in
Julia 1.12's ``Random`` standard library (the reference ``Manifest.toml:3``
pins julia_version 1.12.6) and the dSFMT C library it calls; neither is under
the reference tree, so this file restates their published algorithms:

* Seeding (``Random`` stdlib, ``hash_seed`` + ``initstate!`` of the
  MersenneTwister): a non-negative integer seed is cut into 32-bit words, least
  significant first; the little-endian bytes of the words are hashed with
  SHA2-256; the 32-byte digest, read as eight little-endian UInt32 words, is
  the key of ``dsfmt_init_by_array``.
* dSFMT-19937 (Saito & Matsumoto, "SIMD-oriented Fast Mersenne Twister", the
  double-precision variant, version 2.2): the ``init_by_array`` key schedule
  over the 768 32-bit words of the state, the initial mask that puts every
  state word in [1, 2), the period certification, and the recursion
  ``do_recursion`` (shift 19, shift 12, the two 52-bit masks, the 64-bit
  rotation of the "lung" word) with the pick-up position 117 of N = 191.
* ``rand(rng, n, n)`` on a freshly seeded generator fills the array with the
  first n*n values of the stream in memory order (Julia's array fill calls
  ``dsfmt_fill_array_close1_open2`` on the fresh state and subtracts 1), each
  value in [0, 1).

Pinned: with this stream the oracle reproduces the reference's recorded
initial energies 329.48858453024934 (64^2, radius 16) exactly and
4406.5104552251505 (256^2) to 2e-16, and after the runs of ``checks.jl`` the
recorded final energies, ranges and RMS differences of ``check-results.txt:2-7``
(``tests/test_oracle.py``).  Only even n*n >= 382 (both cases of the reference)
is pinned against the reference; the stream is the same for any count.
"""
from __future__ import annotations

import hashlib
import struct

import numpy as np

__all__ = ["julia_seed_key", "dsfmt_init_by_array", "dsfmt_stream", "rand_uniform", "rand_matrix"]

_M32 = 0xFFFFFFFF
_M64 = 0xFFFFFFFFFFFFFFFF

# dSFMT-19937 parameters (published parameter set of the 19937 exponent)
_N = 191             # 128-bit state words
_POS1 = 117
_SL1 = 19
_SR = 12
_MSK = (0x000FFAFFFFFFFB3F, 0x000FFDFFFC90FFFD)
_FIX = (0x90014964B32F4329, 0x3B8D12AC548A7C7A)
_PCV = (0x3D84E1AC0DC82880, 0x0000000000000001)
_LOW = 0x000FFFFFFFFFFFFF
_HIGH = 0x3FF0000000000000


def julia_seed_key(seed: int) -> list[int]:
    """The dSFMT key of ``MersenneTwister(seed)``: SHA2-256 over the seed's
    32-bit words (least significant first, little-endian bytes), read back as
    eight little-endian UInt32 words."""
    if seed < 0:
        raise ValueError("only non-negative seeds are restated")
    h = hashlib.sha256()
    while True:
        h.update(struct.pack("<I", seed & _M32))
        seed >>= 32
        if seed == 0:
            break
    return list(struct.unpack("<8I", h.digest()))


def _ini1(x: int) -> int:
    return ((x ^ (x >> 27)) * 1664525) & _M32


def _ini2(x: int) -> int:
    return ((x ^ (x >> 27)) * 1566083941) & _M32


def dsfmt_init_by_array(key: list[int]) -> np.ndarray:
    """dSFMT ``init_by_array``: returns the (N + 1) x 2 uint64 state, the last
    row being the lung, ready for the first fill (index at the end of the state)."""
    size = (_N + 1) * 4          # 32-bit words, lung included
    lag = 11                     # size >= 623
    mid = (size - lag) // 2
    s = [0x8B8B8B8B] * size
    count = max(len(key) + 1, size)

    r = _ini1(s[0] ^ s[mid] ^ s[size - 1])
    s[mid] = (s[mid] + r) & _M32
    r = (r + len(key)) & _M32
    s[(mid + lag) % size] = (s[(mid + lag) % size] + r) & _M32
    s[0] = r
    count -= 1
    i, j = 1, 0
    while j < count:
        r = _ini1(s[i] ^ s[(i + mid) % size] ^ s[(i + size - 1) % size])
        s[(i + mid) % size] = (s[(i + mid) % size] + r) & _M32
        r = (r + (key[j] if j < len(key) else 0) + i) & _M32
        s[(i + mid + lag) % size] = (s[(i + mid + lag) % size] + r) & _M32
        s[i] = r
        i = (i + 1) % size
        j += 1
    for _ in range(size):
        r = _ini2((s[i] + s[(i + mid) % size] + s[(i + size - 1) % size]) & _M32)
        s[(i + mid) % size] ^= r
        r = (r - i) & _M32
        s[(i + mid + lag) % size] ^= r
        s[i] = r
        i = (i + 1) % size

    u = [s[2 * k] | (s[2 * k + 1] << 32) for k in range(size // 2)]
    for k in range(2 * _N):                       # initial mask: state words in [1, 2)
        u[k] = (u[k] & _LOW) | _HIGH
    inner = ((u[2 * _N] ^ _FIX[0]) & _PCV[0]) ^ ((u[2 * _N + 1] ^ _FIX[1]) & _PCV[1])
    sh = 32
    while sh:                                     # parity of inner
        inner ^= inner >> sh
        sh >>= 1
    if inner & 1 != 1:                            # period certification
        u[2 * _N + 1] ^= 1
    return np.array(u, dtype=np.uint64).reshape(_N + 1, 2)


def _rot32(x: np.ndarray) -> np.ndarray:
    return (x >> np.uint64(32)) | (x << np.uint64(32))


def dsfmt_stream(state: np.ndarray, count: int) -> np.ndarray:
    """The next ``count`` (rounded up to even) raw 64-bit outputs of a fresh state.

    The recursion for output i reads outputs i - N and i - N + POS1 and the lung.
    The lung update  lung_i = swap-rotate(lung_{i-1}) XOR v_i  (v_i built from
    the two earlier outputs) is linear over GF(2) and the swap-rotate is an
    involution, so within a run of N - POS1 = 74 outputs, whose inputs are all
    earlier outputs, the lungs follow from one prefix XOR.
    """
    nw = (count + 1) // 2
    x = np.empty((_N + nw, 2), dtype=np.uint64)
    x[:_N] = state[:_N]
    lung = state[_N].copy()
    sl1, sr = np.uint64(_SL1), np.uint64(_SR)
    msk = np.array(_MSK, dtype=np.uint64)
    blk = _N - _POS1
    i0 = 0
    while i0 < nw:
        m = min(blk, nw - i0)
        a = x[i0:i0 + m]                           # output i - N   (row i0 + k of x)
        b = x[i0 + _POS1:i0 + _POS1 + m]           # output i - N + POS1
        v = (a << sl1) ^ b
        # lung_k (k = 1..m) = R^k(lung_0) ^ XOR_{t<=k} R^{k-t}(v_t), R = swap lanes + rotate 32
        # with R^2 = identity: write w_t = R^t(v_t), lung_k = R^k(lung_0 ^ XOR_{t<=k} w_t)
        w = v.copy()
        odd = (np.arange(1, m + 1) % 2) == 1
        w[odd] = _rot32(v[odd][:, ::-1])
        acc = np.bitwise_xor.accumulate(w, axis=0) ^ lung
        lk = acc.copy()
        lk[odd] = _rot32(acc[odd][:, ::-1])
        r = (lk >> sr) ^ (lk & msk) ^ a
        x[_N + i0:_N + i0 + m] = r
        lung = lk[-1].copy()
        i0 += m
    return x[_N:].reshape(-1)[:count]


def rand_uniform(seed: int, count: int) -> np.ndarray:
    """The first ``count`` Float64 values of ``rand(MersenneTwister(seed), count)``, in [0, 1)."""
    raw = dsfmt_stream(dsfmt_init_by_array(julia_seed_key(seed)), count)
    return raw.view(np.float64) - 1.0


def rand_matrix(seed: int, n: int, m: int | None = None) -> np.ndarray:
    """``rand(MersenneTwister(seed), n, m)`` as a C-ordered array ``a[j, i]``
    (the bytes of the column-major Julia matrix, first index i contiguous)."""
    m = n if m is None else m
    return rand_uniform(seed, n * m).reshape(m, n)
