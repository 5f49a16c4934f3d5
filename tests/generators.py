"""Deterministic input generators restated from the reference's tests and bench.

Each generator names the reference function it mirrors.  Plain numpy: these make
INPUTS, they compute nothing that is checked.
"""
from __future__ import annotations

import numpy as np

P = 2147483647


def sha3_pattern(length: int, mul: int = 11, add: int = 7) -> bytes:
    """SHA3OracleTests.swift:54-66 (byte i = i*11 + 7)."""
    return bytes(((i * mul + add) & 0xFF) for i in range(length))


def make_batch_messages(count, stride, length, salt=0) -> bytes:
    """SHA3OracleTests.swift:767-775."""
    b = bytearray([0xA5] * (count * stride))
    for m in range(count):
        for o in range(length):
            b[m * stride + o] = (m * 31 + o * 9 + salt + 11) & 0xFF
    return bytes(b)


def make_permutation_states(count, stride, salt) -> np.ndarray:
    """SHA3OracleTests.swift:776-795 (lane = state*0x1f1f0101 ^ lane*0x01020305 ^ salt*0x10001 ^ lane<<40 ^ state<<56)."""
    b = np.full(count * stride, 0xA5, np.uint8)
    M = (1 << 64) - 1
    for s in range(count):
        for lane in range(25):
            v = ((s * 0x1F1F0101) & M) ^ ((lane * 0x01020305) & M) ^ ((salt * 0x10001) & M) ^ ((lane << 40) & M) ^ ((s << 56) & M)
            b[s * stride + lane * 8: s * stride + lane * 8 + 8] = np.frombuffer(int(v).to_bytes(8, "little"), np.uint8)
    return b


def make_leaves(count, stride, length, salt=0) -> bytes:
    """MerkleTests.swift:588-599 (byte = leaf*29 + j*7 + salt + 3, fill 0xa5)."""
    b = bytearray([0xA5] * (count * stride))
    for leaf in range(count):
        base = leaf * stride
        for j in range(length):
            b[base + j] = (leaf * 29 + j * 7 + salt + 3) & 0xFF
    return bytes(b)


def make_bench_leaves(count, length) -> bytes:
    """zkmetal-bench main.swift:1300-1314 (byte = leaf*131 + j*17 + 0x5a)."""
    if length == 0:
        return b""
    leaf = np.arange(count, dtype=np.int64)[:, None]
    j = np.arange(length, dtype=np.int64)[None, :]
    return ((leaf * 131 + j * 17 + 0x5A) & 0xFF).astype(np.uint8).tobytes()


def deterministic_m31(count, salt) -> np.ndarray:
    """zkmetal-bench main.swift:1316-1324."""
    i = np.arange(count, dtype=np.uint64)
    v = (i + 1) * np.uint64(1048573) + np.uint64(salt) * np.uint64(65537) + i * np.uint64(17) * np.uint64(salt | 1)
    return (v % np.uint64(P)).astype(np.uint32)


def deterministic_qm31(count, salts) -> np.ndarray:
    """zkmetal-bench main.swift:1342-1356."""
    return np.stack([deterministic_m31(count, s) for s in salts], axis=1).astype(np.uint32)


def stable_circle_evaluations(count) -> np.ndarray:
    """CircleDomainTests.swift:2825-2837."""
    i = np.arange(count, dtype=np.uint64)
    return np.stack([17 + i * 3, 29 + i * 5, 31 + i * 7, 43 + i * 11], axis=1).astype(np.uint32)


def deterministic_qm31_coefficients(count, salt) -> np.ndarray:
    """CircleDomainTests.swift:2839-2849."""
    i = np.arange(count, dtype=np.uint64)
    s = np.uint64(salt)
    M = np.uint64(0xFFFFFFFF)
    return np.stack([(3 + s + i * 5) & M, (7 + s + i * 11) & M, (13 + s + i * 17) & M, (19 + s + i * 23) & M], axis=1).astype(np.uint32)


def circle_fri_challenges(rounds) -> np.ndarray:
    """zkmetal-bench main.swift:1414-1423."""
    r = np.arange(rounds, dtype=np.uint32)
    return np.stack([41 + r * 18, 43 + r * 22, 47 + r * 26, 53 + r * 30], axis=1).astype(np.uint32)


def bench_codeword_polynomial(domain_size):
    """zkmetal-bench main.swift:1376-1395 (8 x-coefficients, 7 y-coefficients)."""
    nx = max(1, min(8, domain_size // 2))
    ny = max(1, min(7, domain_size // 2))
    return deterministic_qm31(nx, [0xE01, 0xE03, 0xE07, 0xE0B]), deterministic_qm31(ny, [0xE11, 0xE17, 0xE1D, 0xE23])


def splitmix64(seed):
    """SplitMix64 stream (seeded synthetic inputs for the large configs)."""
    state = seed & 0xFFFFFFFFFFFFFFFF
    while True:
        state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        yield z ^ (z >> 31)


def splitmix64_array(seed, n) -> np.ndarray:
    """Vectorised SplitMix64: element k is the (k+1)-th output of the stream."""
    GOLD = np.uint64(0x9E3779B97F4A7C15)
    k = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + k * GOLD
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform_m31(seed, n) -> np.ndarray:
    """Uniform canonical M31: low 31 bits of a u32 draw, rejecting 0x7fffffff."""
    out = np.empty(0, np.uint32)
    draw = 0
    while len(out) < n:
        need = n - len(out)
        words = splitmix64_array(seed + draw * 0x51ED27, need + need // 16 + 16)
        draw += 1
        v = (words & np.uint64(0x7FFFFFFF)).astype(np.uint32)
        v = v[v != np.uint32(P)]
        out = np.concatenate([out, v])
    return out[:n]


# --- seeded inputs of the benchmark configurations ---------------------------
# Seeds per configuration: C1 0xA11CE001, C2 0xA11CE002, C3 0xA11CE003,
# C4 0xA11CE004 (bench.py), C5 0xA11CE005.  Uniform bytes are the little-endian
# bytes of the SplitMix64 stream; uniform M31 values are the low 31 bits of a
# draw with 0x7fffffff rejected (uniform_m31 above).
C1_SEED, C2_SEED, C3_SEED = 0xA11CE001, 0xA11CE002, 0xA11CE003


def splitmix64_range(seed, start, stop) -> np.ndarray:
    """Outputs start+1 ... stop of the SplitMix64 stream (element k of the result is
    output start + k + 1), so a long stream can be made in chunks."""
    GOLD = np.uint64(0x9E3779B97F4A7C15)
    k = np.arange(start + 1, stop + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + k * GOLD
        z ^= z >> np.uint64(30)
        z *= np.uint64(0xBF58476D1CE4E5B9)
        z ^= z >> np.uint64(27)
        z *= np.uint64(0x94D049BB133111EB)
        z ^= z >> np.uint64(31)
    return z


def config_bytes(seed, nbytes) -> np.ndarray:
    """`nbytes` uniform bytes: the little-endian bytes of the SplitMix64 stream."""
    words = (nbytes + 7) // 8
    out = np.empty(words, np.uint64)
    chunk = 1 << 24
    for s in range(0, words, chunk):
        e = min(words, s + chunk)
        out[s:e] = splitmix64_range(seed, s, e)
    return out.view(np.uint8)[:nbytes]


def config_indices(seed, count, modulus) -> np.ndarray:
    """`count` seeded leaf indices in [0, modulus) (a power of two)."""
    return (splitmix64_array(seed ^ 0x1D, count) % np.uint64(modulus)).astype(np.uint64)


def config_c1():
    """C1: 2^16 leaves of 64 uniform bytes and 16 opening indices."""
    n = 1 << 16
    return config_bytes(C1_SEED, n * 64), config_indices(C1_SEED, 16, n)


def config_c3(log_size=22, log_blowup=2):
    """C3: FFT-basis coefficient prefix of a log-22 codeword at blowup 4 -- x-line and
    y-line indices below 2^19 carry uniform M31 values lifted to QM31 (the first
    2^20 interleaved positions), the rest of the 2^22 coefficients are zero -- and a
    32-byte public-input digest."""
    count = (1 << log_size) >> log_blowup
    coeffs = np.zeros((count, 4), np.uint32)
    coeffs[:, 0] = uniform_m31(C3_SEED, count)
    pub = config_bytes(C3_SEED ^ 0x9B, 32).tobytes()
    return coeffs, pub
