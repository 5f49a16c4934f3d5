"""ctypes wrapper over oracle/liboracle.so -- the CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
bench's cpu_baseline / reference arm, always as the checker.  The CUDA library
(apple_b200) never imports this module.

Each function mirrors a reference CPU oracle; the C++ it calls cites the Swift
file:line it restates (oracle/azk_oracle.hpp).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

u8p = ctypes.POINTER(ctypes.c_uint8)
u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)
c_u32 = ctypes.c_uint32
c_u64 = ctypes.c_uint64
c_int = ctypes.c_int


class OracleError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"oracle error {code}: {message}")
        self.code = code


def build() -> None:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.azko_last_error.restype = ctypes.c_char_p
    return _lib


def _p8(a):
    return a.ctypes.data_as(u8p)


def _p32(a):
    return a.ctypes.data_as(u32p)


def _p64(a):
    return a.ctypes.data_as(u64p)


def _check(rc: int) -> None:
    if rc != 0:
        raise OracleError(rc, lib().azko_last_error().decode())


def _bytes(b) -> np.ndarray:
    return np.frombuffer(bytes(b), dtype=np.uint8).copy() if not isinstance(b, np.ndarray) else np.ascontiguousarray(b, dtype=np.uint8)


def _q(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32).reshape(-1, 4))


def num_threads() -> int:
    return lib().azko_num_threads()


def set_num_threads(n: int) -> None:
    lib().azko_set_num_threads(c_int(n))


# --- hashing -----------------------------------------------------------------
def sha3_256(data: bytes) -> bytes:
    buf = _bytes(data)
    out = np.zeros(32, np.uint8)
    _check(lib().azko_sha3_256(_p8(buf), c_u64(len(buf)), _p8(out)))
    return out.tobytes()


def keccak_256(data: bytes) -> bytes:
    buf = _bytes(data)
    out = np.zeros(32, np.uint8)
    _check(lib().azko_keccak_256(_p8(buf), c_u64(len(buf)), _p8(out)))
    return out.tobytes()


def keccak_f1600(states: np.ndarray, stride: int = 200) -> np.ndarray:
    """Permute `count` states stored at byte `stride` (returns a new array)."""
    buf = np.ascontiguousarray(states, dtype=np.uint8).reshape(-1).copy()
    count = len(buf) // stride
    _check(lib().azko_keccak_f1600(_p8(buf), c_u64(count), c_u64(stride)))
    return buf


def hash_batch(messages, count, stride, length, out_stride=32, keccak=False) -> bytes:
    buf = _bytes(messages) if count * stride > 0 else np.zeros(1, np.uint8)
    out = np.zeros(count * out_stride, np.uint8)
    _check(lib().azko_hash_batch(_p8(buf), c_u64(count), c_u64(stride), c_u64(length), _p8(out), c_u64(out_stride), c_int(1 if keccak else 0)))
    return out.tobytes()


# --- Merkle ------------------------------------------------------------------
def merkle_root(leaves, count, stride, length) -> bytes:
    buf = _bytes(leaves) if len(leaves) else np.zeros(1, np.uint8)
    root = np.zeros(32, np.uint8)
    _check(lib().azko_merkle_root(_p8(buf), c_u64(len(leaves)), c_u64(count), c_u64(stride), c_u64(length), _p8(root)))
    return root.tobytes()


def merkle_openings(leaves, count, stride, length, indices):
    """Returns (root, [list of sibling digests per index]) with the tree built once."""
    buf = _bytes(leaves) if len(leaves) else np.zeros(1, np.uint8)
    idx = np.ascontiguousarray(indices, dtype=np.uint64)
    depth = int(count).bit_length() - 1
    sib = np.zeros(max(1, len(idx) * depth * 32), np.uint8)
    root = np.zeros(32, np.uint8)
    _check(lib().azko_merkle_openings(_p8(buf), c_u64(len(leaves)), c_u64(count), c_u64(stride), c_u64(length), _p64(idx), c_u64(len(idx)), _p8(sib), _p8(root)))
    out = []
    for k in range(len(idx)):
        out.append([sib[(k * depth + l) * 32:(k * depth + l + 1) * 32].tobytes() for l in range(depth)])
    return root.tobytes(), out


def merkle_opening_literal(leaves, count, stride, length, index):
    buf = _bytes(leaves) if len(leaves) else np.zeros(1, np.uint8)
    depth = int(count).bit_length() - 1
    sib = np.zeros(max(1, depth * 32), np.uint8)
    root = np.zeros(32, np.uint8)
    _check(lib().azko_merkle_opening_literal(_p8(buf), c_u64(len(leaves)), c_u64(count), c_u64(stride), c_u64(length), c_u64(index), _p8(sib), _p8(root)))
    return root.tobytes(), [sib[l * 32:(l + 1) * 32].tobytes() for l in range(depth)]


def merkle_verify(leaf: bytes, index: int, siblings, root: bytes) -> bool:
    lb = _bytes(leaf) if len(leaf) else np.zeros(1, np.uint8)
    sb = _bytes(b"".join(siblings)) if siblings else np.zeros(1, np.uint8)
    rb = _bytes(root)
    rc = lib().azko_merkle_verify(_p8(lb), c_u64(len(leaf)), c_u64(index), _p8(sb), c_u64(len(siblings)), _p8(rb))
    if rc < 0:
        raise OracleError(1, lib().azko_last_error().decode())
    return rc == 1


def merkle_root_prehashed(digests: bytes) -> bytes:
    buf = _bytes(digests)
    root = np.zeros(32, np.uint8)
    _check(lib().azko_merkle_root_prehashed(_p8(buf), c_u64(len(buf) // 32), _p8(root)))
    return root.tobytes()


def merkle_qm31_levels(layer) -> np.ndarray:
    q = _q(layer)
    n = len(q)
    out = np.zeros((2 * n - 1) * 32, np.uint8)
    _check(lib().azko_merkle_qm31_levels(_p32(q), c_u64(n), _p8(out)))
    return out


# --- transcript --------------------------------------------------------------
def transcript_squeeze(frames, count, modulus):
    data = _bytes(b"".join(frames)) if any(len(f) for f in frames) else np.zeros(1, np.uint8)
    lens = np.array([len(f) for f in frames], dtype=np.uint64)
    out = np.zeros(max(1, count), np.uint32)
    _check(lib().azko_transcript_squeeze(_p8(data), _p64(lens), c_u64(len(frames)), c_u64(count), c_u32(modulus), _p32(out)))
    return [int(v) for v in out[:count]]


def transcript_state(frames) -> np.ndarray:
    data = _bytes(b"".join(frames)) if any(len(f) for f in frames) else np.zeros(1, np.uint8)
    lens = np.array([len(f) for f in frames], dtype=np.uint64)
    out = np.zeros(25, np.uint64)
    _check(lib().azko_transcript_state(_p8(data), _p64(lens), c_u64(len(frames)), _p64(out)))
    return out


# --- fields / circle ---------------------------------------------------------
def qm31_mul(x, y):
    a, b, out = _q(x), _q(y), np.zeros(4, np.uint32)
    _check(lib().azko_qm31_mul(_p32(a), _p32(b), _p32(out)))
    return tuple(int(v) for v in out)


def qm31_inv(x):
    a, out = _q(x), np.zeros(4, np.uint32)
    _check(lib().azko_qm31_inv(_p32(a), _p32(out)))
    return tuple(int(v) for v in out)


def domain_points(log_size: int) -> np.ndarray:
    out = np.zeros(2 << log_size, np.uint32)
    _check(lib().azko_domain_points(c_u32(log_size), _p32(out)))
    return out.reshape(-1, 2)


def domain_encode(log_size: int) -> bytes:
    out = np.zeros(44, np.uint8)
    _check(lib().azko_domain_encode(c_u32(log_size), _p8(out)))
    return out.tobytes()


def fft_twiddles(log_size: int) -> np.ndarray:
    out = np.zeros(max(1, (1 << log_size) - 1), np.uint32)
    _check(lib().azko_fft_twiddles(c_u32(log_size), _p32(out)))
    return out[: (1 << log_size) - 1]


def inverse_layers(log_size: int, rounds: int) -> list:
    n = 1 << log_size
    total = sum(n >> (r + 1) for r in range(rounds))
    out = np.zeros(max(1, total), np.uint32)
    _check(lib().azko_inverse_layers(c_u32(log_size), c_u32(rounds), _p32(out)))
    layers, off = [], 0
    for r in range(rounds):
        m = n >> (r + 1)
        layers.append(out[off:off + m].copy())
        off += m
    return layers


def _poly(x, y):
    xq = _q(x) if len(x) else np.zeros((1, 4), np.uint32)
    yq = _q(y) if len(y) else np.zeros((1, 4), np.uint32)
    return xq, len(x), yq, len(y)


def fft_basis_coefficients(log_size: int, x, y) -> np.ndarray:
    xq, nx, yq, ny = _poly(x, y)
    out = np.zeros((1 << log_size, 4), np.uint32)
    _check(lib().azko_fft_basis_coefficients(c_u32(log_size), _p32(xq), c_u64(nx), _p32(yq), c_u64(ny), _p32(out)))
    return out


def evaluate_direct(log_size: int, x, y) -> np.ndarray:
    xq, nx, yq, ny = _poly(x, y)
    out = np.zeros((1 << log_size, 4), np.uint32)
    _check(lib().azko_evaluate_direct(c_u32(log_size), _p32(xq), c_u64(nx), _p32(yq), c_u64(ny), _p32(out)))
    return out


def fft_evaluate(log_size: int, coefficients) -> np.ndarray:
    v = _q(coefficients).copy()
    _check(lib().azko_fft_evaluate(c_u32(log_size), _p32(v)))
    return v


def fold(evaluations, inverse_points, challenge) -> np.ndarray:
    ev, inv, ch = _q(evaluations), _q(inverse_points), _q(challenge)
    out = np.zeros((len(ev) // 2, 4), np.uint32)
    _check(lib().azko_fold(_p32(ev), c_u64(len(ev)), _p32(inv), _p32(ch), _p32(out)))
    return out


def circle_fold_chain(log_size: int, evaluations, challenges) -> np.ndarray:
    ev, ch = _q(evaluations), _q(challenges)
    rounds = len(ch)
    out = np.zeros(((1 << log_size) >> rounds, 4), np.uint32)
    _check(lib().azko_circle_fold_chain(c_u32(log_size), _p32(ev), _p32(ch), c_u32(rounds), _p32(out)))
    return out


def qm31_transcript_challenges(input_count: int, commitments) -> np.ndarray:
    cm = _bytes(b"".join(commitments))
    out = np.zeros((len(commitments), 4), np.uint32)
    _check(lib().azko_qm31_transcript_challenges(c_u64(input_count), _p8(cm), c_u32(len(commitments)), _p32(out)))
    return out


def qm31_merkle_fold_chain(evaluations, inverse_layers_qm31):
    ev = _q(evaluations)
    inv = _q(np.concatenate([_q(l) for l in inverse_layers_qm31]))
    rounds = len(inverse_layers_qm31)
    fin = np.zeros((len(ev) >> rounds, 4), np.uint32)
    cm = np.zeros(32 * rounds, np.uint8)
    ch = np.zeros((rounds, 4), np.uint32)
    _check(lib().azko_qm31_merkle_fold_chain(_p32(ev), c_u64(len(ev)), _p32(inv), c_u32(rounds), _p32(fin), _p8(cm), _p32(ch)))
    return fin, [cm[32 * r:32 * r + 32].tobytes() for r in range(rounds)], ch


# --- PCS proof ---------------------------------------------------------------
class ProofResult:
    def __init__(self, proof, commitments, challenges, final_layer, query_pairs):
        self.proof = proof
        self.commitments = commitments
        self.challenges = challenges
        self.final_layer = final_layer
        self.query_pairs = query_pairs


def prove(log_size: int, evaluations, log_blowup: int, queries: int, public_digest: bytes, rounds: int,
          grinding_bits: int = 0, claimed=()) -> ProofResult:
    ev = _q(evaluations)
    pub = _bytes(public_digest)
    cl = np.ascontiguousarray(list(claimed) or [0], dtype=np.uint64)
    n = 1 << log_size
    cap = 64 + 44 + 64 + 32 * rounds + 16 * n + queries * rounds * 2 * (16 + 32 * log_size + 32) + len(claimed) * (32 + 32 * log_size) + 64
    out = np.zeros(cap, np.uint8)
    plen = c_u64(cap)
    cm = np.zeros(32 * rounds, np.uint8)
    ch = np.zeros((rounds, 4), np.uint32)
    fin = np.zeros((n >> rounds, 4), np.uint32)
    qp = np.zeros(queries, np.uint32)
    _check(lib().azko_prove(c_u32(log_size), _p32(ev), c_u32(log_blowup), c_u32(queries), c_u32(grinding_bits), _p8(pub), c_u32(rounds),
                            _p64(cl), c_u64(len(claimed)), _p8(out), ctypes.byref(plen), _p8(cm), _p32(ch), _p32(fin), _p32(qp)))
    return ProofResult(out[: plen.value].tobytes(), [cm[32 * r:32 * r + 32].tobytes() for r in range(rounds)], ch, fin, [int(v) for v in qp])


def prove_literal(log_size: int, coefficients, log_blowup: int, queries: int, public_digest: bytes, rounds: int) -> bytes:
    """FFT-basis coefficients -> proof bytes through the reference's literal builder on
    one thread (stage-by-stage FFT, transcript replayed per challenge, a full Merkle
    rebuild per opening); the same bytes as fft_evaluate + prove."""
    c = _q(coefficients)
    pub = _bytes(public_digest)
    n = 1 << log_size
    cap = 64 + 44 + 64 + 32 * rounds + 16 * n + queries * rounds * 2 * (16 + 32 * log_size + 32) + 64
    out = np.zeros(cap, np.uint8)
    plen = c_u64(cap)
    _check(lib().azko_prove_literal(c_u32(log_size), _p32(c), c_u32(log_blowup), c_u32(queries), _p8(pub), c_u32(rounds), _p8(out),
                                    ctypes.byref(plen)))
    return out[: plen.value].tobytes()


def commit_fold_chain_leaf64(log_size: int, evaluations, log_blowup: int, queries: int, public_digest: bytes, rounds: int):
    """Commitments, challenges and final layer of the chain with 64-byte (4 x QM31) Merkle leaves."""
    ev = _q(evaluations)
    pub = _bytes(public_digest)
    cm = np.zeros(32 * rounds, np.uint8)
    ch = np.zeros((rounds, 4), np.uint32)
    fl = np.zeros(((1 << log_size) >> rounds, 4), np.uint32)
    _check(lib().azko_commit_fold_chain_leaf64(c_u32(log_size), _p32(ev), c_u32(log_blowup), c_u32(queries), _p8(pub), c_u32(rounds), _p8(cm),
                                               _p32(ch), _p32(fl)))
    return [cm[32 * k:32 * k + 32].tobytes() for k in range(rounds)], ch, fl


def verify(proof: bytes, public_digest: bytes) -> bool:
    pb, pub = _bytes(proof), _bytes(public_digest)
    rc = lib().azko_verify(_p8(pb), c_u64(len(pb)), _p8(pub))
    if rc < 0:
        raise OracleError(1, lib().azko_last_error().decode())
    return rc == 1


def proof_roundtrip(proof: bytes) -> None:
    pb = _bytes(proof)
    _check(lib().azko_proof_roundtrip(_p8(pb), c_u64(len(pb))))


def verify_contract(proof: bytes, log_size: int, x, y, claimed, log_blowup, queries, grinding_bits=0) -> int:
    pb = _bytes(proof)
    xq, nx, yq, ny = _poly(x, y)
    idx = np.ascontiguousarray(claimed, dtype=np.uint64)
    return lib().azko_verify_contract(_p8(pb), c_u64(len(pb)), c_u32(log_size), _p32(xq), c_u64(nx), _p32(yq), c_u64(ny), _p64(idx), c_u64(len(idx)),
                                      c_u32(log_blowup), c_u32(queries), c_u32(grinding_bits))


def claim_digest(log_size: int, x, y, claimed) -> bytes:
    xq, nx, yq, ny = _poly(x, y)
    idx = np.ascontiguousarray(claimed, dtype=np.uint64)
    out = np.zeros(32, np.uint8)
    _check(lib().azko_claim_digest(c_u32(log_size), _p32(xq), c_u64(nx), _p32(yq), c_u64(ny), _p64(idx), c_u64(len(idx)), _p8(out)))
    return out.tobytes()


# --- sum-check ---------------------------------------------------------------
def sumcheck_chunk(evaluations, rounds: int):
    ev = np.ascontiguousarray(evaluations, dtype=np.uint32)
    n = len(ev)
    fin = np.zeros(n >> rounds, np.uint32)
    total = sum(n >> r for r in range(rounds))
    co = np.zeros(total, np.uint32)
    ch = np.zeros(rounds, np.uint32)
    _check(lib().azko_sumcheck_chunk(_p32(ev), c_u64(n), c_u32(rounds), _p32(fin), _p32(co), _p32(ch)))
    return [int(v) for v in fin], [int(v) for v in co], [int(v) for v in ch]


def sumcheck_multilinear(evaluations):
    ev = np.ascontiguousarray(evaluations, dtype=np.uint32)
    rounds = len(ev).bit_length() - 1
    r0, r1, ch = (np.zeros(rounds, np.uint32) for _ in range(3))
    cs, fe = c_u32(0), c_u32(0)
    dg = np.zeros(32, np.uint8)
    _check(lib().azko_sumcheck_multilinear(_p32(ev), c_u64(len(ev)), _p32(r0), _p32(r1), _p32(ch), ctypes.byref(cs), ctypes.byref(fe), _p8(dg)))
    return {"r0": r0, "r1": r1, "challenges": ch, "claimed_sum": cs.value, "final": fe.value, "initial_digest": dg.tobytes()}
