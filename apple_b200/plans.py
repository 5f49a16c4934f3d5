"""Plan objects mirroring AppleZKProver's Swift plan API over the C ABI.

Names follow the reference (MetalContext -> Context, KeccakF1600PermutationBatchPlan
-> KeccakF1600PermutationPlan, SHA3FixedOneBlockHashPlan, SHA3RawLeavesMerkleCommitPlan,
CircleCodewordPlan, CirclePCSFRIResidentProverV1 -> CirclePCSFRIProver); each call
goes straight to libazk_cuda.so.  Errors raise AZKError carrying the
AppleZKProverError case name.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._capi import AZKError, Schedule, Stats, check, lib

_vp = ctypes.c_void_p


def _ptr(a) -> int:
    return a.ctypes.data if a is not None else None


def _u8(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    return np.frombuffer(bytes(data), dtype=np.uint8)


def _q(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32).reshape(-1, 4))


class Context:
    """One CUDA device (MetalContext.swift:62-112).  Raises AZKError(unavailableOnThisPlatform)
    when no sm_100 device is present."""

    def __init__(self, device: int = 0):
        self._h = _vp()
        check(lib().azk_ctx_create(device, ctypes.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().azk_ctx_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_info(self):
        sm, mem, ma, mi = ctypes.c_int(), ctypes.c_uint64(), ctypes.c_int(), ctypes.c_int()
        check(lib().azk_ctx_device_info(self._h, ctypes.byref(sm), ctypes.byref(mem), ctypes.byref(ma), ctypes.byref(mi)), self._h)
        return {"sm_count": sm.value, "total_bytes": mem.value, "cc": (ma.value, mi.value)}

    def alloc(self, nbytes: int) -> "DeviceBuffer":
        return DeviceBuffer(self, nbytes)

    def synchronize(self):
        check(lib().azk_synchronize(self._h), self._h)


class DeviceBuffer:
    """Device allocation owned by a context (MetalBufferFactory.makePrivateBuffer)."""

    def __init__(self, ctx: Context, nbytes: int):
        self.ctx = ctx
        self.nbytes = int(nbytes)
        self.ptr = _vp()
        check(lib().azk_buf_alloc(ctx.handle, self.nbytes, ctypes.byref(self.ptr)), ctx.handle)

    def upload(self, data, offset: int = 0):
        b = _u8(data)
        check(lib().azk_buf_upload(self.ctx.handle, self.ptr, offset, _ptr(b), b.nbytes), self.ctx.handle)

    def download(self, nbytes: int | None = None, offset: int = 0) -> bytes:
        n = self.nbytes - offset if nbytes is None else nbytes
        out = np.empty(n, np.uint8)
        check(lib().azk_buf_download(self.ctx.handle, _ptr(out), self.ptr, offset, n), self.ctx.handle)
        return out.tobytes()

    def zero(self):
        check(lib().azk_buf_zero(self.ctx.handle, self.ptr, self.nbytes), self.ctx.handle)

    def free(self):
        if self.ptr:
            lib().azk_buf_free(self.ctx.handle, self.ptr)
            self.ptr = _vp()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class _Plan:
    _destroy = None

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self._h = _vp()
        self.last_stats = Stats()

    def close(self):
        if self._h and self._destroy:
            getattr(lib(), self._destroy)(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        check(rc, self.ctx.handle)


class KeccakF1600PermutationPlan(_Plan):
    """KeccakF1600PermutationBatchPlan (KeccakF1600PermutationBatcher.swift:73-294)."""

    _destroy = "azk_keccakf_plan_destroy"

    def __init__(self, ctx: Context, count: int, input_stride: int = 200, output_stride: int = 200, threads: int = 0):
        super().__init__(ctx)
        self.count, self.input_stride, self.output_stride = count, input_stride, output_stride
        self._check(lib().azk_keccakf_plan_create(ctx.handle, count, input_stride, output_stride, threads, ctypes.byref(self._h)))

    def permute(self, states) -> bytes:
        b = _u8(states)
        if b.nbytes < self.count * self.input_stride:
            raise AZKError(1, "state bytes shorter than count * inputStride")
        out = np.empty(self.count * self.output_stride, np.uint8)
        self._check(lib().azk_keccakf_plan_permute(self._h, _ptr(b), _ptr(out), ctypes.byref(self.last_stats)))
        return out.tobytes()

    def permute_resident(self, dev_in, dev_out, in_offset=0, out_offset=0) -> Stats:
        st = Stats()
        self._check(lib().azk_keccakf_plan_permute_resident(self._h, dev_in, in_offset, dev_out, out_offset, ctypes.byref(st)))
        return st

    def clear_reusable_buffers(self):
        self._check(lib().azk_keccakf_plan_clear(self._h))


class SHA3FixedOneBlockHashPlan(_Plan):
    """SHA3FixedOneBlockHashPlan (SHA3BatchHasher.swift:81-264); keccak=True gives the
    Keccak-256 twin (Keccak256BatchHasher.swift)."""

    _destroy = "azk_hash_plan_destroy"

    def __init__(self, ctx: Context, count: int, message_stride: int, message_length: int, output_stride: int = 32, keccak: bool = False,
                 threads: int = 0):
        super().__init__(ctx)
        self.count, self.message_stride, self.message_length, self.output_stride = count, message_stride, message_length, output_stride
        suffix = 0x01 if keccak else 0x06
        self._check(lib().azk_hash_plan_create(ctx.handle, count, message_stride, message_length, output_stride, suffix, threads,
                                               ctypes.byref(self._h)))

    def hash(self, messages) -> bytes:
        b = _u8(messages) if self.count * self.message_stride else np.zeros(1, np.uint8)
        if self.count * self.message_stride and b.nbytes < self.count * self.message_stride:
            raise AZKError(1, "message bytes shorter than count * messageStride")
        out = np.empty(self.count * self.output_stride, np.uint8)
        self._check(lib().azk_hash_plan_hash(self._h, _ptr(b), _ptr(out), ctypes.byref(self.last_stats)))
        return out.tobytes()

    def hash_resident(self, dev_in, dev_out, in_offset=0, out_offset=0) -> Stats:
        st = Stats()
        self._check(lib().azk_hash_plan_hash_resident(self._h, dev_in, in_offset, dev_out, out_offset, ctypes.byref(st)))
        return st

    def clear_reusable_buffers(self):
        self._check(lib().azk_hash_plan_clear(self._h))


class SHA3RawLeavesMerkleCommitPlan(_Plan):
    """SHA3RawLeavesMerkleCommitPlan (MerkleCommitter.swift:526-1182).  treelet_log 0 = automatic."""

    _destroy = "azk_merkle_plan_destroy"

    def __init__(self, ctx: Context, leaf_count: int, leaf_stride: int, leaf_length: int, treelet_log: int = 0):
        super().__init__(ctx)
        self.leaf_count, self.leaf_stride, self.leaf_length = leaf_count, leaf_stride, leaf_length
        self._check(lib().azk_merkle_plan_create(ctx.handle, leaf_count, leaf_stride, leaf_length, treelet_log, ctypes.byref(self._h)))
        d, t = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(lib().azk_merkle_plan_info(self._h, ctypes.byref(d), ctypes.byref(t)))
        self.tree_depth, self.treelet_leaf_count = d.value, t.value

    def _leaves(self, leaves):
        need = self.leaf_count * self.leaf_stride
        if need == 0:
            return np.zeros(1, np.uint8)
        b = _u8(leaves)
        if b.nbytes < need:
            raise AZKError(1, "leaf bytes shorter than leafCount * leafStride")
        return b

    def commit(self, leaves) -> bytes:
        b = self._leaves(leaves)
        root = np.empty(32, np.uint8)
        self._check(lib().azk_merkle_plan_commit(self._h, _ptr(b), _ptr(root), ctypes.byref(self.last_stats)))
        return root.tobytes()

    def commit_resident(self, dev_leaves, offset: int = 0) -> bytes:
        root = np.empty(32, np.uint8)
        self._check(lib().azk_merkle_plan_commit_resident(self._h, dev_leaves, offset, _ptr(root), ctypes.byref(self.last_stats)))
        return root.tobytes()

    def open_raw_leaf(self, leaves, leaf_index: int):
        """Returns (leaf bytes, sibling digests bottom-up, root)."""
        b = self._leaves(leaves)
        leaf = np.zeros(max(1, self.leaf_length), np.uint8)
        sib = np.zeros(max(1, self.tree_depth * 32), np.uint8)
        root = np.empty(32, np.uint8)
        self._check(lib().azk_merkle_plan_open(self._h, _ptr(b), leaf_index, _ptr(leaf), _ptr(sib), _ptr(root), ctypes.byref(self.last_stats)))
        return leaf[: self.leaf_length].tobytes(), [sib[32 * l:32 * l + 32].tobytes() for l in range(self.tree_depth)], root.tobytes()

    def open_resident(self, indices):
        """Sibling paths of several leaves of the last committed tree (no recomputation)."""
        idx = np.ascontiguousarray(indices, dtype=np.uint64)
        sib = np.zeros(max(1, len(idx) * self.tree_depth * 32), np.uint8)
        self._check(lib().azk_merkle_plan_open_resident(self._h, _ptr(idx), len(idx), _ptr(sib), ctypes.byref(self.last_stats)))
        d = self.tree_depth
        return [[sib[(k * d + l) * 32:(k * d + l + 1) * 32].tobytes() for l in range(d)] for k in range(len(idx))]

    def clear_reusable_buffers(self):
        self._check(lib().azk_merkle_plan_clear(self._h))


def commit_prehashed_leaves(ctx: Context, digests) -> bytes:
    """SHA3MerkleCommitter.commitPrehashedLeaves (MerkleCommitter.swift:225-304)."""
    b = _u8(digests)
    root = np.empty(32, np.uint8)
    check(lib().azk_merkle_commit_prehashed(ctx.handle, _ptr(b) if b.nbytes else None, b.nbytes, _ptr(root), None), ctx.handle)
    return root.tobytes()


def circle_domain_points(ctx: Context, log_size: int) -> np.ndarray:
    out = np.empty((1 << log_size, 2), np.uint32)
    check(lib().azk_circle_domain_points(ctx.handle, log_size, _ptr(out)), ctx.handle)
    return out


def circle_fft_twiddles(ctx: Context, log_size: int) -> np.ndarray:
    out = np.empty(max(1, (1 << log_size) - 1), np.uint32)
    check(lib().azk_circle_fft_twiddles(ctx.handle, log_size, _ptr(out)), ctx.handle)
    return out[: (1 << log_size) - 1]


def circle_inverse_layers(ctx: Context, log_size: int, rounds: int) -> list:
    n = 1 << log_size
    out = np.empty(max(1, n - (n >> rounds)), np.uint32)
    check(lib().azk_circle_inverse_layers(ctx.handle, log_size, rounds, _ptr(out)), ctx.handle)
    layers, off = [], 0
    for r in range(rounds):
        m = n >> (r + 1)
        layers.append(out[off:off + m].copy())
        off += m
    return layers


class CircleCodewordPlan(_Plan):
    """CircleCodewordPlan (CircleCodeword.swift:411-887)."""

    _destroy = "azk_codeword_plan_destroy"

    def __init__(self, ctx: Context, log_size: int):
        super().__init__(ctx)
        self.log_size = log_size
        self._check(lib().azk_codeword_plan_create(ctx.handle, log_size, ctypes.byref(self._h)))

    def execute_coefficients(self, coefficients) -> np.ndarray:
        c = _q(coefficients)
        out = np.empty((1 << self.log_size, 4), np.uint32)
        self._check(lib().azk_codeword_plan_execute(self._h, _ptr(c), len(c), _ptr(out), ctypes.byref(self.last_stats)))
        return out

    def execute(self, x_coefficients, y_coefficients=()) -> np.ndarray:
        x = _q(x_coefficients) if len(x_coefficients) else np.zeros((1, 4), np.uint32)
        y = _q(y_coefficients) if len(y_coefficients) else np.zeros((1, 4), np.uint32)
        out = np.empty((1 << self.log_size, 4), np.uint32)
        self._check(lib().azk_codeword_plan_execute_polynomial(self._h, _ptr(x), len(x_coefficients), _ptr(y), len(y_coefficients), _ptr(out),
                                                               ctypes.byref(self.last_stats)))
        return out

    def execute_resident(self, dev_in, dev_out, in_offset=0, out_offset=0) -> Stats:
        st = Stats()
        self._check(lib().azk_codeword_plan_execute_resident(self._h, dev_in, in_offset, dev_out, out_offset, ctypes.byref(st)))
        return st


class CircleWitnessToFFTBasisPlan(_Plan):
    """CircleWitnessToFFTBasisPlanV1 (CircleWitnessFFTBasis.swift:226-590): monomial
    witness columns -> interleaved Circle FFT-basis coefficients, on the device."""

    _destroy = "azk_witness_plan_destroy"

    def __init__(self, ctx: Context, log_size: int):
        super().__init__(ctx)
        self.log_size = log_size
        self._check(lib().azk_witness_plan_create(ctx.handle, log_size, ctypes.byref(self._h)))

    def execute(self, x_coefficients, y_coefficients=()) -> np.ndarray:
        x = _q(x_coefficients) if len(x_coefficients) else np.zeros((0, 4), np.uint32)
        y = _q(y_coefficients) if len(y_coefficients) else np.zeros((0, 4), np.uint32)
        out = np.empty((1 << self.log_size, 4), np.uint32)
        st = Stats()
        self._check(lib().azk_witness_plan_execute(self._h, _ptr(x) if len(x) else None, len(x), _ptr(y) if len(y) else None, len(y), _ptr(out),
                                                   ctypes.byref(st)))
        self.last_stats = st
        return out

    def execute_resident(self, dev_x, x_count, dev_y, y_count, dev_out, x_offset=0, y_offset=0, out_offset=0) -> Stats:
        st = Stats()
        self._check(lib().azk_witness_plan_execute_resident(self._h, dev_x, x_offset, x_count, dev_y, y_offset, y_count, dev_out, out_offset,
                                                            ctypes.byref(st)))
        return st


def qm31_fold(ctx: Context, evaluations, inverse_points, challenge) -> np.ndarray:
    """QM31FRIFoldPlan.execute (QM31FRIFold.swift:960-1117)."""
    ev, inv, ch = _q(evaluations), _q(inverse_points), _q(challenge)
    out = np.empty((len(ev) // 2, 4), np.uint32)
    check(lib().azk_qm31_fold(ctx.handle, _ptr(ev), len(ev), _ptr(inv), _ptr(ch), _ptr(out), None), ctx.handle)
    return out


def circle_fold_chain(ctx: Context, log_size: int, evaluations, challenges) -> np.ndarray:
    """CircleFRIFoldChainPlan.execute (CircleFRIFoldPlan.swift:132-280)."""
    ev, ch = _q(evaluations), _q(challenges)
    out = np.empty(((1 << log_size) >> len(ch), 4), np.uint32)
    check(lib().azk_circle_fold_chain(ctx.handle, log_size, _ptr(ev), _ptr(ch), len(ch), _ptr(out), None), ctx.handle)
    return out


def qm31_merkle_fold_chain(ctx: Context, evaluations, inverse_layers):
    """QM31FRIFoldChainPlan Merkle-transcript mode: (final layer, commitments, challenges)."""
    ev = _q(evaluations)
    inv = np.concatenate([_q(l) for l in inverse_layers])
    r = len(inverse_layers)
    fin = np.empty((len(ev) >> r, 4), np.uint32)
    cm = np.empty(32 * r, np.uint8)
    ch = np.empty((r, 4), np.uint32)
    check(lib().azk_qm31_merkle_fold_chain(ctx.handle, _ptr(ev), len(ev), _ptr(inv), r, _ptr(fin), _ptr(cm), _ptr(ch), None), ctx.handle)
    return fin, [cm[32 * k:32 * k + 32].tobytes() for k in range(r)], ch


def qm31_transcript_challenges(ctx: Context, input_count: int, commitments) -> np.ndarray:
    cm = _u8(b"".join(commitments))
    out = np.empty((len(commitments), 4), np.uint32)
    check(lib().azk_qm31_transcript_challenges(ctx.handle, input_count, _ptr(cm), len(commitments), _ptr(out)), ctx.handle)
    return out


def circle_merkle_fold_chain(ctx: Context, log_size: int, evaluations, log_blowup: int, queries: int, public_digest: bytes, rounds: int,
                             grinding_bits: int = 0):
    """CircleFRIMerkleTranscriptFoldChainPlan (CircleFRIFoldPlan.swift:301-518)."""
    ev = _q(evaluations)
    pub = _u8(public_digest)
    fin = np.empty(((1 << log_size) >> rounds, 4), np.uint32)
    cm = np.empty(32 * rounds, np.uint8)
    ch = np.empty((rounds, 4), np.uint32)
    check(lib().azk_circle_merkle_fold_chain(ctx.handle, log_size, _ptr(ev), log_blowup, queries, grinding_bits, _ptr(pub), rounds, _ptr(fin),
                                             _ptr(cm), _ptr(ch), None), ctx.handle)
    return fin, [cm[32 * k:32 * k + 32].tobytes() for k in range(rounds)], ch


class QM31FRIFoldPlan(_Plan):
    """QM31FRIFoldPlan (QM31FRIFold.swift:960-1338): one fold of `input_count` values."""

    _destroy = "azk_qm31_fold_plan_destroy"

    def __init__(self, ctx: Context, input_count: int):
        super().__init__(ctx)
        self.input_count, self.output_count = input_count, input_count // 2
        self._check(lib().azk_qm31_fold_plan_create(ctx.handle, input_count, ctypes.byref(self._h)))

    def execute(self, evaluations, inverse_points, challenge) -> np.ndarray:
        ev, inv, ch = _q(evaluations), _q(inverse_points), _q(challenge)
        if len(ev) != self.input_count or len(inv) != self.output_count or len(ch) != 1:
            raise AZKError(1, "evaluations / inverse points do not match the plan's counts")
        out = np.empty((self.output_count, 4), np.uint32)
        self._check(lib().azk_qm31_fold_plan_execute(self._h, _ptr(ev), _ptr(inv), _ptr(ch), _ptr(out), ctypes.byref(self.last_stats)))
        return out

    def execute_resident(self, dev_evaluations, dev_inverse_points, dev_out, challenge, evaluations_offset=0, inverse_offset=0, out_offset=0) -> Stats:
        ch = _q(challenge)
        st = Stats()
        self._check(lib().azk_qm31_fold_plan_execute_resident(self._h, dev_evaluations, evaluations_offset, dev_inverse_points, inverse_offset, dev_out,
                                                              out_offset, _ptr(ch), ctypes.byref(st)))
        return st

    def clear_reusable_buffers(self):
        self._check(lib().azk_qm31_fold_plan_clear(self._h))


class QM31FRIFoldChainPlan(_Plan):
    """QM31FRIFoldChainPlan (QM31FRIFold.swift:1359-2931): `round_count` folds with
    explicit challenges, transcript-derived challenges from given commitments, or
    Merkle-bound commitments and challenges; host and resident forms."""

    _destroy = "azk_fold_chain_plan_destroy"

    def __init__(self, ctx: Context, input_count: int, round_count: int):
        super().__init__(ctx)
        self.input_count, self.round_count = input_count, round_count
        self._check(lib().azk_fold_chain_plan_create(ctx.handle, input_count, round_count, ctypes.byref(self._h)))
        o, i, l = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._check(lib().azk_fold_chain_plan_info(self._h, ctypes.byref(o), ctypes.byref(i), ctypes.byref(l)))
        self.output_count, self.total_inverse_domain_count, self.layer_log_count = o.value, i.value, l.value

    def _inputs(self, evaluations, inverse_layers):
        ev = _q(evaluations)
        inv = np.concatenate([_q(l) for l in inverse_layers]) if len(inverse_layers) else np.zeros((0, 4), np.uint32)
        if len(ev) != self.input_count or len(inverse_layers) != self.round_count or len(inv) != self.total_inverse_domain_count:
            raise AZKError(1, "evaluations / inverse-domain layers do not match the plan's counts")
        return ev, np.ascontiguousarray(inv)

    def execute(self, evaluations, inverse_layers, challenges) -> np.ndarray:
        ev, inv = self._inputs(evaluations, inverse_layers)
        ch = _q(challenges)
        if len(ch) != self.round_count:
            raise AZKError(1, "one challenge per round")
        out = np.empty((self.output_count, 4), np.uint32)
        self._check(lib().azk_fold_chain_plan_execute(self._h, _ptr(ev), _ptr(inv), _ptr(ch), _ptr(out), ctypes.byref(self.last_stats)))
        return out

    def execute_resident(self, dev_evaluations, dev_inverse_layers, dev_final, challenges, evaluations_offset=0, inverse_offset=0,
                         final_offset=0) -> Stats:
        ch = _q(challenges)
        st = Stats()
        self._check(lib().azk_fold_chain_plan_execute_resident(self._h, dev_evaluations, evaluations_offset, dev_inverse_layers, inverse_offset,
                                                               dev_final, final_offset, _ptr(ch), ctypes.byref(st)))
        return st

    def execute_transcript_derived(self, evaluations, inverse_layers, commitments):
        """Returns (final layer, challenges)."""
        ev, inv = self._inputs(evaluations, inverse_layers)
        cm = _u8(b"".join(commitments))
        if len(commitments) != self.round_count or any(len(c) != 32 for c in commitments):
            raise AZKError(1, "one 32-byte commitment per round")
        out = np.empty((self.output_count, 4), np.uint32)
        ch = np.empty((self.round_count, 4), np.uint32)
        self._check(lib().azk_fold_chain_plan_execute_transcript(self._h, _ptr(ev), _ptr(inv), _ptr(cm), _ptr(out), _ptr(ch),
                                                                 ctypes.byref(self.last_stats)))
        return out, ch

    def execute_transcript_derived_resident(self, dev_evaluations, dev_inverse_layers, dev_commitments, dev_final, commitment_stride=32,
                                            evaluations_offset=0, inverse_offset=0, commitments_offset=0, final_offset=0) -> Stats:
        st = Stats()
        self._check(lib().azk_fold_chain_plan_execute_transcript_resident(self._h, dev_evaluations, evaluations_offset, dev_inverse_layers, inverse_offset,
                                                                          dev_commitments, commitments_offset, commitment_stride, dev_final,
                                                                          final_offset, ctypes.byref(st)))
        return st

    def _merkle_out(self):
        return (np.empty((self.output_count, 4), np.uint32), np.empty(32 * self.round_count, np.uint8),
                np.empty((self.round_count, 4), np.uint32))

    def _split(self, cm):
        return [cm[32 * k:32 * k + 32].tobytes() for k in range(self.round_count)]

    def execute_merkle_transcript_derived(self, evaluations, inverse_layers):
        """Returns (final layer, commitments, challenges)."""
        ev, inv = self._inputs(evaluations, inverse_layers)
        out, cm, ch = self._merkle_out()
        self._check(lib().azk_fold_chain_plan_execute_merkle(self._h, _ptr(ev), _ptr(inv), _ptr(out), _ptr(cm), _ptr(ch), ctypes.byref(self.last_stats)))
        return out, self._split(cm), ch

    def execute_merkle_transcript_derived_readback(self, dev_evaluations, dev_inverse_layers, evaluations_offset=0, inverse_offset=0):
        out, cm, ch = self._merkle_out()
        self._check(lib().azk_fold_chain_plan_execute_merkle_readback(self._h, dev_evaluations, evaluations_offset, dev_inverse_layers, inverse_offset,
                                                                      _ptr(out), _ptr(cm), _ptr(ch), ctypes.byref(self.last_stats)))
        return out, self._split(cm), ch

    def execute_merkle_transcript_derived_resident(self, dev_evaluations, dev_inverse_layers, dev_commitments, dev_final, dev_layer_log=None,
                                                   dev_first_commitment=None, commitment_stride=32, evaluations_offset=0, inverse_offset=0,
                                                   commitments_offset=0, layer_log_offset=0, first_commitment_offset=0, final_offset=0) -> Stats:
        st = Stats()
        self._check(lib().azk_fold_chain_plan_execute_merkle_resident(self._h, dev_evaluations, evaluations_offset, dev_inverse_layers, inverse_offset,
                                                                      dev_commitments, commitments_offset, commitment_stride, dev_layer_log,
                                                                      layer_log_offset, dev_first_commitment, first_commitment_offset, dev_final,
                                                                      final_offset, ctypes.byref(st)))
        return st

    def challenges(self) -> np.ndarray:
        ch = np.empty((self.round_count, 4), np.uint32)
        self._check(lib().azk_fold_chain_plan_challenges(self._h, _ptr(ch)))
        return ch

    def clear_reusable_buffers(self):
        self._check(lib().azk_fold_chain_plan_clear(self._h))


class SHA3PrehashedLeavesMerkleCommitPlan(_Plan):
    """SHA3PrehashedLeavesMerkleCommitPlan (MerkleCommitter.swift:314-524): the Merkle
    root over `leaf_count` 32-byte leaf digests."""

    _destroy = "azk_merkle_prehashed_plan_destroy"

    def __init__(self, ctx: Context, leaf_count: int):
        super().__init__(ctx)
        self.leaf_count = leaf_count
        self._check(lib().azk_merkle_prehashed_plan_create(ctx.handle, leaf_count, ctypes.byref(self._h)))

    def commit(self, digests) -> bytes:
        d = _u8(digests)
        if d.nbytes != 32 * self.leaf_count:
            raise AZKError(1, "32 bytes per leaf digest")
        root = np.empty(32, np.uint8)
        self._check(lib().azk_merkle_prehashed_plan_commit(self._h, _ptr(d), _ptr(root), ctypes.byref(self.last_stats)))
        return root.tobytes()

    def commit_resident(self, dev_digests, offset: int = 0) -> bytes:
        root = np.empty(32, np.uint8)
        self._check(lib().azk_merkle_prehashed_plan_commit_resident(self._h, dev_digests, offset, _ptr(root), ctypes.byref(self.last_stats)))
        return root.tobytes()


class CircleDomainMaterializationPlan(_Plan):
    """CircleDomainMaterializationPlan (CircleDomainMaterializationPlan.swift:52-219):
    domain points, FFT twiddles and QM31 inverse-domain layers built once on the
    device, with their device addresses and read-back accessors."""

    _destroy = "azk_domain_plan_destroy"

    def __init__(self, ctx: Context, log_size: int, materialize_points: bool = False, materialize_twiddles: bool = False,
                 inverse_round_count: int = 0):
        super().__init__(ctx)
        self.log_size, self.inverse_round_count = log_size, inverse_round_count
        self._check(lib().azk_domain_plan_create(ctx.handle, log_size, int(materialize_points), int(materialize_twiddles), inverse_round_count,
                                                 ctypes.byref(self._h)))
        tw, inv, out = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self.materialization_stats = Stats()
        self._check(lib().azk_domain_plan_info(self._h, ctypes.byref(tw), ctypes.byref(inv), ctypes.byref(out), ctypes.byref(self.materialization_stats)))
        self.codeword_twiddle_count, self.total_inverse_domain_count, self.output_count = tw.value, inv.value, out.value
        self.inverse_domain_layer_counts = [(1 << log_size) >> (k + 1) for k in range(inverse_round_count)]

    def buffers(self):
        """(points, twiddles, inverse layers) device addresses; None where not built."""
        a, b, c = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        self._check(lib().azk_domain_plan_buffers(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def read_domain_points(self) -> np.ndarray:
        out = np.empty((1 << self.log_size, 2), np.uint32)
        self._check(lib().azk_domain_plan_read_points(self._h, _ptr(out)))
        return out

    def read_codeword_twiddles(self) -> np.ndarray:
        out = np.empty(self.codeword_twiddle_count, np.uint32)
        self._check(lib().azk_domain_plan_read_twiddles(self._h, _ptr(out)))
        return out

    def read_inverse_domain_layers(self):
        flat = np.empty((max(1, self.total_inverse_domain_count), 4), np.uint32)
        self._check(lib().azk_domain_plan_read_inverse_layers(self._h, _ptr(flat)))
        out, off = [], 0
        for c in self.inverse_domain_layer_counts:
            out.append(flat[off:off + c])
            off += c
        return out


class CircleFRIFoldPlan(_Plan):
    """CircleFRIFoldPlan (CircleFRIFoldPlan.swift:5-130): the circle -> line fold of
    a canonical domain's evaluations, inverse y twiddles materialised by the plan."""

    _destroy = "azk_circle_fold_plan_destroy"

    def __init__(self, ctx: Context, log_size: int):
        super().__init__(ctx)
        self.log_size, self.input_count, self.output_count = log_size, 1 << log_size, 1 << (log_size - 1)
        self._check(lib().azk_circle_fold_plan_create(ctx.handle, log_size, ctypes.byref(self._h)))

    def execute(self, evaluations, challenge) -> np.ndarray:
        ev, ch = _q(evaluations), _q(challenge)
        if len(ev) != self.input_count or len(ch) != 1:
            raise AZKError(1, "evaluations must cover the domain; one challenge")
        out = np.empty((self.output_count, 4), np.uint32)
        self._check(lib().azk_circle_fold_plan_execute(self._h, _ptr(ev), _ptr(ch), _ptr(out), ctypes.byref(self.last_stats)))
        return out

    def execute_resident(self, dev_evaluations, dev_out, challenge, evaluations_offset=0, out_offset=0) -> Stats:
        ch = _q(challenge)
        st = Stats()
        self._check(lib().azk_circle_fold_plan_execute_resident(self._h, dev_evaluations, evaluations_offset, dev_out, out_offset, _ptr(ch),
                                                                ctypes.byref(st)))
        return st

    def read_inverse_y_twiddles(self) -> np.ndarray:
        out = np.empty((self.output_count, 4), np.uint32)
        self._check(lib().azk_circle_fold_plan_read_inverse(self._h, _ptr(out)))
        return out

    def clear_reusable_buffers(self):
        self._check(lib().azk_circle_fold_plan_clear(self._h))


class CircleFRIFoldChainPlan(_Plan):
    """CircleFRIFoldChainPlan (CircleFRIFoldPlan.swift:132-280): `round_count` folds of
    a canonical domain's evaluations with explicit challenges."""

    _destroy = "azk_circle_fold_chain_plan_destroy"

    def __init__(self, ctx: Context, log_size: int, round_count: int):
        super().__init__(ctx)
        self.log_size, self.round_count = log_size, round_count
        self.input_count, self.output_count = 1 << log_size, (1 << log_size) >> round_count
        self._check(lib().azk_circle_fold_chain_plan_create(ctx.handle, log_size, round_count, ctypes.byref(self._h)))

    def execute(self, evaluations, challenges) -> np.ndarray:
        ev, ch = _q(evaluations), _q(challenges)
        if len(ev) != self.input_count or len(ch) != self.round_count:
            raise AZKError(1, "evaluations must cover the domain; one challenge per round")
        out = np.empty((self.output_count, 4), np.uint32)
        self._check(lib().azk_circle_fold_chain_plan_execute(self._h, _ptr(ev), _ptr(ch), _ptr(out), ctypes.byref(self.last_stats)))
        return out

    def execute_resident(self, dev_evaluations, dev_final, challenges, evaluations_offset=0, final_offset=0) -> Stats:
        ch = _q(challenges)
        st = Stats()
        self._check(lib().azk_circle_fold_chain_plan_execute_resident(self._h, dev_evaluations, evaluations_offset, dev_final, final_offset, _ptr(ch),
                                                                      ctypes.byref(st)))
        return st

    def read_inverse_domain_layers(self):
        flat = np.empty(((1 << self.log_size) - self.output_count, 4), np.uint32)
        self._check(lib().azk_circle_fold_chain_plan_read_inverse_layers(self._h, _ptr(flat)))
        out, off = [], 0
        for k in range(self.round_count):
            c = (1 << self.log_size) >> (k + 1)
            out.append(flat[off:off + c])
            off += c
        return out

    def clear_reusable_buffers(self):
        self._check(lib().azk_circle_fold_chain_plan_clear(self._h))


class CircleFRIMerkleTranscriptFoldChainPlan(_Plan):
    """CircleFRIMerkleTranscriptFoldChainPlan (CircleFRIFoldPlan.swift:301-518): every
    round's layer committed as a SHA3 Merkle tree and its challenge drawn from the
    Circle PCS V1 transcript (domain, security parameters, public digest)."""

    _destroy = "azk_circle_merkle_chain_plan_destroy"

    def __init__(self, ctx: Context, log_size: int, log_blowup: int, queries: int, public_digest: bytes, round_count: int, grinding_bits: int = 0):
        super().__init__(ctx)
        if len(public_digest) != 32:
            raise AZKError(1, "the public-input digest is 32 bytes")
        self.log_size, self.round_count, self.input_count = log_size, round_count, 1 << log_size
        pub = _u8(public_digest)
        self._check(lib().azk_circle_merkle_chain_plan_create(ctx.handle, log_size, log_blowup, queries, grinding_bits, _ptr(pub), round_count,
                                                              ctypes.byref(self._h)))
        o, l = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(lib().azk_circle_merkle_chain_plan_info(self._h, ctypes.byref(o), ctypes.byref(l)))
        self.output_count, self.total_committed_layer_count = o.value, l.value
        self.committed_layer_counts = [(1 << log_size) >> k for k in range(round_count)]

    def execute(self, evaluations):
        """Returns (final layer, commitments, challenges)."""
        ev = _q(evaluations)
        if len(ev) != self.input_count:
            raise AZKError(1, "evaluations must cover the domain")
        out = np.empty((self.output_count, 4), np.uint32)
        cm = np.empty(32 * self.round_count, np.uint8)
        ch = np.empty((self.round_count, 4), np.uint32)
        self._check(lib().azk_circle_merkle_chain_plan_execute(self._h, _ptr(ev), _ptr(out), _ptr(cm), _ptr(ch), ctypes.byref(self.last_stats)))
        return out, [cm[32 * k:32 * k + 32].tobytes() for k in range(self.round_count)], ch

    def execute_resident(self, dev_evaluations, dev_commitments, dev_final, dev_committed_layers=None, dev_first_commitment=None, commitment_stride=32,
                         evaluations_offset=0, committed_layers_offset=0, commitments_offset=0, first_commitment_offset=0, final_offset=0) -> Stats:
        """executeResident, executeMaterializedResident (with `dev_committed_layers`) and
        ...WithPrecomputedFirstCommitment (with `dev_first_commitment` as well)."""
        st = Stats()
        self._check(lib().azk_circle_merkle_chain_plan_execute_resident(self._h, dev_evaluations, evaluations_offset, dev_committed_layers,
                                                                        committed_layers_offset, dev_commitments, commitments_offset, commitment_stride,
                                                                        dev_first_commitment, first_commitment_offset, dev_final, final_offset,
                                                                        ctypes.byref(st)))
        return st

    def challenges(self) -> np.ndarray:
        ch = np.empty((self.round_count, 4), np.uint32)
        self._check(lib().azk_circle_merkle_chain_plan_challenges(self._h, _ptr(ch)))
        return ch

    def read_inverse_domain_layers(self):
        flat = np.empty(((1 << self.log_size) - self.output_count, 4), np.uint32)
        self._check(lib().azk_circle_merkle_chain_plan_read_inverse_layers(self._h, _ptr(flat)))
        out, off = [], 0
        for k in range(self.round_count):
            c = (1 << self.log_size) >> (k + 1)
            out.append(flat[off:off + c])
            off += c
        return out

    def clear_reusable_buffers(self):
        self._check(lib().azk_circle_merkle_chain_plan_clear(self._h))


class CircleFRIResidentQueryExtractor(_Plan):
    """CircleFRIResidentQueryExtractorV1 (CircleFRIFoldPlan.swift:1027-1231): query
    openings from committed layers on the device, in the proof codec's encoding."""

    _destroy = "azk_query_extractor_destroy"

    def __init__(self, ctx: Context, log_size: int, round_count: int):
        super().__init__(ctx)
        self.log_size, self.round_count = log_size, round_count
        self.query_bytes = int(lib().azk_query_extractor_query_bytes(log_size, round_count))
        self._check(lib().azk_query_extractor_create(ctx.handle, log_size, round_count, ctypes.byref(self._h)))

    def extract_queries(self, dev_layers, commitments, query_pair_indices, layers_offset=0) -> bytes:
        cm = _u8(b"".join(commitments))
        if len(commitments) != self.round_count or any(len(c) != 32 for c in commitments):
            raise AZKError(1, "one 32-byte commitment per round")
        idx = np.ascontiguousarray(query_pair_indices, dtype=np.uint64)
        out = np.empty(max(1, len(idx) * self.query_bytes), np.uint8)
        n = ctypes.c_uint64(out.nbytes)
        self._check(lib().azk_query_extractor_extract(self._h, dev_layers, layers_offset, _ptr(cm), _ptr(idx), len(idx), _ptr(out), ctypes.byref(n),
                                                      ctypes.byref(self.last_stats)))
        return out[: n.value].tobytes()


def probe_int_issue(ctx: Context) -> float:
    """Sustained LOP3+SHF 32-bit op rate of the device (ops/s)."""
    v = ctypes.c_double()
    check(lib().azk_probe_int_issue(ctx.handle, ctypes.byref(v)), ctx.handle)
    return v.value


def pcs_proof_size(log_size, rounds, queries, claimed=0, grinding_bits=0) -> int:
    return int(lib().azk_pcs_proof_size(log_size, rounds, queries, claimed, grinding_bits))


def _sched(schedule):
    if schedule is None:
        return None
    if isinstance(schedule, Schedule):
        return ctypes.byref(schedule)
    s = Schedule(schedule.get("treelet_log", 0), schedule.get("group_log", 0), schedule.get("threads", 0), schedule.get("use_graph", 1))
    for lg, tl in dict(schedule.get("layer_treelet", {})).items():
        s.layer_treelet[int(lg)] = int(tl)
    for lg, th in dict(schedule.get("layer_threads", {})).items():
        s.layer_threads[int(lg)] = int(th)
    s.persistent_trees = int(schedule.get("persistent_trees", 0))
    _keep.append(s)
    return ctypes.byref(s)


_keep = []  # Schedule structs passed by reference stay alive until the call returns


class CirclePCSFRIProver(_Plan):
    """CirclePCSFRIResidentProverV1 + CircleCodewordPCSFRIProverV1: evaluations or FFT-basis
    coefficients -> CirclePCSFRIProofCodecV1 bytes, all on the device."""

    _destroy = "azk_pcs_prover_destroy"

    def __init__(self, ctx: Context, log_size: int, log_blowup: int, queries: int, rounds: int, grinding_bits: int = 0, schedule=None):
        super().__init__(ctx)
        self.log_size, self.log_blowup, self.queries, self.rounds, self.grinding_bits = log_size, log_blowup, queries, rounds, grinding_bits
        self._check(lib().azk_pcs_prover_create(ctx.handle, log_size, log_blowup, queries, grinding_bits, rounds, _sched(schedule),
                                                ctypes.byref(self._h)))

    def _buf(self, claimed=0):
        n = pcs_proof_size(self.log_size, self.rounds, self.queries, claimed, self.grinding_bits)
        return np.empty(n, np.uint8), ctypes.c_uint64(n)

    def prove_evaluations(self, evaluations, public_digest: bytes, claimed_indices=()) -> bytes:
        ev, pub = _q(evaluations), _u8(public_digest)
        cl = np.ascontiguousarray(list(claimed_indices) or [0], dtype=np.uint64)
        out, n = self._buf(len(claimed_indices))
        self._check(lib().azk_pcs_prover_prove_evaluations(self._h, _ptr(ev), _ptr(pub), _ptr(cl), len(claimed_indices), _ptr(out), ctypes.byref(n),
                                                           ctypes.byref(self.last_stats)))
        return out[: n.value].tobytes()

    def prove_coefficients(self, coefficients, public_digest: bytes) -> bytes:
        c, pub = _q(coefficients), _u8(public_digest)
        out, n = self._buf()
        self._check(lib().azk_pcs_prover_prove_coefficients(self._h, _ptr(c), len(c), _ptr(pub), _ptr(out), ctypes.byref(n),
                                                            ctypes.byref(self.last_stats)))
        return out[: n.value].tobytes()

    def prove_resident(self, dev_input, public_digest: bytes, dev_proof, input_is_coefficients=True, in_offset=0) -> int:
        pub = _u8(public_digest)
        n = ctypes.c_uint64(pcs_proof_size(self.log_size, self.rounds, self.queries, 0, self.grinding_bits))
        self._check(lib().azk_pcs_prover_prove_resident(self._h, dev_input, in_offset, 1 if input_is_coefficients else 0, _ptr(pub), dev_proof,
                                                        ctypes.byref(n), ctypes.byref(self.last_stats)))
        return n.value

    def prove_polynomial(self, x_coefficients, y_coefficients, public_digest: bytes) -> bytes:
        """prove(polynomial:): monomial columns, converted to the FFT basis on the device."""
        x, y, pub = _q(x_coefficients), _q(y_coefficients), _u8(public_digest)
        out, n = self._buf()
        self._check(lib().azk_pcs_prover_prove_polynomial(self._h, _ptr(x) if len(x) else None, len(x), _ptr(y) if len(y) else None, len(y),
                                                          _ptr(pub), _ptr(out), ctypes.byref(n), ctypes.byref(self.last_stats)))
        return out[: n.value].tobytes()

    def prove_resident_witness(self, dev_x, x_count, dev_y, y_count, public_digest: bytes, dev_proof, x_offset=0, y_offset=0) -> int:
        """proveResidentWitnessCoefficients: monomial columns already on the device."""
        pub = _u8(public_digest)
        n = ctypes.c_uint64(pcs_proof_size(self.log_size, self.rounds, self.queries, 0, self.grinding_bits))
        self._check(lib().azk_pcs_prover_prove_resident_witness(self._h, dev_x, x_offset, x_count, dev_y, y_offset, y_count, _ptr(pub), dev_proof,
                                                                ctypes.byref(n), ctypes.byref(self.last_stats)))
        return n.value

    def trace(self):
        """(commitments, challenges, final layer, query pairs) of the last proof."""
        cm = np.empty(32 * self.rounds, np.uint8)
        ch = np.empty((self.rounds, 4), np.uint32)
        fl = np.empty(((1 << self.log_size) >> self.rounds, 4), np.uint32)
        qp = np.empty(self.queries, np.uint32)
        self._check(lib().azk_pcs_prover_trace(self._h, _ptr(cm), _ptr(ch), _ptr(fl), _ptr(qp)))
        return [cm[32 * k:32 * k + 32].tobytes() for k in range(self.rounds)], ch, fl, [int(v) for v in qp]


class BatchProver(_Plan):
    """Batched commit-and-fold superstep over uneven instances (azk_batch_*)."""

    _destroy = "azk_batch_destroy"

    def __init__(self, ctx: Context, log_sizes, rounds, log_blowup: int, queries: int, schedule=None, leaf_bytes: int = 16):
        super().__init__(ctx)
        self.log_sizes = [int(v) for v in log_sizes]
        self.rounds = [int(v) for v in rounds]
        self.queries = queries
        self.leaf_bytes = leaf_bytes
        ls = np.ascontiguousarray(self.log_sizes, dtype=np.uint32)
        rs = np.ascontiguousarray(self.rounds, dtype=np.uint32)
        self._check(lib().azk_batch_create_leaves(ctx.handle, len(ls), _ptr(ls), _ptr(rs), log_blowup, queries, leaf_bytes, _sched(schedule),
                                                  ctypes.byref(self._h)))
        sizes = np.empty(len(ls), np.uint64)
        total = ctypes.c_uint64()
        self._check(lib().azk_batch_proof_sizes(self._h, _ptr(sizes), ctypes.byref(total)))
        self.proof_sizes = [int(v) for v in sizes]
        self.proof_total = total.value

    def upload(self, coefficients_flat, offsets, counts):
        """coefficients_flat: (M, 4) u32; instance i uses rows offsets[i] : offsets[i] + counts[i]."""
        c = _q(coefficients_flat)
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        cnt = np.ascontiguousarray(counts, dtype=np.uint64)
        self._check(lib().azk_batch_upload(self._h, _ptr(c), _ptr(off), _ptr(cnt)))

    def input_pointer(self, index: int) -> int:
        p = _vp()
        self._check(lib().azk_batch_input(self._h, index, ctypes.byref(p)))
        return p.value

    def prove(self, public_digests: bytes, plain: bool = False) -> Stats:
        pub = _u8(public_digests)
        st = Stats()
        self._check(lib().azk_batch_prove(self._h, _ptr(pub), 1 if plain else 0, ctypes.byref(st)))
        self.last_stats = st
        return st

    def proofs(self):
        out = np.empty(max(1, self.proof_total), np.uint8)
        self._check(lib().azk_batch_download_proofs(self._h, _ptr(out), self.proof_total))
        res, pos = [], 0
        for n in self.proof_sizes:
            res.append(out[pos:pos + n].tobytes())
            pos += n
        return res

    def set_profiling(self, enabled: bool = True):
        self._check(lib().azk_batch_set_profiling(self._h, 1 if enabled else 0))

    def profile(self) -> dict:
        sec = np.zeros(4, np.float64)
        self._check(lib().azk_batch_profile(self._h, _ptr(sec)))
        return {"fft_s": float(sec[0]), "tree_s": float(sec[1]), "fold_s": float(sec[2]), "transcript_s": float(sec[3])}

    def work(self) -> dict:
        t, f, d, l = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        self._check(lib().azk_batch_work(self._h, ctypes.byref(t), ctypes.byref(f), ctypes.byref(d), ctypes.byref(l)))
        return {"tree_permutations": t.value, "fft_bytes": f.value, "fold_bytes": d.value, "launches": l.value}

    def trace(self, index: int):
        r, logn = self.rounds[index], self.log_sizes[index]
        cm = np.empty(32 * r, np.uint8)
        ch = np.empty((r, 4), np.uint32)
        fl = np.empty(((1 << logn) >> r, 4), np.uint32)
        qp = np.empty(self.queries, np.uint32)
        self._check(lib().azk_batch_trace(self._h, index, _ptr(cm), _ptr(ch), _ptr(fl), _ptr(qp)))
        return [cm[32 * k:32 * k + 32].tobytes() for k in range(r)], ch, fl, [int(v) for v in qp]


def sumcheck_prove(ctx: Context, evaluations) -> dict:
    """M31MultilinearSumcheckProofBuilderV1.prove (SumcheckOracle.swift:797-868) on the device."""
    ev = np.ascontiguousarray(evaluations, dtype=np.uint32).reshape(-1)
    rounds = max(0, len(ev).bit_length() - 1)
    r0, r1, ch = (np.zeros(max(1, rounds), np.uint32) for _ in range(3))
    cs, fe = ctypes.c_uint32(), ctypes.c_uint32()
    dg = np.zeros(32, np.uint8)
    st = Stats()
    check(lib().azk_sumcheck_prove(ctx.handle, _ptr(ev), len(ev), _ptr(r0), _ptr(r1), _ptr(ch), ctypes.byref(cs), ctypes.byref(fe), _ptr(dg),
                                   ctypes.byref(st)), ctx.handle)
    return {"r0": r0[:rounds], "r1": r1[:rounds], "challenges": ch[:rounds], "claimed_sum": cs.value, "final": fe.value,
            "initial_digest": dg.tobytes(), "gpu_s": st.gpu_s, "wall_s": st.cpu_wall_s}


def _sumcheck_words(words: np.ndarray) -> dict:
    rounds = (len(words) - 10) // 3
    return {"claimed_sum": int(words[0]), "final": int(words[1]), "initial_digest": words[2:10].tobytes(),
            "r0": words[10:10 + rounds], "r1": words[10 + rounds:10 + 2 * rounds], "challenges": words[10 + 2 * rounds:10 + 3 * rounds]}


class ProofServer:
    """Continuous-batching server over one device (azk_server_*).

    Jobs are queued in arrival order and admitted when a worker slot is free and
    their device memory fits the HBM budget; a job larger than the whole budget
    raises AZKError(hbmBudget) at submission.  `poll` returns None while a
    job is queued or running, else (result, latency_seconds): proof bytes for a
    PCS job, a dict like `sumcheck_prove`'s for a sum-check job.

    `copy=False` on a submission hands the array to the server without copying it
    (azk_server_submit_*_nocopy): the server keeps a reference to it until `poll`
    sees the job finished, and the caller must not change it meanwhile."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int, slots: int = 4, schedule=None):
        self.ctx = ctx
        self._h = _vp()
        self._kind = {}
        self._borrowed = {}  # job id -> the array a no-copy submission reads
        self._pollbuf = np.empty(0, np.uint8)
        check(lib().azk_server_create(ctx.handle, int(hbm_budget_bytes), int(slots), _sched(schedule), ctypes.byref(self._h)), ctx.handle)

    def _check(self, rc):
        check(rc, self.ctx.handle)

    def group_stats(self) -> dict:
        g, j = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(lib().azk_server_group_stats(self._h, ctypes.byref(g), ctypes.byref(j)))
        return {"groups": g.value, "grouped_jobs": j.value, "mean_group": j.value / g.value if g.value else 0.0}

    def submit_pcs(self, log_size: int, log_blowup: int, queries: int, rounds: int, coefficients, public_digest: bytes,
                   copy: bool = True) -> int:
        c = _q(coefficients)
        pub = _u8(public_digest)
        jid = ctypes.c_uint64()
        fn = lib().azk_server_submit_pcs if copy else lib().azk_server_submit_pcs_nocopy
        self._check(fn(self._h, log_size, log_blowup, queries, rounds, _ptr(c), len(c), _ptr(pub), ctypes.byref(jid)))
        self._kind[jid.value] = 0
        if not copy:
            self._borrowed[jid.value] = c
        return jid.value

    def warm(self, pcs_shapes=(), log_blowup: int = 2, queries: int = 64, sumcheck_logs=()):
        """Run, on every worker, one job of zeros of each shape before serving:
        `pcs_shapes` = [(log_size, rounds), ...], `sumcheck_logs` = [log2(count), ...].
        Afterwards no real job pays for creating its worker's device memory or
        pinned staging.  Shapes over the HBM budget are skipped."""
        logs = np.array([int(a) for a, _ in pcs_shapes], np.uint32)
        rounds = np.array([int(b) for _, b in pcs_shapes], np.uint32)
        sc = np.array([int(x) for x in sumcheck_logs], np.uint32)
        self._check(lib().azk_server_warm(self._h, _ptr(logs) if len(logs) else None, _ptr(rounds) if len(rounds) else None, len(logs),
                                          log_blowup, queries, _ptr(sc) if len(sc) else None, len(sc)))

    def submit_sumcheck(self, evaluations, copy: bool = True) -> int:
        ev = np.ascontiguousarray(evaluations, dtype=np.uint32).reshape(-1)
        jid = ctypes.c_uint64()
        fn = lib().azk_server_submit_sumcheck if copy else lib().azk_server_submit_sumcheck_nocopy
        self._check(fn(self._h, _ptr(ev), len(ev), ctypes.byref(jid)))
        self._kind[jid.value] = 1
        if not copy:
            self._borrowed[jid.value] = ev
        return jid.value

    def poll(self, job_id: int, release: bool = True):
        st, lat, n = ctypes.c_int(), ctypes.c_double(), ctypes.c_uint64()
        try:
            self._check(lib().azk_server_poll(self._h, job_id, ctypes.byref(st), ctypes.byref(lat), None, ctypes.byref(n)))
        except AZKError:
            self._borrowed.pop(job_id, None)  # a failed job reads nothing more
            raise
        if st.value != 2:
            return None
        self._borrowed.pop(job_id, None)
        # one reused landing buffer (a fresh one per result would take new pages for
        # every proof); the result handed back is its own copy
        if len(self._pollbuf) < max(1, n.value):
            self._pollbuf = np.empty(max(1, n.value), np.uint8)
        out = self._pollbuf
        self._check(lib().azk_server_poll(self._h, job_id, ctypes.byref(st), None, _ptr(out), ctypes.byref(n)))
        if release:
            self._check(lib().azk_server_release(self._h, job_id))
        kind = self._kind.pop(job_id, 0) if release else self._kind.get(job_id, 0)
        res = out[:n.value].tobytes() if kind == 0 else _sumcheck_words(out[:n.value].copy().view(np.uint32))
        return res, lat.value

    def wait_all(self):
        self._check(lib().azk_server_wait_all(self._h))

    def stats(self) -> dict:
        c, e, h, span = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_double()
        self._check(lib().azk_server_stats(self._h, ctypes.byref(c), ctypes.byref(e), ctypes.byref(span), ctypes.byref(h)))
        return {"completed": c.value, "pcs_elements": e.value, "span_s": span.value, "held_bytes": h.value}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().azk_server_destroy(self._h)
            self._h = _vp()
            self._borrowed.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
