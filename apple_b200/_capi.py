"""ctypes prototypes for libazk_cuda.so (include/azk_cuda.h)."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_NAME = "libazk_cuda.so"

AZK_STATUS_NAMES = {
    0: "ok",
    1: "invalidInputLayout",
    2: "invalidLeafCount",
    3: "unsupportedOneBlockLength",
    4: "invalidPrehashedLeafLength",
    5: "correctnessValidationFailed",
    6: "commandExecutionFailed",
    7: "unavailableOnThisPlatform",
    8: "invalidKernelConfiguration",
    9: "failedToCreateBuffer",
    10: "deviceTimeout",
    11: "hbmBudget",
}


class AZKError(RuntimeError):
    """A non-OK azk_status; `.code` is the status, `.name` its AppleZKProverError case."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.name = AZK_STATUS_NAMES.get(code, f"status{code}")
        super().__init__(f"{self.name}: {message}")


class Stats(ctypes.Structure):
    _fields_ = [("cpu_wall_s", ctypes.c_double), ("gpu_s", ctypes.c_double), ("cpu_submit_ns", ctypes.c_uint64)]


class Schedule(ctypes.Structure):
    _fields_ = [("treelet_log", ctypes.c_uint32), ("group_log", ctypes.c_uint32), ("threads", ctypes.c_uint32), ("use_graph", ctypes.c_uint32),
                ("layer_treelet", ctypes.c_uint8 * 32), ("layer_threads", ctypes.c_uint16 * 32), ("persistent_trees", ctypes.c_uint32)]


class TunerCandidate(ctypes.Structure):
    _fields_ = [("tile_log", ctypes.c_uint32), ("group_log", ctypes.c_uint32), ("threads", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class TunerMeasurement(ctypes.Structure):
    _fields_ = [("median_gpu_s", ctypes.c_double), ("p95_gpu_s", ctypes.c_double), ("median_submit_s", ctypes.c_double),
                ("passed_gate", ctypes.c_uint32), ("runs", ctypes.c_uint32)]


def library_path() -> str:
    return os.path.join(HERE, _LIB_NAME)


_lib = None

P = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
I32 = ctypes.c_int
PP = ctypes.POINTER(ctypes.c_void_p)
U32P = ctypes.POINTER(ctypes.c_uint32)
U64P = ctypes.POINTER(ctypes.c_uint64)
STATS = ctypes.POINTER(Stats)
SCHED = ctypes.POINTER(Schedule)
IP = ctypes.POINTER(ctypes.c_int)

# name -> (restype, argtypes)
PROTOTYPES = {
    "azk_ctx_create": (I32, [I32, PP]),
    "azk_ctx_destroy": (None, [P]),
    "azk_last_error_message": (ctypes.c_char_p, [P]),
    "azk_ctx_device_info": (I32, [P, IP, U64P, IP, IP]),
    "azk_buf_alloc": (I32, [P, U64, PP]),
    "azk_buf_free": (I32, [P, P]),
    "azk_buf_upload": (I32, [P, P, U64, P, U64]),
    "azk_buf_download": (I32, [P, P, P, U64, U64]),
    "azk_buf_zero": (I32, [P, P, U64]),
    "azk_synchronize": (I32, [P]),
    "azk_keccakf_plan_create": (I32, [P, U64, U64, U64, U32, PP]),
    "azk_keccakf_plan_permute": (I32, [P, P, P, STATS]),
    "azk_keccakf_plan_permute_resident": (I32, [P, P, U64, P, U64, STATS]),
    "azk_keccakf_plan_clear": (I32, [P]),
    "azk_keccakf_plan_destroy": (None, [P]),
    "azk_hash_plan_create": (I32, [P, U64, U64, U64, U64, U32, U32, PP]),
    "azk_hash_plan_hash": (I32, [P, P, P, STATS]),
    "azk_hash_plan_hash_resident": (I32, [P, P, U64, P, U64, STATS]),
    "azk_hash_plan_clear": (I32, [P]),
    "azk_hash_plan_destroy": (None, [P]),
    "azk_merkle_plan_create": (I32, [P, U64, U64, U64, U32, PP]),
    "azk_merkle_plan_commit": (I32, [P, P, P, STATS]),
    "azk_merkle_plan_commit_resident": (I32, [P, P, U64, P, STATS]),
    "azk_merkle_plan_open": (I32, [P, P, U64, P, P, P, STATS]),
    "azk_merkle_plan_open_resident": (I32, [P, P, U64, P, STATS]),
    "azk_merkle_plan_info": (I32, [P, U32P, U32P]),
    "azk_merkle_plan_clear": (I32, [P]),
    "azk_merkle_plan_destroy": (None, [P]),
    "azk_merkle_commit_prehashed": (I32, [P, P, U64, P, STATS]),
    "azk_merkle_root_noalloc": (I32, [P, U64, U64, U64, P, P]),
    "azk_circle_domain_points": (I32, [P, U32, P]),
    "azk_circle_fft_twiddles": (I32, [P, U32, P]),
    "azk_circle_inverse_layers": (I32, [P, U32, U32, P]),
    "azk_codeword_plan_create": (I32, [P, U32, PP]),
    "azk_codeword_plan_execute": (I32, [P, P, U64, P, STATS]),
    "azk_codeword_plan_execute_polynomial": (I32, [P, P, U64, P, U64, P, STATS]),
    "azk_codeword_plan_execute_resident": (I32, [P, P, U64, P, U64, STATS]),
    "azk_codeword_plan_destroy": (None, [P]),
    "azk_qm31_fold": (I32, [P, P, U64, P, P, P, STATS]),
    "azk_circle_fold_chain": (I32, [P, U32, P, P, U32, P, STATS]),
    "azk_qm31_merkle_fold_chain": (I32, [P, P, U64, P, U32, P, P, P, STATS]),
    "azk_qm31_transcript_challenges": (I32, [P, U64, P, U32, P]),
    "azk_circle_merkle_fold_chain": (I32, [P, U32, P, U32, U32, U32, P, U32, P, P, P, STATS]),
    "azk_check_canonical": (I32, [P, P, U64, U32P]),
    "azk_qm31_fold_plan_create": (I32, [P, U64, PP]),
    "azk_qm31_fold_plan_execute": (I32, [P, P, P, P, P, STATS]),
    "azk_qm31_fold_plan_execute_resident": (I32, [P, P, U64, P, U64, P, U64, P, STATS]),
    "azk_qm31_fold_plan_clear": (I32, [P]),
    "azk_qm31_fold_plan_destroy": (None, [P]),
    "azk_fold_chain_plan_create": (I32, [P, U64, U32, PP]),
    "azk_fold_chain_plan_info": (I32, [P, U64P, U64P, U64P]),
    "azk_fold_chain_plan_execute": (I32, [P, P, P, P, P, STATS]),
    "azk_fold_chain_plan_execute_resident": (I32, [P, P, U64, P, U64, P, U64, P, STATS]),
    "azk_fold_chain_plan_execute_transcript": (I32, [P, P, P, P, P, P, STATS]),
    "azk_fold_chain_plan_execute_transcript_resident": (I32, [P, P, U64, P, U64, P, U64, U64, P, U64, STATS]),
    "azk_fold_chain_plan_execute_merkle": (I32, [P, P, P, P, P, P, STATS]),
    "azk_fold_chain_plan_execute_merkle_readback": (I32, [P, P, U64, P, U64, P, P, P, STATS]),
    "azk_fold_chain_plan_execute_merkle_resident": (I32, [P, P, U64, P, U64, P, U64, U64, P, U64, P, U64, P, U64, STATS]),
    "azk_fold_chain_plan_challenges": (I32, [P, P]),
    "azk_fold_chain_plan_clear": (I32, [P]),
    "azk_fold_chain_plan_destroy": (None, [P]),
    "azk_query_extractor_create": (I32, [P, U32, U32, PP]),
    "azk_query_extractor_query_bytes": (U64, [U32, U32]),
    "azk_query_extractor_extract": (I32, [P, P, U64, P, P, U64, P, U64P, STATS]),
    "azk_query_extractor_destroy": (None, [P]),
    "azk_merkle_prehashed_plan_create": (I32, [P, U64, PP]),
    "azk_merkle_prehashed_plan_commit": (I32, [P, P, P, STATS]),
    "azk_merkle_prehashed_plan_commit_resident": (I32, [P, P, U64, P, STATS]),
    "azk_merkle_prehashed_plan_destroy": (None, [P]),
    "azk_domain_plan_create": (I32, [P, U32, U32, U32, U32, PP]),
    "azk_domain_plan_info": (I32, [P, U64P, U64P, U64P, STATS]),
    "azk_domain_plan_buffers": (I32, [P, PP, PP, PP]),
    "azk_domain_plan_read_points": (I32, [P, P]),
    "azk_domain_plan_read_twiddles": (I32, [P, P]),
    "azk_domain_plan_read_inverse_layers": (I32, [P, P]),
    "azk_domain_plan_destroy": (None, [P]),
    "azk_circle_fold_plan_create": (I32, [P, U32, PP]),
    "azk_circle_fold_plan_execute": (I32, [P, P, P, P, STATS]),
    "azk_circle_fold_plan_execute_resident": (I32, [P, P, U64, P, U64, P, STATS]),
    "azk_circle_fold_plan_read_inverse": (I32, [P, P]),
    "azk_circle_fold_plan_clear": (I32, [P]),
    "azk_circle_fold_plan_destroy": (None, [P]),
    "azk_circle_fold_chain_plan_create": (I32, [P, U32, U32, PP]),
    "azk_circle_fold_chain_plan_execute": (I32, [P, P, P, P, STATS]),
    "azk_circle_fold_chain_plan_execute_resident": (I32, [P, P, U64, P, U64, P, STATS]),
    "azk_circle_fold_chain_plan_read_inverse_layers": (I32, [P, P]),
    "azk_circle_fold_chain_plan_clear": (I32, [P]),
    "azk_circle_fold_chain_plan_destroy": (None, [P]),
    "azk_circle_merkle_chain_plan_create": (I32, [P, U32, U32, U32, U32, P, U32, PP]),
    "azk_circle_merkle_chain_plan_info": (I32, [P, U64P, U64P]),
    "azk_circle_merkle_chain_plan_execute": (I32, [P, P, P, P, P, STATS]),
    "azk_circle_merkle_chain_plan_execute_resident": (I32, [P, P, U64, P, U64, P, U64, U64, P, U64, P, U64, STATS]),
    "azk_circle_merkle_chain_plan_challenges": (I32, [P, P]),
    "azk_circle_merkle_chain_plan_read_inverse_layers": (I32, [P, P]),
    "azk_circle_merkle_chain_plan_clear": (I32, [P]),
    "azk_circle_merkle_chain_plan_destroy": (None, [P]),
    "azk_pcs_prover_create": (I32, [P, U32, U32, U32, U32, U32, SCHED, PP]),
    "azk_pcs_proof_size": (U64, [U32, U32, U32, U32, U32]),
    "azk_pcs_prover_prove_evaluations": (I32, [P, P, P, P, U64, P, U64P, STATS]),
    "azk_pcs_prover_prove_coefficients": (I32, [P, P, U64, P, P, U64P, STATS]),
    "azk_pcs_prover_prove_resident": (I32, [P, P, U64, I32, P, P, U64P, STATS]),
    "azk_pcs_prover_prove_polynomial": (I32, [P, P, U64, P, U64, P, P, U64P, STATS]),
    "azk_pcs_prover_prove_resident_witness": (I32, [P, P, U64, U64, P, U64, U64, P, P, U64P, STATS]),
    "azk_pcs_prover_trace": (I32, [P, P, P, P, P]),
    "azk_pcs_prover_destroy": (None, [P]),
    "azk_batch_create": (I32, [P, U32, P, P, U32, U32, SCHED, PP]),
    "azk_batch_create_leaves": (I32, [P, U32, P, P, U32, U32, U32, SCHED, PP]),
    "azk_batch_input": (I32, [P, U32, PP]),
    "azk_batch_upload": (I32, [P, P, P, P]),
    "azk_batch_prove": (I32, [P, P, I32, STATS]),
    "azk_batch_proof_sizes": (I32, [P, P, U64P]),
    "azk_batch_download_proofs": (I32, [P, P, U64]),
    "azk_batch_trace": (I32, [P, U32, P, P, P, P]),
    "azk_batch_set_profiling": (I32, [P, I32]),
    "azk_batch_profile": (I32, [P, P]),
    "azk_batch_work": (I32, [P, U64P, U64P, U64P, U32P]),
    "azk_batch_destroy": (None, [P]),
    "azk_probe_int_issue": (I32, [P, ctypes.POINTER(ctypes.c_double)]),
    "azk_sumcheck_prove": (I32, [P, P, U64, P, P, P, U32P, U32P, P, STATS]),
    "azk_witness_plan_create": (I32, [P, U32, PP]),
    "azk_witness_plan_execute": (I32, [P, P, U64, P, U64, P, STATS]),
    "azk_witness_plan_execute_resident": (I32, [P, P, U64, U64, P, U64, U64, P, U64, STATS]),
    "azk_witness_plan_destroy": (None, [P]),
    "azk_server_create": (I32, [P, U64, U32, SCHED, PP]),
    "azk_server_submit_pcs": (I32, [P, U32, U32, U32, U32, P, U64, P, U64P]),
    "azk_server_submit_sumcheck": (I32, [P, P, U64, U64P]),
    "azk_server_submit_pcs_nocopy": (I32, [P, U32, U32, U32, U32, P, U64, P, U64P]),
    "azk_server_submit_sumcheck_nocopy": (I32, [P, P, U64, U64P]),
    "azk_server_warm": (I32, [P, P, P, U32, U32, U32, P, U32]),
    "azk_server_poll": (I32, [P, U64, IP, ctypes.POINTER(ctypes.c_double), P, U64P]),
    "azk_server_release": (I32, [P, U64]),
    "azk_server_wait_all": (I32, [P]),
    "azk_server_stats": (I32, [P, U64P, U64P, ctypes.POINTER(ctypes.c_double), U64P]),
    "azk_server_group_stats": (I32, [P, U64P, U64P]),
    "azk_server_destroy": (None, [P]),
    "azk_tuner_time_tree": (I32, [P, U32, U32, U32, U32, U32, U32, U32, U32, ctypes.POINTER(ctypes.c_double)]),
    "azk_tuner_race_tree": (I32, [P, U32, U32, U32, U32, P, U32, U32, U32, U64, P, U32P]),
    "azk_tuner_validate_tree": (I32, [P, U32, U32, U32, U32, P, U32, U64]),
    "azk_mlp_create": (I32, [P, U32, P, U64, PP]),
    "azk_mlp_param_count": (U64, [P]),
    "azk_mlp_get_params": (I32, [P, P, U64]),
    "azk_mlp_set_params": (I32, [P, P, U64]),
    "azk_mlp_forward": (I32, [P, P, U64, P]),
    "azk_mlp_gradients": (I32, [P, P, P, U64, ctypes.POINTER(ctypes.c_float), P]),
    "azk_mlp_train": (I32, [P, P, P, U64, U32, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]),
    "azk_mlp_destroy": (None, [P]),
}


def lib():
    """Load libazk_cuda.so (built in-tree by apple_b200.build)."""
    global _lib
    if _lib is None:
        path = library_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python -m apple_b200.build` (nvcc, sm_100a); there is no CPU fallback")
        _lib = ctypes.CDLL(path)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def check(rc: int, ctx=None) -> None:
    if rc != 0:
        msg = lib().azk_last_error_message(ctx)
        raise AZKError(rc, (msg or b"").decode(errors="replace"))
