"""apple_b200: B200 (sm_100a) commit-and-fold superstep behind a C ABI.

Python mirror of AppleZKProver's plan API over libazk_cuda.so (include/azk_cuda.h).
The CUDA library is the product; this module only marshals arguments.  Importing
it loads the in-tree shared library and fails loudly when it is missing: there is
no CPU fallback.
"""
from __future__ import annotations

import os as _os

# Every plan, batch and server worker runs on its own CUDA stream.  With the
# driver's default of 8 hardware work queues, streams share queues and work on one
# waits behind another's whole CUDA graph (a prover's upload stalls until another
# prover's superstep ends).  The queue count is read when CUDA initialises in the
# process, so it is set here, at import, before torch or anything else starts
# CUDA; a value the caller set is kept.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from ._capi import (  # noqa: E402,F401
    AZK_STATUS_NAMES,
    AZKError,
    Schedule,
    Stats,
    lib,
    library_path,
)
from .plans import (  # noqa: E402,F401
    BatchProver,
    CircleCodewordPlan,
    CircleDomainMaterializationPlan,
    CircleFRIFoldChainPlan,
    CircleFRIFoldPlan,
    CircleFRIMerkleTranscriptFoldChainPlan,
    CircleFRIResidentQueryExtractor,
    CirclePCSFRIProver,
    CircleWitnessToFFTBasisPlan,
    Context,
    ProofServer,
    KeccakF1600PermutationPlan,
    QM31FRIFoldChainPlan,
    QM31FRIFoldPlan,
    SHA3FixedOneBlockHashPlan,
    SHA3PrehashedLeavesMerkleCommitPlan,
    SHA3RawLeavesMerkleCommitPlan,
    circle_domain_points,
    circle_fft_twiddles,
    circle_fold_chain,
    circle_inverse_layers,
    circle_merkle_fold_chain,
    commit_prehashed_leaves,
    pcs_proof_size,
    probe_int_issue,
    qm31_fold,
    qm31_merkle_fold_chain,
    qm31_transcript_challenges,
    sumcheck_prove,
)
