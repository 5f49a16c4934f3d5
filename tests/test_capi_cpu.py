"""CPU-only checks of the C-ABI library: it loads, exports every symbol that
include/azk_cuda.h declares, and refuses to run without an sm_100 device (no CPU
fallback).  The device helpers (Keccak, fields, transcript) are also compiled for
the host and compared with the CPU oracle."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "azk_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(azk_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_api():
    names = declared_functions()
    assert "azk_ctx_create" in names and "azk_batch_prove" in names and len(names) > 40


def test_library_exports_every_declared_symbol():
    import apple_b200

    path = apple_b200.library_path()
    assert os.path.exists(path)
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    lib = ctypes.CDLL(path)
    for n in declared_functions():
        assert getattr(lib, n) is not None


def test_python_prototypes_cover_header():
    from apple_b200 import _capi

    assert set(declared_functions()) == set(_capi.PROTOTYPES)


def test_context_fails_loudly_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import apple_b200

    with pytest.raises(apple_b200.AZKError) as e:
        apple_b200.Context(0)
    assert e.value.name == "unavailableOnThisPlatform"


def test_proof_size_formula_matches_reference_bench_sizes(golden):
    # CirclePCSFRIProofCodecV1 sizes from the reference's bench reports (log 14 and 10, 3 rounds, 4 queries)
    import apple_b200

    assert apple_b200.pcs_proof_size(14, 3, 4) == golden["bench_codeword_prover_log14"]["proof_bytes"]
    assert apple_b200.pcs_proof_size(10, 3, 4) == golden["bench_codeword_prover_log10"]["proof_bytes"]
    assert apple_b200.pcs_proof_size(6, 2, 36, claimed=3) == golden["corpus"]["valid_bytes"]


def test_device_helpers_compiled_for_host(tmp_path):
    exe = tmp_path / "host_check"
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-fopenmp", "-I", os.path.join(ROOT, "oracle"), "-I", os.path.join(ROOT, "apple_b200", "csrc"),
                    os.path.join(ROOT, "tests", "host_check.cpp"), "-o", str(exe)], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "host check ok" in r.stdout
