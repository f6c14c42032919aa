"""The C++20 drop-in (include/qlassical_b200/cuda_engine.hpp, gpu_runner.hpp):
CUDAEngine / CUDAStateVector derive from the reference's ExecutionEngine /
StateVector and GPUCircuitRunner mirrors CircuitRunner.  The test program
tests/cpp/test_cuda_engine.cpp restates the reference's backend, frontend and
integration Catch2 cases against them and checks them differentially against
the reference CPUOpenMPEngine compiled into the same binary."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP_DIR = os.path.join(ROOT, "tests", "cpp")
BIN = os.path.join(CPP_DIR, "_bin", "test_cuda_engine")
from oracle.oracle import REFERENCE_DIR  # noqa: E402  ($QLB_REFERENCE_DIR or `reference` beside the repo)

REFERENCE_INCLUDE = os.path.join(REFERENCE_DIR, "include")


@pytest.mark.skipif(not os.path.isdir(REFERENCE_INCLUDE), reason="reference headers absent")
def test_dropin_compiles_against_reference_headers():
    """The headers compile in the reference's own include tree (C++20, -Wall)
    and the program links libqlassical_b200.so."""
    r = subprocess.run(["make", "-s", "-C", CPP_DIR, f"REF={REFERENCE_DIR}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert os.path.isfile(BIN)


@pytest.mark.gpu
def test_dropin_program_passes_on_gpu():
    if not os.path.isfile(BIN):
        pytest.skip("C++ drop-in test program not built (needs the reference headers at build time)")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-4000:]
    assert " 0 failures" in r.stdout
