"""The drop-in: LELA code with Context<Modular<uint32>, CUDAModule<uint32>>
(include/lela_cuda/cuda-module.h) compiled against LELA's own headers and run
next to LELA's ZpModule / GenericModule / FaugereLachartre
(tests/cuda_module/test_cuda_module.C)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "cuda_module", "build.sh")
BIN = os.path.join(HERE, "cuda_module", "_build", "test_cuda_module")
REF = os.environ.get("REF", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def test_cuda_module_header_compiles_against_lela():
    """Compile-only check on the CPU (needs the reference headers)."""
    if not os.path.isdir(os.path.join(REF, "lela")):
        pytest.skip("LELA headers not present on this machine")
    r = subprocess.run(["sh", BUILD], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert os.path.exists(BIN)


@pytest.mark.gpu
def test_cuda_module_matches_lela_modules():
    # the binary is built with the library (__graft_entry__.build) and travels
    # with it; a GPU run without it has lost the drop-in check, which fails
    assert os.path.exists(BIN), \
        "tests/cuda_module/_build/test_cuda_module missing: build it with the LELA headers (build.sh)"
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all passed" in r.stdout
