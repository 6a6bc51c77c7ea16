"""The transposed streaming push of the plasma adjoint (csrc/k_adj_stream.cuh), checked on the CPU: a host harness
(tests/stream_reverse_check.cu) built with nvcc differentiates one particle's push through a half-cell (Boris pushes,
the half-cell time, the midpoint gather, the deposit) with analytic fields and current adjoints, and compares the
hand-written reverse with central differences of the forward (state and field adjoints)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "gem-pic-3d_b200", "csrc")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc is not installed")
def test_transposed_streaming_push_matches_central_differences(tmp_path):
    exe = tmp_path / "stream_reverse_check"
    subprocess.run([NVCC, "-std=c++17", "-O2", "-I", CSRC, "-I", os.path.join(HERE, "..", "include"), "-o", str(exe),
                    os.path.join(HERE, "stream_reverse_check.cu")], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "worst" in r.stdout
