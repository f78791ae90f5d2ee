"""Host-side check of the device modular arithmetic header: the Barrett
product for every modulus bit length up to 62 and the Montgomery fallback
above, against exact 128-bit arithmetic (tests/modarith_check.cu)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_modarith_host(tmp_path):
    nvcc = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)
    if nvcc is None:
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "modarith_check")
    subprocess.run([nvcc, "-O2", "-Wno-deprecated-gpu-targets", "-o", exe, os.path.join(HERE, "modarith_check.cu")],
                   check=True, capture_output=True, timeout=300)
    out = subprocess.run([exe], check=False, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr
