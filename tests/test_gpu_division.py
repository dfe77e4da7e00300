"""The per-pixel loops divide with a branch-free correctly rounded scheme
(rcp_markstein / div_markstein in word2world_b200/csrc/common.cuh) where the
operands allow it.  This compiles tests/kernels/division_check.cu and checks
it against CUDA's __frcp_rn (every significand, several exponents) and
__fdiv_rn (about 2.5e9 seeded random pairs in the admitted range): bit-identical."""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(not _gpu(), reason="needs a GPU")
def test_division_matches_ieee(tmp_path):
    if not os.path.exists(NVCC) and not shutil.which("nvcc"):
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "division_check")
    subprocess.run([NVCC if os.path.exists(NVCC) else "nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                    "-std=c++17", "--expt-relaxed-constexpr", "-o", exe,
                    os.path.join(HERE, "kernels", "division_check.cu")], check=True)
    r = subprocess.run([exe, "1"], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
