"""Drop-in C++ API on the GPU (tests/cxx/api_checks.cu): the fused Solver path
against the unfused reference sequence, bit for bit, for AC and CH
single-equation RK4, the multi-step CH form, Dirichlet sides and 3-D, plus a
coupled VectorSolver run that must conserve c to 1e-12."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "api_checks.cu")
BIN = os.path.join(ROOT, "phix_b200", "_build", "api_checks")


def build_api_checks() -> str:
    """Compile api_checks.cu against include/phix + libphix_cxx.so (cached)."""
    from phix_b200.build import build_cxx, json_include
    lib = build_cxx()
    if os.path.exists(BIN) and os.path.getmtime(BIN) >= max(os.path.getmtime(SRC), os.path.getmtime(lib)):
        return BIN
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    libdir = os.path.join(ROOT, "phix_b200")
    cmd = ["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "--expt-extended-lambda",
           "--expt-relaxed-constexpr", f"-I{ROOT}/include", f"-I{ROOT}/include/phix", f"-I{json_include()}", SRC,
           "-o", BIN, f"-L{libdir}", "-lphix_cxx", "-lphix_b200", "-Xlinker", "-rpath,$ORIGIN/.."]
    subprocess.run(cmd, check=True, capture_output=True)
    return BIN


def test_cxx_api_fused_matches_unfused(cuda, tmp_path):
    exe = build_api_checks()
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0 and "ALL CHECKS PASSED" in r.stdout, r.stdout + r.stderr
