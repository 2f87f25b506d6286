"""Accuracy of the FP64 reciprocal the RHS kernels use for divisions that share a denominator.

rcp64 (ablate_b200/csrc/fv_physics.cuh) refines the PTX rcp.approx.ftz.f64 approximation with two
Newton-Raphson steps and sends zero, infinite, NaN and extreme inputs (|x| outside 1e-300..1e300) to the
IEEE division. The check (tests/rcp64_check.cu, compiled here with nvcc for sm_100a) evaluates it on
about 2.5 million inputs spanning the whole exponent range, the cut-offs and their neighbours, every
power of two and the special values: the special values must equal the host's 1/x exactly, and every
other result must lie within one unit in the last place of the exact reciprocal (faithful rounding).
"""
import shutil
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent


def test_rcp64_within_one_ulp_of_ieee_division(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "rcp64_check"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
                    "-I", str(HERE.parent / "include"), str(HERE / "rcp64_check.cu"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=120).stdout.split()
    fields = dict(zip(out[0::2], out[1::2]))
    assert int(fields["n"]) > 2_500_000
    assert int(fields["mismatched_specials"]) == 0, out
    # faithful: below one unit in the last place of the exact reciprocal (the result is the correctly rounded
    # quotient or its neighbour; not_nearest counts the neighbours)
    assert float(fields["max_ulp"]) < 1.0, out
