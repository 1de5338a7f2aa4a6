"""The walker's exact shortcuts checked on the device: Markstein division by
S + 1 against __ddiv_rn (bit for bit) and the FP32 pre-test of the trace rule
against the FP64 rule, via tests/cuda/walk_math_check.cu (built with nvcc from
the walker's own header)."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_walk_division_and_trace_shortcuts_are_exact(tmp_path):
    exe = str(tmp_path / "walk_math_check")
    subprocess.run(["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "info-centric_ge_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "cuda", "walk_math_check.cu")], check=True)
    out = subprocess.run([exe, str(1 << 28), str(1 << 26)], check=True, capture_output=True, text=True, timeout=300)
    n_div, bad_div, n_trace, bad_trace = map(int, out.stdout.split())
    print(f"division: {n_div} cases, {bad_div} mismatches; trace rule: {n_trace} cases, {bad_trace} mismatches")
    assert n_div == 1 << 28 and bad_div == 0
    assert n_trace == 1 << 26 and bad_trace == 0
