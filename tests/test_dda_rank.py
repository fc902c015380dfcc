"""The cell walk's face-time ranking, on the CPU.

The walk (flexrt_imaging_reion_b200/csrc/frt_dda.cuh) evaluates the reference's exact face-time
quotients only for the axes whose approximate time lies within 2^-18 of the smallest. It is
compiled here as host code (tests/dda_rank_test.cu) and compared ray by ray with the walk that
evaluates all three exact quotients at every face (advance_ray's expressions,
ray_tracing.cc:1254-1400): segment counts, cells, distances and end states bit for bit, over
random rays in boxes of the S, M and L sizes and edge cases with exact ties between axes.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="needs nvcc to compile the walk header for the host")
def test_ranked_walk_matches_three_quotients(tmp_path):
    exe = str(tmp_path / "dda_rank_test")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-Xcompiler", "-ffp-contract=off", "-fmad=false",
                    "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets", "-x", "cu",
                    os.path.join(HERE, "dda_rank_test.cu"), "-o", exe], check=True)
    out = subprocess.run([exe, "1000000"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:]
    tok = out.stdout.split()
    assert tok[0] == "ok", out.stdout
    rays, segs, ties = int(tok[1]), int(tok[2]), int(tok[3])
    assert rays == 3_000_000 and segs > 3 * rays and ties > 10_000
