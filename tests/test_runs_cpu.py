"""The host check and run coding of sorted arc sources (zog_b200/csrc/runs.h),
which decides whether a chunk of a host arc list crosses PCIe as run offsets,
compiled with g++ and run against a plain loop on 4,000 random chunks
(tests/runs_check.cpp): the offsets must match, a chunk that is not
non-decreasing or holds a source >= V must be refused, and no write may leave
the chunk's offset range.  No GPU."""
import os
import subprocess

from conftest import ROOT


def test_run_coding_matches_a_plain_loop(tmp_path):
    exe = str(tmp_path / "runs_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-pthread",
                    "-I", os.path.join(ROOT, "zog_b200", "csrc"),
                    os.path.join(ROOT, "tests", "runs_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "runs ok"
