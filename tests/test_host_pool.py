"""The host thread pool of the chunked transfers (dasha_b200/csrc/host_pool.h): compiled on its
own with g++ and run; every row of every job is visited exactly once, for job sizes below and
above the threading threshold, many jobs in a row and four host threads calling at once."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_host_pool_visits_every_row_once(tmp_path):
    exe = str(tmp_path / "host_pool_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I" + os.path.join(ROOT, "dasha_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "host_pool_check.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "bad=0" in r.stdout
