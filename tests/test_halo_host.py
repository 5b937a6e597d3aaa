"""Host side of the slab group (dasha_b200/csrc/halo.h): the time-limited barrier of the
in-process exchange and the partition, compiled on their own with g++ and run (no GPU): threads
pass 2000 generations in step, a failing member releases every waiter, a missing member makes
the others give up after the limit, reset() makes the barrier usable again, and the partition
covers the interior rows in order."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_group_barrier_and_partition(tmp_path):
    exe = str(tmp_path / "halo_barrier_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I" + os.path.join(ROOT, "dasha_b200", "csrc"),
                    "-I/usr/local/cuda/include", "-o", exe, os.path.join(ROOT, "tests", "halo_barrier_check.cpp"),
                    "-ldl"], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "bad=0" in r.stdout
