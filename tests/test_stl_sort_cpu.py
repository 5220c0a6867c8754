"""The device stages' sorts leave elements in the same order as the host library's std::sort, equal keys included,
so the device searcher keeps the same candidate among equal scores as the host searcher and the reference: the
sequential form (csrc/stl_sort.h) and the block-parallel form (csrc/stl_sort_par.h, run here as one emulated
thread).  Compiled with the host compiler and checked on 8,000 arrays with many equal keys, some of them built by
McIlroy's adversary so that the depth budget runs out and the heapsort fallback is taken."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_device_sort_order_equals_std_sort():
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "stl_sort_check")
        subprocess.check_call(["g++", "-O2", "-std=c++20", "-I" + os.path.join(ROOT, "desert-search_b200", "csrc"),
                               os.path.join(ROOT, "tests", "cpp", "stl_sort_check.cpp"), "-o", exe])
        out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
        assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr
