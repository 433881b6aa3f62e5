"""The tie-exact heap routines keep std::priority_queue's element layout
(host compile of the same header the kernel uses; CPU only)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_heap_layout_matches_libstdcxx(tmp_path):
    exe = tmp_path / "heapchk"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "hnsw_rabitq_b200", "csrc"),
                           os.path.join(ROOT, "tests", "heap_layout_check.cpp"), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout
