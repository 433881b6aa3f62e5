"""The C++ shim (include/hnswgpu.hpp) compiled with g++ against
libhnswgpu.so, driven like hnswlib's C++ tests; its searchKnn results must
equal the reference's recorded outputs (needs a B200)."""
import os
import subprocess

import numpy as np
import pytest

from tests.helpers import GOLDEN, golden

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_shim_matches_reference(tmp_path):
    exe = tmp_path / "shim"
    libdir = os.path.join(ROOT, "hnsw_rabitq_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp_shim_check.cpp"), "-o", str(exe),
                           "-L", libdir, "-l:libhnswgpu.so", f"-Wl,-rpath,{libdir}"])
    g = golden()
    q = g["hnsw_l2_d16/queries"]
    qf = tmp_path / "q.f32"
    q.astype(np.float32).tofile(qf)
    e = np.load(f"{GOLDEN}/epsilon.npz")
    key = "hnsw_l2_d16/q10_min50_max128/plain"
    eps, mn, mx = e[key + "/params"]
    out = subprocess.run([str(exe), f"{GOLDEN}/hnsw_l2_d16.bin", str(qf), "16", str(q.shape[0]), "10", "32",
                          repr(float(np.float32(eps))), str(int(mn)), str(int(mx))],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stderr)
    lines = out.stdout.splitlines()
    cut = lines.index("EPS")
    # searchStopConditionClosest through the shim == the reference's recorded results
    for i, ln in enumerate(lines[cut + 1:]):
        t = ln.split()
        c = int(e[key + "/counts"][i])
        assert len(t) == 2 * c
        assert [int(v) for v in t[0::2]] == [int(v) for v in e[key + "/labels"][i, :c]]
        assert np.array_equal(np.array([float(v) for v in t[1::2]], np.float32), e[key + "/dists"][i, :c])
    rows = [r.split() for r in lines[:cut]]
    labels = np.array([[int(t) for t in r[0::2]] for r in rows], np.uint64)
    dists = np.array([[float(t) for t in r[1::2]] for r in rows], np.float32)
    assert np.array_equal(labels, g["hnsw_l2_d16/ef32_k10/labels"])
    assert np.array_equal(dists, g["hnsw_l2_d16/ef32_k10/dists"])
