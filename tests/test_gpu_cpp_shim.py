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


def _compile(tmp_path):
    exe = tmp_path / "shim"
    libdir = os.path.join(ROOT, "hnsw_rabitq_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp_shim_check.cpp"), "-o", str(exe),
                           "-L", libdir, "-l:libhnswgpu.so", f"-Wl,-rpath,{libdir}"])
    return exe


def test_cpp_shim_matches_reference(tmp_path):
    exe = _compile(tmp_path)
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


def test_cpp_shim_filtered_single_queries(tmp_path):
    """1,000 single-query filtered searchKnn calls through the shim on a
    100,000-row index, with a functor of hnswlib's shape (not derived from the
    shim's): the functor is evaluated once and its mask stays on the device,
    so the calls finish inside a time bound; every result equals the
    reference's own filtered search; saveIndex writes the reference's file
    with the delete mark set."""
    from tests.helpers import build_hnsw, ref_or_skip
    hnswlib = ref_or_skip()
    rng = np.random.default_rng(5)
    x = rng.standard_normal((100000, 32)).astype(np.float32)
    q = rng.standard_normal((1000, 32)).astype(np.float32)
    path = tmp_path / "big.bin"
    ref = build_hnsw(path, x, "l2", M=16, efc=100, num_threads=8)
    exe = _compile(tmp_path)
    qf = tmp_path / "q.f32"
    q.tofile(qf)
    out = subprocess.run([str(exe), "--timed", str(path), str(qf), "32", "1000", "10", "64", str(tmp_path / "s.bin")],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, (out.returncode, out.stderr)
    lines = out.stdout.splitlines()
    secs = float(lines[-1].split()[1])
    assert secs < 2.0, secs
    rows = [r.split() for r in lines[:-1]]
    labels = np.array([[int(t) for t in r[0::2]] for r in rows], np.uint64)
    dists = np.array([[float(t) for t in r[1::2]] for r in rows], np.float32)
    ref.set_ef(64)
    rl, rd = ref.knn_query(q, k=10, filter=lambda l: l % 2 == 0, num_threads=1)
    assert np.array_equal(labels, rl.astype(np.uint64)) and np.array_equal(dists, rd)
    # saveIndex: the reference's file with the first result marked deleted
    ref.mark_deleted(int(labels[0, 0]))
    ref.save_index(str(tmp_path / "r.bin"))
    assert (tmp_path / "s.bin").read_bytes() == (tmp_path / "r.bin").read_bytes()
