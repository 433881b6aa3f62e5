"""C ABI checks that need no GPU: the library loads, exports every symbol the
header declares with matching struct layouts, and the Python surface keeps
the reference's argument checks.  No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from hnsw_rabitq_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hnswgpu.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"HNSWGPU_API\s+[\w\s\*]+?\b(hnswgpu_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    names = declared()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
        assert n in _capi.SIGNATURES, n
    assert set(_capi.SIGNATURES) == set(names)


def test_struct_layouts_match_header(tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text('#include <stdio.h>\n#include "hnswgpu.h"\n#include <stddef.h>\n'
                    'int main(void){printf("%zu %zu %zu %zu %zu %zu %d\\n", sizeof(hnswgpu_info), sizeof(hnswgpu_search_opts),'
                    ' offsetof(hnswgpu_info, device_bytes), offsetof(hnswgpu_search_opts, stream),'
                    ' sizeof(hnswgpu_term_train_opts), offsetof(hnswgpu_term_train_opts, seed),'
                    ' HNSWGPU_TERM_PARAMS);return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)])
    a, b, c, d, e, f, g = map(int, subprocess.check_output([str(exe)]).split())
    assert a == C.sizeof(_capi.Info) and b == C.sizeof(_capi.SearchOpts)
    assert c == _capi.Info.device_bytes.offset and d == _capi.SearchOpts.stream.offset
    assert e == C.sizeof(_capi.TermTrainOpts) and f == _capi.TermTrainOpts.seed.offset
    assert g == _capi.TERM_PARAMS


def test_server_struct_layouts(tmp_path):
    prog = tmp_path / "sv.c"
    prog.write_text('#include <stdio.h>\n#include "hnswgpu.h"\n#include <stddef.h>\n'
                    'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(hnswgpu_server_opts),'
                    ' sizeof(hnswgpu_request), sizeof(hnswgpu_server_stats), offsetof(hnswgpu_request, rerank),'
                    ' offsetof(hnswgpu_server_stats, max_us));return 0;}\n')
    exe = tmp_path / "sv"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)])
    a, b, c, d, e = map(int, subprocess.check_output([str(exe)]).split())
    assert (a, b, c) == (C.sizeof(_capi.ServerOpts), C.sizeof(_capi.Request), C.sizeof(_capi.ServerStats))
    assert d == _capi.Request.rerank.offset and e == _capi.ServerStats.max_us.offset


def test_version_and_error_string():
    lib = _capi.lib()
    assert b"sm_100a" in lib.hnswgpu_version()
    # a null handle is rejected before any CUDA call
    rc = lib.hnswgpu_set_ef(None, 5)
    assert rc == _capi.ERR_ARG
    assert lib.hnswgpu_last_error() == b"invalid argument"
    info = _capi.Info()
    assert lib.hnswgpu_get_info(None, C.byref(info)) == _capi.ERR_ARG


def test_python_surface_argument_checks():
    with pytest.raises(RuntimeError, match="Space name must be one of l2, ip, or cosine."):
        H.Index("hamming", 8)
    with pytest.raises(RuntimeError, match="Space name must be one of l2, ip, or cosine."):
        H.BFIndex("dot", 8)
    with pytest.raises(RuntimeError, match="Space name must be one of l2, ip, or cosine."):
        H.BFIndex("l2_uint8", 8)  # L2SpaceI: HNSW indexes only
    assert H.Index("l2_uint8", 8).space == "l2_uint8"
    idx = H.Index("l2", 8)
    assert idx.ef == 10 and idx.get_current_count() == 0
    idx.set_ef(77)
    assert idx.ef == 77
    with pytest.raises(RuntimeError, match="load_index"):
        idx.knn_query(np.zeros((1, 8), np.float32))
    with pytest.raises(NotImplementedError):
        idx.add_items(np.zeros((1, 8), np.float32))
    bf = H.BFIndex("l2", 4)
    bf.init_index(3)
    bf.add_items(np.eye(4, dtype=np.float32)[:3])
    assert bf.get_current_count() == 3
    with pytest.raises(RuntimeError, match="exceeds the specified limit"):
        bf.add_items(np.ones((1, 4), np.float32), ids=[99])
    with pytest.raises(RuntimeError, match="wrong shape"):
        bf.knn_query(np.zeros((1, 1, 4), np.float32))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_fails_loudly_without_gpu(tmp_path):
    """No CPU fallback: without a device the load reports a CUDA error."""
    gold = os.path.join(ROOT, "tests", "golden", "hnsw_l2_d16.bin")
    idx = H.Index("l2", 16)
    with pytest.raises(_capi.HnswGpuError) as e:
        idx.load_index(gold)
    assert e.value.code == _capi.ERR_CUDA


def test_datasets_deterministic_and_shaped():
    from hnsw_rabitq_b200 import datasets as D
    x1, q1 = D.gmm_1m_128(n=2000, nq=50)
    x2, q2 = D.gmm_1m_128(n=2000, nq=50)
    assert np.array_equal(x1, x2) and np.array_equal(q1, q2)
    assert x1.dtype == np.float32 and x1.min() >= 0 and x1.max() <= 255
    assert np.array_equal(x1, np.rint(x1))
    x, q = D.uniform_10k()
    assert x.shape == (10000, 128) and q.shape == (1000, 128)
    x, q = D.gmm_unit_ip(n=500, nq=10)
    assert np.allclose(np.linalg.norm(x, axis=1), 1, atol=1e-5)
    x, q = D.gmm_lognormal_sigma(n=1000, nq=10)
    assert x.shape == (1000, 96)


def test_newer_entry_points_reject_bad_arguments():
    """Argument checks that run before any device work (no GPU needed)."""
    lib = _capi.lib()
    u64 = C.c_uint64()
    # learned termination
    assert lib.hnswgpu_set_termination_model(None, None, 4, C.c_float(0.0)) == _capi.ERR_ARG
    opts = _capi.SearchOpts()
    assert lib.hnswgpu_search_checkpoints(None, None, 1, 10, C.byref(opts), 4, 8, 0, None, None, None, None, None,
                                          None, None) == _capi.ERR_ARG
    to = _capi.TermTrainOpts(epochs=1, batch=16, lr=1e-3, pos_weight=1.0, weight_decay=0.0, reserved=0, seed=0)
    assert lib.hnswgpu_term_train(0, None, None, 0, C.byref(to), None, None) == _capi.ERR_ARG
    assert lib.hnswgpu_term_loss_grad(0, None, None, None, 0, C.c_float(1.0), None, None) == _capi.ERR_ARG
    assert lib.hnswgpu_term_logits(0, None, None, 3, None) == _capi.ERR_ARG
    h = C.c_void_p()
    assert lib.hnswgpu_load_hnsw_buffer(None, 16, 0, 16, 0, 0, C.byref(h)) == _capi.ERR_ARG
    assert lib.hnswgpu_load_hnsw_buffer(C.c_char_p(b"x" * 16), 16, 7, 16, 0, 0, C.byref(h)) == _capi.ERR_ARG
    # float64 oracle, serving loop
    assert lib.hnswgpu_fp64_distances(None, None, 1, None, 1, None) == _capi.ERR_ARG
    srv = C.c_void_p()
    assert lib.hnswgpu_server_create(None, None, C.byref(srv)) == _capi.ERR_ARG
    req = _capi.Request(k=10, ef=0, filter=-1, flags=0, precision=0, rerank=0)
    assert lib.hnswgpu_server_submit(None, None, C.byref(req), C.byref(u64)) == _capi.ERR_ARG
    assert lib.hnswgpu_server_wait(None, 1, None, None, None, None) == _capi.ERR_ARG
    st = _capi.ServerStats()
    assert lib.hnswgpu_server_get_stats(None, C.byref(st), 0) == _capi.ERR_ARG
    assert lib.hnswgpu_server_destroy(None) == _capi.ERR_ARG
    assert lib.hnswgpu_build_traversal_copy(None, 2) == _capi.ERR_ARG
    assert lib.hnswgpu_search_epsilon(None, None, 1, C.c_float(1.0), 1, 4, C.byref(opts), None, None,
                                      None) == _capi.ERR_ARG
    h = C.c_void_p()
    assert lib.hnswgpu_load_bf(b"none.bin", _capi.SPACE_L2_UINT8, 8, 0, C.byref(h)) == _capi.ERR_UNSUPPORTED
    assert lib.hnswgpu_create_bf(_capi.SPACE_L2_UINT8, 8, None, None, 0, 0, 0, C.byref(h)) == _capi.ERR_UNSUPPORTED
    assert lib.hnswgpu_last_error() != b""


def test_termination_model_file_round_trip(tmp_path):
    from hnsw_rabitq_b200 import learned
    rng = np.random.default_rng(0)
    m = learned.TerminationModel(learned.init_params(rng.normal(size=(50, _capi.TERM_FEATURES)), 1), 8, 1.25, 96, "fp8", 40,
                                 {"note": "x"})
    m.save(str(tmp_path / "t.npz"))
    r = learned.TerminationModel.load(str(tmp_path / "t.npz"))
    assert np.array_equal(r.params, m.params)
    assert (r.period, r.threshold, r.ef_cap, r.precision, r.rerank, r.info) == (8, 1.25, 96, "fp8", 40, {"note": "x"})


def test_serving_helpers():
    from hnsw_rabitq_b200.serving import Server, poisson_arrivals
    a = poisson_arrivals(20000, 100_000, seed=1)
    assert np.all(np.diff(a) > 0) and abs(a[-1] / 20000 - 10.0) < 0.5  # mean gap 10 us
    r = Server.request(k=5, ef=64, filter=2, tie_order="reference", precision="bf16", rerank=7)
    assert (r.k, r.ef, r.filter, r.flags, r.precision, r.rerank) == (5, 64, 2, _capi.EXACT_TIES, _capi.PREC_BF16, 7)
    assert Server.request(learned=True).flags == _capi.LEARNED_STOP


def test_flag_and_status_constants_match_header():
    src = open(HEADER).read()
    defs = {m.group(1): int(m.group(2), 16) for m in re.finditer(r"#define HNSWGPU_(\w+)\s+0x([0-9a-fA-F]+)u", src)}
    for name in ("DEVICE_PTRS", "TRACE", "EXACT_TIES", "LEARNED_STOP", "EXACT_SCAN", "REPLAY_ALL", "STATUS_TIMEOUT",
                 "STATUS_OVERFLOW"):
        assert defs[name] == getattr(_capi, name), name
    flags = [defs[n] for n in ("DEVICE_PTRS", "TRACE", "EXACT_TIES", "LEARNED_STOP", "EXACT_SCAN", "REPLAY_ALL")]
    assert len(set(flags)) == len(flags) and all(f & (f - 1) == 0 for f in flags)


def test_tie_order_values():
    idx = H.Index("l2", 8)
    with pytest.raises(ValueError, match="tie_order"):
        idx.knn_query_traced(np.zeros((1, 8), np.float32), tie_order="heap")


def test_tie_order_flags_reach_the_c_abi(monkeypatch):
    """knn_query / knn_query_traced pass the tie order as flags: "reference"
    (default) -> HNSWGPU_EXACT_TIES, "replay" -> EXACT_TIES | REPLAY_ALL,
    "id" -> neither; low precision and the learned stop use the id order.
    The search call is replaced by a recorder, so no GPU is needed."""
    seen = []

    class FakeLib:
        def hnswgpu_search(self, h, q, nq, k, opts, labels, dists, counts):
            o = opts._obj
            seen.append(o.flags)
            C.memset(counts, 0, 4 * nq)
            return 0

    monkeypatch.setattr(_capi, "lib", lambda: FakeLib())
    idx = H.Index("l2", 8)
    idx._h = C.c_void_p(1)  # never dereferenced by the recorder
    try:
        q = np.zeros((2, 8), np.float32)
        for order, want in (("reference", _capi.EXACT_TIES), ("replay", _capi.EXACT_TIES | _capi.REPLAY_ALL),
                            ("id", 0)):
            idx.knn_query_traced(q, k=3, tie_order=order)
            assert seen[-1] & (_capi.EXACT_TIES | _capi.REPLAY_ALL) == want, order
        idx.knn_query_traced(q, k=3, tie_order="reference", precision="fp8")
        assert seen[-1] & _capi.EXACT_TIES == 0
    finally:
        idx._h = None
