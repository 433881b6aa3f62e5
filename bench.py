#!/usr/bin/env python
"""Benchmark of the GPU HNSW query path on the 1M x 128 L2 workload.

Workload (seeded synthetic stand-in; the reference ships no dataset):
1,000,000 x 128 float32 vectors from a 1,024-component isotropic Gaussian
mixture (centres U[0,255], sigma 20) rounded to integers in [0,255]; 10,000
queries from the same mixture; graph built by the reference (hnswlib 0.9.0,
M=16, ef_construction=200); k=10.

Metric: queries/s at recall@10 >= 0.95.  Recall is measured against exact
top-10 from the GPU brute force (bit-identical to the reference's
BruteforceSearch).  The smallest ef of the sweep 10..400 that reaches the
target is the operating point.

* ``value``  -- device-resident throughput: K launches over the 10,000
  resident queries, timed with CUDA events on the launch stream.
* ``e2e``    -- the same through the C ABI (hnswgpu_search) with pinned host
  buffers: host->device copy of the queries, search, device->host copy of the
  labels/distances/counts every step, wall-clock timed.
* ``roofline`` -- HBM bound: algorithmic bytes per query from the oracle's
  trace at the same ef (link lists read x their size + distance evaluations x
  512 B), divided by the kernel time.
* ``cpu_baseline`` -- the reference's own knn_query (oracle/_ref) on the
  host cores of this machine, all threads, same index / queries / ef.

``--impl reference`` times the reference's knn_query instead (CPU, all host
threads; rank 0 only under torchrun).

Multi-GPU (torchrun): replicas only -- every rank loads the full index and
searches its own copy of the query batch; no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CACHE = os.path.join(ROOT, ".cache")
EFS = [10, 16, 24, 32, 40, 44, 48, 52, 56, 64, 80, 96, 128, 192, 256, 320, 400]
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--nq", type=int, default=10_000)
    ap.add_argument("--ef", type=int, default=0, help="fixed ef (skip the sweep)")
    ap.add_argument("--target-recall", type=float, default=0.95)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", action="store_true", help="only run the timed loop (for ncu)")
    ap.add_argument("--tie-order", default="reference", choices=["reference", "id"],
                    help="reference: heap replay, results identical to hnswlib; id: ties by internal id")
    return ap.parse_args()


# ----------------------------------------------------------------- plumbing
class Dist:
    def __init__(self, n_gpus):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", self.local))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{self.local}")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# ----------------------------------------------------------------- workload
def workload(n, nq):
    from hnsw_rabitq_b200.datasets import gmm_1m_128
    return gmm_1m_128(n=n, nq=nq)


def ref_module():
    """The reference's own compiled extension (builds the graph the workload
    names; times the CPU baseline).  Never on the measured GPU path."""
    from oracle import oracle as O
    mod = O.ref_module()
    if mod is None:
        raise SystemExit("the reference extension (oracle/_ref) is not built: run `make -C oracle ref`")
    return mod


def ensure_index(x, dist: Dist):
    os.makedirs(CACHE, exist_ok=True)
    n = x.shape[0]
    path = os.path.join(CACHE, f"gmm_{n}_128_M16_efc200.bin")
    if dist.rank == 0 and not os.path.exists(path):
        hnswlib = ref_module()
        t = time.time()
        p = hnswlib.Index("l2", 128)
        p.init_index(n, M=16, ef_construction=200, random_seed=100)
        p.add_items(x, num_threads=os.cpu_count())
        p.save_index(path + ".tmp")
        os.replace(path + ".tmp", path)
        print(f"[bench] built reference index in {time.time() - t:.1f}s -> {path}", file=sys.stderr)
    dist.barrier()
    return path


def ground_truth(x, q, k=10):
    """Exact top-k on the GPU (bit-identical to the reference brute force)."""
    path = os.path.join(CACHE, f"gt_{x.shape[0]}_{q.shape[0]}_{k}.npy")
    if os.path.exists(path):
        return np.load(path)
    from hnsw_rabitq_b200 import BFIndex
    bf = BFIndex("l2", x.shape[1])
    bf.init_index(x.shape[0])
    bf.add_items(x)
    labels, _ = bf.knn_query(q, k=k)
    tmp = f"{path}.{os.getpid()}.npy"
    np.save(tmp, labels)
    os.replace(tmp, path)
    return labels


def recall(found, gt):
    k = gt.shape[1]
    hit = sum(len(np.intersect1d(found[i, :k], gt[i])) for i in range(gt.shape[0]))
    return hit / gt.size


# -------------------------------------------------------------- our GPU arm
def run_ours(args, dist: Dist):
    import ctypes as C

    import torch

    from hnsw_rabitq_b200 import Index, _capi

    dev = dist.local
    torch.cuda.set_device(dev)
    x, q = workload(args.n, args.nq)
    path = ensure_index(x, dist)
    gt = None if args.profile_steps else ground_truth(x, q)
    idx = Index("l2", 128)
    idx.device = dev
    idx.tie_order = args.tie_order
    idx.load_index(path)
    info = idx._info()
    if args.profile_steps and not args.ef:
        raise SystemExit("--profile-steps needs --ef")

    # ---- operating point: smallest ef with recall@10 >= target
    sweep = []
    ef_star = args.ef
    if not ef_star:
        for ef in EFS:
            idx.set_ef(ef)
            t = time.perf_counter()
            lab, _ = idx.knn_query(q, k=10)
            dt = time.perf_counter() - t
            r = recall(lab, gt)
            sweep.append({"ef": ef, "recall": round(r, 5), "qps_e2e_untimed": round(q.shape[0] / dt, 1)})
            if r >= args.target_recall and not ef_star:
                ef_star = ef
                break
        if not ef_star:
            ef_star = EFS[-1]
    idx.set_ef(ef_star)
    lab, _ = idx.knn_query(q, k=10)
    rec = recall(lab, gt) if gt is not None else None

    # ---- device-resident timed loop
    lib = _capi.lib()
    nq, k = q.shape[0], 10
    stream = torch.cuda.Stream(device=dev)
    dq = torch.from_numpy(q).to(f"cuda:{dev}")
    dl = torch.empty((nq, k), dtype=torch.int64, device=f"cuda:{dev}")
    dd = torch.empty((nq, k), dtype=torch.float32, device=f"cuda:{dev}")
    dc = torch.empty((nq,), dtype=torch.int32, device=f"cuda:{dev}")
    tie_flag = _capi.EXACT_TIES if args.tie_order == "reference" else 0
    opts = _capi.SearchOpts()
    opts.flags = _capi.DEVICE_PTRS | tie_flag
    opts.ef = ef_star
    opts.stream = stream.cuda_stream

    def step():
        _capi.check(lib.hnswgpu_search(idx._h, C.c_void_p(dq.data_ptr()), nq, k, C.byref(opts),
                                       C.c_void_p(dl.data_ptr()), C.c_void_p(dd.data_ptr()),
                                       C.c_void_p(dc.data_ptr())))

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    # the device results equal the host-path results
    assert np.array_equal(dl.cpu().numpy().view(np.uint64), lab)
    dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                step()
            ev1.record(stream)
        torch.cuda.synchronize()
    dist.barrier()
    ms_local = ev0.elapsed_time(ev1)
    ms_total = dist.max(ms_local)
    ms_step = ms_total / args.steps
    value = dist.world * nq * args.steps / (ms_total / 1e3)
    if args.profile_steps:
        return None

    # ---- e2e through the C ABI with pinned host buffers
    hq = torch.from_numpy(q).pin_memory()
    hl = torch.empty((nq, k), dtype=torch.int64).pin_memory()
    hd = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    hc = torch.empty((nq,), dtype=torch.int32).pin_memory()
    eopts = _capi.SearchOpts()
    eopts.flags = tie_flag
    eopts.ef = ef_star

    def e2e_step():
        _capi.check(lib.hnswgpu_search(idx._h, C.c_void_p(hq.data_ptr()), nq, k, C.byref(eopts),
                                       C.c_void_p(hl.data_ptr()), C.c_void_p(hd.data_ptr()),
                                       C.c_void_p(hc.data_ptr())))

    for _ in range(args.warmup):
        e2e_step()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = dist.max(time.perf_counter() - t0)
    e2e_qps = dist.world * nq * args.steps / e2e_s
    assert np.array_equal(hl.numpy().view(np.uint64), lab)

    out = None
    if dist.rank == 0:
        peak, peak_kind = peaks()
        cpu, bytes_per_q = cpu_baseline(args, path, q, ef_star, info) if not args.no_cpu_baseline else (None, None)
        roof = None
        if bytes_per_q:
            per_launch = bytes_per_q * nq
            achieved = per_launch / (ms_step / 1e3) / 1e9
            roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(achieved / peak, 4), "traffic": committed_traffic(args.tie_order, ef_star),
                    "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                    else "fallback 6.65 TB/s",
                    "algorithmic_bytes_per_query": round(bytes_per_q, 1)}
        out = {
            "metric": "QPS at recall@10>=0.95 (plain FP32 GPU HNSW, 1M x 128 L2)",
            "value": round(value, 1), "unit": "queries/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "gmm_1m_128: 1,000,000 x 128 L2 (1024-comp. GMM, integer-valued), reference-built "
                                   "HNSW M=16 efc=200, 10,000 queries, k=10",
                       "method": "plain fp32 beam, reference semantics, tie order: " + args.tie_order,
                       "ef": ef_star,
                       "recall@10": round(rec, 5), "global_batch": nq, "parallelism": f"replicas x{dist.world}",
                       "l2_flush": "not needed: index data 640 MB > 126 MB L2",
                       "index_device_bytes": info.device_bytes},
            "sweep": sweep,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_qps, 1), "unit": "queries/s", "h2d_bytes_per_step": int(q.nbytes),
                    "d2h_bytes_per_step": int(nq * k * 8 + nq * k * 4 + nq * 4)},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
        }
    return out


def committed_traffic(tie_order, ef):
    """DRAM bytes per launch of hnsw_search_kernel from the committed ncu
    summary (profiles/), for the same tie order and ef, or None."""
    p = os.path.join(ROOT, "profiles", "hnsw_search_gmm1m_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d.get(tie_order, {}).get(str(ef))
    except (OSError, ValueError, AttributeError):
        return None


def cpu_baseline(args, path, q, ef, info):
    """The reference's knn_query on this host (all threads), plus the oracle's
    work trace at the same ef for the roofline's algorithmic bytes."""
    from oracle import oracle as O
    hnswlib = ref_module()
    p = hnswlib.Index("l2", 128)
    p.load_index(path)
    p.set_ef(ef)
    threads = os.cpu_count()
    p.knn_query(q[:1000], k=10, num_threads=threads)
    times = []
    for _ in range(5):
        t = time.perf_counter()
        p.knn_query(q, k=10, num_threads=threads)
        times.append(time.perf_counter() - t)
    qps = q.shape[0] / statistics.median(times)
    cpu = {"value": round(qps, 1), "unit": "queries/s", "cores": threads, "kind": "reference",
           "sample": f"all {q.shape[0]} queries x 5 runs (median), ef={ef}, k=10"}
    o = O.Hnsw(path, "l2", 128)
    _, _, _, tr = o.search(q, 10, ef, mode=O.CANONICAL, trace=True, nthreads=threads)
    up_links = 4 + 4 * info.maxM
    l0_links = 4 + 4 * info.maxM0
    bytes_q = (tr[:, 0] * up_links + tr[:, 2] * l0_links + (tr[:, 1] + tr[:, 3]) * 128 * 4).mean()
    return cpu, float(bytes_q)


# --------------------------------------------------------- reference arm
def run_reference(args, dist: Dist):
    if dist.rank != 0:
        return None
    x, q = workload(args.n, args.nq)
    path = ensure_index(x, _Solo())
    hnswlib = ref_module()
    threads = os.cpu_count()
    p = hnswlib.Index("l2", 128)
    p.load_index(path)
    # operating point from a 500-query sample against the reference's own brute force
    sample = q[:500]
    bf = hnswlib.BFIndex("l2", 128)
    bf.init_index(x.shape[0])
    bf.add_items(x)
    gt, _ = bf.knn_query(sample, k=10, num_threads=threads)
    ef_star = args.ef
    if not ef_star:
        for ef in EFS:
            p.set_ef(ef)
            lab, _ = p.knn_query(sample, k=10, num_threads=threads)
            if recall(lab, gt) >= args.target_recall:
                ef_star = ef
                break
        ef_star = ef_star or EFS[-1]
    p.set_ef(ef_star)
    for _ in range(args.warmup):
        p.knn_query(q, k=10, num_threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lab, _ = p.knn_query(q, k=10, num_threads=threads)
    dt = time.perf_counter() - t0
    qps = q.shape[0] * args.steps / dt
    return {"impl": "reference", "metric": "QPS at recall@10>=0.95 (plain FP32 GPU HNSW, 1M x 128 L2)",
            "value": round(qps, 1), "unit": "queries/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "gmm_1m_128: 1,000,000 x 128 L2 (1024-comp. GMM, integer-valued), reference-built "
                                   "HNSW M=16 efc=200, 10,000 queries, k=10",
                       "method": "hnswlib 0.9.0 knn_query (CPU)", "ef": ef_star,
                       "recall@10_sample500": round(recall(lab[:500], gt), 5)},
            "cpu_baseline": {"value": round(qps, 1), "unit": "queries/s", "cores": threads, "kind": "reference",
                             "sample": f"{q.shape[0]} queries per step"},
            "e2e": {"value": round(qps, 1), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


class _Solo:
    rank = 0

    def barrier(self):
        pass


def main():
    args = parse()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0
        out = run_reference(args, _Solo())
        print(json.dumps(out), flush=True)
        return 0
    dist = Dist(args.gpus)
    try:
        out = run_ours(args, dist)
    finally:
        dist.close()
    if out is not None and dist.rank == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
