#!/usr/bin/env python
"""Benchmark of the GPU HNSW query path on the 1M x 128 L2 workload.

Workload (seeded synthetic stand-in; the reference ships no dataset):
1,000,000 x 128 float32 vectors from a 1,024-component isotropic Gaussian
mixture (centres U[0,255], sigma 20) rounded to integers in [0,255]; 10,000
queries from the same mixture; graph built by the reference (hnswlib 0.9.0,
M=16, ef_construction=200); k=10.

Metric: queries/s at recall@10 >= 0.95 of the learned-termination + FP8
search, with the plain FP32 beam (both tie orders) measured beside it in the
same run.  Recall is measured against exact top-10 from the GPU brute force
(bit-identical to the reference's BruteforceSearch).

* plain FP32: every ef of the sweep 10..400 timed (QPS and recall@10 per
  ef, both tie orders); the operating point is the smallest ef whose recall
  meets the target, timed over the full K steps.  The reference tie order
  returns hnswlib's own results (the parity contract); the id order breaks
  exact distance ties by internal id, and the share of its rows identical to
  the reference order is reported.
* fp8 at fixed ef: the same sweep over the fp8 beam (the learned stop's
  fallback and cap).
* learned + FP8 (``value``): the termination network is trained on the GPU
  from checkpoint traces of 12,000 training queries (a query stream disjoint
  from the 10,000 evaluation queries), its cap and logit threshold
  calibrated on a held-out third of them at the target recall; a second
  held-out stream of 5,000 queries checks the calibrated recall and, if it
  falls short, the calibration target is raised (no retraining).  The
  evaluation queries never inform a choice.  K launches over the 10,000
  resident queries, timed with CUDA events on the launch stream.
* ``e2e``    -- the learned + FP8 search through the C ABI (hnswgpu_search)
  with pinned host buffers: host->device copy of the queries, search,
  device->host copy of the labels/distances/counts every step, wall clock;
  the asynchronous form, steps double-buffered on three streams so that a
  step's copies overlap its neighbours' searches.  ``e2e_sync``: the
  synchronous host-pointer call (copy in, search, copy out, synchronise).
* ``roofline`` -- HBM bound: algorithmic bytes per query of the headline
  kernel from its own work counters (link lists x their size, fp8 rows of
  136 B -- 128 e4m3 bytes, scale and squared norm -- for upper-layer and
  level-0 distances, float32 re-rank rows of 512 B), divided by the kernel
  time; the plain beam's fraction (bytes from the oracle's trace at
  the same ef) sits under ``plain_fp32``.
* ``cpu_baseline`` -- the reference's own knn_query (oracle/_ref) on the
  host cores of this machine, all threads, same index / queries, at the
  plain operating point's ef.

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
EFS = [10, 16, 24, 32, 40, 44, 48, 50, 52, 54, 56, 60, 64, 80, 96, 128, 192, 256, 320, 400]
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    # --rows / --queries: the same, for launchers whose own options start with --n
    ap.add_argument("--n", "--rows", dest="n", type=int, default=1_000_000)
    ap.add_argument("--nq", "--queries", dest="nq", type=int, default=10_000)
    ap.add_argument("--ef", type=int, default=0, help="fixed ef (skip the sweep)")
    ap.add_argument("--target-recall", type=float, default=0.95)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", action="store_true", help="only run the timed loop (for ncu)")
    ap.add_argument("--profile-precision", default="fp32", choices=["fp32", "bf16", "fp8"],
                    help="traversal precision of --profile-steps")
    ap.add_argument("--profile-learned", type=float, default=None, metavar="LOGIT",
                    help="train the termination network, then only run the learned + FP8 loop with this logit "
                         "threshold at ef = --term-cap (for ncu; no calibration sweep)")
    ap.add_argument("--tie-order", default="reference", choices=["reference", "id"],
                    help="tie order of --profile-steps: reference (heap replay, results identical to hnswlib) "
                         "or id (ties by internal id)")
    ap.add_argument("--train-queries", type=int, default=12_000, help="learned termination: training queries")
    ap.add_argument("--term-cap", type=int, default=96, help="learned termination: ef of the training traces")
    ap.add_argument("--term-period", type=int, default=4, help="learned termination: expansions per checkpoint")
    ap.add_argument("--rerank", type=int, default=0, help="FP8 beam: candidates re-ranked in FP32 (0: the pool)")
    ap.add_argument("--workload", default="gmm1m128", choices=["gmm1m128", "bf768", "serve768", "learned96"],
                    help="gmm1m128: the HNSW headline (default); bf768: tensor-core brute force, 1M x 768 IP, "
                         "k=100, over-fetch 400, recall against float64 exact top-k; serve768: serving mix on a "
                         "1M x 768 IP HNSW index (5%% deleted, 30%% filtered, k in {1,10,100}, ef in 32..512, "
                         "learned stop, Poisson arrivals); learned96: learned termination vs fixed ef on the "
                         "heterogeneous 96-d mixture (M=32, ef_construction=400, ef cap 512)")
    ap.add_argument("--serve-rates-mix", type=int, nargs="*", default=[5_000, 50_000, 200_000],
                    help="serve768: Poisson arrival rates (requests/s)")
    ap.add_argument("--serve-rates", type=int, nargs="*", default=[200_000, 1_000_000],
                    help="Poisson arrival rates (requests/s) of the serving-latency measurement")
    return ap.parse_args()


# ----------------------------------------------------------------- plumbing
class Dist:
    """One process per GPU (replicas: no data-path collective).  The process
    group only times the run: a barrier around the timed region and the max
    over ranks.  NCCL on GPUs; gloo when the backend is given as "gloo" (the
    CPU tests of this plumbing)."""

    def __init__(self, n_gpus, backend: str = "nccl", timeout_s: int = 600):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                        device_id=torch.device("cuda", self.local))
            else:
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
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
        raise SystemExit("the reference extension (oracle/_ref) is not built: run `make -C oracle ref REF=<hnswlib source tree>`")
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
class DeviceLoop:
    """Device-resident batch search through the C ABI (HNSWGPU_DEVICE_PTRS):
    queries and outputs stay in HBM; one kernel launch per step (two for the
    reference tie order, whose two-pass search lists then replays)."""

    def __init__(self, idx, q, dev, k=10):
        import torch
        from hnsw_rabitq_b200 import _capi
        self.idx, self.k, self.nq, self.dev = idx, k, q.shape[0], dev
        self.lib, self.capi = _capi.lib(), _capi
        self.stream = torch.cuda.Stream(device=dev)
        self.dq = torch.from_numpy(q).to(f"cuda:{dev}")
        self.dl = torch.empty((self.nq, k), dtype=torch.int64, device=f"cuda:{dev}")
        self.dd = torch.empty((self.nq, k), dtype=torch.float32, device=f"cuda:{dev}")
        self.dc = torch.empty((self.nq,), dtype=torch.int32, device=f"cuda:{dev}")

    def opts(self, ef, flags=0, precision=0, rerank=0):
        o = self.capi.SearchOpts()
        o.flags = self.capi.DEVICE_PTRS | flags
        o.ef, o.precision, o.rerank = ef, precision, rerank
        o.stream = self.stream.cuda_stream
        return o

    def step(self, o):
        import ctypes as C
        self.capi.check(self.lib.hnswgpu_search(self.idx._h, C.c_void_p(self.dq.data_ptr()), self.nq, self.k,
                                                C.byref(o), C.c_void_p(self.dl.data_ptr()),
                                                C.c_void_p(self.dd.data_ptr()), C.c_void_p(self.dc.data_ptr())))

    def labels(self):
        self.stream.synchronize()  # the search ran on this (non-blocking) stream
        return self.dl.cpu().numpy().view(np.uint64)

    def time(self, o, steps, warmup, dist, clocks=False):
        """ms per step (max over ranks), CUDA events on the launch stream."""
        import torch
        with torch.cuda.stream(self.stream):
            for _ in range(warmup):
                self.step(o)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clk = ClockSampler(self.dev) if clocks else None
        if clk:
            clk.__enter__()
        with torch.cuda.stream(self.stream):
            ev0.record(self.stream)
            for _ in range(steps):
                self.step(o)
            ev1.record(self.stream)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__()
        dist.barrier()
        return dist.max(ev0.elapsed_time(ev1)) / steps, (clk.summary() if clk else None)


def e2e_qps(idx, q, o_flags, ef, precision, rerank, steps, warmup, dist, expect, k=10):
    """Same search through the public C ABI with pinned HOST buffers: the
    call copies the queries in, searches and copies labels / distances /
    counts out every step (wall clock, max over ranks)."""
    import ctypes as C

    import torch
    from hnsw_rabitq_b200 import _capi
    lib = _capi.lib()
    nq = q.shape[0]
    hq = torch.from_numpy(q).pin_memory()
    hl = torch.empty((nq, k), dtype=torch.int64).pin_memory()
    hd = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    hc = torch.empty((nq,), dtype=torch.int32).pin_memory()
    o = _capi.SearchOpts()
    o.flags, o.ef, o.precision, o.rerank = o_flags, ef, precision, rerank

    def call():
        _capi.check(lib.hnswgpu_search(idx._h, C.c_void_p(hq.data_ptr()), nq, k, C.byref(o),
                                       C.c_void_p(hl.data_ptr()), C.c_void_p(hd.data_ptr()),
                                       C.c_void_p(hc.data_ptr())))

    for _ in range(warmup):
        call()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        call()
    dt = dist.max(time.perf_counter() - t0)
    assert np.array_equal(hl.numpy().view(np.uint64), expect)
    return dist.world * nq * steps / dt, int(q.nbytes), int(nq * k * 8 + nq * k * 4 + nq * 4)


def e2e_pipelined_qps(idx, q, o_flags, ef, precision, rerank, steps, warmup, dist, expect, k=10):
    """The same search through the public C ABI's asynchronous form
    (HNSWGPU_DEVICE_PTRS on a caller stream), as a throughput client drives
    it: every step copies its queries in from pinned host memory and reads
    its labels / distances / counts back into pinned host memory, inside the
    timed region, with double buffers on three streams, so that step i + 1's
    copy-in and step i - 1's read-back overlap step i's search (wall clock,
    max over ranks)."""
    import ctypes as C

    import torch
    from hnsw_rabitq_b200 import _capi
    lib = _capi.lib()
    nq, dim = q.shape
    dev = torch.cuda.current_device()
    hq = torch.from_numpy(q).pin_memory()
    hl = [torch.empty((nq, k), dtype=torch.int64).pin_memory() for _ in range(2)]
    hd = [torch.empty((nq, k), dtype=torch.float32).pin_memory() for _ in range(2)]
    hc = [torch.empty((nq,), dtype=torch.int32).pin_memory() for _ in range(2)]
    dq = [torch.empty((nq, dim), dtype=torch.float32, device=dev) for _ in range(2)]
    dl = [torch.empty((nq, k), dtype=torch.int64, device=dev) for _ in range(2)]
    dd = [torch.empty((nq, k), dtype=torch.float32, device=dev) for _ in range(2)]
    dc = [torch.empty((nq,), dtype=torch.int32, device=dev) for _ in range(2)]
    s_in, s_run, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_run = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    o = _capi.SearchOpts()
    o.flags, o.ef, o.precision, o.rerank = _capi.DEVICE_PTRS | o_flags, ef, precision, rerank
    o.stream = s_run.cuda_stream

    def step(i):
        b = i & 1
        s_in.wait_event(ev_run[b])  # the search of step i - 2 has read dq[b]
        with torch.cuda.stream(s_in):
            dq[b].copy_(hq, non_blocking=True)
            ev_in[b].record(s_in)
        s_run.wait_event(ev_in[b])
        s_run.wait_event(ev_out[b])  # step i - 2's results have left dl[b]
        _capi.check(lib.hnswgpu_search(idx._h, C.c_void_p(dq[b].data_ptr()), nq, k, C.byref(o),
                                       C.c_void_p(dl[b].data_ptr()), C.c_void_p(dd[b].data_ptr()),
                                       C.c_void_p(dc[b].data_ptr())))
        ev_run[b].record(s_run)
        s_out.wait_event(ev_run[b])
        with torch.cuda.stream(s_out):
            hl[b].copy_(dl[b], non_blocking=True)
            hd[b].copy_(dd[b], non_blocking=True)
            hc[b].copy_(dc[b], non_blocking=True)
            ev_out[b].record(s_out)

    for i in range(warmup):
        step(i)
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    for i in range(steps):
        step(i)
    torch.cuda.synchronize()
    dt = dist.max(time.perf_counter() - t0)
    for b in range(min(2, steps)):
        assert np.array_equal(hl[b].numpy().view(np.uint64), expect)
    return dist.world * nq * steps / dt


def plain_sweep(idx, loop, q, gt, target, tie_order, fixed_ef=0, precision=0, dist=None):
    """Every ef of the sweep, timed (5 steps after 2 warm-up steps, device
    events): recall@10 and QPS per ef.  Returns the smallest ef whose
    recall meets the target, the flags and the curve."""
    from hnsw_rabitq_b200 import _capi
    flags = _capi.EXACT_TIES if tie_order == "reference" else 0
    sweep, ef_star = [], fixed_ef
    for ef in ([fixed_ef] if fixed_ef else EFS):
        o = loop.opts(ef, flags, precision)
        loop.step(o)
        r = recall(loop.labels(), gt) if gt is not None else None
        ms, _ = loop.time(o, 5, 2, dist or _Solo())
        sweep.append({"ef": ef, "recall": None if r is None else round(r, 5),
                      "qps": round(loop.nq / (ms / 1e3), 1)})
        if r is not None and r >= target and not ef_star:
            ef_star = ef
    return (ef_star or EFS[-1]), flags, sweep


def train_termination(idx, args):
    """Learned termination for the FP8 beam: trained on queries drawn from the
    same mixture (a stream disjoint from the evaluation queries), cap and
    threshold calibrated on a held-out share of them."""
    from hnsw_rabitq_b200 import learned
    from hnsw_rabitq_b200.datasets import gmm_1m_128_queries
    tq = gmm_1m_128_queries(args.train_queries, stream_seed=1000)
    t0 = time.perf_counter()
    model, rep = learned.fit(idx, tq, k=10, ef_cap=args.term_cap, period=args.term_period,
                             target_recall=args.target_recall, precision="fp8", rerank=args.rerank,
                             epochs=20, seed=0)
    return model, rep, tq, time.perf_counter() - t0


def run_ours(args, dist: Dist):
    import torch

    from hnsw_rabitq_b200 import Index, _capi, learned

    dev = dist.local
    torch.cuda.set_device(dev)
    x, q = workload(args.n, args.nq)
    path = ensure_index(x, dist)
    gt = None if args.profile_steps else ground_truth(x, q)
    idx = Index("l2", 128)
    idx.device = dev
    idx.load_index(path)
    info = idx._info()
    _capi.check(_capi.lib().hnswgpu_build_traversal_copy(idx._h, _capi.PREC_FP8))
    loop = DeviceLoop(idx, q, dev)
    nq, k = q.shape[0], 10
    if args.profile_learned is not None:
        from hnsw_rabitq_b200.datasets import gmm_1m_128_queries
        tq = gmm_1m_128_queries(args.train_queries, stream_seed=1000)
        tgt = idx.knn_query_exact(tq, 10)[0]
        ck = learned.traces(idx, tq, 10, args.term_cap, args.term_period,
                            max(16, 2 * args.term_cap // args.term_period + 8), "fp8", args.rerank)
        params, _ = learned.train(*learned.checkpoint_dataset(idx, ck, tgt), epochs=20, seed=0)
        idx.set_termination_model(learned.TerminationModel(params, args.term_period, args.profile_learned,
                                                           args.term_cap, "fp8", args.rerank))
        loop.time(loop.opts(args.term_cap, _capi.LEARNED_STOP, _capi.PREC_FP8, args.rerank), args.steps,
                  args.warmup, dist)
        return None
    if args.profile_steps:
        if not args.ef:
            raise SystemExit("--profile-steps needs --ef")
        prec = {"fp32": 0, "bf16": 1, "fp8": 2}[args.profile_precision]
        tie = _capi.EXACT_TIES if args.tie_order == "reference" and prec == 0 else 0
        loop.time(loop.opts(args.ef, tie, prec), args.steps, args.warmup, dist)
        return None

    # ---- plain FP32 beam (the comparison), both tie orders
    plain = {}
    rows = {}
    for order in ("id", "reference"):
        ef_p, fl_p, sw = plain_sweep(idx, loop, q, gt, args.target_recall, order, args.ef, dist=dist)
        o = loop.opts(ef_p, fl_p)
        loop.step(o)
        lab_p = loop.labels()
        rows[order] = lab_p
        ms_p, _ = loop.time(o, args.steps, args.warmup, dist)
        plain[order] = {"ef": ef_p, "recall@10": round(recall(lab_p, gt), 5), "ms_per_step": round(ms_p, 4),
                        "qps": round(dist.world * nq / (ms_p / 1e3), 1), "sweep": sw}
        if order == "reference":
            # the same results by the one-pass heap replay of every query (the
            # default replays only the queries whose id-order run met a tie)
            o = loop.opts(ef_p, fl_p | _capi.REPLAY_ALL)
            loop.step(o)
            same = bool(np.array_equal(loop.labels(), lab_p))
            ms_r, _ = loop.time(o, args.steps, args.warmup, dist)
            plain[order]["replay_all"] = {"ms_per_step": round(ms_r, 4), "qps": round(dist.world * nq / (ms_r / 1e3), 1),
                                          "same_labels": same}

    # the parity contract: the reference tie order returns hnswlib's own
    # results; the id order differs only where distances tie exactly
    same_rows = float(np.mean(np.all(rows["id"] == rows["reference"], axis=1))) \
        if plain["id"]["ef"] == plain["reference"]["ef"] else None
    plain["id"]["rows_identical_to_reference_order"] = None if same_rows is None else round(same_rows, 5)

    # ---- fp8 traversal at fixed ef (the learned stop's fallback), swept
    ef_f, _, sw_f = plain_sweep(idx, loop, q, gt, args.target_recall, "id", 0, precision=_capi.PREC_FP8,
                                dist=dist)

    # ---- learned termination + FP8 traversal + FP32 re-rank (the headline).
    # Trained and calibrated on training-stream queries; a second held-out
    # stream (never the evaluation queries) checks the calibrated recall and,
    # if it falls short, tightens the calibration target (no retraining).
    model, rep, tq, fit_s = train_termination(idx, args)
    flags = _capi.LEARNED_STOP
    from hnsw_rabitq_b200.datasets import gmm_1m_128_queries
    vq = gmm_1m_128_queries(5000, stream_seed=2000)
    vgt = idx.knn_query_exact(vq, 10)[0]
    hold = tq[: max(1, len(tq) // 3)]
    hgt = idx.knn_query_exact(hold, 10)[0]
    tgt = args.target_recall
    val_rec = None
    for _ in range(6):
        vl, _, _, _ = idx.knn_query_traced(vq, 10, ef=model.ef_cap, tie_order="id", precision="fp8",
                                           rerank=args.rerank, learned=np.isfinite(model.threshold))
        val_rec = recall(vl, vgt)
        if val_rec >= args.target_recall:
            break
        tgt += 0.005
        cap, thr, _ = learned.calibrate(idx, hold, hgt, 10, model, tgt, caps=sorted({c for c, *_ in rep["curve"]}))
        model.ef_cap, model.threshold = cap, thr
        idx.set_termination_model(model)
    o = loop.opts(model.ef_cap, flags, _capi.PREC_FP8, args.rerank)
    loop.step(o)
    lab = loop.labels()
    rec = recall(lab, gt)
    ms_step, clk = loop.time(o, args.steps, args.warmup, dist, clocks=True)
    value = dist.world * nq * args.steps / (ms_step * args.steps / 1e3)
    _, _, _, trace = idx.knn_query_traced(q, 10, ef=model.ef_cap, tie_order="id", precision="fp8",
                                          rerank=args.rerank, learned=True)
    e2e_sync, h2d, d2h = e2e_qps(idx, q, flags, model.ef_cap, _capi.PREC_FP8, args.rerank, args.steps, args.warmup,
                                 dist, lab)
    e2e = e2e_pipelined_qps(idx, q, flags, model.ef_cap, _capi.PREC_FP8, args.rerank, args.steps, args.warmup,
                            dist, lab)
    latency = serving_latency(idx, q, model, args, lab)

    out = None
    if dist.rank == 0:
        peak, peak_kind = peaks()
        # algorithmic bytes of the headline kernel from its own work counters:
        # upper-layer link lists (4 + 4 maxM) and float32 rows; level-0 link
        # lists (4 + 4 maxM0) and fp8 rows (128 B + 16 B scale block); the
        # float32 re-rank of the pool (at most ef_cap rows of 512 B)
        fp8_row = 128 + 8  # e4m3 data, scale and squared norm of the dequantized row
        rr = args.rerank or model.ef_cap
        bq = (trace[:, 0] * (4 + 4 * info.maxM) + trace[:, 1] * fp8_row + trace[:, 2] * (4 + 4 * info.maxM0)
              + trace[:, 3] * fp8_row).mean() + min(rr, model.ef_cap) * 512
        achieved = bq * nq / (ms_step / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                # with threshold +inf the calibrated search is the plain fp8 beam
                "traffic": committed_traffic("learned_fp8" if np.isfinite(model.threshold) else "fp8",
                                             model.ef_cap),
                "traffic_source": "committed ncu capture (profiles/), not measured in this run",
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_query": round(float(bq), 1),
                "kernel": "hnsw_lean_kernel<L2, fp8 traversal, " +
                          ("learned stop>" if np.isfinite(model.threshold) else "fixed ef (calibrated: no stop)>")}
        cpu, bytes_q = (cpu_baseline(args, path, q, plain["id"]["ef"], info) if not args.no_cpu_baseline
                        else (None, None))
        if bytes_q:
            ms_id = plain["id"]["ms_per_step"]
            plain["id"]["roofline_hbm_frac"] = round(bytes_q * nq / (ms_id / 1e3) / 1e9 / peak, 4)
            plain["id"]["algorithmic_bytes_per_query"] = round(bytes_q, 1)
        out = {
            "metric": "QPS at recall@10>=0.95, learned termination + FP8 traversal (FP32 re-rank) GPU HNSW, "
                      "1M x 128 L2",
            "value": round(value, 1), "unit": "queries/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp8 traversal, f32 accumulation and re-rank", "data": "synthetic",
            "config": {"workload": gmm128_label(args),
                       "method": (f"learned early termination ({learned.F}-64-64-1 fp16 MLP every "
                                  f"{model.period} expansions) over an fp8 e4m3 per-row-scaled beam, fp32 re-rank")
                       if np.isfinite(model.threshold) else
                       ("fixed ef: the calibrated logit threshold is +inf (the network never stops a query "
                        "earlier than the cap), fp8 e4m3 per-row-scaled beam, fp32 re-rank"),
                       "ef_cap": model.ef_cap, "logit_threshold": model.threshold,
                       "recall@10": round(rec, 5), "validation_recall@10": round(val_rec, 5),
                       "calibration_target": round(tgt, 4),
                       "mean_l0_expansions": round(float(trace[:, 2].mean()), 2),
                       "global_batch": nq, "parallelism": f"replicas x{dist.world}",
                       "l2_flush": "not needed: index data 640 MB + fp8 copy 144 MB > 126 MB L2",
                       "index_device_bytes": int(idx._info().device_bytes),
                       "training": {"queries": int(tq.shape[0]), "samples": rep["samples"],
                                    "positive_share": round(rep["positive"], 4),
                                    "loss_first_last": [round(rep["loss"][0], 4), round(rep["loss"][-1], 4)],
                                    "trained_cap": rep["trained_cap"], "fit_seconds": round(fit_s, 1)}},
            "plain_fp32": plain,
            "parity_contract_arm": "plain_fp32.reference (results identical to hnswlib's searchKnn, "
                                   "including exact ties)",
            "fp8_fixed_ef": {"ef": ef_f, "sweep": sw_f},
            "speedup_vs_plain_fp32": {o2: round(value / plain[o2]["qps"], 3) for o2 in plain},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e, 1), "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "mode": "public C ABI, asynchronous form on a caller stream: every step copies its queries "
                            "in from pinned host memory and its results out to pinned host memory inside the "
                            "timed region; double buffers on three streams overlap step i+1's copy-in and step "
                            "i-1's read-back with step i's search"},
            "e2e_sync": {"value": round(e2e_sync, 1), "unit": "queries/s", "h2d_bytes_per_step": h2d,
                         "d2h_bytes_per_step": d2h,
                         "mode": "public C ABI, synchronous host-pointer call (copy in, search, copy out, "
                                 "synchronise) per step"},
            "gpu_launches": args.steps,
            "clocks": clk,
            "latency": latency,
        }
    return out


def serving_latency(idx, q, model, args, expect):
    """Per-request latency through the serving loop (continuous batching):
    the evaluation queries arrive one by one as a Poisson process and are
    submitted natively at their arrival times, each with the headline
    configuration (k=10, learned stop, FP8 beam, cap ef); latency = submission
    to results on the host."""
    from hnsw_rabitq_b200.serving import Server, poisson_arrivals
    out = []
    req = Server.request(k=10, ef=model.ef_cap, learned=True, precision="fp8", rerank=args.rerank)
    with Server(idx) as srv:
        srv.replay(q[:2000], [req] * 2000, poisson_arrivals(2000, 200_000, seed=11))  # warm-up
        for rate in args.serve_rates:
            srv.stats(reset=True)
            arr = poisson_arrivals(q.shape[0], rate, seed=rate)
            t0 = time.perf_counter()
            lab, _, cnt, lat = srv.replay(q, [req] * q.shape[0], arr)
            wall = time.perf_counter() - t0
            st = srv.stats()
            assert np.array_equal(lab, expect)  # same results as the batch launch
            out.append({"arrival_rate_qps": rate, "p50_us": round(float(np.percentile(lat, 50)), 1),
                        "p99_us": round(float(np.percentile(lat, 99)), 1),
                        "mean_us": round(float(lat.mean()), 1), "served_qps": round(q.shape[0] / wall, 1),
                        "mean_batch": round(st["mean_batch"], 2), "requests": int(q.shape[0])})
    return out


def measured_tflops():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def run_bf768(args, dist: Dist):
    """Tensor-core brute force on 1,000,000 unit vectors (dim 768, 256-component
    mixture, inner product), 10,000 queries, k = 100, over-fetch 4 k = 400,
    float32 re-rank; recall against the float64 exact top-100."""
    import ctypes as C

    import torch

    from hnsw_rabitq_b200 import BFIndex, _capi
    from hnsw_rabitq_b200.datasets import gmm_unit_ip
    from hnsw_rabitq_b200.groundtruth import fp64_distances, fp64_topk
    dev = dist.local
    torch.cuda.set_device(dev)
    n = args.n
    x, q = gmm_unit_ip(n=n, nq=args.nq, dim=768)
    g = BFIndex("ip", 768)
    g.device = dev
    g.init_index(n)
    g.add_items(x)
    g._sync()  # upload the rows now, outside any timed region
    del x
    k, R = 100, 400
    if not args.profile_steps:
        t0 = time.perf_counter()
        gt, d64, cert = fp64_topk(g, q, k)
        gt_s = time.perf_counter() - t0
    lib = _capi.lib()
    nq = q.shape[0]
    dq = torch.from_numpy(q).to(f"cuda:{dev}")
    dl = torch.empty((nq, k), dtype=torch.int64, device=f"cuda:{dev}")
    dd = torch.empty((nq, k), dtype=torch.float32, device=f"cuda:{dev}")
    dc = torch.empty((nq,), dtype=torch.int32, device=f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)

    def timed(prec, steps, warmup):
        o = _capi.SearchOpts()
        o.flags, o.precision, o.rerank, o.stream = _capi.DEVICE_PTRS, prec, R, stream.cuda_stream
        call = lambda: _capi.check(lib.hnswgpu_search(g._h, C.c_void_p(dq.data_ptr()), nq, k, C.byref(o),
                                                      C.c_void_p(dl.data_ptr()), C.c_void_p(dd.data_ptr()),
                                                      C.c_void_p(dc.data_ptr())))
        for _ in range(warmup):
            call()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            call()
        ev1.record(stream)
        torch.cuda.synchronize()
        stream.synchronize()
        return ev0.elapsed_time(ev1) / steps, dl.cpu().numpy().view(np.uint64), dd.cpu().numpy()

    if args.profile_steps:  # one tensor-core form (for ncu): fp8 with --profile-precision fp8, else bf16
        timed(_capi.PREC_FP8 if args.profile_precision == "fp8" else _capi.PREC_BF16, args.steps, args.warmup)
        return None
    peak, kind = measured_tflops()
    arms = {}
    for name, prec in (("bf16", _capi.PREC_BF16), ("fp8", _capi.PREC_FP8)):
        ms, lab, dist_ = timed(prec, args.steps, args.warmup)
        r = float(np.mean([len(np.intersect1d(lab[i], gt[i])) for i in range(nq)]) / k)
        d64r = fp64_distances(g, q, lab)
        err = np.abs(dist_.astype(np.float64) - d64r) / np.maximum(np.abs(d64r), 1e-30)
        flops = 2.0 * nq * n * 768
        arms[name] = {"qps": round(nq / (ms / 1e3), 1), "ms_per_step": round(ms, 3), "recall@100_vs_fp64": round(r, 5),
                      "max_rel_err_vs_fp64": float(err.max()), "mean_rel_err_vs_fp64": float(err.mean()),
                      "tensor_tflops": round(flops / (ms / 1e3) / 1e12, 1),
                      "frac_of_bf16_peak": round(flops / (ms / 1e3) / 1e12 / peak, 4)}
    ms32, lab32, _ = timed(_capi.PREC_FP32, 1, 1)
    r32 = float(np.mean([len(np.intersect1d(lab32[i], gt[i])) for i in range(nq)]) / k)
    best = arms["fp8"] if arms["fp8"]["qps"] > arms["bf16"]["qps"] else arms["bf16"]
    return {"metric": "QPS at recall@100 vs float64 exact top-100, tensor-core brute force (bf16 / fp8 scores, "
                      "fp32 re-rank), 1M x 768 IP",
            "value": best["qps"], "unit": "queries/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": best["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 / fp8 e4m3 tensor-core scores, f32 re-rank", "data": "synthetic",
            "config": {"workload": f"gmm_unit_ip: {n:,} x 768 unit vectors (256-component mixture, noise norm 0.3), "
                                   f"{args.nq:,} queries, inner product, k=100, over-fetch 400",
                       "fp64_gt_seconds": round(gt_s, 1), "fp64_gt_certified": float(cert.mean())},
            "arms": arms,
            "exact_fp32": {"qps": round(nq / (ms32 / 1e3), 1), "ms_per_step": round(ms32, 2),
                           "recall@100_vs_fp64": round(r32, 5)},
            "roofline": {"bound": "tensor", "achieved": best["tensor_tflops"], "peak": peak, "unit": "TFLOP/s",
                         "frac": best["frac_of_bf16_peak"], "traffic": None,
                         "peak_source": f"{kind} bf16 (MEASURED_PEAKS.json bf16_tflops); fp8 nominal peak is 2x"},
            # per search call: query prep, sample-helper gather, threshold
            # pass, scores pass, select + re-rank
            "gpu_launches": 5 * args.steps}


def ensure_index_ip768(x, dist):
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"unit_{x.shape[0]}_768_ip_M16_efc200.bin")
    if dist.rank == 0 and not os.path.exists(path):
        hnswlib = ref_module()
        t = time.time()
        p = hnswlib.Index("ip", 768)
        p.init_index(x.shape[0], M=16, ef_construction=200, random_seed=100)
        p.add_items(x, num_threads=os.cpu_count())
        p.save_index(path + ".tmp")
        os.replace(path + ".tmp", path)
        print(f"[bench] built reference index in {time.time() - t:.1f}s -> {path}", file=sys.stderr)
    dist.barrier()
    return path


def run_serve768(args, dist: Dist):
    """Serving mix (continuous batching) on a reference-built HNSW index over
    1,000,000 x 768 unit vectors (inner product, M=16, ef_construction=200):
    5 % of labels deleted, 30 % of requests with a label-parity filter, k
    uniform over {1, 10, 100}, ef over {32, 64, 128, 256, 512}, learned
    termination enabled; Poisson arrivals; latency = submission to results
    on the host; recall@k against the exact scan of the admissible rows."""
    import torch

    from hnsw_rabitq_b200 import Index, learned
    from hnsw_rabitq_b200.datasets import gmm_unit_ip
    from hnsw_rabitq_b200.serving import Server, poisson_arrivals
    dev = dist.local
    torch.cuda.set_device(dev)
    n = args.n
    x, q = gmm_unit_ip(n=n, nq=args.nq, dim=768)
    path = ensure_index_ip768(x, dist)
    del x
    idx = Index("ip", 768)
    idx.device = dev
    idx.load_index(path)
    rng = np.random.default_rng(5)
    for lab in rng.choice(n, n // 20, replace=False):
        idx.mark_deleted(int(lab))
    # learned termination for the general (delete / filter aware) beam
    _, tq = gmm_unit_ip(n=0, nq=8000, dim=768, query_seed=1000)
    t0 = time.perf_counter()
    model, rep = learned.fit(idx, tq, k=10, ef_cap=128, period=4, target_recall=0.95, precision="fp32",
                             epochs=20, seed=0, caps=[128])
    fit_s = time.perf_counter() - t0
    idx.set_termination_model(model)
    # the request mix and its ground truth
    nq = q.shape[0]
    ks = rng.choice([1, 10, 100], nq)
    efs = rng.choice([32, 64, 128, 256, 512], nq)
    filt = rng.random(nq) < 0.3
    gt = np.empty((nq, 100), np.uint64)
    gt[~filt] = idx.knn_query_exact(q[~filt], 100)[0]
    gt[filt] = idx.knn_query_exact(q[filt], 100, filter=lambda l: l % 2 == 0)[0]
    lines = []
    with Server(idx) as srv:
        parity = srv.add_filter(lambda l: l % 2 == 0)
        reqs = [Server.request(k=int(ks[i]), ef=int(efs[i]), filter=parity if filt[i] else -1, learned=True)
                for i in range(nq)]
        srv.replay(q[:2000], reqs[:2000], poisson_arrivals(2000, 50_000, seed=3))  # warm-up
        for rate in args.serve_rates_mix:
            srv.stats(reset=True)
            t0 = time.perf_counter()
            lab, _, cnt, lat = srv.replay(q, reqs, poisson_arrivals(nq, rate, seed=rate))
            wall = time.perf_counter() - t0
            st = srv.stats()
            hits = [len(np.intersect1d(lab[i, :ks[i]], gt[i, :ks[i]])) / ks[i] for i in range(nq)]
            lines.append({"arrival_rate_qps": rate, "served_qps": round(nq / wall, 1),
                          "p50_us": round(float(np.percentile(lat, 50)), 1),
                          "p99_us": round(float(np.percentile(lat, 99)), 1), "mean_batch": round(st["mean_batch"], 2),
                          "recall@k": round(float(np.mean(hits)), 4)})
    top = lines[-1]
    return {"metric": "serving mix p99 latency (continuous batching, learned stop), 1M x 768 IP HNSW",
            "value": top["p99_us"], "unit": "us", "n_gpus": dist.world, "steps": len(lines), "warmup": 1,
            "ms_per_step": None, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"gmm_unit_ip {n:,} x 768 inner product, reference-built HNSW M=16 efc=200; "
                                   f"5% of labels deleted; {args.nq:,} requests: k in {{1,10,100}}, ef in {{32..512}}, "
                                   "30% label-parity filter, learned termination (trained cap 128)",
                       "termination": {"threshold": model.threshold, "samples": rep["samples"],
                                       "fit_seconds": round(fit_s, 1)}},
            "rates": lines, "gpu_launches": None}


def run_learned96(args, dist: Dist):
    """Learned termination on the mixture with per-component sigma log-uniform
    in [0.05, 0.5] (queries of very different difficulty): n x 96 L2,
    reference-built HNSW M=32, ef_construction=400, k=10, ef cap 512.  QPS at
    recall@10 >= target of the plain fixed-ef beam (smallest ef of the sweep)
    and of the learned stop (cap and threshold calibrated on held-out
    training queries), over float32 rows and over the fp8 copy (the lean
    beam, one 64-slot link row per iteration for M = 32) with a float32
    re-rank."""
    import torch

    from hnsw_rabitq_b200 import Index, _capi, learned
    from hnsw_rabitq_b200.datasets import gmm_lognormal_sigma
    dev = dist.local
    torch.cuda.set_device(dev)
    n = args.n
    x, q = gmm_lognormal_sigma(n=n, nq=args.nq, dim=96)
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"lognormal_{n}_96_M32_efc400.bin")
    if dist.rank == 0 and not os.path.exists(path):
        hnswlib = ref_module()
        t = time.time()
        p = hnswlib.Index("l2", 96)
        p.init_index(n, M=32, ef_construction=400, random_seed=100)
        p.add_items(x, num_threads=os.cpu_count())
        p.save_index(path + ".tmp")
        os.replace(path + ".tmp", path)
        print(f"[bench] built reference index in {time.time() - t:.1f}s -> {path}", file=sys.stderr)
    dist.barrier()
    del x
    idx = Index("l2", 96)
    idx.device = dev
    idx.load_index(path)
    gt = idx.knn_query_exact(q, 10)[0]
    loop = DeviceLoop(idx, q, dev)
    nq = q.shape[0]
    target = args.target_recall
    sweep, ef_p = [], None
    for ef in [16, 24, 32, 40, 48, 56, 64, 80, 96, 128, 160, 192, 256, 320, 384, 448, 512]:
        loop.step(loop.opts(ef))
        r = recall(loop.labels(), gt)
        sweep.append({"ef": ef, "recall": round(r, 5)})
        if r >= target:
            ef_p = ef
            break
    ef_p = ef_p or 512
    ms_p, _ = loop.time(loop.opts(ef_p), args.steps, args.warmup, dist)
    _, _, _, tr_p = idx.knn_query_traced(q, 10, ef=ef_p, tie_order="id")
    _, tq = gmm_lognormal_sigma(n=0, nq=args.train_queries, dim=96, query_seed=1000)
    t0 = time.perf_counter()
    model, rep = learned.fit(idx, tq, k=10, ef_cap=512, period=4, target_recall=target, precision="fp32",
                             epochs=20, seed=0)
    fit_s = time.perf_counter() - t0
    tgt = target
    for _ in range(6):
        o = loop.opts(model.ef_cap, _capi.LEARNED_STOP)
        loop.step(o)
        rec = recall(loop.labels(), gt)
        if rec >= target:
            break
        tgt += 0.005
        hold = tq[: max(1, len(tq) // 3)]
        cap, thr, _ = learned.calibrate(idx, hold, idx.knn_query_exact(hold, 10)[0], 10, model, tgt,
                                        caps=sorted({c for c, *_ in rep["curve"]}))
        model.ef_cap, model.threshold = cap, thr
        idx.set_termination_model(model)
    ms_l, clk = loop.time(o, args.steps, args.warmup, dist, clocks=True)
    _, _, _, tr_l = idx.knn_query_traced(q, 10, ef=model.ef_cap, tie_order="id", learned=True)
    qps_l, qps_p = nq / (ms_l / 1e3), nq / (ms_p / 1e3)

    # ---- FP8 traversal + float32 re-rank: fixed ef, then the learned stop
    # (traces at ef 128, labelled by what the re-rank returns; calibrated on
    # measured time, so it falls back to fixed ef when the network does not pay)
    _capi.check(_capi.lib().hnswgpu_build_traversal_copy(idx._h, _capi.PREC_FP8))
    sweep8, ef_8 = [], None
    for ef in [16, 24, 32, 40, 48, 56, 64, 80, 96, 128, 160, 192, 256, 320, 384, 448, 512]:
        loop.step(loop.opts(ef, 0, _capi.PREC_FP8))
        r = recall(loop.labels(), gt)
        sweep8.append({"ef": ef, "recall": round(r, 5)})
        if r >= target:
            ef_8 = ef
            break
    ef_8 = ef_8 or 512
    ms_8, _ = loop.time(loop.opts(ef_8, 0, _capi.PREC_FP8), args.steps, args.warmup, dist)
    _, _, _, tr_8 = idx.knn_query_traced(q, 10, ef=ef_8, tie_order="id", precision="fp8")
    t0 = time.perf_counter()
    model8, rep8 = learned.fit(idx, tq[: min(len(tq), 6000)], k=10, ef_cap=128, period=4, target_recall=target,
                               precision="fp8", epochs=20, seed=0)
    fit8_s = time.perf_counter() - t0
    o8 = loop.opts(model8.ef_cap, _capi.LEARNED_STOP, _capi.PREC_FP8)
    loop.step(o8)
    rec8 = recall(loop.labels(), gt)
    ms_l8, _ = loop.time(o8, args.steps, args.warmup, dist)
    _, _, _, tr_l8 = idx.knn_query_traced(q, 10, ef=model8.ef_cap, tie_order="id", precision="fp8", learned=True)
    fp8 = {"fixed": {"ef": ef_8, "qps": round(nq / (ms_8 / 1e3), 1), "recall@10": sweep8[-1]["recall"],
                     "mean_l0_expansions": round(float(tr_8[:, 2].mean()), 1), "sweep": sweep8},
           "learned": {"ef_cap": model8.ef_cap, "threshold": model8.threshold, "recall@10": round(rec8, 5),
                       "qps": round(nq / (ms_l8 / 1e3), 1),
                       "mean_l0_expansions": round(float(tr_l8[:, 2].mean()), 1), "samples": rep8["samples"],
                       "fit_seconds": round(fit8_s, 1)},
           "speedup_fp8_learned_vs_fp32_plain": round(ms_p / ms_l8, 3)}
    return {"metric": "QPS at recall@10>=0.95, learned termination vs fixed ef, heterogeneous 96-d mixture",
            "value": round(qps_l, 1), "unit": "queries/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_l, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"gmm_lognormal_sigma {n:,} x 96 L2 (4096 components, sigma log-uniform "
                                   "[0.05, 0.5]), reference-built HNSW M=32 efc=400, 10,000 queries, k=10",
                       "learned": {"ef_cap": model.ef_cap, "threshold": model.threshold, "recall@10": round(rec, 5),
                                   "mean_l0_expansions": round(float(tr_l[:, 2].mean()), 1),
                                   "p99_l0_expansions": float(np.percentile(tr_l[:, 2], 99)),
                                   "training_queries": int(tq.shape[0]), "samples": rep["samples"],
                                   "fit_seconds": round(fit_s, 1)},
                       "plain": {"ef": ef_p, "qps": round(qps_p, 1), "recall@10": sweep[-1]["recall"],
                                 "mean_l0_expansions": round(float(tr_p[:, 2].mean()), 1),
                                 "p99_l0_expansions": float(np.percentile(tr_p[:, 2], 99)), "sweep": sweep}},
            "speedup_vs_plain": round(qps_l / qps_p, 3), "fp8": fp8, "clocks": clk, "gpu_launches": args.steps}


def gmm128_label(args):
    """The headline workload's name in the bench line, with its sizes."""
    return (f"gmm_1m_128: {args.n:,} x 128 L2 (1024-comp. GMM, integer-valued), reference-built HNSW M=16 "
            f"efc=200, {args.nq:,} queries, k=10")


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
    return {"impl": "reference",
            "metric": "QPS at recall@10>=0.95, learned termination + FP8 traversal (FP32 re-rank) GPU HNSW, "
                      "1M x 128 L2",
            "value": round(qps, 1), "unit": "queries/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": gmm128_label(args),
                       "method": "hnswlib 0.9.0 knn_query (CPU, fixed ef: the reference has no learned or "
                                 "FP8 search)", "ef": ef_star,
                       "recall@10_sample500": round(recall(lab[:500], gt), 5)},
            "cpu_baseline": {"value": round(qps, 1), "unit": "queries/s", "cores": threads, "kind": "reference",
                             "sample": f"{q.shape[0]} queries per step"},
            "e2e": {"value": round(qps, 1), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


class _Solo:
    """Rank 0 alone, no process group (the reference arm and setup helpers);
    `world` is the launch's rank count, which the reference arm reports."""
    rank = 0
    local = 0

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))

    def barrier(self):
        pass

    def max(self, v: float) -> float:
        return v


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
        out = (run_bf768(args, dist) if args.workload == "bf768" else
               run_serve768(args, dist) if args.workload == "serve768" else
               run_learned96(args, dist) if args.workload == "learned96" else run_ours(args, dist))
    finally:
        dist.close()
    if out is not None and dist.rank == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
