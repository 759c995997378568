"""Benchmark of the exact FP32 top-k search path on B200 (one JSON line on rank 0).

Workload (default): exact FP32 cosine top-k in the memory-bound regime — a base of 1,000,000 ×
768 float32 rows drawn from a 1,024-centre Gaussian mixture (centres ~ N(0, 1), points = centre
+ 0.3·N(0, 1)), unit-normalised and indexed with normalized=true; query batches of 16 drawn from
the same mixture; k = 100. One step = one batch of queries through the fused scan (K1 query prep
→ K2 scan with fused top-k → merge). Batches of 1 and 4 are reported beside it.

  value : queries/s with queries and outputs resident in HBM (device C-ABI entry point);
  e2e   : queries/s through nndex_cuda_search_batch with host buffers (H2D of the queries and
          D2H of the results inside the timed region);
  roofline : the scan kernel's algorithmic bytes per launch (N·D·4 + B·D·4 + B·k·12) ÷ its
          CUDA-event duration, against the measured HBM copy bandwidth;
  cpu_baseline : the CPU restatement of the reference's exact path (oracle/, its Gemm strategy
          for batches, src/cpu.rs:256-284) on the host cores, on a bounded sample.

`--impl reference` times that CPU restatement alone on the same workload (the reference is Rust
and cannot be built here). Under torchrun each rank runs an independent replica on its own GPU
(the path does not shard; one GPU per index), with a barrier around the timed region and the max
of the per-rank times.
"""
from __future__ import annotations

import argparse
import ctypes as C
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

METRIC = "top-k queries/s & % roofline; BF16/FP8+rerank vs FP32 at equal recall@k"


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--rows", type=int, default=1_000_000)
    p.add_argument("--dims", type=int, default=768)
    p.add_argument("--centers", type=int, default=1024)
    p.add_argument("--sigma", type=float, default=0.3)
    p.add_argument("--batch", type=int, default=16)
    p.add_argument("--k", type=int, default=100)
    p.add_argument("--seed", type=int, default=42)
    p.add_argument("--extra-batches", default="1,4", help="batch sizes reported beside the headline")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--autotune", choices=["on", "off"], default="on",
                   help="off: the fixed path rules for the headline index (profiling a given kernel)")
    p.add_argument("--cpu-sample-batches", type=int, default=2)
    p.add_argument("--c1", choices=["on", "off", "only"], default="on",
                   help="the 50,000 x 128 plain exact section (single query and batch 64, k=10)")
    p.add_argument("--c1-calls", type=int, default=300)
    p.add_argument("--mixed", choices=["on", "off", "only"], default="on",
                   help="also measure the mixed-precision workload (BF16/FP8 scan + FP32 rerank vs FP32)")
    p.add_argument("--mixed-rows", type=int, default=10_000_000)
    p.add_argument("--mixed-dims", type=int, default=256)
    p.add_argument("--mixed-centers", type=int, default=4096)
    p.add_argument("--mixed-sigma", type=float, default=0.25)
    p.add_argument("--mixed-batch", type=int, default=4096)
    p.add_argument("--mixed-k", type=int, default=10)
    p.add_argument("--mixed-steps", type=int, default=5)
    p.add_argument("--mixed-oracle-queries", type=int, default=512)
    p.add_argument("--mixed-stride", type=int, default=0,
                   help="fix the tensor-core scans' pass-1 tile stride (installed as the tuner's plan); 0 = tuned")
    p.add_argument("--mixed-qb", type=int, default=0, choices=[0, 1, 2, 3],
                   help="fix the tensor-core pass 2's query blocks per CTA (3 = CTA pairs; installed as the "
                        "tuner's plan); 0 = tuned")
    p.add_argument("--ivf", choices=["on", "off", "only"], default="on",
                   help="also measure the IVF workload (GPU k-means build + probe + ragged list scan)")
    p.add_argument("--ivf-rows", type=int, default=2_000_000)
    p.add_argument("--ivf-dims", type=int, default=384)
    p.add_argument("--ivf-centers", type=int, default=8192)
    p.add_argument("--ivf-zipf", type=float, default=1.1)
    p.add_argument("--ivf-sigma", type=float, default=0.25)
    p.add_argument("--ivf-nlist", type=int, default=1414)
    p.add_argument("--ivf-iters", type=int, default=10)
    p.add_argument("--ivf-seed", type=int, default=42)
    p.add_argument("--ivf-nprobe", default="8,32,64")
    p.add_argument("--ivf-batch", type=int, default=1024)
    p.add_argument("--ivf-k", type=int, default=10)
    p.add_argument("--ivf-steps", type=int, default=10)
    p.add_argument("--ivf-cpu-queries", type=int, default=64)
    p.add_argument("--serve", choices=["on", "off", "only"], default="on",
                   help="also measure the serving loop (Poisson arrivals, continuous batching)")
    p.add_argument("--serve-rows", type=int, default=5_000_000)
    p.add_argument("--serve-dims", type=int, default=512)
    p.add_argument("--serve-centers", type=int, default=2048)
    p.add_argument("--serve-sigma", type=float, default=0.25)
    p.add_argument("--serve-rates", default="20000,50000,100000,200000", help="offered queries/s")
    p.add_argument("--serve-seconds", type=float, default=2.0)
    p.add_argument("--serve-slots", type=int, default=3)
    p.add_argument("--serve-nprobe", type=int, default=32)
    p.add_argument("--serve-latency-ms", type=int, default=100,
                   help="server latency budget: requests are refused while the oldest queued one has waited longer")
    return p.parse_args(argv)


# ---------------------------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------------------------

def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def dist_init(backend: str):
    import torch.distributed as dist
    from datetime import timedelta
    rank, world, _ = dist_env()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend=backend, timeout=timedelta(seconds=120))
    return rank, world


def replica_seed(seed: int, rank: int) -> int:
    """Each replica indexes its own synthetic base (independent objects, no exchange)."""
    return seed + 1000003 * rank


def aggregate(local_ms: float, local_queries: int, world: int, device=None):
    """Max of the per-rank times and the sum of queries over ranks → (max_ms, total_queries)."""
    if world == 1:
        return local_ms, local_queries
    import torch
    import torch.distributed as dist
    t = torch.tensor([local_ms], dtype=torch.float64, device=device)
    q = torch.tensor([float(local_queries)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(q, op=dist.ReduceOp.SUM)
    return float(t.item()), int(q.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------------------------
# synthetic data (seeded; generated on the GPU when one is present)
# ---------------------------------------------------------------------------------------------

def make_mixture(rows, dims, centers, sigma, seed, device, center_seed=None, zipf=None):
    """Unit rows x = c_a + sigma·N(0, I), centres c ~ N(0, I); the centre a is uniform, or drawn with
    power-law (Zipf, exponent `zipf`) cluster sizes."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(center_seed if center_seed is not None else seed)
    c = torch.randn((centers, dims), generator=g, device=device, dtype=torch.float32)
    cdf = None
    if zipf:
        # cluster sizes ∝ rank^-zipf; each row's centre from one uniform draw through the CDF
        # (a plain inverse-CDF lookup: the same rows on every run and GPU configuration)
        w = torch.arange(1, centers + 1, device=device, dtype=torch.float64).pow(-float(zipf))
        cdf = torch.cumsum(w / w.sum(), 0)
    g.manual_seed(seed + 1)
    out = torch.empty((rows, dims), device=device, dtype=torch.float32)
    step = 1 << 18
    for r0 in range(0, rows, step):
        r1 = min(rows, r0 + step)
        if cdf is not None:
            u = torch.rand((r1 - r0,), generator=g, device=device, dtype=torch.float64)
            a = torch.searchsorted(cdf, u).clamp_(max=centers - 1)
        else:
            a = torch.randint(0, centers, (r1 - r0,), generator=g, device=device)
        x = torch.randn((r1 - r0, dims), generator=g, device=device, dtype=torch.float32)
        x.mul_(sigma).add_(c[a])
        x.div_(torch.linalg.vector_norm(x, dim=1, keepdim=True))
        out[r0:r1] = x
    return out


# ---------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(rows, dims, batch, k, kernel=""):
    """DRAM bytes per scan launch from the committed ncu summary (profiles/scan_fp32_traffic.txt),
    scaled to this workload by the rows streamed; the line must be for the same kernel family."""
    family = kernel.split("<")[0].split(" ")[0]
    path = os.path.join(ROOT, "profiles", "scan_fp32_traffic.txt")
    try:
        lines = open(path).read().splitlines()
    except OSError:
        return None
    for line in lines:
        f = line.split()
        if not f or f[0].startswith("#") or len(f) < 6:
            continue
        r, d, b, kk, kern, dram = f[:6]
        if int(d) == dims and int(b) == batch and int(kk) == k and kern.split("<")[0] == family:
            return int(dram) * rows / int(r)
    return None


# ---------------------------------------------------------------------------------------------
# CPU restatement timing (oracle port)
# ---------------------------------------------------------------------------------------------

def cpu_reference_time(base_np, queries_np, k, batches: int):
    from oracle import oracle as O
    O.lib()
    threads = O.num_threads()
    times = []
    for b in range(batches):
        q = queries_np[b % len(queries_np)]
        t0 = time.perf_counter()
        O.bench_search_batch(base_np, q, k)
        times.append(time.perf_counter() - t0)
    return times, threads


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------

def run_ours(args):
    import torch
    from nndex_b200 import _lib, kernel_launch_count
    from nndex_b200._lib import NNDEX_FLAG_NORMALIZED

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rank, world = dist_init("nccl")
    dev = torch.device("cuda", local)
    seed = replica_seed(args.seed, rank)
    L = _lib.lib()
    if args.c1 == "only":
        return {"c1": run_c1(args, dev, L, world)} if rank == 0 else None
    if args.mixed == "only":
        # the mixed-precision section alone (profiling runs of the tensor-core scan)
        mixed = run_mixed(args, dev, L, world)
        return {"mixed_precision": mixed} if rank == 0 else None
    if args.ivf == "only":
        ivf = run_ivf(args, dev, L, world)
        return {"ivf": ivf} if rank == 0 else None
    if args.serve == "only":
        serve = run_serve(args, dev, L, world)
        return {"serving": serve} if rank == 0 else None

    base = make_mixture(args.rows, args.dims, args.centers, args.sigma, seed, dev, center_seed=args.seed)
    opts = _lib.Opts()
    opts.device = local
    h = C.c_void_p()
    st = L.nndex_cuda_create_from_device(base.data_ptr(), base.numel(), args.rows, args.dims,
                                         NNDEX_FLAG_NORMALIZED, C.byref(opts), C.byref(h))
    if st != 0:
        raise RuntimeError(_lib.last_error())
    if args.autotune == "off":
        L.nndex_cuda_set_autotune(h, 0)
    base_host = base.cpu().numpy() if (rank == 0 and not args.no_cpu_baseline) else None
    del base
    torch.cuda.empty_cache()

    batches = [args.batch] + [int(b) for b in args.extra_batches.split(",") if b and int(b) != args.batch]
    pool = 8
    qall = make_mixture(pool * max(batches), args.dims, args.centers, args.sigma, seed + 7, dev,
                        center_seed=args.seed)
    k = min(args.k, args.rows)
    # A dedicated stream: the library launches on it and the CUDA events below are recorded on it.
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    sptr = C.c_void_p(stream.cuda_stream)
    out_i = torch.empty((max(batches), k), dtype=torch.int64, device=dev)
    out_s = torch.empty((max(batches), k), dtype=torch.float32, device=dev)
    out_c = torch.empty((max(batches),), dtype=torch.int32, device=dev)

    def step(b, i):
        q = qall[(i % pool) * b:(i % pool) * b + b]
        r = L.nndex_cuda_search_batch_device(h, q.data_ptr(), b, args.dims, k, out_i.data_ptr(), out_s.data_ptr(),
                                             out_c.data_ptr(), sptr, 0)
        if r != 0:
            raise RuntimeError(_lib.last_error())

    results = {}
    clocks = None
    launches = 0
    for bi, b in enumerate(batches):
        for i in range(args.warmup):
            step(b, i)
        torch.cuda.synchronize(dev)
        L.nndex_cuda_set_scan_timing(h, 1)
        sampler = ClockSampler(local) if bi == 0 else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        barrier(world)
        torch.cuda.synchronize(dev)
        n0 = kernel_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            step(b, i)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        n1 = kernel_launch_count()
        barrier(world)
        if sampler:
            clocks = sampler.stop()
        L.nndex_cuda_set_scan_timing(h, 0)
        ms = e0.elapsed_time(e1)
        scan_ms = C.c_double(0.0)
        scan_n = C.c_uint64(0)
        L.nndex_cuda_scan_timing(h, C.byref(scan_ms), C.byref(scan_n))
        sst = _lib.SearchStats()
        L.nndex_cuda_last_search_stats(h, C.byref(sst))
        serr = score_error_report(L, h, lambda: L.nndex_cuda_search_batch_device(
            h, qall[:b].data_ptr(), b, args.dims, k, out_i.data_ptr(), out_s.data_ptr(), out_c.data_ptr(), sptr, 1))
        max_ms, total_q = aggregate(ms, b * args.steps, world, dev)
        results[b] = {
            "ms_per_step": max_ms / args.steps,
            "queries_per_s": total_q / (max_ms / 1e3),
            "scan_ms": scan_ms.value / max(scan_n.value, 1),
            "launches": n1 - n0,
            "score_error_vs_fp64": serr,
            "kernel": ("scan_tf32_kernel (TF32 candidates + exact FP32 rerank)" if sst.path == 6
                       else f"scan_fp32_wide_kernel<{sst.scan_qb},{sst.scan_wide}>" if sst.scan_wide
                       else f"scan_fp32_kernel<{sst.scan_qb},4>"),
        }
        if bi == 0:
            launches = n1 - n0

    # e2e through the host-buffer C-ABI call (pinned staging inside the library)
    b = args.batch
    qhost = [qall[i * b:(i + 1) * b].cpu().numpy().copy() for i in range(pool)]
    oi = np.zeros((b, k), np.uint64)
    os_ = np.zeros((b, k), np.float32)
    oc = np.zeros(b, np.uint64)

    def host_step(i):
        q = qhost[i % pool]
        r = L.nndex_cuda_search_batch(h, q.ctypes.data, q.size, b, k, oi.ctypes.data, os_.ctypes.data,
                                      oc.ctypes.data)
        if r != 0:
            raise RuntimeError(_lib.last_error())

    for i in range(args.warmup):
        host_step(i)
    barrier(world)
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        host_step(i)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    wall_ms = (time.perf_counter() - t0) * 1e3
    ev_ms = e0.elapsed_time(e1)
    e2e_ms = max(wall_ms, ev_ms)
    e2e_max_ms, e2e_q = aggregate(e2e_ms, b * args.steps, world, dev)
    barrier(world)

    cpu = None
    if rank == 0 and base_host is not None:
        qs = [qall[i * b:(i + 1) * b].cpu().numpy() for i in range(args.cpu_sample_batches)]
        times, threads = cpu_reference_time(base_host, qs, k, args.cpu_sample_batches)
        cpu = {"value": b * len(times) / sum(times), "unit": "queries/s", "cores": threads, "kind": "port",
               "sample": f"{len(times)} batches of {b} queries over the full {args.rows}x{args.dims} base "
                         f"(oracle restatement of src/cpu.rs Gemm strategy, {threads} threads)"}

    L.nndex_cuda_destroy(h)
    del qall
    torch.cuda.empty_cache()
    c1 = run_c1(args, dev, L, world) if args.c1 != "off" else None
    mixed = run_mixed(args, dev, L, world) if args.mixed != "off" else None
    ivf = run_ivf(args, dev, L, world) if args.ivf != "off" else None
    serve = run_serve(args, dev, L, world) if args.serve != "off" else None
    if rank != 0:
        return None
    head = results[args.batch]
    bytes_per_launch = args.rows * args.dims * 4 + args.batch * args.dims * 4 + args.batch * k * 12
    achieved = bytes_per_launch / (head["scan_ms"] / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic(args.rows, args.dims, args.batch, k, head["kernel"])
    line = {
        "metric": METRIC,
        "value": head["queries_per_s"],
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": f"exact-fp32 top-k, base {args.rows}x{args.dims} f32 ({args.centers}-centre Gaussian "
                        f"mixture, sigma={args.sigma}, unit rows, normalized=true), batch {args.batch}, k={k}",
            "rows": args.rows, "dims": args.dims, "batch": args.batch, "k": k,
            "parallelism": f"replicas{world}" if world > 1 else "single-gpu",
            "l2": f"inputs larger than L2 (base {args.rows * args.dims * 4 / 1e9:.2f} GB per step vs 126 MB L2)",
        },
        "e2e": {"value": e2e_q / (e2e_max_ms / 1e3), "unit": "queries/s",
                "h2d_bytes_per_step": b * args.dims * 4, "d2h_bytes_per_step": b * k * 12 + b * 8},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{peak_kind} hbm_gbs",
                     "kernel": head["kernel"],
                     "bytes_per_launch": bytes_per_launch, "avg_launch_ms": head["scan_ms"]},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "c1": c1,
        "mixed_precision": mixed,
        "ivf": ivf,
        "serving": serve,
        "batches": {str(bb): {"queries_per_s": r["queries_per_s"], "ms_per_step": r["ms_per_step"],
                              "scan_ms": r["scan_ms"], "kernel": r["kernel"],
                              "score_error_vs_fp64": r["score_error_vs_fp64"],
                              "hbm_gbs": (args.rows * args.dims * 4 + bb * args.dims * 4 + bb * k * 12)
                              / (r["scan_ms"] / 1e3) / 1e9}
                    for bb, r in results.items()},
    }
    return line


# ---------------------------------------------------------------------------------------------
# plain exact search on 50,000 x 128: the one configuration with published reference numbers
# ---------------------------------------------------------------------------------------------

def l2_copy_gbs(dev, nbytes=24 << 20, iters=200):
    """Copy bandwidth (read + write bytes) of a buffer pair that stays in the 126 MB L2."""
    import torch
    a = torch.empty(nbytes // 4, dtype=torch.float32, device=dev).fill_(1.0)
    b = torch.empty_like(a)
    for _ in range(10):
        b.copy_(a)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(iters):
        b.copy_(a)
    e1.record()
    torch.cuda.synchronize(dev)
    return 2.0 * nbytes * iters / (e0.elapsed_time(e1) / 1e3) / 1e9


def run_c1(args, dev, L, world):
    """50,000 x 128 N(0, 1) (numpy default_rng(42)), normalized=false, k=10: the golden single query
    of the reference's demo notebook and a batch of 64 from the same generator; host-buffer calls
    (the reference-facing API) and device-resident calls, beside the reference's published CPU
    latencies and the CPU restatement on this host."""
    import numpy as np
    import torch
    from nndex_b200 import NNdex, _lib
    from oracle import oracle as O
    rng = np.random.default_rng(42)
    m = rng.normal(size=(50_000, 128)).astype(np.float32)
    q1 = rng.normal(size=(128,)).astype(np.float32)
    q64 = rng.normal(size=(64, 128)).astype(np.float32)
    k = 10
    index = NNdex(m, gpu_device_index=dev.index)
    gi, _ = index.search(q1, k=5)
    golden = gi.tolist() == [43576, 14100, 15993, 35409, 38916]
    if not golden:
        raise RuntimeError(f"50k x 128 golden query answered {gi.tolist()}")
    out = {"golden_top5_matches": golden}
    # host-buffer calls: wall time per call (the latency a caller sees)
    for name, q in (("batch_1", q1), ("batch_64", q64)):
        for _ in range(20):
            index.search(q, k=k)
        lat = []
        for _ in range(args.c1_calls):
            t0 = time.perf_counter()
            index.search(q, k=k)
            lat.append((time.perf_counter() - t0) * 1e3)
        lat = np.array(lat)
        nq = 1 if q.ndim == 1 else q.shape[0]
        out[name] = {"host_call_ms_p50": float(np.median(lat)), "host_call_ms_p99": float(np.percentile(lat, 99)),
                     "host_queries_per_s": nq / (np.median(lat) / 1e3)}
    # device-resident: CUDA events over back-to-back calls on one stream (the base stays in L2)
    stream = torch.cuda.Stream(device=dev)
    sptr = C.c_void_p(stream.cuda_stream)
    l2 = l2_copy_gbs(dev)
    peak, peak_kind = measured_peaks()
    h = index.handle
    for name, q in (("batch_1", q1.reshape(1, -1)), ("batch_64", q64)):
        nq = q.shape[0]
        qd = torch.from_numpy(q).to(dev)
        oi = torch.empty((nq, k), dtype=torch.int64, device=dev)
        os_ = torch.empty((nq, k), dtype=torch.float32, device=dev)

        def call():
            if L.nndex_cuda_search_batch_device(h, qd.data_ptr(), nq, 128, k, oi.data_ptr(), os_.data_ptr(), None,
                                                sptr, 0) != 0:
                raise RuntimeError(_lib.last_error())
        for _ in range(20):
            call()
        torch.cuda.synchronize(dev)
        L.nndex_cuda_set_scan_timing(h, 1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.c1_calls):
                call()
            e1.record(stream)
        torch.cuda.synchronize(dev)
        L.nndex_cuda_set_scan_timing(h, 0)
        scan_ms, scan_n = C.c_double(0.0), C.c_uint64(0)
        L.nndex_cuda_scan_timing(h, C.byref(scan_ms), C.byref(scan_n))
        ms = e0.elapsed_time(e1) / args.c1_calls
        scan = scan_ms.value / max(scan_n.value, 1)
        gbs = 50_000 * 128 * 4 / (scan / 1e3) / 1e9
        st = index.last_search_stats()
        out[name].update({"device_ms_per_call": ms, "device_queries_per_s": nq / (ms / 1e3), "scan_ms": scan,
                          "path": st["path"], "scan_gbs": gbs, "frac_of_hbm": gbs / peak,
                          "frac_of_l2_copy": gbs / l2})
    # the CPU restatement on this host: single query (ParallelChunked) and the batch (Gemm)
    st_, base = O.prepare_index(m, False)
    _, qn1 = O.prepare_queries(q1.reshape(1, -1), False, base.shape[1])
    _, qn64 = O.prepare_queries(q64, False, base.shape[1])
    ts = []
    for _ in range(30):
        t0 = time.perf_counter()
        O.bench_search_single(base, qn1[0], k)
        ts.append(time.perf_counter() - t0)
    tb = []
    for _ in range(5):
        t0 = time.perf_counter()
        O.bench_search_batch(base, qn64, k)
        tb.append(time.perf_counter() - t0)
    out["cpu_restatement"] = {"single_ms_p50": float(np.median(ts)) * 1e3,
                              "batch_64_queries_per_s": 64 / float(np.median(tb)), "cores": O.num_threads()}
    out["published_reference_cpu_single_ms"] = {
        "accuracy_vs_numpy notebook (k=20, seed 7)": 0.31, "python_bindings_demo notebook (k=5, seed 42)": 0.28962,
        "hardware": "unstated"}
    out["roofline"] = {"bytes_per_batch": 50_000 * 128 * 4, "l2_copy_gbs_measured": l2, "hbm_peak_gbs": peak,
                       "hbm_peak_kind": peak_kind,
                       "note": "the 25.6 MB base stays in the 126 MB L2 across calls: a latency case"}
    del index
    return out


# ---------------------------------------------------------------------------------------------
# mixed-precision workload: BF16 / FP8 tensor-core scan + FP32 rerank vs the FP32 scan
# ---------------------------------------------------------------------------------------------

def fp64_topk(base, queries, k, chunk_rows=1 << 20):
    """FP64 ground truth (verification only): top-k rows by float64 dot product, ties → lower row."""
    import torch
    qd = queries.double()
    best_s = None
    best_i = None
    for r0 in range(0, base.shape[0], chunk_rows):
        s = qd @ base[r0:r0 + chunk_rows].double().T
        v, i = torch.topk(s, min(k + 1, s.shape[1]), dim=1)
        i = i + r0
        if best_s is None:
            best_s, best_i = v, i
        else:
            cs = torch.cat([best_s, v], 1)
            ci = torch.cat([best_i, i], 1)
            v2, j = torch.topk(cs, k + 1, dim=1)
            best_s, best_i = v2, torch.gather(ci, 1, j)
    return best_i[:, :k], best_s


def run_mixed(args, dev, L, world):
    import torch
    from nndex_b200 import _lib, kernel_launch_count
    from nndex_b200._lib import (NNDEX_FLAG_BF16, NNDEX_FLAG_FP8, NNDEX_FLAG_NORMALIZED, NNDEX_PRECISION_BF16,
                                 NNDEX_PRECISION_FP32, NNDEX_PRECISION_FP8)
    rank, _, local = dist_env()
    seed = replica_seed(args.seed + 100, rank)
    rows, dims, nq, k = args.mixed_rows, args.mixed_dims, args.mixed_batch, args.mixed_k
    base = make_mixture(rows, dims, args.mixed_centers, args.mixed_sigma, seed, dev, center_seed=args.seed + 100)
    opts = _lib.Opts()
    opts.device = local
    h = C.c_void_p()
    flags = NNDEX_FLAG_NORMALIZED | NNDEX_FLAG_BF16 | NNDEX_FLAG_FP8
    st = L.nndex_cuda_create_from_device(base.data_ptr(), base.numel(), rows, dims, flags, C.byref(opts), C.byref(h))
    if st != 0:
        raise RuntimeError(_lib.last_error())
    q = make_mixture(nq, dims, args.mixed_centers, args.mixed_sigma, seed + 7, dev, center_seed=args.seed + 100)
    stream = torch.cuda.current_stream(dev)
    sptr = C.c_void_p(stream.cuda_stream)
    oi = torch.empty((nq, k), dtype=torch.int64, device=dev)
    os_ = torch.empty((nq, k), dtype=torch.float32, device=dev)
    stats = _lib.SearchStats()
    out = {}
    if args.mixed_stride or args.mixed_qb:
        # the tuner's cache with the given stride / blocks for both tensor-core precisions at this shape
        n = C.c_uint64(0)
        L.nndex_cuda_autotune_export(h, None, 0, C.byref(n))
        buf = C.create_string_buffer(n.value)
        L.nndex_cuda_autotune_export(h, buf, n.value, C.byref(n))
        nqb, kb = 1 << (nq - 1).bit_length(), 1 << (k - 1).bit_length()
        text = buf.value.decode() + "".join(
            f"shape ivf=0 nq={nqb} k={kb} precision={p} nprobe=0 plan path={p} stride={args.mixed_stride} "
            f"qb={args.mixed_qb} ms=0\n"
            for p in (2, 3))
        if L.nndex_cuda_autotune_import(h, text.encode()) != 0:
            raise RuntimeError(_lib.last_error())
    sample = min(args.mixed_oracle_queries, nq)
    ref_i, ref_s = fp64_topk(base, q[:sample], k)
    for name, prec in (("fp32", NNDEX_PRECISION_FP32), ("bf16", NNDEX_PRECISION_BF16), ("fp8", NNDEX_PRECISION_FP8)):
        L.nndex_cuda_set_precision(h, prec, 0)
        steps = max(1, min(args.mixed_steps, 2 if name == "fp32" else args.mixed_steps))
        for _ in range(2):  # warm-up (the second also runs with the autotuned k′)
            if L.nndex_cuda_search_batch_device(h, q.data_ptr(), nq, dims, k, oi.data_ptr(), os_.data_ptr(), None,
                                                sptr, 1) != 0:
                raise RuntimeError(_lib.last_error())
        torch.cuda.synchronize(dev)
        L.nndex_cuda_set_scan_timing(h, 1)
        barrier(world)
        n0 = kernel_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        second = 0
        fallbacks = 0
        flops = 0.0
        p2rows = 0
        for _ in range(steps):
            if L.nndex_cuda_search_batch_device(h, q.data_ptr(), nq, dims, k, oi.data_ptr(), os_.data_ptr(), None,
                                                sptr, 1) != 0:
                raise RuntimeError(_lib.last_error())
            L.nndex_cuda_last_search_stats(h, C.byref(stats))
            if stats.path in (2, 3):
                second += stats.second_pass_queries
                fallbacks += stats.fp32_fallback_queries
                p2rows += stats.pass2_rows
                # tensor-core FLOPs executed: pass 1 over 1/stride of the rows, pass 2 over all rows
                flops += 2.0 * rows * dims * (nq / max(stats.pass1_tile_stride, 1) + stats.second_pass_queries)
            else:
                flops += 2.0 * rows * dims * nq
        e1.record(stream)
        torch.cuda.synchronize(dev)
        n1 = kernel_launch_count()
        L.nndex_cuda_set_scan_timing(h, 0)
        ms = e0.elapsed_time(e1)
        scan_ms = C.c_double(0.0)
        scan_n = C.c_uint64(0)
        L.nndex_cuda_scan_timing(h, C.byref(scan_ms), C.byref(scan_n))
        max_ms, total_q = aggregate(ms, nq * steps, world, dev)
        got = oi[:sample]
        hits = sum(len(set(got[i].tolist()) & set(ref_i[i].tolist())) for i in range(sample))
        # every result's score error against the FP64 oracle, from the library's own report (one
        # untimed batch with the report on)
        serr = score_error_report(L, h, lambda: L.nndex_cuda_search_batch_device(
            h, q.data_ptr(), nq, dims, k, oi.data_ptr(), os_.data_ptr(), None, sptr, 1))
        scan_total = scan_ms.value  # all scan-kernel launches of the timed batches
        out[name] = {
            "queries_per_s": total_q / (max_ms / 1e3),
            "ms_per_batch": max_ms / steps,
            "scan_ms_per_batch": scan_total / steps,
            "scan_launches_per_batch": scan_n.value / steps,
            "scan_tflops": flops / (scan_total / 1e3) / 1e12,
            "pass1_tile_stride": int(stats.pass1_tile_stride),
            "recall_at_k_vs_fp64": hits / (sample * k),
            "score_error_vs_fp64": serr,
            "algorithmic_tflops": 2.0 * rows * dims * nq / (max_ms / steps / 1e3) / 1e12,
            "rerank_width": int(stats.rerank_width),
            "second_pass_queries_per_batch": second / steps,
            "pass2_rows_per_query": p2rows / second if second else 0.0,
            "pass2_query_blocks": int(stats.pass2_query_blocks),
            "fp32_fallback_queries_per_batch": fallbacks / steps,
            "kernel_launches_per_batch": (n1 - n0) / steps,
        }
    L.nndex_cuda_destroy(h)
    del base
    torch.cuda.empty_cache()
    fp32 = out["fp32"]["queries_per_s"]
    for name in ("bf16", "fp8"):
        out[name]["speedup_vs_fp32"] = out[name]["queries_per_s"] / fp32
    bf16_peak = measured_bf16_peak()
    bf16_sus = measured_bf16_peak(sustained=True)
    alg = {name: out[name]["algorithmic_tflops"] for name in ("bf16", "fp8")}
    return {
        "workload": f"exact top-{k}, base {rows}x{dims} ({args.mixed_centers}-centre Gaussian mixture, "
                    f"sigma={args.mixed_sigma}, unit rows), batch {nq}; BF16/FP8 tensor-core scan + FP32 rerank "
                    f"vs the FP32 scan; recall on {sample} queries vs a float64 brute force",
        "results": out,
        "roofline": {"bound": "tensor", "kernel": "scan_tc_kernel",
                     "flops": "algorithmic 2*N*D*batch per batch, over the whole batch time (both passes, "
                              "merge, rerank)",
                     "achieved_bf16_tflops": alg["bf16"], "peak_bf16_tflops": bf16_peak[0],
                     "frac_bf16": alg["bf16"] / bf16_peak[0],
                     "achieved_fp8_tflops": alg["fp8"], "peak_fp8_tflops": 2 * bf16_peak[0],
                     "frac_fp8": alg["fp8"] / (2 * bf16_peak[0]),
                     "peak_kind": bf16_peak[1] + "; FP8 peak taken as twice the BF16 figure",
                     "executed_scan_tflops": {name: out[name]["scan_tflops"] for name in ("bf16", "fp8")},
                     # the batches run back to back for about 0.1 s: the power-capped figure is the
                     # ceiling of a scan that long, the burst figure that of a single launch
                     "peak_bf16_tflops_sustained": bf16_sus[0],
                     "executed_scan_frac_bf16_sustained": out["bf16"]["scan_tflops"] / bf16_sus[0],
                     "peak_sustained_kind": bf16_sus[1]},
    }


def run_ivf(args, dev, L, world):
    """IVF ANN with exact rerank: the k-means build on the GPU, then probe + ragged list scan."""
    import numpy as np
    import torch
    from nndex_b200 import _lib, kernel_launch_count
    from nndex_b200._lib import NNDEX_FLAG_APPROX, NNDEX_FLAG_NORMALIZED
    rank, _, local = dist_env()
    seed = replica_seed(args.seed + 200, rank)
    rows, dims, nq, k = args.ivf_rows, args.ivf_dims, args.ivf_batch, args.ivf_k
    base = make_mixture(rows, dims, args.ivf_centers, args.ivf_sigma, seed, dev, center_seed=args.seed + 200,
                        zipf=args.ivf_zipf)
    q = make_mixture(nq, dims, args.ivf_centers, args.ivf_sigma, seed + 7, dev, center_seed=args.seed + 200,
                     zipf=args.ivf_zipf)
    # exact checksum of the synthetic base (its bits as integers), so runs can be compared
    data_fp = int(base.view(torch.int32).to(torch.int64).sum().item())
    opts = _lib.Opts()
    opts.device = local
    opts.nlist = args.ivf_nlist
    opts.kmeans_iters = args.ivf_iters
    opts.has_seed = 1
    opts.seed = args.ivf_seed
    h = C.c_void_p()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    st = L.nndex_cuda_create_from_device(base.data_ptr(), base.numel(), rows, dims,
                                         NNDEX_FLAG_NORMALIZED | NNDEX_FLAG_APPROX, C.byref(opts), C.byref(h))
    build_wall = time.perf_counter() - t0
    if st != 0:
        raise RuntimeError(_lib.last_error())
    bst = _lib.IvfStats()
    L.nndex_cuda_ivf_stats_get(h, C.byref(bst))
    # exact reference results (the FP32 exact path, parity-tested against the FP64 oracle)
    hx = C.c_void_p()
    ox = _lib.Opts()
    ox.device = local
    if L.nndex_cuda_create_from_device(base.data_ptr(), base.numel(), rows, dims, NNDEX_FLAG_NORMALIZED,
                                       C.byref(ox), C.byref(hx)) != 0:
        raise RuntimeError(_lib.last_error())
    stream = torch.cuda.current_stream(dev)
    sptr = C.c_void_p(stream.cuda_stream)
    ei = torch.empty((nq, k), dtype=torch.int64, device=dev)
    es = torch.empty((nq, k), dtype=torch.float32, device=dev)
    if L.nndex_cuda_search_batch_device(hx, q.data_ptr(), nq, dims, k, ei.data_ptr(), es.data_ptr(), None, sptr, 1):
        raise RuntimeError(_lib.last_error())
    ex0, ex1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ex0.record(stream)
    L.nndex_cuda_search_batch_device(hx, q.data_ptr(), nq, dims, k, ei.data_ptr(), es.data_ptr(), None, sptr, 1)
    ex1.record(stream)
    torch.cuda.synchronize(dev)
    exact_ms = ex0.elapsed_time(ex1)
    L.nndex_cuda_destroy(hx)
    exact_sets = [set(r) for r in ei.cpu().tolist()]
    oi = torch.empty((nq, k), dtype=torch.int64, device=dev)
    os_ = torch.empty((nq, k), dtype=torch.float32, device=dev)
    cnt = torch.empty((nq,), dtype=torch.int32, device=dev)
    stats = _lib.SearchStats()
    peak, peak_kind = measured_peaks()
    per = {}
    layout = None
    from nndex_b200._lib import NNDEX_PRECISION_AUTO, NNDEX_PRECISION_FP32
    runs = [(str(n), n, NNDEX_PRECISION_AUTO) for n in [int(x) for x in args.ivf_nprobe.split(",") if x]]
    runs += [(f"{n}_fp32_list_scan", n, NNDEX_PRECISION_FP32) for n in [int(x) for x in args.ivf_nprobe.split(",") if x]]
    for name, np_, prec in runs:
        L.nndex_cuda_set_nprobe(h, np_)
        L.nndex_cuda_set_precision(h, prec, 0)
        for _ in range(3):
            if L.nndex_cuda_search_batch_device(h, q.data_ptr(), nq, dims, k, oi.data_ptr(), os_.data_ptr(),
                                                cnt.data_ptr(), sptr, 1) != 0:
                raise RuntimeError(_lib.last_error())
        L.nndex_cuda_last_search_stats(h, C.byref(stats))
        torch.cuda.synchronize(dev)
        L.nndex_cuda_set_scan_timing(h, 1)
        barrier(world)
        n0 = kernel_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.ivf_steps):
            L.nndex_cuda_search_batch_device(h, q.data_ptr(), nq, dims, k, oi.data_ptr(), os_.data_ptr(),
                                             cnt.data_ptr(), sptr, 0)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        n1 = kernel_launch_count()
        L.nndex_cuda_set_scan_timing(h, 0)
        if L.nndex_cuda_stream_status(h) != 0:
            raise RuntimeError(_lib.last_error())
        ms = e0.elapsed_time(e1)
        scan_ms = C.c_double(0.0)
        scan_n = C.c_uint64(0)
        L.nndex_cuda_scan_timing(h, C.byref(scan_ms), C.byref(scan_n))
        max_ms, total_q = aggregate(ms, nq * args.ivf_steps, world, dev)
        got = oi.cpu().tolist()
        hits = sum(len(set(got[i]) & exact_sets[i]) for i in range(nq))
        tc = stats.path == 5
        serr = score_error_report(L, h, lambda: L.nndex_cuda_search_batch_device(
            h, q.data_ptr(), nq, dims, k, oi.data_ptr(), os_.data_ptr(), cnt.data_ptr(), sptr, 1))
        scan_avg = scan_ms.value / args.ivf_steps  # all scan launches of a batch (the tensor-core scan: 2 passes)
        passes = (scan_n.value / args.ivf_steps) if tc else 1.0
        streamed_b = stats.ivf_rows_streamed * dims * (2 if tc else 4) * passes
        union_b = stats.ivf_rows_union * dims * 4
        per[name] = {
            "path": "tensor-core list scan" if stats.path == 5 else "FP32 list scan",
            "second_pass_queries": stats.second_pass_queries,
            "pass2_rows_per_query": stats.pass2_rows / stats.second_pass_queries if stats.second_pass_queries else 0.0,
            "pass1_tile_stride": int(stats.pass1_tile_stride) if tc else None,
            "fp32_fallback_queries": stats.fp32_fallback_queries,
            "queries_per_s": total_q / (max_ms / 1e3),
            "ms_per_batch": max_ms / args.ivf_steps,
            "recall_at_k_vs_exact": hits / (nq * k),
            "score_error_vs_fp64": serr,
            "rows_probed_per_query": stats.rows_scanned / nq,
            "rows_streamed": stats.ivf_rows_streamed,
            "rows_union": stats.ivf_rows_union,
            "scan_ms": scan_avg,
            "scan_gbs_streamed": streamed_b / (scan_avg / 1e3) / 1e9,
            "scan_frac_of_hbm_streamed": streamed_b / (scan_avg / 1e3) / 1e9 / peak,
            "scan_gbs_union": union_b / (scan_avg / 1e3) / 1e9,
            "scan_fp32_tflops": None if tc else 2.0 * stats.rows_scanned * dims / (scan_avg / 1e3) / 1e12,
            # tensor-core scan: executed MMA work, 128-query blocks × streamed rows × D, per pass
            "scan_tensor_tflops": (2.0 * 128 * stats.ivf_rows_streamed * dims * passes / (scan_avg / 1e3) / 1e12
                                   if tc else None),
            "kernel_launches_per_batch": (n1 - n0) / args.ivf_steps,
        }
    # CPU baseline: the reference's IVF search restated (oracle/) on the same index, host threads.
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        n_lay = C.c_uint64(0)
        L.nndex_cuda_ivf_layout(h, C.byref(n_lay), None, None, None, None)
        nl = n_lay.value
        cent = np.zeros((nl, (dims + 7) // 8 * 8), dtype=np.float32)
        off = np.zeros(nl + 1, dtype=np.uint64)
        orig = np.zeros(rows, dtype=np.uint64)
        L.nndex_cuda_ivf_layout(h, C.byref(n_lay), cent.ctypes.data, off.ctypes.data, orig.ctypes.data, None)
        storage = base.cpu().numpy()
        if storage.shape[1] != cent.shape[1]:
            storage = np.ascontiguousarray(np.pad(storage, ((0, 0), (0, cent.shape[1] - storage.shape[1]))))
        ref = O.IvfIndex(storage, layout={"centroids": cent, "cluster_offsets": off, "original_indices": orig})
        qs = q[:args.ivf_cpu_queries].cpu().numpy()
        if qs.shape[1] != cent.shape[1]:
            qs = np.ascontiguousarray(np.pad(qs, ((0, 0), (0, cent.shape[1] - qs.shape[1]))))
        cpu = {}
        for np_ in [int(x) for x in args.ivf_nprobe.split(",") if x]:
            t0 = time.perf_counter()
            ri, _, _ = ref.search(qs, k, np_)
            dt = time.perf_counter() - t0
            cpu[str(np_)] = {"queries_per_s": qs.shape[0] / dt, "cores": O.num_threads(),
                             "sample": f"{qs.shape[0]} queries, same index (restated src/cpu.rs:456-502)"}
        del ref, storage
    # The saved layout installed into a second index over the same rows instead of building it.
    n_lay = C.c_uint64(0)
    L.nndex_cuda_ivf_layout(h, C.byref(n_lay), None, None, None, None)
    nl = n_lay.value
    r_cent = np.zeros((nl, (dims + 7) // 8 * 8), dtype=np.float32)
    r_off, r_orig, r_init = (np.zeros(nl + 1, dtype=np.uint64), np.zeros(rows, dtype=np.uint64),
                             np.zeros(nl, dtype=np.uint64))
    L.nndex_cuda_ivf_layout(h, C.byref(n_lay), r_cent.ctypes.data, r_off.ctypes.data, r_orig.ctypes.data,
                            r_init.ctypes.data)
    hr = C.c_void_p()
    if L.nndex_cuda_create_from_device(base.data_ptr(), base.numel(), rows, dims, NNDEX_FLAG_NORMALIZED,
                                       C.byref(opts), C.byref(hr)) != 0:
        raise RuntimeError(_lib.last_error())
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    if L.nndex_cuda_ivf_restore(hr, nl, r_cent.ctypes.data, r_off.ctypes.data, r_orig.ctypes.data,
                                r_init.ctypes.data) != 0:
        raise RuntimeError(_lib.last_error())
    restore_wall = time.perf_counter() - t0
    rst = _lib.IvfStats()
    L.nndex_cuda_ivf_stats_get(hr, C.byref(rst))
    restored_equal = True
    ri_, rs_ = torch.empty_like(oi), torch.empty_like(os_)
    for np_ in [int(x) for x in args.ivf_nprobe.split(",") if x]:
        for hh in (h, hr):
            L.nndex_cuda_set_nprobe(hh, np_)
            L.nndex_cuda_set_precision(hh, NNDEX_PRECISION_AUTO, 0)
        L.nndex_cuda_search_batch_device(h, q.data_ptr(), nq, dims, k, oi.data_ptr(), os_.data_ptr(), None, sptr, 1)
        L.nndex_cuda_search_batch_device(hr, q.data_ptr(), nq, dims, k, ri_.data_ptr(), rs_.data_ptr(), None, sptr, 1)
        restored_equal &= bool(torch.equal(oi, ri_)) and bool(torch.equal(os_.view(torch.int32), rs_.view(torch.int32)))
    L.nndex_cuda_destroy(hr)
    L.nndex_cuda_destroy(h)
    del base
    torch.cuda.empty_cache()
    return {
        "workload": f"IVF top-{k}, base {rows}x{dims} ({args.ivf_centers}-centre Gaussian mixture, Zipf "
                    f"s={args.ivf_zipf} sizes, sigma={args.ivf_sigma}, unit rows), nlist={args.ivf_nlist}, "
                    f"{args.ivf_iters} k-means iterations, seed {args.ivf_seed}, batch {nq}",
        "build": {"device_ms": bst.build_ms, "seed_ms": bst.seed_ms, "kmeans_ms": bst.kmeans_ms,
                  "layout_ms": bst.layout_ms, "wall_s_with_upload": build_wall, "max_list": bst.max_list,
                  "ambiguous_rows_all_iters": bst.ambiguous_rows,
                  "candidate_rows_all_iters": bst.candidate_rows, "seed_exact_rows": bst.seed_exact_rows},
        "restore_saved_layout": {"device_ms": rst.build_ms, "wall_s": restore_wall,
                                 "results_equal_built_index": restored_equal},
        "data_fingerprint": data_fp,
        "exact_fp32_ms_per_batch": exact_ms,
        "by_nprobe": per,
        "cpu_baseline": cpu,
        "roofline": {"bound": "hbm", "kernel": "ivf_scan_kernel", "peak": peak, "peak_kind": peak_kind,
                     "bytes": "rows_streamed * D * 4 per batch (a list is read once per group of queries)"},
    }


def run_serve(args, dev, L, world):
    """Serving loop: Poisson arrivals of mixed requests against a device-resident index."""
    import numpy as np
    import torch
    from nndex_b200 import _lib
    from nndex_b200._lib import NNDEX_FLAG_APPROX, NNDEX_FLAG_BF16, NNDEX_FLAG_NORMALIZED, NNDEX_PENDING
    rank, _, local = dist_env()
    seed = replica_seed(args.seed + 300, rank)
    rows, dims = args.serve_rows, args.serve_dims
    base = make_mixture(rows, dims, args.serve_centers, args.serve_sigma, seed, dev, center_seed=args.seed + 300)
    pool = make_mixture(1 << 16, dims, args.serve_centers, args.serve_sigma, seed + 7, dev,
                        center_seed=args.seed + 300).cpu().numpy()
    opts = _lib.Opts()
    opts.device = local
    h = C.c_void_p()
    t0 = time.perf_counter()
    if L.nndex_cuda_create_from_device(base.data_ptr(), base.numel(), rows, dims,
                                       NNDEX_FLAG_NORMALIZED | NNDEX_FLAG_APPROX | NNDEX_FLAG_BF16, C.byref(opts),
                                       C.byref(h)) != 0:
        raise RuntimeError(_lib.last_error())
    create_s = time.perf_counter() - t0
    del base
    torch.cuda.empty_cache()
    bst = _lib.IvfStats()
    L.nndex_cuda_ivf_stats_get(h, C.byref(bst))
    so = _lib.ServerOpts()
    so.slots = args.serve_slots
    so.latency_budget_ms = args.serve_latency_ms
    srv = C.c_void_p()
    t_start = time.perf_counter()
    if L.nndex_cuda_server_start(h, C.byref(so), C.byref(srv)) != 0:
        raise RuntimeError(_lib.last_error())
    start_s = time.perf_counter() - t_start  # the slots' warm-up batches included
    rng = np.random.default_rng(seed)
    mean_size = (1 + 256) / 2
    out = {}
    rates = [float(x) for x in args.serve_rates.split(",") if x]
    # a warm-up phase first (not reported): every slot meets every request kind and grows its scratch
    phases = [(None, max(rates), 0.5)] + [(str(int(r)), r, args.serve_seconds) for r in rates]
    for name, rate, seconds in phases:
        nreq = max(1, int(rate * seconds / mean_size))
        gaps = rng.exponential(mean_size / rate, size=nreq)
        sizes = rng.integers(1, 257, size=nreq)
        ks = rng.choice([1, 10, 100], size=nreq)
        approx = rng.integers(0, 2, size=nreq).astype(bool)
        starts = rng.integers(0, pool.shape[0] - 256, size=nreq)
        tickets = [None] * nreq
        lat = []
        batches_seen = {}  # batch id → (slot, start_ns, done_ns, queries)
        done_q = [0]
        refused = [0]
        first_last = [None, None]
        ready = threading.Semaphore(0)

        def collect():
            for i in range(nreq):
                ready.acquire()
                t = tickets[i]
                if t is None:
                    continue
                n, k = int(sizes[i]), int(ks[i])
                idx = np.empty((n, k), dtype=np.uint64)
                sim = np.empty((n, k), dtype=np.float32)
                cnt = np.empty(n, dtype=np.uint64)
                info = _lib.RequestInfo()
                st = L.nndex_cuda_server_poll(srv, t, -1, idx.ctypes.data, sim.ctypes.data, cnt.ctypes.data,
                                              C.byref(info))
                if st != 0:
                    raise RuntimeError(_lib.last_error())
                lat.append((info.done_ns - info.submit_ns) / 1e6)
                batches_seen[info.batch_id] = (info.slot, info.start_ns, info.done_ns, info.batch_queries)
                done_q[0] += n
                first_last[0] = info.submit_ns if first_last[0] is None else min(first_last[0], info.submit_ns)
                first_last[1] = info.done_ns if first_last[1] is None else max(first_last[1], info.done_ns)

        s0 = _lib.ServerStats()
        L.nndex_cuda_server_stats_get(srv, C.byref(s0))
        th = threading.Thread(target=collect)
        th.start()
        tk = C.c_uint64(0)
        t_begin = time.perf_counter()
        due = t_begin
        for i in range(nreq):
            due += gaps[i]
            while time.perf_counter() < due:
                pass
            q = pool[starts[i]:starts[i] + sizes[i]]
            st = L.nndex_cuda_server_submit(srv, q.ctypes.data, int(sizes[i]), dims, int(ks[i]),
                                            NNDEX_FLAG_APPROX if approx[i] else 0,
                                            args.serve_nprobe if approx[i] else 0, C.byref(tk))
            if st == 0:
                tickets[i] = tk.value
            else:
                refused[0] += 1
            ready.release()
        th.join()
        s1 = _lib.ServerStats()
        L.nndex_cuda_server_stats_get(srv, C.byref(s1))
        elapsed = (first_last[1] - first_last[0]) / 1e9 if first_last[1] else float("nan")
        # per-slot timeline: batches, mean batch time and the share of the phase each slot was busy
        slots_tl = {}
        for sl, b0, b1, bq in batches_seen.values():
            d = slots_tl.setdefault(sl, [0, 0.0, 0])
            d[0] += 1
            d[1] += (b1 - b0) / 1e6
            d[2] += bq
        lat_a = np.array(lat) if lat else np.array([float("nan")])
        if name is None:
            continue
        out[name] = {
            "offered_queries_per_s": rate,
            "requests": nreq,
            "refused": refused[0],
            "queries_per_s": done_q[0] / elapsed if elapsed > 0 else None,
            "latency_ms_p50": float(np.percentile(lat_a, 50)),
            "latency_ms_p99": float(np.percentile(lat_a, 99)),
            "latency_ms_max": float(lat_a.max()),
            "refused_by_latency_budget": int(s1.refused_latency - s0.refused_latency),
            "us_per_query_estimate": float(s1.us_per_query),
            "slots": {str(sl): {"batches": d[0], "mean_batch_ms": d[1] / d[0], "mean_batch_queries": d[2] / d[0],
                                "busy_frac": d[1] / 1e3 / elapsed if elapsed > 0 else None}
                      for sl, d in sorted(slots_tl.items())},
        }
    sst = _lib.ServerStats()
    L.nndex_cuda_server_stats_get(srv, C.byref(sst))
    L.nndex_cuda_server_stop(srv)
    L.nndex_cuda_destroy(h)
    return {
        "workload": f"serving: base {rows}x{dims} ({args.serve_centers}-centre mixture, sigma={args.serve_sigma}, "
                    f"unit rows; FP32 + BF16 copies + IVF nlist={bst.nlist}), Poisson arrivals, requests of "
                    f"U{{1..256}} queries, k in {{1,10,100}}, 50/50 exact / IVF(nprobe={args.serve_nprobe}), "
                    f"{args.serve_slots} slots, admission by free HBM and a {args.serve_latency_ms} ms "
                    f"queue-drain budget",
        "create_s_with_ivf_build": create_s,
        "server_start_s_with_warmup": start_s,
        "by_offered_rate": out,
        "batches": sst.batches,
        "mean_batch_queries": sst.queries_done / max(sst.batches, 1),
        "max_queued_queries": sst.max_queued_queries,
        "slot_bytes": sst.slot_bytes,
        "fp32_fallback_queries": sst.fp32_fallback_queries,
        "slowest_batch": {"ms": sst.slowest_batch_ms, "queries": sst.slowest_batch_queries,
                          "k": sst.slowest_batch_k, "path": sst.slowest_batch_path,
                          "approx": bool(sst.slowest_batch_approx)},
    }


def score_error_report(L, h, search):
    """Runs `search` once with the library's per-result error report on; max and mean error of all
    its results against the FP64 oracle."""
    from nndex_b200 import _lib
    L.nndex_cuda_set_error_report(h, 1)
    if search() != 0:
        raise RuntimeError(_lib.last_error())
    st = _lib.SearchStats()
    L.nndex_cuda_last_search_stats(h, C.byref(st))
    L.nndex_cuda_set_error_report(h, 0)
    return {"max": st.max_score_error, "mean": st.mean_score_error, "results": "every result of one batch"}


def measured_bf16_peak(sustained=False):
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        if sustained:
            return float(d["bf16_tflops_sustained"]), "measured bf16_tflops_sustained (power-capped loop)"
        return float(d["bf16_tflops"]), "measured bf16_tflops (burst)"
    except (OSError, KeyError, ValueError):
        return (1400.0, "fallback (sustained)") if sustained else (1590.0, "fallback")


# ---------------------------------------------------------------------------------------------
# reference arm: the CPU restatement of the reference's exact path on the host cores
# ---------------------------------------------------------------------------------------------

def run_reference(args):
    rank, world, local = dist_env()
    if world > 1 and rank != 0:
        return None
    import torch
    dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
    base = make_mixture(args.rows, args.dims, args.centers, args.sigma, replica_seed(args.seed, 0), dev,
                        center_seed=args.seed).cpu().numpy()
    b = args.batch
    k = min(args.k, args.rows)
    qall = make_mixture(8 * b, args.dims, args.centers, args.sigma, args.seed + 7, dev,
                        center_seed=args.seed).cpu().numpy()
    qs = [qall[i * b:(i + 1) * b] for i in range(8)]
    from oracle import oracle as O
    O.lib()
    threads = O.num_threads()
    # Each step is a bounded sample: a row subsample when a full pass would exceed ~2 s.
    t0 = time.perf_counter()
    O.bench_search_batch(base, qs[0], k)
    full = time.perf_counter() - t0
    rows = args.rows if full <= 2.0 else max(100_000, int(args.rows * 2.0 / full))
    sub = np.ascontiguousarray(base[:rows])
    for i in range(args.warmup):
        O.bench_search_batch(sub, qs[i % 8], k)
    times = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        O.bench_search_batch(sub, qs[i % 8], k)
        times.append(time.perf_counter() - t0)
    scale = rows / args.rows
    step_s = statistics.mean(times) / scale
    value = b / step_s
    sample = (f"each step: {b} queries over {rows} of {args.rows} rows, scaled to the full base"
              if rows < args.rows else f"each step: {b} queries over the full {args.rows}-row base")
    return {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"exact-fp32 top-k, base {args.rows}x{args.dims} f32 ({args.centers}-centre "
                               f"Gaussian mixture, sigma={args.sigma}, unit rows, normalized=true), batch {b}, k={k}",
                   "rows": args.rows, "dims": args.dims, "batch": b, "k": k, "parallelism": "host-cores"},
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "port",
                         "sample": sample + " (CPU restatement of src/cpu.rs:256-341 + src/topk.rs, oracle/)"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main(argv=None):
    args = parse_args(argv)
    line = run_reference(args) if args.impl == "reference" else run_ours(args)
    if line is not None:
        print(json.dumps(line), flush=True)
    rank, world, _ = dist_env()
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
