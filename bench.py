#!/usr/bin/env python
"""Benchmark of the sieve query path on B200: QPS at R@10 >= 0.90 with p50/p99 latency, and the
scan kernel's HBM roofline.

Workloads (seeded synthetic Gaussian mixtures standing in for the reference's datasets, which are
not available; shapes, sizes and noise model as the workloads name them):
  c1  1M x 768, 1024 centres, 1024 clusters, SOAR, 10k queries   (the reference's CPU-sized case)
  c2  18.4M x 768, 16384 centres, 4096 clusters, SOAR + 2-bit tier, 50k queries   (default)
  c3  113.5M x 768, 65536 centres, 16384 clusters, SOAR + 2-bit tier, 100k queries (~105 GB HBM)
  c4  bigann L2: int8 x 100 rows (100M by default, --rows up to the 1B shape), 131,072 leaves
      (512 x 256), 2-bit refinement, 64 probes, 10k queries

One step = one batch of queries through the whole path (route, scan, cut, rerank) with the
inputs resident in HBM (sg_search_device). `e2e` runs the same batches through the host API
(sg_search) from pinned host memory, copies included. `plain` is the one-query-per-launch form.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2] [--impl ours|reference]
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

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "a-game-of-vectors_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402
import torch  # noqa: E402

# `search` is the headline search of a workload: the stated probing with enough candidates that
# recall reaches the corpus's int8 ceiling (on these mixtures 500 candidates leave most true
# neighbours behind: ~1,150 near-equidistant rows sit around each centre). `stated` is the
# workload's search exactly as stated (500 candidates, the 2-bit tier picking 200 int8 rows),
# measured beside it.
WORKLOADS = {
    "c1": dict(n=1_000_000, centers=1024, k=1024, queries=10_000, search="32:1000:full",
               stated="32:500:full"),
    "c2": dict(n=18_400_000, centers=16384, k=4096, queries=50_000, search="32:2000:full",
               stated="32:500:tiered200", serve="5000,20000,50000,100000,150000,200000"),
    # margin probing: 0.35 gives a median of ~46 probes (cap 128) on this mixture
    "c3": dict(n=113_500_000, centers=65536, k=16384, queries=100_000, search="128:2000:full:p0.35",
               stated="128:500:tiered200:p0.35",
               serve="5000,10000,20000,25000,30000,40000,50000,100000,150000,200000",
               secondary="c2"),
    # billion-scale L2 (bigann): 512 x 256 = 131,072 leaves, 2-bit refinement. The bench default
    # is a 100M-row cut of the 1B shape (--rows sets it): the 1B build does not fit the run's time.
    "c4": dict(n=100_000_000, centers=131072, k1=512, k2=256, bits=2, queries=10_000,
               search="64:300:2000"),
}
BG_SCAN_BYTES_PER_SLOT = 24  # 16 B code + 8 B [mul, |x|^2] per scanned slot
SCAN_BYTES_PER_SLOT = 40  # 32 B code + 8 B [mul, err] factors per scanned slot


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---- clocks during the timed region ------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value: float, world: int, device) -> float:
    """The largest of every rank's `value` (a timed region's length): each GPU runs an independent
    replica of the workload (no data-path collective), so the job's time is its slowest rank's."""
    if world <= 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_qps(per_rank_queries: int, seconds: float, world: int, device) -> float:
    """Whole-job throughput of `world` replicas: all ranks' queries over the slowest rank's time."""
    return world * per_rank_queries / max_over_ranks(seconds, world, device)


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


# ---- workload ----------------------------------------------------------------------------------
def build_workload(name: str, device: str, rows: int | None, nq_pool: int, n_eval: int):
    from sieve_gpu import builder, synth

    w = dict(WORKLOADS[name])
    if rows:
        w["n"] = rows
    t0 = time.time()
    mix = synth.Mixture(n=w["n"], n_centers=w["centers"], dim=768, spread=1.0, sigma=0.3, seed=1,
                        device=device)
    corpus = builder.ingest(mix)
    t_ingest = time.time() - t0
    index = builder.build_ivf(corpus, k=w["k"], sample_n=min(w["n"], 262144), iters=10,
                              soar_lambda=1.0, device=device)
    t_build = time.time() - t0 - t_ingest
    arrays = {**corpus, **index}
    del corpus, index
    torch.cuda.empty_cache()  # the index upload needs the build's cached device memory back
    queries = mix.queries(nq_pool, sigma=0.35).float()
    arrays["domain"] = domain_ids(mix, w["n"])  # per-row domains of the serving filters
    t1 = time.time()
    gt = builder.ground_truth(mix, queries[:n_eval], k=10)
    torch.cuda.empty_cache()
    t_gt = time.time() - t1
    log(f"workload {name}: n={w['n']} k={w['k']} ingest {t_ingest:.1f}s build {t_build:.1f}s "
        f"gt {t_gt:.1f}s nblocks={int(arrays['block_off'][-1])}")
    return w, arrays, queries, gt, {"ingest_s": round(t_ingest, 1), "build_s": round(t_build, 1)}


def prefix256(q768: np.ndarray) -> np.ndarray:
    """quant::prefix (src/quant.rs:17-20) of each row: the first 256 dims renormalised."""
    p = q768[:, :256].astype(np.float32)
    return (p / np.sqrt((p * p).sum(1, keepdims=True))).astype(np.float32)


def probe_stats(index, q768: np.ndarray, params, batch: int) -> tuple[dict, list]:
    """Probe counts of the queries (Index::route with the search's own margin, budget and cap)
    and, per `batch`-query window, the distinct clusters the window probes."""
    routes = index.route(prefix256(q768), params)
    counts = np.array([len(c) for _, c in routes])
    stats = {"min": int(counts.min()), "median": float(np.median(counts)), "max": int(counts.max()),
             "mean": float(counts.mean())}
    return stats, [c for _, c in routes]


def distinct_slots(routes: list, lo: int, batch: int, slots_per_cluster: np.ndarray) -> int:
    """Slots of the distinct clusters queries [lo, lo + batch) probe: what a batch must read at
    least once."""
    cl = np.unique(np.concatenate(routes[lo:lo + batch]))
    return int(slots_per_cluster[cl].sum())


def parity_check(gpu_ids, gpu_sc, gpu_cnt, cpu: dict) -> dict:
    """Per query, the GPU's (score, row) list against the CPU leg's, bit for bit. A query whose
    lists differ is counted as tied, not mismatched, when a cut on its oracle path was tied (the
    reference leaves the survivors of a tie unspecified)."""
    m = min(len(gpu_cnt), len(cpu["cnt"]))
    same = np.array([int(gpu_cnt[i]) == int(cpu["cnt"][i])
                     and np.array_equal(gpu_ids[i, :gpu_cnt[i]], cpu["ids"][i, :cpu["cnt"][i]])
                     and np.array_equal(gpu_sc[i, :gpu_cnt[i]], cpu["sc"][i, :cpu["cnt"][i]])
                     for i in range(m)], dtype=bool)
    tied = cpu["tied"][:m]
    return {"queries": int(m), "mismatched": int((~same & ~tied).sum()),
            "tied_boundary": int(tied.sum()), "tied_and_differing": int((~same & tied).sum()),
            "rule": "bit-exact (score, row) lists; canonical ties (score desc, row asc)"}


def time_search(index, q768: torch.Tensor, params, batch: int, nq_pool: int, warmup: int, steps: int) -> dict:
    """Device-timed batches of one search config (inputs resident in HBM, CUDA events on the
    launching stream): queries/s, ms per batch and the mean stage times."""
    dev = q768.device
    out_sc = torch.empty((batch, params.k), dtype=torch.float32, device=dev)
    out_id = torch.empty((batch, params.k), dtype=torch.int32, device=dev)
    out_n = torch.empty((batch,), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    ms, stats = [], []
    for i in range(warmup + steps):
        lo = (i * batch) % (nq_pool - batch + 1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        index.search_device(batch, q768[lo].data_ptr(), None, params, out_sc.data_ptr(), out_id.data_ptr(),
                            out_n.data_ptr(), stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        if i >= warmup:
            ms.append(a.elapsed_time(b))
            stats.append(index.last_stats())
    stage = {k: round(float(np.mean([s[k] for s in stats])), 4)
             for k in ("ms_route_gemm", "ms_route_select", "ms_scan", "ms_cut", "ms_rerank", "ms_tier2", "ms_total")}
    return {"qps": batch * len(ms) / (float(np.sum(ms)) / 1e3), "ms_per_batch": float(np.mean(ms)),
            "stage_ms": stage, "batches": len(ms)}


def search_line(index, arrays, queries, gt, t8, config: str, nclusters: int, batch: int, nq_pool: int,
                warmup: int, steps: int) -> dict:
    """Recall (float and int8 truth), probe counts and device-timed QPS of one search config."""
    from sieve_gpu import parse_config

    _, p = parse_config(config, nclusters)
    p.k = 10
    q_host = queries.cpu().numpy()
    ev = q_host[: gt.shape[0]]
    _, ids, cnt = index.search_batch(ev, None, p)
    probes, _ = probe_stats(index, q_host[:batch], p, batch)
    index.set_timing(True)
    t = time_search(index, queries.to(index_device(index)).contiguous(), p, batch, nq_pool, warmup, steps)
    return {"search": config, "recall_at_10": recall10(ids, cnt, gt), "recall_at_10_int8_truth": recall10(ids, cnt, t8),
            "probes": probes, **t}


def index_device(index) -> str:
    return f"cuda:{index.device}"


def recall10(ids: np.ndarray, cnt: np.ndarray, gt: np.ndarray) -> float:
    r = []
    for i in range(gt.shape[0]):
        got = set(int(x) for x in ids[i, : min(10, int(cnt[i]))])
        truth = set(int(x) for x in gt[i, :10])
        r.append(len(got & truth) / max(min(10, len(truth)), 1))
    return float(np.mean(r))


def int8_truth(arrays, q768: torch.Tensor, k: int = 10) -> np.ndarray:
    """Exact top-k by the rerank's own int8 score (the ground truth filter::truth uses,
    src/filter.rs:112-151): (query_i8(q / scale) . row) in exact integer arithmetic."""
    dev = q768.device
    scale = torch.as_tensor(arrays["quant_scale"], device=dev)
    w = q768.float() / scale
    m = torch.clamp(w.abs().amax(1, keepdim=True), min=1e-12)
    s = 127.0 / m
    v = w * s
    wq = torch.where((v - torch.trunc(v)).abs() == 0.5, torch.trunc(v) + torch.sign(v), torch.round(v))
    rows = arrays["rerank"]
    best_v = torch.full((q768.shape[0], k), -float("inf"), device=dev)
    best_i = torch.zeros((q768.shape[0], k), dtype=torch.int64, device=dev)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False  # products and sums stay exact integers in f32
    try:
        for s0 in range(0, rows.shape[0], 1 << 20):
            x = torch.as_tensor(rows[s0:s0 + (1 << 20)], device=dev).float()
            sc = wq @ x.T
            v_, i_ = torch.topk(sc, min(k, sc.shape[1]), dim=1)
            allv, alli = torch.cat((best_v, v_), 1), torch.cat((best_i, i_ + s0), 1)
            # ties by ascending row id, as the reference's TopK order
            order = torch.argsort(alli, dim=1, stable=True)
            allv, alli = allv.gather(1, order), alli.gather(1, order)
            tv, ti = torch.sort(allv, dim=1, descending=True, stable=True)
            best_v, best_i = tv[:, :k], alli.gather(1, ti[:, :k])
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return best_i.cpu().numpy().astype(np.uint32)


def cpu_reference(arrays, q768_host: np.ndarray, params, seconds: float, threads: int):
    """The reference's portable CPU path (oracle restatement, -march=native, OpenMP over queries)
    on a sample of queries sized to run about `seconds`."""
    import oracle as O

    oi = O.OracleIndex(arrays, native=True)
    q256 = np.stack([O.prefix(v)[0] for v in q768_host]).astype(np.float32)
    p = params.to_c()
    probe = min(q768_host.shape[0], max(threads * 4, 64))
    t = time.perf_counter()
    oi.search_batch(q768_host[:probe], q256[:probe], p, threads=threads)
    per_q = (time.perf_counter() - t) / probe
    # the sample cycles through the query pool until it holds about `seconds` of work
    n = int(max(probe, seconds / max(per_q, 1e-9)))
    sel = np.arange(n) % q768_host.shape[0]
    t = time.perf_counter()
    s, o, c, scanned, tied = oi.search_batch(q768_host[sel], q256[sel], p, threads=threads, tied=True)
    dt = time.perf_counter() - t
    k = min(n, q768_host.shape[0])
    return {"qps": n / dt, "queries": n, "seconds": dt, "ids": o[:k], "cnt": c[:k], "sc": s[:k],
            "tied": tied[:k]}


N_DOMAINS = 10_000
GOLDEN = 0x9E3779B97F4A7C15


def domain_ids(mix, n: int, seed: int = 23) -> np.ndarray:
    """Seeded per-row domain ids over 10,000 domains. A row's domain follows its mixture centre
    (centre mod 10,000) with probability 0.8 and is uniform otherwise, so a domain's rows cluster
    by topic as a real site's pages do."""
    out = np.empty(n, np.uint16)
    rng = np.random.default_rng(seed)
    for s in range(0, n, 1 << 22):
        e = min(n, s + (1 << 22))
        d = (mix.centres_of(s, e - s).cpu().numpy() % N_DOMAINS).astype(np.uint16)
        flip = rng.random(e - s) < 0.2
        d[flip] = rng.integers(0, N_DOMAINS, int(flip.sum()))
        out[s:e] = d
    return out


def domain_allowlist(dom: np.ndarray, selectivity: float) -> np.ndarray:
    """The search binary's filter allowlists (src/bin/search.rs:598-620): domains in the fixed
    pseudo-random order of (h * 0x9E3779B97F4A7C15).rotate_left(17), whole domains allowed until
    they hold `selectivity` of the rows. Returns the allow bitset (u64 words)."""
    counts = np.bincount(dom, minlength=N_DOMAINS)
    h = np.arange(N_DOMAINS, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = h * np.uint64(GOLDEN)
    key = (x << np.uint64(17)) | (x >> np.uint64(47))
    order = np.argsort(key, kind="stable")
    want = int(selectivity * dom.size)
    allowed, rows = np.zeros(N_DOMAINS, bool), 0
    for d in order:
        if rows >= want:
            break
        allowed[d] = True
        rows += int(counts[d])
    mask = allowed[dom]
    pad = (-mask.size) % 64
    bits = np.packbits(np.concatenate([mask, np.zeros(pad, bool)]), bitorder="little")
    return bits.view(np.uint64).copy()


def serve_load(index, arrays, queries_host: np.ndarray, params, rates, seconds: float, dom=None,
               seed: int = 7, warmup_s: float = 0.3, contexts: int = 3):
    """Open-loop Poisson arrivals into the serving loop (continuous batching), replayed by the
    library's own submitter thread (sg_server_replay): for each rate, the achieved QPS and the
    p50/p99 latency from submit to results on the host. One request in ten carries a domain
    allowlist (whole domains at 0.1%, 1%, 10% and 50% of the rows). Each rate first replays
    `warmup_s` of the same process unmeasured: a fresh server sizes its contexts' scratch on
    first use."""
    from sieve_gpu import Server
    from sieve_gpu import filter as F

    rng = np.random.default_rng(seed)
    sels = (0.001, 0.01, 0.1, 0.5)
    filters = []
    if dom is not None:
        filters = [F.Filter(domain_allowlist(dom, s), index) for s in sels]
    out = []
    try:
        for rate in rates:
            srv = Server(index, max_batch=4096, contexts=contexts)
            try:
                def trace(n):
                    t = np.cumsum(rng.exponential(1.0 / rate, n))
                    which = rng.integers(0, queries_host.shape[0], n)
                    fo = np.where(rng.random(n) < 0.1, rng.integers(0, max(len(filters), 1), n), -1)
                    return t, which, fo if filters else None
                t, wh, fo = trace(max(int(rate * warmup_s), 1))
                srv.replay(t, queries_host, wh, params, filters, fo)
                st0 = srv.stats()
                nreq = int(rate * seconds)
                t, wh, fo = trace(nreq)
                lat, bat, wall = srv.replay(t, queries_host, wh, params, filters, fo)
                st = srv.stats()
            finally:
                srv.stop()
            out.append({"offered_qps": rate, "achieved_qps": nreq / wall,
                        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                        "requests": nreq, "filtered": int((fo >= 0).sum()) if fo is not None else 0,
                        "mean_batch": (st["queries_batched"] - st0["queries_batched"])
                        / max(st["batches"] - st0["batches"], 1),
                        "retried": st["retried"] - st0["retried"]})
            log(f"serve {rate}/s: {out[-1]}")
    finally:
        for f in filters:
            f.close()
    return out


def serving_knee(serving, plain_ms) -> dict | None:
    """The highest offered rate whose p99 stays within 5 ms and whose achieved rate keeps up
    (>= 95% of offered), and its ratio to the plain one-query-per-launch path."""
    if not serving:
        return None
    ok = [s for s in serving if s["p99_ms"] <= 5.0 and s["achieved_qps"] >= 0.95 * s["offered_qps"]]
    if not ok:
        return {"offered_qps": None, "note": "no rate met p99 <= 5 ms"}
    best = max(ok, key=lambda s: s["achieved_qps"])
    plain_qps = float(1e3 / np.mean(plain_ms))
    return {"offered_qps": best["offered_qps"], "achieved_qps": best["achieved_qps"], "p99_ms": best["p99_ms"],
            "vs_plain": best["achieved_qps"] / plain_qps}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--rows", type=int, default=None, help="override the corpus size (smoke runs)")
    ap.add_argument("--config", default=None, help="search config nprobe:cand:rerank[:...]")
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--route", default="bf16", choices=["bf16", "fp32"])
    ap.add_argument("--eval", type=int, default=1000, help="queries with exact ground truth")
    ap.add_argument("--plain", type=int, default=512, help="queries timed one per launch")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--serve", default=None,
                    help="Poisson arrival rates (queries/s) for the serving loop (default: the "
                         "workload's); empty: skip")
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--serve-contexts", type=int, default=6, help="execution contexts of the serving loop")
    ap.add_argument("--no-tune", action="store_true", help="keep the default shapes (no autotuner)")
    ap.add_argument("--tuning", default=None,
                    help="pin the batched path's shapes instead of autotuning: "
                         "tc_min_queries:chunk_blocks:scan_ctas_per_sm:seed_blocks:tc_split")
    ap.add_argument("--stated", default=None,
                    help="search config measured beside the headline (default: the workload's "
                         "stated search); empty: skip")
    ap.add_argument("--secondary", default=None,
                    help="a second workload measured after the first (its headline and stated "
                         "searches; default: the workload's, c2 for c3); empty: skip")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    if args.impl == "reference" and rank != 0:
        return finish(world)

    if args.workload == "c4":
        return main_bigann(args, rank, world, local, dev)

    from sieve_gpu import Index, parse_config

    wl = WORKLOADS[args.workload]
    config = args.config or wl["search"]
    nq_pool = max(args.batch, args.eval, args.plain)
    nq_pool = min(max(nq_pool, args.batch * 2), wl["queries"])
    w, arrays, queries, gt, build_info = build_workload(args.workload, dev, args.rows, nq_pool, args.eval)
    label, params = parse_config(config, w["k"])
    params.k = 10
    threads = os.cpu_count() or 1
    # the workload and search as stated; build times and tuning are outcomes, reported apart
    cfg = {"workload": f"{args.workload}: {w['n']} x 768, {w['centers']} centres, {w['k']} clusters",
           "search": config, "batch": args.batch, "route": args.route, "queries_pool": nq_pool,
           "l2": "inputs larger than L2 (index and per-batch scan far above 126 MB)"}
    metric = "QPS at R@10>=0.90 (p50/p99 ms, scan GB/s vs HBM peak)"

    if args.impl == "reference":
        q_host = queries.cpu().numpy()
        times = []
        res = None
        for i in range(args.warmup + args.steps):
            res = cpu_reference(arrays, q_host[: max(args.eval, 256)], params,
                                args.cpu_seconds / max(args.steps, 1), threads)
            if i >= args.warmup:
                times.append(res["qps"])
        qps = float(np.mean(times))
        m = min(res["ids"].shape[0], gt.shape[0])
        rec = recall10(res["ids"][:m], res["cnt"][:m], gt[:m])
        line = {"metric": metric, "impl": "reference",
                "value": qps, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u8 LUT / f32 estimate / i8 rerank", "data": "synthetic", "config": cfg,
                "recall_at_10": rec, "build": build_info,
                "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": threads, "kind": "port",
                                 "sample": f"{res['queries']} queries per step on {threads} threads "
                                           f"(the reference's portable path restated in C, "
                                           f"-march=native, OpenMP over queries)"},
                "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return finish(world)

    index = Index.from_arrays(arrays, device=local)
    index.set_route_precision(args.route == "bf16")
    index.set_timing(True)
    q768 = queries.to(dev).contiguous()
    q_pool_host = queries.cpu().numpy()
    B = args.batch
    out_sc = torch.empty((B, params.k), dtype=torch.float32, device=dev)
    out_id = torch.empty((B, params.k), dtype=torch.int32, device=dev)
    out_n = torch.empty((B,), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()

    # recall on the ground-truth queries, against float truth and against exact int8 truth; the
    # ceiling is exact int8 brute force (the rerank's own arithmetic over every row) scored
    # against float truth: no candidate list can do better than the rows' own quantisation
    ev = q_pool_host[: args.eval]
    ev_sc, ev_ids, ev_cnt = index.search_batch(ev, None, params)
    rec = recall10(ev_ids, ev_cnt, gt)
    t8 = int8_truth(arrays, q768[: args.eval])
    rec_i8 = recall10(ev_ids, ev_cnt, t8)
    ceiling = recall10(t8, np.full(t8.shape[0], 10), gt)
    probes, routes = probe_stats(index, q_pool_host, params, B)
    slots_pc = np.diff(np.asarray(arrays["block_off"], np.int64)) * 32
    log(f"{label}: recall@10 {rec:.4f} (float truth), {rec_i8:.4f} (int8 truth), int8 ceiling "
        f"{ceiling:.4f}; probes {probes}")

    def window(i):
        return (i * B) % (nq_pool - B + 1)

    def step(i):
        index.search_device(B, q768[window(i)].data_ptr(), None, params, out_sc.data_ptr(),
                            out_id.data_ptr(), out_n.data_ptr(), stream.cuda_stream)

    # the autotuner picks the batched path's shapes on this batch size (untimed; results are
    # identical under every shape)
    tuning = None
    if args.tuning:
        # shapes given on the command line (a profiling run that repeats a tuned bench's launches)
        names = ("tc_min_queries", "chunk_blocks", "scan_ctas_per_sm", "seed_blocks", "tc_split")
        tuning = dict(zip(names, (int(x) for x in args.tuning.split(":"))))
        index.set_tuning(**tuning)
    elif B >= 64 and not args.no_tune:
        index.set_timing(False)
        tuning = index.autotune(B, q768[nq_pool - B].data_ptr(), params, reps=2)
        index.set_timing(True)
        log(f"autotune: {tuning}")
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    step_ms, stats = [], []
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        for i in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(args.warmup + i)
            b.record(stream)
            b.synchronize()
            step_ms.append(a.elapsed_time(b))
            stats.append(index.last_stats())
        torch.cuda.synchronize()
    total_ms = max_over_ranks(float(np.sum(step_ms)), world, dev)
    qps = world * args.steps * B / (total_ms / 1e3)

    # The scan stage's roofline. Algorithmic bytes of one batch: every distinct cluster its queries
    # probe, read once (32 B code + 8 B factors per slot), plus the row id of every entry admitted
    # to a candidate buffer (4 B); over the stage's CUDA-event time on the library's stream.
    scan_ms = np.array([s["ms_scan"] for s in stats])
    scanned = np.array([s["scanned"] for s in stats], dtype=np.float64)
    dslots = np.array([distinct_slots(routes, window(args.warmup + i), B, slots_pc)
                       for i in range(args.steps)], dtype=np.float64)
    buffered = np.array([s["buffered"] for s in stats], dtype=np.float64)
    alg_bytes = dslots * SCAN_BYTES_PER_SLOT + buffered * 4
    achieved = float(np.mean(alg_bytes / (scan_ms / 1e3)) / 1e9)
    peaks = measured_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "scan_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            t = json.load(f)
        if (t.get("workload") == args.workload and t.get("config") == config
                and t.get("batch") == args.batch and not args.rows):
            traffic = float(t["dram_bytes_per_slot"]) * float(np.mean(scanned))
    stage = {k: round(float(np.mean([s[k] for s in stats])), 4)
             for k in ("ms_prep", "ms_route_gemm", "ms_route_select", "ms_seed", "ms_scan", "ms_cut",
                       "ms_rerank", "ms_tier2", "ms_total")}

    # one query per launch (timing off: repeated call shapes replay their captured CUDA graph)
    index.set_timing(False)
    plain_ms = []
    for i in range(args.plain):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        index.search_device(1, q768[i].data_ptr(), None, params, out_sc.data_ptr(), out_id.data_ptr(),
                            out_n.data_ptr(), stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        plain_ms.append(a.elapsed_time(b))
    plain_ms = np.array(plain_ms[min(8, len(plain_ms) // 4):] or [float("nan")])

    # end to end through the host API from pinned memory
    qh = torch.empty((B, 768), dtype=torch.float32).pin_memory()
    osc = torch.empty((B, params.k), dtype=torch.float32).pin_memory()
    oid = torch.empty((B, params.k), dtype=torch.int32).pin_memory()
    ocn = torch.empty((B,), dtype=torch.int32).pin_memory()
    host_pool = queries.cpu()
    e2e_s = []
    for i in range(args.warmup + args.steps):
        lo = window(i)
        qh.copy_(host_pool[lo:lo + B])
        t = time.perf_counter()
        index.search_into(qh.numpy(), params, osc.numpy(), oid.numpy().view(np.uint32), ocn.numpy().view(np.uint32))
        if i >= args.warmup:
            e2e_s.append(time.perf_counter() - t)
    e2e_qps = replica_qps(args.steps * B, float(np.sum(e2e_s)), world, dev)

    serving = None
    rates = args.serve if args.serve is not None else wl.get("serve", "")
    if rates:
        rates = [float(x) for x in rates.split(",") if x]
        serving = serve_load(index, arrays, q_pool_host, params, rates, args.serve_seconds,
                             dom=arrays.get("domain"), contexts=args.serve_contexts)

    # the workload's search exactly as stated, beside the headline
    stated = None
    stated_cfg = args.stated if args.stated is not None else wl.get("stated", "")
    if stated_cfg and stated_cfg != config and rank == 0:
        stated = search_line(index, arrays, queries[:nq_pool], gt, t8, stated_cfg, w["k"], B, nq_pool, 3, 5)
        log(f"stated {stated_cfg}: {stated}")

    cpu, parity = None, None
    if rank == 0 and world == 1 and args.cpu_seconds > 0:
        r = cpu_reference(arrays, q_pool_host[: max(args.eval, 256)], params, args.cpu_seconds, threads)
        cpu = {"value": r["qps"], "unit": "queries/s", "cores": threads, "kind": "port",
               "sample": f"{r['queries']} queries of the same workload, {r['seconds']:.1f} s, "
                         f"OpenMP over queries, oracle built -march=native"}
        parity = parity_check(ev_ids, ev_sc, ev_cnt, r)
        log(f"parity against the CPU leg: {parity}")
    line = {
        "metric": metric,
        "value": qps, "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8 LUT / f32 estimate / i8 rerank", "data": "synthetic",
        "config": cfg, "recall_at_10": rec, "recall_at_10_int8_truth": rec_i8,
        "recall_ceiling_int8": ceiling,
        "recall_note": "float truth = exact FP32 top-10 over the unit 768-d vectors; int8 truth = "
                       "exact top-10 of the int8 rerank score over every row; ceiling = that int8 "
                       "top-10 scored against float truth (the best any candidate list can reach "
                       "with the corpus's int8 rows)",
        "probes": probes,
        "parity": parity,
        "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
        "latency_note": "batched form: every query of a batch completes with its batch",
        "plain": {"qps": float(1e3 / np.mean(plain_ms)), "p50_ms": float(np.percentile(plain_ms, 50)),
                  "p99_ms": float(np.percentile(plain_ms, 99)), "queries": int(plain_ms.size)},
        "stage_ms": stage,
        "serving": serving,
        "serving_note": f"continuous batching (sg_server, {args.serve_contexts} contexts, batches up to 4096): open-loop "
                        "Poisson arrivals replayed by the library's submitter thread "
                        "(sg_server_replay), 10% of requests on domain allowlists (10,000 seeded "
                        "domains, whole domains at 0.1/1/10/50% of the rows, Post plan), after 0.3 s "
                        "of unmeasured warm-up at the same rate; latency = submit to results on the "
                        "host, on the library's clock",
        "serving_knee": serving_knee(serving, plain_ms),
        "scanned_per_query": float(np.mean(scanned) / B),
        "distinct_probed_slots_per_step": float(np.mean(dslots)),
        "retried_queries_per_step": float(np.mean([s["retried"] for s in stats])),
        "stated": stated,
        "roofline": {"bound": "hbm",
                     "kernel": "the scan stage: k_scan_seed + k_scan (ALU chunks) + k_filter_prep + "
                               "k_scan_tcf (tcgen05 bound) + k_tc_recheck",
                     "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback",
                     "traffic": traffic,
                     "traffic_frac": (traffic / (float(np.mean(scan_ms)) / 1e3) / 1e9 / peak) if traffic else None,
                     "bytes": "distinct probed slots x 40 B (32 B code + 8 B factors) + buffered entries "
                              "x 4 B (row ids), per batch",
                     "note": "a batch reads each probed cluster once for all its queries; traffic = ncu "
                             "dram bytes of the scan kernels per batch (profiles/scan_traffic.json)"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_qps, "unit": "queries/s", "h2d_bytes_per_step": B * 768 * 4,
                "d2h_bytes_per_step": B * params.k * 8 + B * 4},
        "gpu_launches": int(sum(s["launches"] for s in stats)),
        "clocks": clocks.summary(),
        "build": build_info,
        "tuning": tuning,
    }
    index.close()
    sec_name = args.secondary if args.secondary is not None else wl.get("secondary", "")
    if sec_name and rank == 0 and not args.rows:
        del arrays
        torch.cuda.empty_cache()
        line["secondary"] = secondary_workload(sec_name, dev, local, B, args.route)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return finish(world)


def secondary_workload(name: str, dev: str, local: int, batch: int, route: str) -> dict:
    """A second workload after the first: its headline and stated searches, device-timed (the
    autotuner off: the default shapes)."""
    from sieve_gpu import Index

    wl = WORKLOADS[name]
    nq_pool = min(max(batch * 2, 1000), wl["queries"])
    w, arrays, queries, gt, build_info = build_workload(name, dev, None, nq_pool, 1000)
    index = Index.from_arrays(arrays, device=local)
    index.set_route_precision(route == "bf16")
    t8 = int8_truth(arrays, queries[:1000].to(dev))
    out = {"workload": f"{name}: {w['n']} x 768, {w['centers']} centres, {w['k']} clusters", "batch": batch,
           "recall_ceiling_int8": recall10(t8, np.full(t8.shape[0], 10), gt), "build": build_info}
    for key in ("search", "stated"):
        out[key] = search_line(index, arrays, queries, gt, t8, wl[key], w["k"], batch, nq_pool, 3, 10)
        log(f"secondary {name} {key}: {out[key]}")
    index.close()
    return out


# ---- bigann (billion-scale L2 over int8 rows) ----------------------------------------------------
def recall10_ties(ids, cnt, gt_ids, gt_sc) -> tuple[float, float]:
    """big-ann recall@10 with ties (any true row at most as far as the 10th nearest) and strict
    recall@10 (src/bin/spacev.rs:108-119)."""
    rt, rs = [], []
    for i in range(gt_ids.shape[0]):
        got = [int(x) for x in ids[i, : min(10, int(cnt[i]))]]
        cut = gt_sc[i, 9]
        ok = set(int(x) for x, sc in zip(gt_ids[i], gt_sc[i]) if sc >= cut)
        rt.append(sum(g in ok for g in got) / 10.0)
        rs.append(sum(g in set(int(x) for x in gt_ids[i, :10]) for g in got) / 10.0)
    return float(np.mean(rt)), float(np.mean(rs))


def bigann_launches(K: int, params, batch: int) -> int:
    """Kernels one sg_search_bigann call launches (bg_run in csrc/bigann.cu): per pass of queries,
    prep, the routing kernels (tensor-core: queries to bf16, the subset GEMM when the plan has one,
    thresholds, the filtered GEMM, select; FP32: scores, select), the scan, rerank and top-k."""
    P = max(min(params.nprobe, K), 1)
    ksub = -(-K // 16)
    subset, cap = False, K
    if not params.route_fp32 and K > 8192 and ksub >= 2 * P and max(8192, 32 * P) < K:
        subset, cap = True, max(8192, 32 * P)
    per_query = (ksub * 4 if subset else 0) + cap * 8 if not params.route_fp32 else K * 4
    per = max(1, min((1 << 30) // per_query, 65535))
    route = (5 if subset else 4) if not params.route_fp32 else 2
    return (1 + route + 1 + 2) * -(-batch // per)


def main_bigann(args, rank: int, world: int, local: int, dev: str):
    from sieve_gpu import bigann_builder as BB
    from sieve_gpu.bigann import BigannIndex, BigannTiming, parse_config as bg_parse

    wl = dict(WORKLOADS["c4"])
    if args.rows:
        wl["n"] = args.rows
    config = args.config or wl["search"]
    params = bg_parse(config, 10)
    nq_pool = min(max(args.batch * 2, args.eval, args.plain), wl["queries"])
    t0 = time.time()
    sp = BB.Spacev(wl["n"], wl["centers"], spread=40.0, sigma=12.0, seed=1, device=dev)
    base = sp.rows(0, wl["n"])
    t_ingest = time.time() - t0
    arrays = BB.build_bigann(base, wl["k1"], wl["k2"], bits=wl["bits"],
                             sample_n=min(wl["n"], max(2_000_000, wl["n"] // 10)), iters=6)
    t_build = time.time() - t0 - t_ingest
    queries = sp.queries(nq_pool)
    gt_ids, gt_sc = BB.ground_truth(base, queries[: args.eval], k=100)
    del base
    torch.cuda.empty_cache()
    log(f"workload c4: n={wl['n']} leaves={arrays['k']} ingest {t_ingest:.1f}s build {t_build:.1f}s "
        f"leaf sizes mean {arrays['sizes'].mean():.0f} max {arrays['sizes'].max()}")
    threads = os.cpu_count() or 1
    cfg = {"workload": f"c4: {wl['n']} x 100 int8 (1B shape cut to {wl['n']} rows), "
                       f"{wl['centers']} centres, {wl['k1']}x{wl['k2']} leaves, {wl['bits']}-bit refine",
           "search": config, "batch": args.batch, "queries_pool": nq_pool,
           "l2": "inputs larger than L2 (records and base far above 126 MB)"}
    build_info = {"ingest_s": round(t_ingest, 1), "build_s": round(t_build, 1)}
    metric = "QPS at R@10>=0.90 (p50/p99 ms, scan GB/s vs HBM peak)"
    qh_all = queries.cpu().numpy()

    def cpu_ref(seconds: float):
        import oracle as O

        ob = O.OracleBigann(arrays, native=True)
        p = params.to_c()
        probe = min(qh_all.shape[0], max(threads * 4, 64))
        t = time.perf_counter()
        ob.search_batch(qh_all[:probe], p, threads=threads)
        per_q = (time.perf_counter() - t) / probe
        n = int(min(qh_all.shape[0], max(probe, seconds / max(per_q, 1e-9))))
        t = time.perf_counter()
        s_, o_, c_, _ = ob.search_batch(qh_all[:n], p, threads=threads)
        dt = time.perf_counter() - t
        return {"qps": n / dt, "queries": n, "seconds": dt, "ids": o_, "cnt": c_}

    if args.impl == "reference":
        times, res = [], None
        for i in range(args.warmup + args.steps):
            res = cpu_ref(args.cpu_seconds / max(args.steps, 1))
            if i >= args.warmup:
                times.append(res["qps"])
        qps = float(np.mean(times))
        m = min(res["ids"].shape[0], gt_ids.shape[0])
        rec, rec_strict = recall10_ties(res["ids"][:m], res["cnt"][:m], gt_ids[:m], gt_sc[:m])
        line = {"metric": metric, "impl": "reference", "value": qps, "unit": "queries/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "i8/u8/f32", "data": "synthetic", "config": cfg,
                "recall_at_10": rec, "recall_at_10_strict": rec_strict, "build": build_info,
                "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": threads, "kind": "port",
                                 "sample": f"{res['queries']} queries per step on {threads} threads"},
                "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return finish(world)

    index = BigannIndex.from_arrays(arrays, device=local)
    q = queries.to(dev).contiguous()
    B = min(args.batch, nq_pool)
    k = params.k
    out_sc = torch.empty((B, k), dtype=torch.float32, device=dev)
    out_id = torch.empty((B, k), dtype=torch.int32, device=dev)
    out_n = torch.empty((B,), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    t_eval = BigannTiming()
    sc, ids, cnt = index.search_batch(qh_all[: args.eval], params, t_eval)
    rec, rec_strict = recall10_ties(ids, cnt, gt_ids, gt_sc)
    log(f"{config}: recall@10 {rec:.4f} (ties), {rec_strict:.4f} (strict)")

    def step(i):
        lo = (i * B) % (nq_pool - B + 1)
        index.search_device(B, q[lo].data_ptr(), params, out_sc.data_ptr(), out_id.data_ptr(),
                            out_n.data_ptr(), stream.cuda_stream)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    step_ms = []
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        for i in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(args.warmup + i)
            b.record(stream)
            b.synchronize()
            step_ms.append(a.elapsed_time(b))
    total_ms = max_over_ranks(float(np.sum(step_ms)), world, dev)
    qps = world * args.steps * B / (total_ms / 1e3)
    # stage times of one timed batch (the scan kernel's share and its algorithmic bytes)
    tb = BigannTiming()
    index.search_batch(qh_all[:B], params, tb)
    scan_s = tb.scan / 1e9
    achieved = tb.scanned * BG_SCAN_BYTES_PER_SLOT / scan_s / 1e9 if scan_s > 0 else None
    peaks = measured_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    plain_ms = []
    for i in range(args.plain):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        index.search_device(1, q[i].data_ptr(), params, out_sc.data_ptr(), out_id.data_ptr(),
                            out_n.data_ptr(), stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        plain_ms.append(a.elapsed_time(b))
    plain_ms = np.array(plain_ms[min(8, len(plain_ms) // 4):] or [float("nan")])
    qh = torch.empty((B, 100), dtype=torch.int8).pin_memory()
    osc = torch.empty((B, k), dtype=torch.float32).pin_memory()
    oid = torch.empty((B, k), dtype=torch.int32).pin_memory()
    ocn = torch.empty((B,), dtype=torch.int32).pin_memory()
    e2e_s = []
    for i in range(args.warmup + args.steps):
        lo = (i * B) % (nq_pool - B + 1)
        qh.copy_(queries[lo:lo + B].cpu())
        t = time.perf_counter()
        index.search_into(qh.numpy(), params, osc.numpy(), oid.numpy().view(np.uint32),
                          ocn.numpy().view(np.uint32))
        if i >= args.warmup:
            e2e_s.append(time.perf_counter() - t)
    e2e_qps = replica_qps(args.steps * B, float(np.sum(e2e_s)), world, dev)
    cpu = None
    if rank == 0 and world == 1 and args.cpu_seconds > 0:
        r = cpu_ref(args.cpu_seconds)
        cpu = {"value": r["qps"], "unit": "queries/s", "cores": threads, "kind": "port",
               "sample": f"{r['queries']} queries of the same workload, {r['seconds']:.1f} s, "
                         f"OpenMP over queries, oracle built -march=native"}
    line = {
        "metric": metric, "value": qps, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "i8 route/rerank, u8 LUT, f32 estimate",
        "data": "synthetic", "config": cfg, "recall_at_10": rec, "recall_at_10_strict": rec_strict,
        "recall_note": "big-ann recall@10 with ties (spacev) and strict; truth = exact int8 L2 over every row",
        "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
        "latency_note": "batched form: every query of a batch completes with its batch",
        "plain": {"qps": float(1e3 / np.mean(plain_ms)), "p50_ms": float(np.percentile(plain_ms, 50)),
                  "p99_ms": float(np.percentile(plain_ms, 99)), "queries": int(plain_ms.size)},
        "stage_ms": {"route": tb.route / 1e6, "scan": tb.scan / 1e6, "rerank": tb.rerank / 1e6},
        "scanned_per_query": tb.scanned / B,
        "roofline": {"bound": "hbm", "kernel": "k_bg_scan (the candidate scan)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback",
                     "traffic": None, "bytes_per_slot": BG_SCAN_BYTES_PER_SLOT},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_qps, "unit": "queries/s", "h2d_bytes_per_step": B * 100,
                "d2h_bytes_per_step": B * k * 8 + B * 4},
        "gpu_launches": args.steps * bigann_launches(int(arrays["k"]), params, B),
        "clocks": clocks.summary(),
        "build": build_info,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    index.close()
    return finish(world)


def finish(world: int):
    if world > 1 and torch.distributed.is_initialized():
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
