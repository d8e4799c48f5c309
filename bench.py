#!/usr/bin/env python
"""bench.py -- throughput of the B200 TOPAZ search hot path.

Headline workload (one step): the batched Smith-Waterman microbench --
1,000,000 (query, subject) pairs, query lengths log-normal (median 350,
30..1000), subject lengths log-normal (median 350, 30..5000), 80% background
/ 20% mutated homologues at 25-60% identity, BLOSUM62, gap 11/1, scores and
end coordinates with the u8 -> i16 -> drop semantics of TOPAZ's ssw_align.
Seeded synthetic data (no dataset exists for it).  Metric: GCUPS = sum over
pairs of qlen*slen cells per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]

N > 1 runs as torchrun ranks, one GPU each, every rank aligning its own
1,000,000 pairs (replicas, weak scaling, no data-path collective); the
timed region is bracketed by barriers and the max over ranks is reported.
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

METRIC = ("queries/s + SW GCUPS at identical hits; batched vs per-pair GPU; p50/p99 ms")
WORKLOAD = ("batched Smith-Waterman: 1,000,000 pairs/step, qlen lognormal(350) 30-1000, "
            "slen lognormal(350) 30-5000, 20% homologues 25-60% identity, BLOSUM62 11/1, "
            "scores+ends (ssw_align u8->i16->drop semantics)")
DPX_OPS_PER_CELL = 4      # 8 DPX instructions per int16x2 cell pair in the inner loop


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["native", "reference"], default="native")
    ap.add_argument("--pairs", type=int, default=1_000_000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--search-workers", type=int, default=3,
                    help="host threads issuing search batches concurrently")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop section")
    ap.add_argument("--search-large", action="store_true",
                    help="add a full search on a large DB (default and --fast)")
    ap.add_argument("--large-proteins", type=int, default=10_000_000)
    ap.add_argument("--large-queries", type=int, default=20_000)
    ap.add_argument("--search-proteins", type=int, default=1_000_000,
                    help="DB size of the full-search section (proteins)")
    ap.add_argument("--search-queries", type=int, default=10_000,
                    help="queries of the full-search section")
    ap.add_argument("--search-batch", type=int, default=0,
                    help="queries per tpz_search_batch call in the full-search sections; 0: an "
                         "equal share per worker thread (mid size), 2500 (large)")
    ap.add_argument("--no-search", action="store_true",
                    help="skip the full-search (config 2) section")
    ap.add_argument("--config3", action="store_true",
                    help="run only the large full search (30M proteins, 10^5 queries) through the "
                         "topaz CLI against the reference binary and print its JSON")
    ap.add_argument("--c3-proteins", type=int, default=30_000_000)
    ap.add_argument("--c3-queries", type=int, default=100_000)
    ap.add_argument("--c3-dir", default="/dev/shm/tpz_c3",
                    help="working directory of --config3 (DB files: ~10.5 bytes per residue)")
    ap.add_argument("--c3-ref-seconds", type=float, default=30.0,
                    help="reference run time per mode on its query sample")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


class ClockSampler:
    """nvidia-smi samples (200 ms) of this GPU during the timed region."""

    FIELDS = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str):
        self.bus = bus_id.lower()
        self.rows = []
        self.proc = None
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()
        # nvidia-smi's start-up holds the driver for a moment: wait for its
        # first sample so that it falls outside the timed region
        t0 = time.perf_counter()
        while not self.rows and time.perf_counter() - t0 < 10 and self.proc.poll() is None:
            time.sleep(0.05)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and parts[0].lower().endswith(self.bus[-7:]):
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.th:
            self.th.join(timeout=5)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_baseline_sw(ps, mat, budget_s=12.0):
    """The reference's own ssw_init+ssw_align (oracle/_ref, compiled from the
    TOPAZ sources) over all host threads on a bounded sample of the same
    pairs; falls back to the oracle port when _ref is absent."""
    import oracle
    kind = "reference" if oracle.libref() is not None else "port"
    fn = oracle.reference_sw if kind == "reference" else oracle.oracle_sw
    threads = os.cpu_count() or 1
    m = min(ps.n, 4 * threads * 50)
    t0 = time.perf_counter()
    fn(ps.q, ps.qoff[:m], ps.qlen[:m], ps.s, ps.soff[:m], ps.slen[:m], mat, 11, 1, threads)
    dt = time.perf_counter() - t0
    cells = int((ps.qlen[:m].astype(np.int64) * ps.slen[:m]).sum())
    if dt < budget_s * 0.5 and m < ps.n:
        m2 = int(min(ps.n, m * max(1.0, budget_s / max(dt, 1e-3))))
        t0 = time.perf_counter()
        fn(ps.q, ps.qoff[:m2], ps.qlen[:m2], ps.s, ps.soff[:m2], ps.slen[:m2], mat, 11, 1, threads)
        dt = time.perf_counter() - t0
        m = m2
        cells = int((ps.qlen[:m].astype(np.int64) * ps.slen[:m]).sum())
    return {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": threads, "kind": kind,
            "sample": "first %d of the %d pairs (%.2f Gcells) in %.1f s" % (m, ps.n, cells / 1e9, dt)}


def read_traffic():
    path = os.path.join(ROOT, "profiles", "sw_microbench_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_cell:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


SEARCH_WORKLOAD = ("full search, mid size: 1,000,000-protein synthetic DB (log-normal lengths "
                   "median 300, 50-2000; ~359M residues, int64 SA ~2.9 GB resident in HBM), "
                   "10,000 queries of 50-1500 residues (half mutated from DB proteins at 30-90%% "
                   "identity with indels, half random), SEG on, BLOSUM62 11/1, -H 100 -E 1e-3, "
                   "batches of %d queries")


SERVE_WORKLOAD = ("serving on the resident mid-size DB: Poisson request arrivals at 5 offered "
                  "loads (fractions of the loop's saturated throughput on this mix), each request 1-1000 "
                  "queries (log-uniform count) of 30-3000 residues, continuous batching across "
                  "requests by %d worker threads (batches up to %d queries, both picked by the "
                  "autotuner; admitted by free device memory), -H 100 -E 1e-3")


def serve_bench(ix, mat, res, lens, batch_qps, args, loads=(0.2, 0.4, 0.6, 0.8, 1.0),
                seconds=6.0):
    """p50/p99 request latency and delivered queries/s of the serving loop
    (topaz_b200.serve.SearchServer) at five offered loads."""
    from topaz_b200 import native, serve, synth
    qres, qlens = synth.search_queries_arrays(res, lens, 4000, 4000, seed=args.seed + 21,
                                              lo=30, hi=3000)
    qoff = np.cumsum(qlens) - qlens
    pool = native.prepare_queries([qres[o:o + n].tobytes() for o, n in zip(qoff, qlens)])
    rng = np.random.Generator(np.random.PCG64(args.seed + 22))
    # the loop's shape from the project's autotuner on a sample of this mix,
    # and its capacity: saturated throughput on the same mix
    rep = {"max_evalue": 1e-3}
    (workers, max_batch), tried = serve.autotune(ix, mat, pool[:4000], report=rep)
    capacity_qps = serve.saturated_qps(ix, mat, pool, workers, max_batch, report=rep)
    srv = serve.SearchServer(ix, mat, workers=workers, max_batch=max_batch, report=rep)
    srv.submit(pool[:50]).result()                        # warm-up
    rows = []
    mean_req = float(np.mean(np.exp(rng.uniform(0, np.log(1000), 100000))))
    for load in loads:
        qps = load * capacity_qps
        rate = qps / mean_req                              # requests per second
        futs, nq, t = [], 0, 0.0
        t0 = time.perf_counter()
        while t < seconds:
            t += rng.exponential(1.0 / rate)
            n = int(np.exp(rng.uniform(0, np.log(1000))))
            start = int(rng.integers(0, len(pool) - n))
            while time.perf_counter() - t0 < t:
                time.sleep(0.0005)
            futs.append(srv.submit(pool[start:start + n]))
            nq += n
        for f in futs:
            f.result()
        wall = time.perf_counter() - t0
        lat = np.array([serve.latency_of(f) for f in futs]) * 1e3
        rows.append({"offered_qps": round(qps, 1), "requests": len(futs), "queries": nq,
                     "delivered_qps": round(nq / wall, 1), "p50_ms": round(float(np.percentile(lat, 50)), 2),
                     "p99_ms": round(float(np.percentile(lat, 99)), 2)})
    srv.close()
    return {"workload": SERVE_WORKLOAD % (workers, max_batch), "capacity_qps": round(capacity_qps, 1),
            "capacity": "saturated throughput of the serving loop on this request mix",
            "batch_capacity_qps_config2_mix": round(batch_qps, 1),
            "autotune": {"%dx%d" % k: round(v, 1) for k, v in tried.items()},
            "loads": rows, "api": "topaz_b200.serve.SearchServer over tpz_search_batch report mode"}


def seed_roofline(positions, ms, tsize):
    """Seed lookup against HBM: algorithmic bytes per searched position =
    ceil(log2(Tsize+1)) x (8 B SA entry + 32 B text sector) -- the binary
    search of sa_search; the kernel's prefix table skips most of those steps,
    so the figure is the work it stands in for, not its own traffic."""
    peak, src = measured_hbm_gbs()
    steps = int(np.ceil(np.log2(tsize + 1)))
    gb = positions * steps * 40 / 1e9
    ach = gb / (ms / 1e3) if ms > 0 else None
    return {"positions": int(positions), "device_ms": round(ms, 2),
            "algorithmic_gb": round(gb, 2), "achieved_gbs": round(ach, 1) if ach else None,
            "peak_gbs": peak, "frac": round(ach / peak, 3) if ach and peak else None,
            "peak_source": src}


def extension_roofline(chain_elems, chain_ms, refill_elems, pops):
    """Gapless extension (sa_hsp) of the cursor chains against HBM:
    algorithmic bytes per call = the 8-byte SA entry + the text window's
    32-byte sectors, up to 8 (128 residues each side); the chain kernel's
    calls over its device time.  Also how many of the computed extensions
    the walk used (one per pop)."""
    peak, src = measured_hbm_gbs()
    gb = chain_elems * (8 + 8 * 32) / 1e9
    ach = gb / (chain_ms / 1e3) if chain_ms > 0 else None
    return {"chain_calls": int(chain_elems), "walk_refill_calls": int(refill_elems),
            "device_ms": round(chain_ms, 2), "algorithmic_gb": round(gb, 2),
            "achieved_gbs": round(ach, 1) if ach else None, "peak_gbs": peak,
            "frac": round(ach / peak, 3) if ach and peak else None, "peak_source": src,
            "bytes_per_call": "8 B SA entry + up to 8 x 32 B text sectors",
            "computed_over_used": round((chain_elems + refill_elems) / max(pops, 1), 2),
            "l2_hit_rate": "profiles/search_kernels_small.md (ncu)"}


_HBM_LIVE = []


def measured_hbm_gbs():
    """(peak GB/s, where it comes from): MEASURED_PEAKS.json when present, else a
    device-to-device copy of 2 GiB timed here (bytes read + written), else the
    fallback figure"""
    try:
        return (float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]),
                "measured: MEASURED_PEAKS.json hbm_gbs (copy)")
    except (OSError, KeyError, ValueError):
        pass
    if not _HBM_LIVE:
        try:
            import torch
            n = 1 << 31
            a = torch.empty(n, dtype=torch.uint8, device="cuda")
            b = torch.empty(n, dtype=torch.uint8, device="cuda")
            for _ in range(2):
                b.copy_(a)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(5):
                b.copy_(a)
            e1.record()
            torch.cuda.synchronize()
            _HBM_LIVE.append(2 * n * 5 / (e0.elapsed_time(e1) / 1e3) / 1e9)
            del a, b
            torch.cuda.empty_cache()
        except Exception:                  # no device: the fallback below
            _HBM_LIVE.append(None)
    if _HBM_LIVE[0]:
        return round(_HBM_LIVE[0], 1), "measured live: 2 GiB device-to-device copy (read + write bytes)"
    return 6650.0, "fallback: 6.65 TB/s, an earlier copy measurement on this pool"


def large_bench(args, dev):
    """Full search on a larger DB than the mid-size config: index built on the
    device, default and --fast sensitivity, report mode, 2 host threads."""
    import torch

    from topaz_b200 import dbformat, native, synth
    t0 = time.perf_counter()
    res, lens = synth.protein_db_arrays(args.large_proteins, seed=args.seed + 31)
    db = dbformat.build_from_arrays(res, lens)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    db.SA = native.sa_build(db.T)
    sa_s = time.perf_counter() - t0
    torch.cuda.empty_cache()
    qres, qlens = synth.search_queries_arrays(res, lens, args.large_queries // 2,
                                              args.large_queries - args.large_queries // 2,
                                              seed=args.seed + 32)
    qoff = np.cumsum(qlens) - qlens
    qs = native.prepare_queries([qres[o:o + n].tobytes() for o, n in zip(qoff, qlens)])
    del res
    t0 = time.perf_counter()
    ix = native.Index(db)
    load_s = time.perf_counter() - t0
    mat = synth.matrix("BLOSUM62")
    report = {"max_evalue": 1e-3}
    bsz = args.search_batch or 2500
    out = {"workload": "full search, large: %d-protein synthetic DB (%.2f G residues, log-normal "
                       "lengths median 300, 50-2000), %d queries of 50-1500 residues (half mutated, "
                       "half random), SEG on, BLOSUM62 11/1, -H 100 -E 1e-3, batches of %d from 2 "
                       "host threads" % (args.large_proteins, len(db.T) / 1e9, len(qs), bsz),
           "db_bytes": int(len(db.T)), "generate_s": round(gen_s, 1), "sa_build_s": round(sa_s, 2),
           "index_load_s": round(load_s, 2), "index_device_gb": round(ix.device_bytes / 1e9, 2)}
    for mode, seeds, aligns in (("default", 300000, 5000), ("fast", 100000, 1500)):
        ix.search(qs[:bsz], mat, report=report, seeds=seeds, alignments=aligns)   # warm-up
        starts = list(range(0, len(qs), bsz))
        lock = threading.Lock()
        nh = [0]

        def worker():
            while True:
                with lock:
                    if not starts:
                        return
                    b = starts.pop(0)
                r = ix.search(qs[b:b + bsz], mat, report=report, seeds=seeds, alignments=aligns)
                with lock:
                    nh[0] += len(r["protein"])

        t0 = time.perf_counter()
        th = [threading.Thread(target=worker) for _ in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        wall = time.perf_counter() - t0
        out[mode] = {"queries_per_s": round(len(qs) / wall, 1), "wall_s": round(wall, 2),
                     "seeds": seeds, "alignments": aligns,
                     "reported_hits_per_query": round(nh[0] / len(qs), 2)}
    ix.close()
    return out


def search_bench(args, dev):
    """Full-search throughput (queries/s) through tpz_search_batch with host
    buffers (SEG + internal alphabet on the host, H2D of queries, D2H of
    hit lists inside the timed region), with the reference binary timed on a
    query sample on all host threads and its output compared per query."""
    import subprocess
    import tempfile

    import torch

    import oracle
    from topaz_b200 import build as B, dbformat, native, synth

    t0 = time.perf_counter()
    res, lens = synth.protein_db_arrays(args.search_proteins, seed=args.seed + 11)
    db = dbformat.build_from_arrays(res, lens)
    t1 = time.perf_counter()
    db.SA = native.sa_build(db.T)          # the device SA builder of `topaz index`
    sa_s = time.perf_counter() - t1
    torch.cuda.empty_cache()
    qres, qlens = synth.search_queries_arrays(res, lens, args.search_queries // 2,
                                              args.search_queries - args.search_queries // 2,
                                              seed=args.seed + 12)
    qoff = np.cumsum(qlens) - qlens
    q_aa = [qres[o:o + n].tobytes() for o, n in zip(qoff, qlens)]
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    ix = native.Index(db)
    load_s = time.perf_counter() - t0
    mat = synth.matrix("BLOSUM62")
    report = {"max_evalue": 1e-3}                     # -H 100 -E 1e-3, ranked on the device
    # one batch per worker thread: with more batches than threads the last
    # batch runs alone on a device the other threads have left idle
    bsz = args.search_batch or -(-len(q_aa) // args.search_workers)
    # warm-up: one full-size batch per worker thread, so that the device
    # memory pool of every thread has grown to a batch before the timing
    warm = native.prepare_queries(q_aa[:bsz])

    def warm_one():
        ix.search(warm, mat, report=report)

    th = [threading.Thread(target=warm_one) for _ in range(args.search_workers)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    torch.cuda.synchronize()
    stage = np.zeros(4)
    nh = [0]
    swc = [0, 0, 0.0, 0.0, 0, 0, 0]
    pops = []
    starts = list(range(0, len(q_aa), bsz))
    lock = threading.Lock()

    def worker():
        # batches taken in order by host threads, each thread on its own CUDA
        # default stream, so one batch's SW overlaps another's walk
        while True:
            with lock:
                if not starts:
                    return
                b = starts.pop(0)
            qs = native.prepare_queries(q_aa[b:b + bsz])
            r = ix.search(qs, mat, report=report)
            with lock:
                stage[:] += np.array(r["stage_ms"])
                nh[0] += len(r["protein"])
                swc[0] += r["sw_pairs"]
                swc[1] += r["sw_cells"]
                swc[2] += r["seed_ms"]
                swc[3] += r["chain_ms"]
                swc[4] += r["positions"]
                swc[5] += r["chain_elems"]
                swc[6] += r["refill_elems"]
                pops.extend(r["npops"].tolist())

    t0 = time.perf_counter()
    th = [threading.Thread(target=worker) for _ in range(args.search_workers)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    wall = time.perf_counter() - t0
    nh = nh[0]
    wl = SEARCH_WORKLOAD % bsz
    if (args.search_proteins, args.search_queries) != (1_000_000, 10_000):
        wl = ("smaller full search: %d-protein synthetic DB, %d queries (otherwise as the "
              "mid-size config), batches of %d" % (args.search_proteins, args.search_queries, bsz))
    out = {"workload": wl, "queries": len(q_aa), "queries_per_s": round(len(q_aa) / wall, 1),
           "wall_s": round(wall, 3),
           "api": "tpz_search_batch report mode (host buffers; SEG + alphabet on the host by "
                  "tpz_prepare_queries, "
                  "ranking and -H/-E cut on the device, all inside the timed region; "
                  "batches from %d host threads)" % args.search_workers,
           "device_ms": {"seed": round(stage[0], 2), "walk_hitlist": round(stage[1], 2),
                         "sw_rank_select": round(stage[2], 2), "calls_wall": round(stage[3], 2)},
           "reported_hits_per_query": round(nh / len(q_aa), 2),
           "sw_pairs_per_query": round(swc[0] / len(q_aa), 1),
           "sw_gcells": round(swc[1] / 1e9, 2),
           "seed_lookup": seed_roofline(swc[4], swc[2], len(db.T)),
           "extension": extension_roofline(swc[5], swc[3], swc[6], int(np.sum(pops))),
           "pops_per_query": {"mean": round(float(np.mean(pops)), 1),
                              "p50": int(np.percentile(pops, 50)), "p99": int(np.percentile(pops, 99)),
                              "max": int(np.max(pops))},
           "host_threads": args.search_workers,
           "setup_s": round(setup_s, 1), "index_load_s": round(load_s, 2),
           "sa_build_s": round(sa_s, 2), "sa_bytes": int(len(db.T)),
           "index_device_gb": round(ix.device_bytes / 1e9, 2)}
    if not args.no_serve:
        out["serving"] = serve_bench(ix, mat, res, lens, len(q_aa) / wall, args)
    ix.close()
    if args.no_cpu_baseline or not os.path.exists(oracle.REF_BIN):
        return out
    # the reference binary on a query sample, all host threads; our CLI on the
    # same sample; outputs compared per query block
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as tmp:
        pre = os.path.join(tmp, "db")
        dbformat.write_files(pre, db)
        # both binaries find the DB files in the page cache (cat DB.* > /dev/null)
        for e in (".psq", ".SA", ".phr", ".pin", ".ind"):
            with open(pre + e, "rb") as fh:
                while fh.read(64 << 20):
                    pass

        def run(exe, idx, extra=(), tag="q"):
            fa = os.path.join(tmp, "%s%d.fa" % (tag, len(idx)))
            synth.write_fasta(fa, synth.Proteins(["q%d" % i for i in idx],
                                                 [np.frombuffer(q_aa[i], np.uint8) for i in idx]))
            t = time.perf_counter()
            r = subprocess.run([exe, "search", "-f", fa, "-p", pre, "-T", str(threads), *extra],
                               capture_output=True, cwd=tmp)
            return time.perf_counter() - t, r

        def spread(n):
            # n queries evenly spaced over the whole query set, so that the
            # mutated and the random halves are both represented
            return np.unique(np.linspace(0, len(q_aa) - 1, n).astype(np.int64)).tolist()

        def blocks(text):
            d = {}
            for ln in text.decode().splitlines()[1:]:
                d.setdefault(ln.split("\t", 1)[0], []).append(ln)
            return d

        dt, _ = run(oracle.REF_BIN, spread(4 * threads))
        n = int(min(len(q_aa), max(4 * threads, 4 * threads * 15.0 / max(dt, 1e-3))))
        sample = spread(n)
        dt, rr = run(oracle.REF_BIN, sample)
        dt_cli, rm = run(B.CLI, sample)
        dt_cli_all, r_all = run(B.CLI, list(range(len(q_aa))))
        cli_stages = [ln for ln in r_all.stderr.decode(errors="replace").splitlines()
                      if ln.startswith("timing:")]
        half = len(q_aa) // 2
        out["cpu_reference"] = {"queries_per_s": round(len(sample) / dt, 2), "threads": threads,
                                "kind": "reference", "sample": "%d queries evenly spaced over the %d "
                                "(%d mutated, %d random), topaz search -T %d, DB files in page cache"
                                % (len(sample), len(q_aa), sum(i < half for i in sample),
                                   sum(i >= half for i in sample), threads)}
        out["parity_sample"] = {"default": {"queries": len(sample),
                                            "identical_blocks": blocks(rr.stdout) == blocks(rm.stdout),
                                            "lines": rr.stdout.count(b"\n") - 1}}
        # --fast and --blasttab on smaller evenly spaced samples, each mode
        # compared per query block and timed for both binaries
        for mode, extra, frac in (("fast", ("--fast",), 0.5), ("blasttab", ("--blasttab",), 0.5)):
            sm = spread(max(4 * threads, int(len(sample) * frac)))
            dr, r1 = run(oracle.REF_BIN, sm, extra, tag=mode)
            do, r2 = run(B.CLI, sm, extra, tag=mode)
            out["parity_sample"][mode] = {
                "queries": len(sm), "identical_blocks": blocks(r1.stdout) == blocks(r2.stdout),
                "lines": r1.stdout.count(b"\n") - 1,
                "reference_queries_per_s": round(len(sm) / dr, 2),
                "cli_queries_per_s": round(len(sm) / do, 2)}
        # our `topaz search` as a user runs it: process start to exit (CUDA
        # context, index upload, FASTA, SEG, search, output), -T as above
        # (at most 4 batches in flight), on the sample and on all queries
        out["cli"] = {"queries_per_s_sample": round(len(sample) / dt_cli, 1),
                      "queries_per_s_all": round(len(q_aa) / dt_cli_all, 1),
                      "sample_s": round(dt_cli, 2), "all_s": round(dt_cli_all, 2),
                      "stages_all": cli_stages[0] if cli_stages else None,
                      "threads": threads, "api": "topaz search CLI (whole process)"}
        # `topaz index` on the first 100,000 proteins: the reference (host
        # SA-IS) and ours (SA on the device), files compared
        m = min(100_000, len(lens))
        off = np.cumsum(lens) - lens
        fa = os.path.join(tmp, "idx.fa")
        synth.write_fasta(fa, synth.Proteins(["db%d" % i for i in range(m)],
                                             [res[off[i]:off[i] + lens[i]] for i in range(m)]))
        ti = {}
        for who, exe in (("reference", oracle.REF_BIN), ("ours", B.CLI)):
            pre = os.path.join(tmp, "idx_" + who)
            t = time.perf_counter()
            subprocess.run([exe, "index", "-f", fa, "-p", pre], check=True, capture_output=True)
            ti[who] = time.perf_counter() - t
        same = all(open(os.path.join(tmp, "idx_reference") + e, "rb").read() ==
                   open(os.path.join(tmp, "idx_ours") + e, "rb").read()
                   for e in (".SA", ".psq", ".ind", ".pin", ".phr"))
        out["index_build"] = {"proteins": m, "residues": int(lens[:m].sum()),
                              "reference_s": round(ti["reference"], 2), "ours_s": round(ti["ours"], 2),
                              "identical_files": same, "api": "topaz index (CLI), SA on the device"}
    return out


C3_WORKLOAD = ("full search, large: %d-protein synthetic DB (log-normal lengths median 300, "
               "50-2000, Robinson-Robinson residues; %.2f G residues, int64 SA %.1f GB), %d queries "
               "of 50-1500 residues (half mutated from DB proteins at 30-90%% identity with "
               "indels, half random), SEG on, BLOSUM62 11/1, -H 100 -E 1e-3; default, --fast "
               "and --blasttab")


def config3_bench(args):
    """The large full search end to end through the command line: the DB
    FASTA is written, `topaz index` (ours; suffix array on the device) builds
    the files, our `topaz search` runs all queries in default, --fast and
    --blasttab modes, and the reference binary `topaz search -T nproc` runs
    an evenly spaced query sample of each mode on the same files; outputs
    are compared per query block."""
    import shutil

    import oracle
    from topaz_b200 import build as B, synth
    threads = os.cpu_count() or 1
    d = args.c3_dir
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(d)
    out = {}
    try:
        fa, qfa, pre = os.path.join(d, "db.fa"), os.path.join(d, "q.fa"), os.path.join(d, "db")
        t0 = time.perf_counter()
        lens, sstart = synth.write_db_fasta(fa, args.c3_proteins, seed=args.seed + 41)
        residues = int(lens.sum())
        need = int(11.5 * residues)
        free = shutil.disk_usage(d).free
        if free < need:
            return {"unavailable": "working directory %s has %.0f GB free, the DB needs ~%.0f GB"
                                   % (d, free / 1e9, need / 1e9)}
        mm = np.memmap(fa, np.uint8, mode="r")
        nq = args.c3_queries
        qres, qlens = synth.search_queries_arrays(
            lambda pick: synth.fasta_residues(mm, sstart, lens, pick), lens, nq // 2, nq - nq // 2,
            seed=args.seed + 42)
        del mm
        qoff = np.cumsum(qlens) - qlens
        ids = ["q%d" % i for i in range(nq)]
        synth.write_fasta(qfa, synth.Proteins(ids, [qres[o:o + n] for o, n in zip(qoff, qlens)]))
        gen_s = time.perf_counter() - t0
        out["workload"] = C3_WORKLOAD % (args.c3_proteins, residues / 1e9, 8 * (residues + len(lens)) / 1e9, nq)
        out["generate_s"] = round(gen_s, 1)
        # `topaz index` (ours): FASTA -> .pin/.psq/.phr/.ind, SA on the device
        t0 = time.perf_counter()
        r = subprocess.run([B.CLI, "index", "-f", fa, "-p", pre], capture_output=True)
        out["index"] = {"seconds": round(time.perf_counter() - t0, 1), "rc": r.returncode,
                        "stderr_tail": r.stderr.decode(errors="replace")[-400:],
                        "sa_bytes": os.path.getsize(pre + ".SA") if os.path.exists(pre + ".SA") else 0}
        os.remove(fa)
        if r.returncode != 0:
            return out

        def run(exe, qpath, extra, dst):
            with open(dst, "wb") as fo:
                t = time.perf_counter()
                rr = subprocess.run([exe, "search", "-f", qpath, "-p", pre, "-T", str(threads), *extra],
                                    stdout=fo, stderr=subprocess.PIPE, cwd=d)
                return time.perf_counter() - t, rr

        def blocks(path, keep=None):
            bl = {}
            with open(path, "rb") as fh:
                head = fh.readline()
                for ln in fh:
                    q = ln.split(b"\t", 1)[0]
                    if keep is None or q in keep:
                        bl.setdefault(q, []).append(ln)
            return head, bl

        def spread(n):
            return np.unique(np.linspace(0, nq - 1, n).astype(np.int64)).tolist()

        modes = (("default", []), ("fast", ["--fast"]), ("blasttab", ["--blasttab"]))
        for mode, extra in modes:
            dst = os.path.join(d, "ours_%s.out" % mode)
            dt, rr = run(B.CLI, qfa, extra, dst)
            timing = [ln for ln in rr.stderr.decode(errors="replace").splitlines()
                      if ln.startswith("timing:")]
            out[mode] = {"queries_per_s": round(nq / dt, 1), "wall_s": round(dt, 1),
                         "rc": rr.returncode, "stages": timing[0] if timing else None,
                         "api": "topaz search CLI, whole process, -T %d" % threads}
        if not os.path.exists(oracle.REF_BIN):
            return out
        # the reference on evenly spaced samples (mutated and random halves)
        probe = spread(2 * threads)
        pf = os.path.join(d, "probe.fa")
        synth.write_fasta(pf, synth.Proteins([ids[i] for i in probe],
                                             [qres[qoff[i]:qoff[i] + qlens[i]] for i in probe]))
        dt, _ = run(oracle.REF_BIN, pf, [], os.path.join(d, "probe.out"))
        rate = len(probe) / dt
        for mode, extra in modes:
            n = int(min(nq, max(2 * threads, rate * args.c3_ref_seconds * (2.0 if mode == "fast" else 1.0))))
            sample = spread(n)
            sf = os.path.join(d, "sample_%s.fa" % mode)
            synth.write_fasta(sf, synth.Proteins([ids[i] for i in sample],
                                                 [qres[qoff[i]:qoff[i] + qlens[i]] for i in sample]))
            dst = os.path.join(d, "ref_%s.out" % mode)
            dr, rr = run(oracle.REF_BIN, sf, extra, dst)
            keep = {ids[i].encode() for i in sample}
            h1, b1 = blocks(dst)
            h2, b2 = blocks(os.path.join(d, "ours_%s.out" % mode), keep)
            ref_qps = len(sample) / dr
            out[mode].update({
                "reference_queries_per_s": round(ref_qps, 2),
                "reference_sample": "%d queries evenly spaced over the %d (%d mutated, %d random), "
                                    "topaz search -T %d" % (len(sample), nq,
                                                            sum(i < nq // 2 for i in sample),
                                                            sum(i >= nq // 2 for i in sample), threads),
                "reference_rc": rr.returncode,
                "over_reference": round(out[mode]["queries_per_s"] / ref_qps, 1),
                "identical_blocks": h1 == h2 and b1 == b2,
                "blocks_compared": len(b1), "lines_compared": sum(len(v) for v in b1.values())})
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def per_pair_bench(torch, t, ps, mat, dev, batched_gcups, npairs=20000, nstreams=(1, 16)):
    """GCUPS of one kernel launch per pair (tpz_sw_align_one) on an evenly
    spaced sample of the workload's pairs with qlen <= 1024, launched from
    one host thread round-robin over 1 and over 16 CUDA streams."""
    from topaz_b200 import native
    idx = np.linspace(0, ps.n - 1, npairs).astype(np.int64)
    idx = idx[ps.qlen[idx] <= 1024]
    cells = int((ps.qlen[idx].astype(np.int64) * ps.slen[idx]).sum())
    out = torch.empty((len(idx), 4), dtype=torch.int32, device=dev)
    matc = np.ascontiguousarray(mat, dtype=np.int8)
    L = native.lib()
    qb, sb, ob = t["q"].data_ptr(), t["s"].data_ptr(), out.data_ptr()
    qoff, qlen, soff, slen = ps.qoff[idx], ps.qlen[idx], ps.soff[idx], ps.slen[idx]
    res = {"pairs": len(idx), "cells": cells, "api": "tpz_sw_align_one"}
    for ns in nstreams:
        streams = [torch.cuda.Stream(device=dev) for _ in range(ns)]
        handles = [st.cuda_stream for st in streams]
        for i in range(min(64, len(idx))):            # warm-up
            native.check(L.tpz_sw_align_one(qb + int(qoff[i]), int(qlen[i]), sb + int(soff[i]),
                                            int(slen[i]), matc.ctypes.data, 11, 1, ob + 16 * i,
                                            handles[i % ns]))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(len(idx)):
            native.check(L.tpz_sw_align_one(qb + int(qoff[i]), int(qlen[i]), sb + int(soff[i]),
                                            int(slen[i]), matc.ctypes.data, 11, 1, ob + 16 * i,
                                            handles[i % ns]))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        got = out.cpu().numpy()
        ok = bool((got[:, 0] == t["score"][torch.from_numpy(idx).to(dev)].cpu().numpy()).all())
        res["streams_%d" % ns] = {"gcups": round(cells / dt / 1e9, 3), "seconds": round(dt, 3),
                                  "scores_match_batched": ok,
                                  "batched_over_per_pair": round(batched_gcups / (cells / dt / 1e9), 1)}
    return res


def native_arm(args, rank, local_rank, world):
    import torch
    import torch.distributed as dist

    from topaz_b200 import native, replicas, synth

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        dist.init_process_group("nccl", device_id=dev,
                                timeout=__import__("datetime").timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    ps = synth.sw_pairs(args.pairs, seed=args.seed + 1000 * rank)
    mat = synth.matrix("BLOSUM62")
    cells = ps.cells
    t = {k: torch.from_numpy(np.ascontiguousarray(getattr(ps, k))).to(dev)
         for k in ("q", "qoff", "qlen", "s", "soff", "slen")}
    for k in ("score", "ref_end", "read_end", "status"):
        t[k] = torch.empty(ps.n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()

    # roofline denominator: DPX issue rate on this GPU
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    probe_out = torch.empty(nsm * 8 * 256, dtype=torch.int32, device=dev)
    for _ in range(2):
        native.dpx_probe(nsm * 8, 4096, probe_out.data_ptr(), stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ops = native.dpx_probe(nsm * 8, 65536, probe_out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    dpx_ops_s = ops / (e0.elapsed_time(e1) / 1e3)
    peak_gcups = dpx_ops_s / DPX_OPS_PER_CELL / 1e9

    pr = torch.cuda.get_device_properties(dev)
    bus = "%08X:%02X:%02X.0" % (getattr(pr, "pci_domain_id", 0), getattr(pr, "pci_bus_id", 0),
                                getattr(pr, "pci_device_id", 0))
    clocks = ClockSampler(bus or "")
    clocks.start()
    # warm-up right before the timed steps, so that the clocks do not idle
    # down in between
    barrier()
    for _ in range(args.warmup):
        native.sw_batch_torch(t, mat, 11, 1)
    launches_per_step = native.last_launches()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    torch.cuda.synchronize()
    barrier()
    ev[0].record(stream)
    for i in range(args.steps):
        native.sw_batch_torch(t, mat, 11, 1)
        ev[i + 1].record(stream)
    torch.cuda.synchronize()
    barrier()
    status = t["status"].cpu().numpy()
    assert (status == native.TPZ_SW_OK).all(), "pairs not aligned: %s" % np.unique(status)
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = sum(step_ms)
    max_ms = replicas.max_over_ranks(total_ms, world, dev)
    value = world * cells * args.steps / (max_ms / 1e3) / 1e9
    achieved = cells / (total_ms / args.steps / 1e3) / 1e9

    # end to end: host buffers through the C ABI, H2D + D2H inside the step
    pin = {k: torch.from_numpy(np.ascontiguousarray(getattr(ps, k))).pin_memory()
           for k in ("q", "qoff", "qlen", "s", "soff", "slen")}
    outs = {k: torch.empty(ps.n, dtype=torch.int32).pin_memory()
            for k in ("score", "ref_end", "read_end", "status")}
    matc = np.ascontiguousarray(mat, dtype=np.int8)
    L = native.lib()

    def e2e_step():
        native.check(L.tpz_sw_batch_host(
            ps.n, pin["q"].data_ptr(), pin["qoff"].data_ptr(), pin["qlen"].data_ptr(),
            pin["s"].data_ptr(), pin["soff"].data_ptr(), pin["slen"].data_ptr(),
            matc.ctypes.data, 11, 1, outs["score"].data_ptr(), outs["ref_end"].data_ptr(),
            outs["read_end"].data_ptr(), outs["status"].data_ptr()))

    e2e_step()
    assert (outs["score"].numpy() == t["score"].cpu().numpy()).all()
    barrier()
    for _ in range(args.warmup):
        e2e_step()              # W untimed steps right before the timed ones
    e2e_ms = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        t1 = time.perf_counter()
        e2e_step()
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
    e2e_s = time.perf_counter() - t0
    e2e_max_s = replicas.max_over_ranks(e2e_s, world, dev)
    barrier()
    e2e_val = world * cells * args.steps / e2e_max_s / 1e9
    clk = clocks.stop()         # the samples cover the device-timed and the e2e steps
    h2d = sum(v.numel() * v.element_size() for v in pin.values())
    d2h = sum(v.numel() * v.element_size() for v in outs.values())

    # the plain per-pair-launch GPU form: one tpz_sw_align_one launch per pair
    # (the per-hit ssw_init + ssw_align pattern moved to the GPU) on a sample
    per_pair = None
    if rank == 0:
        per_pair = per_pair_bench(torch, t, ps, mat, dev, achieved)

    line = None
    search = None
    large = None
    if rank == 0 and world == 1 and not args.no_search:
        del t, pin, outs
        torch.cuda.empty_cache()
        search = search_bench(args, dev)
    if rank == 0 and world == 1 and args.search_large:
        torch.cuda.empty_cache()
        large = large_bench(args, dev)
    if rank == 0:
        # the host-core baseline is an N=1 figure: rank 0 of a single-GPU run
        cpu = None if (args.no_cpu_baseline or world > 1) else cpu_baseline_sw(ps, mat)
        traffic_per_cell = read_traffic()
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GCUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16x2",
            "data": "synthetic (seeded PCG64; Robinson-Robinson background, BLOSUM62-conditional homologues)",
            "config": {"workload": WORKLOAD, "pairs_per_step": ps.n, "cells_per_step": cells,
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (%.2f GB resident per step)" % (h2d / 1e9)},
            "e2e": {"value": round(e2e_val, 2), "unit": "GCUPS", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "step_ms": [round(x, 2) for x in e2e_ms],
                    "api": "tpz_sw_batch_host (pinned host buffers)"},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": {"bound": "dpx", "achieved": round(achieved, 2),
                         "peak": round(peak_gcups, 2), "unit": "GCUPS",
                         "frac": round(achieved / peak_gcups, 4),
                         "peak_source": "measured live: __viaddmax_s16x2 issue rate %.3e op/s / %d DPX ops per cell"
                                        % (dpx_ops_s, DPX_OPS_PER_CELL),
                         "traffic": (round(traffic_per_cell * cells) if traffic_per_cell else None),
                         "traffic_source": ("not measured in this run: DRAM bytes per cell of the "
                                            "ncu capture in profiles/sw_microbench_traffic.txt "
                                            "(100,000-pair case), scaled to this step's cells"
                                            if traffic_per_cell else None)},
            "cpu_baseline": cpu,
            "per_pair_gpu": per_pair,
            "clocks": clk,
            "step_ms": [round(x, 3) for x in step_ms],
            "search": search,
        }
        if large is not None:
            line["search_large"] = large
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line


def reference_arm(args, rank, world):
    """The reference's own CPU implementation of the path (ssw_init+ssw_align
    compiled from the TOPAZ sources into oracle/_ref), all host threads, each
    step a bounded sample of the same workload."""
    if rank != 0:
        return None
    import oracle
    from topaz_b200 import synth
    if oracle.libref() is None:
        return {"impl": "reference", "unavailable": "oracle/_ref (reference build) is not present"}
    ps = synth.sw_pairs(args.pairs, seed=args.seed)
    mat = synth.matrix("BLOSUM62")
    threads = os.cpu_count() or 1
    # size one step to about 8 s of work
    m = min(ps.n, 200 * threads)
    t0 = time.perf_counter()
    oracle.reference_sw(ps.q, ps.qoff[:m], ps.qlen[:m], ps.s, ps.soff[:m], ps.slen[:m], mat, 11, 1, threads)
    dt = time.perf_counter() - t0
    m = int(min(ps.n, max(m, m * 8.0 / max(dt, 1e-3))))
    times, cells_l = [], []
    for i in range(args.warmup + args.steps):
        off = (i * m) % max(1, ps.n - m + 1)
        sl = slice(off, off + m)
        t0 = time.perf_counter()
        oracle.reference_sw(ps.q, ps.qoff[sl], ps.qlen[sl], ps.s, ps.soff[sl], ps.slen[sl], mat, 11, 1, threads)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            cells_l.append(int((ps.qlen[sl].astype(np.int64) * ps.slen[sl]).sum()))
    value = sum(cells_l) / sum(times) / 1e9
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GCUPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8/i16 SSE2",
        "data": "synthetic (seeded PCG64)",
        "config": {"workload": WORKLOAD, "pairs_per_step": m,
                   "parallelism": "%d host threads" % threads},
        "cpu_baseline": {"value": round(value, 3), "unit": "GCUPS", "cores": threads,
                         "kind": "reference",
                         "sample": "%d consecutive pairs per step of the 1,000,000-pair workload" % m},
        "e2e": {"value": round(value, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    rank, local_rank, world = dist_env()
    if args.warmup < 3 and args.impl == "native":
        args.warmup = 3
    if args.config3:
        line = {"search_config3": config3_bench(args)} if rank == 0 else None
    elif args.impl == "reference":
        line = reference_arm(args, rank, world)
    else:
        line = native_arm(args, rank, local_rank, world)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
