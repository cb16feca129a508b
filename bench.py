"""Benchmark: all-pairs SW-Gotoh distance matrix on B200 (batched engine), one JSON line.

Workload: 20,000 synthetic DNA sequences, lognormal lengths (median 400, sigma 0.6, clipped
50-1,500), 200 family roots, EDNAFULL, gap open 16 / extend 4, PercentIdentity -> Int16.  A step
is one MPI rank's share of an 8-rank run of that job (the pairs rank b aligns in
MPIComputeLowerTriangularBlocked.Compute), so W = 3 warm-up steps then K = 8 timed steps time the
whole job once on one GPU.  With N GPUs (torchrun) each rank takes a different share per step
(no data-path collective; "weak" scaling: per-GPU work per step is fixed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Besides the headline value (inputs resident in HBM), the line carries: e2e (the same job driven
through host buffers, copies inside the timed region), the integer-pipe roofline of the engine
kernels (peak measured live by a calibration kernel), a CPU baseline (the reference's own
aligner and ComputeDistance, transliterated from its C# and run on the host cores), a parity
spot check of that sample against the GPU matrix, the plain one-launch-per-block kernel versus
the batched engine on the same 2,000-sequence block, and the SM clocks sampled while timing.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = dict(n=20000, median=400, sigma=0.6, lo=50, hi=1500, roots=200, seed=3)
OPS_PER_CELL = 11      # algorithmic integer ops of one SW-Gotoh cell (E, F, H, running best)
LANES_PER_OP = 2       # the engine's score registers hold two 16-bit lanes
SHARES = 8             # steps per whole job: the shares of an 8-rank run
SERVE = dict(db=100000, qmin=1, qmax=512, load=0.7, seconds=40.0, seed=6)
ENGINE_OPTIONS = {}    # engine knobs from the command line (sw_set_option), applied to every engine


def with_options(eng):
    for k, v in ENGINE_OPTIONS.items():
        eng.set_option(k, v)
    return eng


def workload_sequences(n):
    from csharp_b200 import pack_sequences, synth
    rng = np.random.default_rng(WORKLOAD["seed"] + 1000)
    lens = synth.lognormal_lengths(n, WORKLOAD["median"], WORKLOAD["sigma"], WORKLOAD["lo"], WORKLOAD["hi"], rng)
    seqs = synth.dna_family(n, WORKLOAD["roots"], lens, WORKLOAD["seed"])
    return pack_sequences(seqs)


def sample_pairs(n, count, rng):
    """`count` pairs drawn uniformly from the job, oriented (s1, s2) as the SHARES-rank run
    orients them: diagonal blocks align (s_i, s_j) for i > j; block (r, c) is aligned by the rank
    the checkerboard names, with s1 from its rows."""
    from csharp_b200 import block_is_computed, range_partition
    ii = rng.integers(1, n, count)
    jj = (rng.random(count) * ii).astype(np.int64)
    blk = np.zeros(n, dtype=np.int64)
    for r, x in enumerate(range_partition(n, SHARES)):
        blk[x.StartIndex:x.EndIndex + 1] = r
    flip = np.array([bi != bj and not block_is_computed(bi, bj) for bi, bj in zip(blk[ii], blk[jj])], dtype=bool)
    return np.where(flip, jj, ii), np.where(flip, ii, jj), blk


class ClockSampler:
    """nvidia-smi SM clocks and throttle reasons while the timed region runs."""
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[3:]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _cpu_worker(args):
    concat, off, rows, cols = args
    import oracle
    return oracle.ref_distances("EDNAFULL", 1, 0, 16.0, 4.0, concat, off, rows, cols)


def cpu_reference(concat, off, rows, cols, threads):
    """The reference's aligner + ComputeDistance over the pairs, one single-threaded process per
    host core (the reference's one-rank-per-core model).  Returns (distances, seconds)."""
    import multiprocessing as mp
    chunks = np.array_split(np.arange(len(rows)), threads * 4)
    ctx = mp.get_context("spawn")
    with ctx.Pool(threads) as pool:
        pool.map(_cpu_worker, [(concat, off, rows[:1], cols[:1])] * threads)  # warm the workers
        t = time.perf_counter()
        parts = pool.map(_cpu_worker, [(concat, off, rows[c], cols[c]) for c in chunks if len(c)])
        dt = time.perf_counter() - t
    return np.concatenate(parts), dt


def reference_available():
    import oracle
    return oracle.ref_available()


def run_reference_arm(a):
    """--impl reference: the reference's CPU path on this host's cores, same metric/workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    concat, off = workload_sequences(a.n)
    lens = np.diff(off)
    threads = os.cpu_count() or 1
    kind = "reference" if reference_available() else "port"
    rng = np.random.default_rng(11)
    per_step = max(threads * 8, int(a.ref_step_seconds * threads * 0.12e9 / (np.mean(lens) ** 2)))
    cells, secs = 0, 0.0
    for step in range(a.warmup + a.steps):
        r, c, _ = sample_pairs(a.n, per_step, rng)
        if kind == "reference":
            _, dt = cpu_reference(concat, off, r, c, threads)
        else:
            import oracle
            from csharp_b200 import ScoringMatrix
            sc = ScoringMatrix.Load("EDNAFULL").Scores[:127, :127].astype(np.float32)
            t = time.perf_counter()
            oracle.pairs(concat, off, r, c, sc, 16.0, 4.0, threads=threads)
            dt = time.perf_counter() - t
        if step >= a.warmup:
            cells += int((lens[r] * lens[c]).sum())
            secs += dt
    value = cells / secs / 1e9
    line = {"impl": "reference", "metric": "all-pairs SW-Gotoh GCUPS", "value": round(value, 4),
            "unit": "GCUPS", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(secs / a.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"cfg3 uneven SW-Gotoh all-pairs, {a.n} DNA lognormal(400, 0.6) 50-1500, EDNAFULL 16/4",
                       "sample": f"{per_step} pairs per step drawn uniformly from the job"},
            "cpu_baseline": {"value": round(value, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
                             "sample": f"{per_step} uniform pairs x {a.steps} steps of the {a.n}-sequence job"},
            "e2e": {"value": round(value, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def serving(cs, device, seconds, load):
    """Serving workload: a device-resident database of 100,000 DNA sequences (lognormal median
    500, sigma 0.6, clipped 50-2,000), a Poisson stream of query batches (sizes log-uniform in
    1-512, query lengths from the same distribution) aligned SW-Gotoh against the whole database.
    The arrival rate is set from a calibration job so that the offered load is `load` of the GPU.
    Latency of a job = its completion (results in host memory) minus its submission."""
    from csharp_b200 import pack_sequences, synth
    db = synth.config5_db(SERVE["db"])
    concat, off = pack_sequences(db)
    dblen = float(off[-1])
    rng = np.random.default_rng(SERVE["seed"])
    pool = synth.dna_family(4000, 40, synth.lognormal_lengths(4000, 500, 0.6, 50, 2000, rng), SERVE["seed"])
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4, device=device)
    eng.upload(concat=concat, offsets=off)
    # calibration (also builds the database state): 64 queries alone
    cal = [pool[k].tobytes() for k in range(64)]
    r = eng.wait(eng.submit(cal))
    cal_rate = r["cells"] / max(r["done_s"] - r["admit_s"], 1e-9)
    mean_q = (SERVE["qmax"] - SERVE["qmin"]) / np.log(SERVE["qmax"] / SERVE["qmin"])
    mean_cells = mean_q * float(np.mean([len(p) for p in pool])) * dblen
    lam = load * cal_rate / mean_cells           # batches per second
    arrivals = np.cumsum(rng.exponential(1.0 / lam, 10000))
    arrivals = arrivals[arrivals < seconds]
    sizes = np.exp(rng.uniform(np.log(SERVE["qmin"]), np.log(SERVE["qmax"] + 1), len(arrivals))).astype(int)
    sizes = np.clip(sizes, SERVE["qmin"], SERVE["qmax"])
    batches = [[pool[k].tobytes() for k in rng.integers(0, len(pool), n)] for n in sizes]
    outstanding, results = {}, []
    t0 = time.monotonic()
    for at, b in zip(arrivals, batches):
        while True:
            now = time.monotonic() - t0
            if now >= at:
                break
            time.sleep(min(0.005, at - now))
        outstanding[eng.submit(b)] = len(b)
        for t in list(outstanding):
            x = eng.poll(t, 0)
            if x is not None:
                results.append(x)
                del outstanding[t]
    for t in list(outstanding):
        results.append(eng.wait(t))
    st = eng.serve_stats()
    lat = np.array([x["done_s"] - x["submit_s"] for x in results]) * 1e3
    cells = float(sum(x["cells"] for x in results))
    span = max(x["done_s"] for x in results) - min(x["submit_s"] for x in results)
    ok = all(x["status"] == 0 for x in results)
    eng.close()
    return {"workload": "cfg5 serving: 100,000 DNA database lognormal(median 500, sigma 0.6) clipped 50-2000, "
                        "Poisson batches of 1-512 queries (log-uniform sizes), EDNAFULL, open 16 / extend 4",
            "jobs": len(results), "queries": int(sizes.sum()), "offered_load": load,
            "arrival_rate_per_s": round(lam, 3), "p50_ms": round(float(np.percentile(lat, 50)), 1),
            "p99_ms": round(float(np.percentile(lat, 99)), 1), "mean_ms": round(float(lat.mean()), 1),
            "gcups": round(cells / span / 1e9, 1), "calibration_gcups": round(cal_rate / 1e9, 1),
            "max_admitted": st["max_active"], "waves": st["waves"], "all_ok": ok}


def other_configs(cs, device, stream, flush):
    """The other benchmark configurations, each timed with inputs resident (CUDA events, L2
    flushed): the 16-bit engine on the whole job and, on a subset, the same pairs on 32-bit
    lanes (results compared entry by entry; parity with the reference is the tests' job)."""
    import torch
    from csharp_b200 import pack_sequences, synth
    out = {}
    specs = [
        ("cfg1", "plain SW-Gotoh: 1,000 DNA, 20 roots of 500 nt, lengths 200-600, EDNAFULL 16/4",
         lambda: synth.config1(), "EDNAFULL", 16, 4, cs.SWG_MPI, cs.NUCLEIC, 1000),
        ("cfg2", "NW global: 10,000 DNA, lengths uniform 300-500, 100 roots, EDNAFULL 16/4",
         lambda: synth.config2(), "EDNAFULL", 16, 4, cs.NW, cs.NUCLEIC, 1500),
        ("cfg4", "protein SW-Gotoh: 5,000 of the 20,000-sequence set (20 amino acids, lengths 100-1000, "
                 "500 roots), BLOSUM62 10/1",
         lambda: synth.config4(cs.ScoringMatrix.Load("BLOSUM62").Scores, n=5000), "BLOSUM62", 10, 1,
         cs.SWG_MPI, cs.PROTEIN, 1000),
    ]

    def timed(eng, n, dst):
        eng.all_pairs_device(dst.data_ptr(), n, 1)
        torch.cuda.synchronize()
        flush.zero_()
        b, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b.record(stream)
        eng.all_pairs_device(dst.data_ptr(), n, 1)
        e.record(stream)
        torch.cuda.synchronize()
        return b.elapsed_time(e), eng.query("cells")

    for name, desc, gen, matrix, o, e, mode, atype, sub in specs:
        seqs = gen()
        concat, off = pack_sequences(seqs)
        n = len(seqs)
        eng = with_options(cs.Engine(cs.ScoringMatrix.Load(matrix), o, e, mode=mode, alignment_type=atype, device=device))
        eng.upload(concat=concat, offsets=off)
        eng.use_stream(stream.cuda_stream)
        full = torch.zeros((n, n), dtype=torch.int16, device="cuda")
        ms, cells = timed(eng, n, full)
        m = min(sub, n)
        a16 = with_options(cs.Engine(cs.ScoringMatrix.Load(matrix), o, e, mode=mode, alignment_type=atype, device=device))
        a32 = with_options(cs.Engine(cs.ScoringMatrix.Load(matrix), o, e, mode=mode, alignment_type=atype, device=device,
                                     lanes=32))
        r = {}
        for tag, x in (("lanes16", a16), ("lanes32", a32)):
            x.upload(concat=concat[: off[m]], offsets=off[: m + 1])
            x.use_stream(stream.cuda_stream)
            d = torch.zeros((m, m), dtype=torch.int16, device="cuda")
            t, c = timed(x, m, d)
            r[tag] = (t, c, d)
        out[name] = {"workload": desc, "gcups": round(cells / (ms * 1e-3) / 1e9, 1), "ms": round(ms, 1),
                     "cells": int(cells), "pairs": n * (n - 1) // 2,
                     "subset": f"first {m} sequences: 16-bit lanes {r['lanes16'][1] / (r['lanes16'][0] * 1e-3) / 1e9:.1f}"
                               f" vs 32-bit lanes {r['lanes32'][1] / (r['lanes32'][0] * 1e-3) / 1e9:.1f} GCUPS",
                     "subset_identical": bool(torch.equal(r["lanes16"][2], r["lanes32"][2]))}
        for x in (eng, a16, a32):
            x.close()
        del full
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=SHARES)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--n", type=int, default=WORKLOAD["n"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-step-seconds", type=float, default=6.0)
    ap.add_argument("--skip-extras", action="store_true", help="headline only (profiling runs)")
    ap.add_argument("--rows-per-lane", type=int, default=0, help="engine rows per lane (0 = per query)")
    ap.add_argument("--no-autotune", action="store_true", help="built-in rows-per-lane costs instead of measured ones")
    ap.add_argument("--serving-only", action="store_true", help="only the serving workload (one JSON line)")
    ap.add_argument("--configs-only", action="store_true", help="only configurations 1, 2 and 4 (one JSON line)")
    ap.add_argument("--serve-seconds", type=float, default=SERVE["seconds"])
    ap.add_argument("--box-reg", type=int, default=-1, choices=[-1, 0, 1],
                    help="two-pass box step: 1 register box step first, 0 warp box kernel only (-1: engine default)")
    a = ap.parse_args()
    if a.box_reg >= 0:
        ENGINE_OPTIONS["box_reg"] = a.box_reg
    if a.serving_only:
        import csharp_b200 as cs
        print(json.dumps({"serving": serving(cs, 0, a.serve_seconds, SERVE["load"])}))
        return 0
    if a.configs_only:
        import torch
        import csharp_b200 as cs
        st = torch.cuda.Stream()
        torch.cuda.set_stream(st)
        fl = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        print(json.dumps({"configs": other_configs(cs, 0, st, fl)}))
        return 0
    if a.impl == "reference":
        return run_reference_arm(a)

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    import csharp_b200 as cs
    concat, off = workload_sequences(a.n)
    lens = np.diff(off)
    N = a.n
    eng = with_options(cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4, device=local))
    eng.upload(concat=concat, offsets=off)
    if a.rows_per_lane:
        eng.set_option("rows_per_lane", a.rows_per_lane)
    stream = torch.cuda.Stream()  # a real stream handle (the legacy default stream's is 0)
    torch.cuda.set_stream(stream)
    eng.use_stream(stream.cuda_stream)
    out = torch.zeros((N, N), dtype=torch.int16, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def share_of(step):
        return (step * world + rank) % SHARES

    # the autotuner times each rows-per-lane choice on a sample of this job (before any timing)
    tuned = None if (a.no_autotune or a.rows_per_lane) else eng.autotune(out.data_ptr(), N)
    share_cells = {}
    eng.set_option("plan_only", 1)  # plan and capture every share before timing; launch nothing
    for s in range(SHARES):
        eng.rank_blocks_device(s, SHARES, out.data_ptr(), N)
        share_cells[s] = eng.query("cells")
    eng.set_option("plan_only", 0)
    torch.cuda.synchronize()

    for w in range(a.warmup):
        eng.rank_blocks_device(share_of(w), SHARES, out.data_ptr(), N)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    cells = 0
    launches = 0
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for k in range(a.steps):
            flush.zero_()
            s = share_of(a.warmup + k)
            ev[k][0].record(stream)
            eng.rank_blocks_device(s, SHARES, out.data_ptr(), N)
            ev[k][1].record(stream)
            cells += share_cells[s]
            launches += eng.query("launches")
        t1.record(stream)
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    kernel_ms = sum(b.elapsed_time(e) for b, e in ev)
    if world > 1:
        t = torch.tensor([ms, kernel_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, kernel_ms = float(t[0]), float(t[1])
        c = torch.tensor([cells], device="cuda", dtype=torch.float64)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
        total_cells = float(c[0])
    else:
        total_cells = float(cells)
    value = total_cells / (ms * 1e-3) / 1e9

    result = {"metric": "all-pairs SW-Gotoh GCUPS", "value": round(value, 3), "unit": "GCUPS",
              "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 3),
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16x2",
              "data": "synthetic (seeded family generator; no dataset in the reference)",
              "config": {"workload": f"cfg3 batched uneven SW-Gotoh all-pairs: {N} DNA, lognormal(median 400, sigma 0.6) "
                                     f"clipped 50-1500, 200 roots, EDNAFULL, open 16 / extend 4, PercentIdentity Int16",
                         "step": f"one rank's share of an {SHARES}-rank MPI run of the job (whole job = {SHARES} steps)",
                         "l2": "flushed (256 MB write) before every timed step",
                         "cells_per_job": int(sum(share_cells.values())), "pairs_per_job": N * (N - 1) // 2,
                         "engine_options": dict(ENGINE_OPTIONS) or "defaults",
                         "rows_per_lane_costs": (tuned if tuned and any(tuned.values()) else
                                                 "built-in" + (" (kept by the autotuner)" if tuned else ""))},
              "gpu_launches": int(launches), "clocks": clk.summary()}

    if rank == 0:
        peak_max, peak_add = cs.measure_int_peak(local)
        peak_cells = peak_max * LANES_PER_OP / OPS_PER_CELL
        achieved = cells / (kernel_ms * 1e-3)
        traffic = None
        tp = ROOT / "profiles" / "engine_kernel_traffic.json"  # from an ncu capture (see that file)
        if tp.exists():
            traffic = json.loads(tp.read_text()).get("dram_bytes_per_launch")
        result["roofline"] = {"bound": "int_alu", "achieved": round(achieved / 1e9, 2), "peak": round(peak_cells / 1e9, 2),
                              "unit": "Gcell/s", "frac": round(achieved / peak_cells, 4), "traffic": traffic,
                              "peak_basis": f"measured max.s32 {peak_max / 1e12:.2f} Tops/s x {LANES_PER_OP} lanes / {OPS_PER_CELL} ops per cell",
                              "kernel_ms": round(kernel_ms, 2)}
    if not a.skip_extras and rank == 0:
        # e2e: the same shares through host buffers: H2D of the sequences, D2H of the matrix
        pin_seq = torch.from_numpy(concat).pin_memory()
        pin_out = torch.empty((N, N), dtype=torch.int16).pin_memory()
        d_seq = torch.empty_like(pin_seq, device="cuda")
        e_cells, e_ms = 0, 0.0
        for k in range(3):
            s = share_of(k)
            b, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            b.record(stream)
            d_seq.copy_(pin_seq, non_blocking=True)
            eng.rank_blocks_device(s, SHARES, out.data_ptr(), N)
            pin_out.copy_(out, non_blocking=True)
            e.record(stream)
            torch.cuda.synchronize()
            if k >= 1:
                e_ms += b.elapsed_time(e)
                e_cells += share_cells[s]
        result["e2e"] = {"value": round(e_cells / (e_ms * 1e-3) / 1e9, 3), "unit": "GCUPS",
                         "h2d_bytes_per_step": int(concat.nbytes), "d2h_bytes_per_step": int(N * N * 2),
                         "note": "per step: sequences H2D from pinned host, one rank share, full Int16 matrix D2H"}
        # the shares of all steps so far cover the whole job: the matrix of an 8-rank run
        torch.cuda.synchronize()
        full = pin_out.numpy().copy()
        covered = {share_of(k) for k in range(a.warmup + a.steps)} | {share_of(k) for k in range(3)}
        # CPU baseline: the reference's aligner on a uniform sample of the job's pairs, oriented
        # as the 8-rank run orients them (s1 = the row of the share that aligns the pair)
        threads = os.cpu_count() or 1
        ii, jj, blk = sample_pairs(N, 200000, np.random.default_rng(5))
        keep = np.isin(blk[ii], list(covered))
        ii, jj = ii[keep], jj[keep]
        per_pair = float(np.mean(lens[ii] * lens[jj]))
        npairs = int(max(threads * 4, min(len(ii), a.cpu_seconds * threads * 0.12e9 / per_pair)))
        ii, jj = ii[:npairs], jj[:npairs]
        kind = "reference" if reference_available() else "port"
        if kind == "reference":
            d_cpu, dt = cpu_reference(concat, off, ii, jj, threads)
        else:
            import oracle
            sc = cs.ScoringMatrix.Load("EDNAFULL").Scores[:127, :127].astype(np.float32)
            t = time.perf_counter()
            d_cpu = oracle.pairs(concat, off, ii, jj, sc, 16.0, 4.0, threads=threads)
            dt = time.perf_counter() - t
        cpu_cells = float((lens[ii] * lens[jj]).sum())
        result["cpu_baseline"] = {"value": round(cpu_cells / dt / 1e9, 4), "unit": "GCUPS", "cores": threads,
                                  "kind": kind,
                                  "sample": f"{npairs} pairs (i > j) drawn uniformly from the {N}-sequence job, "
                                            f"{cpu_cells:.3g} cells, {dt:.1f} s"}
        mism = int((full[ii, jj] != d_cpu).sum())
        result["parity"] = {"pairs_checked_vs_cpu_reference": npairs, "mismatches": mism,
                            "tolerance": "exact Int16"}
        # plain one-launch-per-block kernel vs the batched engine on the same 2,000-sequence block
        M = min(2000, N)
        sub = with_options(cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4, device=local))
        sub.upload(concat=concat[: off[M]], offsets=off[: M + 1])
        sub.use_stream(stream.cuda_stream)
        o2 = torch.zeros((M, M), dtype=torch.int16, device="cuda")
        o3 = torch.zeros((M, M), dtype=torch.int16, device="cuda")
        sub.all_pairs_device(o2.data_ptr(), M)
        sub.compute_block_device(0, M - 1, 0, M - 1, True, o3.data_ptr(), M)
        torch.cuda.synchronize()
        sub_cells = float(np.tril(np.outer(lens[:M], lens[:M]), -1).sum())
        times = {}
        for name, fn in (("batched", lambda: sub.all_pairs_device(o2.data_ptr(), M)),
                         ("plain", lambda: sub.compute_block_device(0, M - 1, 0, M - 1, True, o3.data_ptr(), M))):
            b, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            flush.zero_()
            b.record(stream)
            fn()
            e.record(stream)
            torch.cuda.synchronize()
            times[name] = b.elapsed_time(e)
        a2, a3 = o2.cpu().numpy(), o3.cpu().numpy()
        offd = ~np.eye(M, dtype=bool)
        result["plain_vs_batched"] = {"block": f"diagonal block of {M} sequences ({M * (M - 1) // 2} pairs)",
                                      "plain_gcups": round(sub_cells / (times["plain"] * 1e-3) / 1e9, 2),
                                      "batched_gcups": round(sub_cells / (times["batched"] * 1e-3) / 1e9, 2),
                                      "speedup": round(times["plain"] / times["batched"], 2),
                                      "identical": bool(np.array_equal(a2[offd], a3[offd]))}
        sub.close()
        result["configs"] = other_configs(cs, local, stream, flush)
        result["serving"] = serving(cs, local, a.serve_seconds, SERVE["load"])
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
