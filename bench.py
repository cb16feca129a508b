"""Benchmark: all-pairs SW-Gotoh distance matrix on B200 (batched engine), one JSON line.

Workload: 20,000 synthetic DNA sequences, lognormal lengths (median 400, sigma 0.6, clipped
50-1,500), 200 family roots, EDNAFULL, gap open 16 / extend 4, PercentIdentity -> Int16.  A step
is one MPI rank's share of an 8-rank run of that job (the pairs rank b aligns in
MPIComputeLowerTriangularBlocked.Compute), so W = 3 warm-up steps then K = 8 timed steps time the
whole job once on one GPU.  With N GPUs (torchrun) each rank takes a different share per step
(no data-path collective; "weak" scaling: per-GPU work per step is fixed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Besides the headline value (inputs resident in HBM, one engine call per share), the line carries:
  e2e              the whole job through the reference-facing C ABI with host buffers, its 8 shares
                   split among the ranks: per share sw_upload_sequences from pinned memory, then one
                   sw_compute_block call per block in the reference driver's order, each copying its
                   block to the host (every rank; the rest below at N = 1 only)
  roofline         the engine kernels' cell rate against the integer-pipe peak measured live
  cpu_baseline     the reference's own aligner and ComputeDistance (transliterated from its C#)
                   on the host cores, over a uniform sample of the job's pairs, with its parity
  plain_vs_batched one 8-rank share block by block: the plain one-thread-per-pair kernel against
                   the engine behind the same block handler, identical results required
  configs          configurations 1, 2 and 4, and configuration 1 with the Kimura2 distance, on
                   the engine, each checked against the oracle (cfg1 every pair, the others
                   uniform samples) by CPU workers that run while the GPU legs run
  serving          configuration 5: Poisson query batches against a 100,000-sequence database
  clocks           the SM clocks sampled while timing
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
SHARES = 8             # steps per whole job: 8 shares of equal DP cells (and an 8-rank run's blocks)
SERVE = dict(db=100000, qmin=1, qmax=512, load=0.7, jobs=100, seed=6)
PARITY_SAMPLE = 100000  # pairs of configurations 2 and 4 checked against the oracle
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


# ---- the reference driver's partition (RangePartitioner.cs:17-55, Program.cs:628-642), in Python
# so that the reference arm loads nothing of this repository's library
def ranges(n, parts):
    """Inclusive (start, end) of each part: the first n % parts parts get one more element."""
    q, r = divmod(n, parts)
    out, s = [], 0
    for k in range(parts):
        ln = q + (1 if k < r else 0)
        out.append((s, s + ln - 1))
        s += ln
    return out


def block_computed(r, c):
    """Rank r computes block (r, c) (the SWG-MPI checkerboard)."""
    return (r > c and (r + c) % 2 == 0) or (r < c and (r + c) % 2 == 1)


def checkerboard_share_cells(lens, share, parts=SHARES):
    """DP cells (sum of m * n) of the pairs rank `share` of a `parts`-rank run aligns."""
    lens = np.asarray(lens, dtype=np.float64)
    tot = 0.0
    for rs, re_, cs_, ce, diag in share_blocks(len(lens), share, parts):
        r = lens[rs:re_ + 1]
        tot += (r.sum() ** 2 - (r * r).sum()) / 2 if diag else r.sum() * lens[cs_:ce + 1].sum()
    return tot


def share_blocks(n, share, parts=SHARES):
    """The blocks rank `share` of a `parts`-rank run hands to its block handler, in the order
    MPIComputeLowerTriangularBlocked.Compute calls it: (row start, row end, col start, col end,
    diagonal)."""
    rr = ranges(n, parts)
    rs, re_ = rr[share]
    return [(rs, re_, cs, ce, c == share) for c, (cs, ce) in enumerate(rr)
            if c == share or block_computed(share, c)]


def sample_pairs(n, count, rng):
    """`count` pairs drawn uniformly from the job, oriented (s1, s2) as the SHARES-rank run
    orients them: diagonal blocks align (s_i, s_j) for i > j; block (r, c) is aligned by the rank
    the checkerboard names, with s1 from its rows."""
    ii = rng.integers(1, n, count)
    jj = (rng.random(count) * ii).astype(np.int64)
    blk = np.zeros(n, dtype=np.int64)
    for r, (a, b) in enumerate(ranges(n, SHARES)):
        blk[a:b + 1] = r
    flip = np.array([bi != bj and not block_computed(bi, bj) for bi, bj in zip(blk[ii], blk[jj])], dtype=bool)
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


# ---- CPU legs (spawned worker processes; the oracle is the checker and the timed CPU reference) --
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


_PARITY_SETS = {}


def _parity_init(sets):
    _PARITY_SETS.update(sets)


def _parity_task(args):
    """One chunk of a parity check: (set name, checker, pairs) -> the oracle's distances."""
    name, kind, rows, cols = args
    import oracle
    concat, off, scores, o, e, atype, dist_fn, mode = _PARITY_SETS[name]
    if kind == "count":    # the in-DP integer checker, one counter word (pinned by the tests)
        return oracle.indp_pairs(concat, off, rows, cols, scores.astype(np.int32), o, e, atype, threads=1, fast=True)
    if kind == "nw":       # the NW traceback restatement
        return oracle.nw_pairs(concat, off, rows, cols, scores.astype(np.float32), float(o), float(e),
                               protein=atype == 0, threads=1)
    if kind == "block":    # the oracle's block restatement, one pair at a time (any distance)
        sc = scores.astype(np.float32)
        return np.array([oracle.block(concat, off, int(i), int(i), int(j), int(j), False, mode, sc, float(o),
                                      float(e), atype, dist_fn)[0][0, 0] for i, j in zip(rows, cols)], dtype=np.int16)
    return oracle.ref_distances("BLOSUM62" if atype == 0 else "EDNAFULL", atype, dist_fn, float(o), float(e),
                                concat, off, rows, cols)  # the transliterated reference


class Parity:
    """Oracle checks of whole configurations on the host cores, in spawned workers that run while
    the GPU legs run.  submit(name, kind, rows, cols) queues one check; result(name) waits."""

    def __init__(self, sets, workers):
        import multiprocessing as mp
        self.pool = mp.get_context("spawn").Pool(max(1, workers), initializer=_parity_init, initargs=(sets,))
        self.jobs = {}
        self.t0 = time.perf_counter()

    def submit(self, name, kind, rows, cols, chunk=1500):
        idx = np.array_split(np.arange(len(rows)), max(1, len(rows) // chunk))
        self.jobs[name] = (kind, self.pool.map_async(_parity_task, [(name, kind, rows[c], cols[c]) for c in idx if len(c)]))

    def result(self, name):
        kind, r = self.jobs[name]
        return kind, np.concatenate(r.get())

    def close(self):
        self.pool.close()
        self.pool.join()
        return time.perf_counter() - self.t0


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
            from csharp_b200 import ScoringMatrix  # only without the transliterated reference
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


# ---- GPU legs -----------------------------------------------------------------------------------
def serving(cs, device, jobs, load):
    """Serving workload: a device-resident database of 100,000 DNA sequences (lognormal median
    500, sigma 0.6, clipped 50-2,000), a Poisson stream of `jobs` query batches (sizes log-uniform
    in 1-512, query lengths from the same distribution) aligned SW-Gotoh against the whole
    database.  The arrival rate is set from the measured capacity (a burst of 8 jobs of 64 queries
    submitted at once: their cells over first submission to last completion) so that the offered
    load is `load` of the GPU; `gcups` is then the cells of the stream over its span, about `load`
    times the capacity.  Latency of a job = its completion (results in host memory) minus its
    submission."""
    from csharp_b200 import pack_sequences, synth
    db = synth.config5_db(SERVE["db"])
    concat, off = pack_sequences(db)
    dblen = float(off[-1])
    rng = np.random.default_rng(SERVE["seed"])
    pool = synth.dna_family(4000, 40, synth.lognormal_lengths(4000, 500, 0.6, 50, 2000, rng), SERVE["seed"])
    eng = with_options(cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4, device=device))
    eng.upload(concat=concat, offsets=off)
    # warm-up (builds the database state), then the capacity: a burst of 8 jobs of 64 queries
    # submitted at once, their cells over first submission to last completion
    eng.wait(eng.submit([pool[k].tobytes() for k in range(16)]))
    burst = [eng.submit([pool[k].tobytes() for k in rng.integers(0, len(pool), 64)]) for _ in range(8)]
    rs = [eng.wait(t) for t in burst]
    cal_rate = sum(x["cells"] for x in rs) / max(max(x["done_s"] for x in rs) - min(x["submit_s"] for x in rs), 1e-9)
    mean_q = (SERVE["qmax"] - SERVE["qmin"]) / np.log(SERVE["qmax"] / SERVE["qmin"])
    mean_cells = mean_q * float(np.mean([len(p) for p in pool])) * dblen
    lam = load * cal_rate / mean_cells           # batches per second
    arrivals = np.cumsum(rng.exponential(1.0 / lam, jobs))
    sizes = np.exp(rng.uniform(np.log(SERVE["qmin"]), np.log(SERVE["qmax"] + 1), jobs)).astype(int)
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
            "arrival_rate_per_s": round(lam, 3), "span_s": round(span, 1),
            "p50_ms": round(float(np.percentile(lat, 50)), 1), "p99_ms": round(float(np.percentile(lat, 99)), 1),
            "mean_ms": round(float(lat.mean()), 1), "gcups": round(cells / span / 1e9, 1),
            "capacity_gcups": round(cal_rate / 1e9, 1), "max_admitted": st["max_active"], "waves": st["waves"],
            "all_ok": ok}


def _timed(stream, fn):
    """fn() between two CUDA events on `stream`, waited for; returns milliseconds."""
    import torch
    b, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    b.record(stream)
    fn()
    e.record(stream)
    torch.cuda.synchronize()
    return b.elapsed_time(e)


def config_sets(cs, only=None, n=None):
    """Configurations 1, 2 and 4, and configuration 1 with the Kimura2 distance: (name, description,
    sequences, matrix, open, extend, mode, type, distance function).
    only: the names to keep; n: the first n sequences of each (a smaller case, for profiling)."""
    from csharp_b200 import synth
    bl = cs.ScoringMatrix.Load("BLOSUM62").Scores
    c1 = synth.config1()
    sets = [
        ("cfg1", "plain SW-Gotoh: 1,000 DNA, 20 roots of 500 nt, lengths 200-600, EDNAFULL 16/4",
         c1, "EDNAFULL", 16, 4, cs.SWG_MPI, cs.NUCLEIC, cs.PERCENT_IDENTITY),
        ("cfg2", "NW global: 10,000 DNA, lengths uniform 300-500, 100 roots, EDNAFULL 16/4",
         synth.config2(), "EDNAFULL", 16, 4, cs.NW, cs.NUCLEIC, cs.PERCENT_IDENTITY),
        ("cfg4", "protein SW-Gotoh: 20,000 sequences (20 amino acids, lengths 100-1000, 500 roots), BLOSUM62 10/1",
         synth.config4(bl), "BLOSUM62", 10, 1, cs.SWG_MPI, cs.PROTEIN, cs.PERCENT_IDENTITY),
        ("cfg1_kimura2", "SW-Gotoh with the Kimura2 distance: the 1,000 DNA of configuration 1, EDNAFULL 16/4",
         c1, "EDNAFULL", 16, 4, cs.SWG_MPI, cs.NUCLEIC, cs.KIMURA2),
    ]
    if only:
        sets = [s for s in sets if s[0] in only]
    if n:
        sets = [(s[0], s[1] + f" (first {n} sequences)", s[2][:n]) + tuple(s[3:]) for s in sets]
    return sets


def config_parity_pairs(n, name, rng):
    """The pairs a configuration's check covers: every pair of cfg1, a uniform sample of the others
    (s1 = the larger index, as a 1-rank run orients them)."""
    if name == "cfg1":
        ii, jj = np.tril_indices(n, -1)
        return ii.astype(np.int64), jj.astype(np.int64)
    ii = rng.integers(1, n, PARITY_SAMPLE)
    jj = (rng.random(PARITY_SAMPLE) * ii).astype(np.int64)
    return ii, jj


def run_configs(cs, device, stream, flush, sets, picks, parity):
    """Each configuration as one whole-job engine call (inputs resident, planned before timing),
    and the oracle's verdict on its checked pairs."""
    import torch
    out, got = {}, {}
    for name, desc, seqs, matrix, o, e, mode, atype, dist_fn in sets:
        concat, off = cs.pack_sequences(seqs)
        n = len(seqs)
        eng = with_options(cs.Engine(cs.ScoringMatrix.Load(matrix), o, e, mode=mode, alignment_type=atype,
                                     distance_fn=dist_fn, device=device))
        eng.upload(concat=concat, offsets=off)
        eng.use_stream(stream.cuda_stream)
        full = torch.zeros((n, n), dtype=torch.int16, device="cuda")
        t = time.perf_counter()
        eng.set_option("plan_only", 1)
        eng.all_pairs_device(full.data_ptr(), n, 1)
        eng.set_option("plan_only", 0)
        plan_s = time.perf_counter() - t
        flush.zero_()
        ms = _timed(stream, lambda: eng.all_pairs_device(full.data_ptr(), n, 1))
        cells = eng.query("cells")
        ii, jj = picks[name]
        gi, gj = torch.from_numpy(ii).cuda(), torch.from_numpy(jj).cuda()
        got[name] = full[gi, gj].cpu().numpy()
        eng.close()
        del full
        out[name] = {"workload": desc, "gcups": round(cells / (ms * 1e-3) / 1e9, 1), "ms": round(ms, 1),
                     "cells": int(cells), "pairs": n * (n - 1) // 2, "plan_s": round(plan_s, 2)}
    for name in got:  # the CPU checks were running meanwhile
        kind, want = parity.result(name)
        out[name]["parity"] = {"pairs_checked": int(len(want)), "mismatches": int((got[name] != want).sum()),
                               "checker": {"count": "oracle in-DP integer restatement (every pair)",
                                           "nw": "oracle NW traceback restatement (uniform sample)",
                                           "ref": "transliterated reference oracle/_ref (uniform sample)",
                                           "block": "oracle block restatement (uniform sample)"}[kind],
                               "tolerance": "exact Int16"}
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
    ap.add_argument("--configs-only", action="store_true", help="only configurations 1, 2, 4 and 1 with Kimura2 (one JSON line)")
    ap.add_argument("--only", default="", help="with --configs-only: comma-separated names (cfg1,cfg2,cfg4,cfg1_kimura2)")
    ap.add_argument("--config-n", type=int, default=0, help="with --configs-only: first N sequences of each")
    ap.add_argument("--serve-jobs", type=int, default=SERVE["jobs"])
    ap.add_argument("--box-reg", type=int, default=-1, choices=[-1, 0, 1],
                    help="two-pass box step: 1 register box step first, 0 warp box kernel only (-1: engine default)")
    ap.add_argument("--third-pass", type=int, default=-1, choices=[-1, 0, 1],
                    help="two-pass give-ups: 1 one-pass 16-bit counter kernel, 0 32-bit lanes (-1: engine default)")
    ap.add_argument("--engine-option", action="append", default=[], metavar="KEY=VALUE",
                    help="any sw_set_option knob for every engine of the run (repeatable)")
    a = ap.parse_args()
    for kv in a.engine_option:
        k, v = kv.split("=", 1)
        ENGINE_OPTIONS[k] = int(v)
    if a.box_reg >= 0:
        ENGINE_OPTIONS["box_reg"] = a.box_reg
    if a.third_pass >= 0:
        ENGINE_OPTIONS["third_pass"] = a.third_pass
    if a.impl == "reference":
        return run_reference_arm(a)
    threads = os.cpu_count() or 1
    if a.serving_only:
        import csharp_b200 as cs
        print(json.dumps({"serving": serving(cs, 0, a.serve_jobs, SERVE["load"])}))
        return 0
    if a.configs_only:
        import torch
        import csharp_b200 as cs
        sets = config_sets(cs, [x for x in a.only.split(",") if x], a.config_n)
        picks = {s[0]: config_parity_pairs(len(s[2]), s[0], np.random.default_rng(21)) for s in sets}
        parity = start_parity(cs, sets, picks, threads)
        st = torch.cuda.Stream()
        torch.cuda.set_stream(st)
        fl = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        res = run_configs(cs, 0, st, fl, sets, picks, parity)
        parity.close()
        print(json.dumps({"configs": res}))
        return 0

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

    # the job's shares: contiguous rows of equal DP cells (the cost-balanced partition of the
    # one-process-per-GPU path), each aligned as a one-rank run orients its pairs
    from csharp_b200.driver import balanced_row_ranges
    bal = balanced_row_ranges(lens, SHARES)
    # the autotuner times each rows-per-lane choice on a sample of this job (before any timing)
    tuned = None if (a.no_autotune or a.rows_per_lane) else eng.autotune(out.data_ptr(), N)
    share_cells = {}
    t_plan = time.perf_counter()
    eng.set_option("plan_only", 1)  # plan and capture every share before timing; launch nothing
    for s in range(SHARES):
        eng.rows_device(*bal[s], out.data_ptr(), N)
        share_cells[s] = eng.query("cells")
    eng.set_option("plan_only", 0)
    plan_s = time.perf_counter() - t_plan
    torch.cuda.synchronize()

    for w in range(a.warmup):
        eng.rows_device(*bal[share_of(w)], out.data_ptr(), N)
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
            eng.rows_device(*bal[s], out.data_ptr(), N)
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
                         "step": f"one of {SHARES} contiguous row shares of equal DP cells, pairs oriented as a "
                                 f"one-rank run (whole job = {SHARES} steps)",
                         "share_cells_max_over_mean": round(max(share_cells.values()) * SHARES / sum(share_cells.values()), 4),
                         "l2": "flushed (256 MB write) before every timed step",
                         "cells_per_job": int(sum(share_cells.values())), "pairs_per_job": N * (N - 1) // 2,
                         "plan_s": round(plan_s, 2),
                         "engine_options": dict(ENGINE_OPTIONS) or "defaults",
                         "rows_per_lane_costs": (tuned if tuned and any(tuned.values()) else
                                                 "built-in" + (" (kept by the autotuner)" if tuned else ""))},
              "gpu_launches": int(launches), "clocks": clk.summary(),
              "engine_counters_last_step": {k: eng.query(k) for k in ("pairs", "lane16_pairs", "tripped", "box_spilled", "box_third_pass",
                                                                      "box_fallbacks")}}

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
    if not a.skip_extras:
        # every rank: the job end to end through the block handler; one GPU only: the CPU
        # reference, the plain-kernel comparison, the configurations and serving
        e2e = e2e_leg(cs, eng, concat, off, lens, N, rank, world)
        if rank == 0:
            result["e2e"] = e2e
        if world == 1:
            covered = {share_of(k) for k in range(a.warmup + a.steps)}
            extras(a, cs, eng, stream, flush, out, concat, off, lens, N, bal, threads, result, covered)
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    eng.close()
    return 0


def start_parity(cs, sets, picks, threads):
    """Queue the oracle checks of configurations 1, 2 and 4 on all but two host cores."""
    tables = {}
    for name, _, seqs, matrix, o, e, mode, atype, dist_fn in sets:
        concat, off = cs.pack_sequences(seqs)
        tables[name] = (concat, off, cs.ScoringMatrix.Load(matrix).Scores[:127, :127].copy(), o, e, atype, dist_fn,
                        mode)
    parity = Parity(tables, threads - 2)
    for name, _, seqs, matrix, o, e, mode, atype, dist_fn in sets:
        ii, jj = picks[name]
        if mode == cs.NW:
            kind = "nw"
        elif dist_fn != cs.PERCENT_IDENTITY:
            kind = "ref" if reference_available() else "block"
        else:
            kind = "ref" if (atype == cs.PROTEIN and reference_available()) else "count"
        parity.submit(name, kind, ii, jj)
    return parity


def e2e_shares(rank, world):
    """The 8-rank shares the end-to-end leg of rank `rank` (of `world`) takes: r, r + world, ..."""
    return [s for s in range(SHARES) if s % world == rank]


def e2e_leg(cs, eng, concat, off, lens, N, rank, world):
    """The reference-facing C ABI with host buffers, over the whole job split among the ranks (rank
    r takes the 8-rank shares r, r + world, ...).  Per share: sw_upload_sequences of the set from
    pinned host memory (same lengths and letters: the engine keeps its plans), then one
    sw_compute_block call per block of the share, in the reference driver's order, each copying its
    block into the share's row slab in pinned host memory.  Host wall clock per rank; the job's
    time is the slowest rank's."""
    import torch
    mine = e2e_shares(rank, world)
    pin_seq = torch.from_numpy(concat).pin_memory().numpy()
    rows = max(b - a_ + 1 for a_, b in ranges(N, SHARES))
    slab = torch.empty((rows, N), dtype=torch.int16).pin_memory().numpy()

    def share_calls(s):
        r0 = ranges(N, SHARES)[s][0]
        for rs, re_, cs_, ce, diag in share_blocks(N, s):
            eng.compute_block(rs, re_, cs_, ce, diag, out=slab[rs - r0:re_ - r0 + 1, cs_:ce + 1])

    t = time.perf_counter()
    eng.set_option("plan_only", 1)
    for s in mine:
        share_calls(s)
    eng.set_option("plan_only", 0)
    plan_s = time.perf_counter() - t
    if mine:  # one untimed share
        eng.upload(concat=pin_seq, offsets=off)
        share_calls(mine[0])
    cells, h2d, d2h = 0, 0, 0
    t = time.perf_counter()
    for s in mine:
        eng.upload(concat=pin_seq, offsets=off)
        share_calls(s)
        cells += checkerboard_share_cells(lens, s)
        h2d += concat.nbytes + off.nbytes
        d2h += sum((re_ - rs + 1) * (ce - cs_ + 1) * 2 for rs, re_, cs_, ce, _ in share_blocks(N, s))
    secs = time.perf_counter() - t
    if world > 1:
        import torch.distributed as dist
        x = torch.tensor([secs, plan_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        y = torch.tensor([cells, h2d, d2h], device="cuda", dtype=torch.float64)
        dist.all_reduce(y, op=dist.ReduceOp.SUM)
        secs, plan_s = float(x[0]), float(x[1])
        cells, h2d, d2h = float(y[0]), float(y[1]), float(y[2])
    return {"value": round(cells / secs / 1e9, 3), "unit": "GCUPS",
            "h2d_bytes_per_step": int(h2d // SHARES), "d2h_bytes_per_step": int(d2h // SHARES),
            "note": f"the whole job as {SHARES} 8-rank shares split over {world} GPU(s); per share: "
                    "sw_upload_sequences from pinned host memory, then one sw_compute_block per block of the "
                    "share (host output) in the reference driver's order; host wall clock, slowest rank",
            "plan_s": round(plan_s, 2)}


def extras(a, cs, eng, stream, flush, out, concat, off, lens, N, bal, threads, result, covered):
    import torch
    # ---- CPU baseline: the reference's aligner on a uniform sample of the job's pairs (s1 = the
    # larger index, as the timed shares orient them), alone on the host cores; its distances
    # against the GPU matrix of the shares the timed run computed
    rng = np.random.default_rng(5)
    ii = rng.integers(1, N, 200000)
    jj = (rng.random(200000) * ii).astype(np.int64)
    share_of_row = np.searchsorted(np.array([lo for lo, _ in bal]), ii, side="right") - 1
    keep = np.isin(share_of_row, list(covered))
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
    got = out[torch.from_numpy(ii).cuda(), torch.from_numpy(jj).cuda()].cpu().numpy()
    result["parity"] = {"pairs_checked_vs_cpu_reference": npairs, "mismatches": int((got != d_cpu).sum()),
                        "tolerance": "exact Int16"}

    # ---- the parity checks of configurations 1, 2 and 4 run on the host cores from here on
    sets = config_sets(cs)
    picks = {s[0]: config_parity_pairs(len(s[2]), s[0], np.random.default_rng(21)) for s in sets}
    parity = start_parity(cs, sets, picks, threads)

    # ---- plain one-launch-per-block kernel vs the engine behind the same block handler, on one
    # whole 8-rank share, block by block in the driver's order, device output
    share = 0
    r0, r1 = ranges(N, SHARES)[share]
    d_plain = torch.zeros((r1 - r0 + 1, N), dtype=torch.int16, device="cuda")
    d_eng = torch.zeros_like(d_plain)
    blocks = share_blocks(N, share)

    def handler_calls(dst):
        for rs, re_, cs_, ce, diag in blocks:
            eng.compute_block_device(rs, re_, cs_, ce, diag, dst.data_ptr() + ((rs - r0) * N + cs_) * 2, N)

    eng.set_option("plan_only", 1)
    handler_calls(d_eng)
    eng.set_option("plan_only", 0)
    times = {}
    for name, mode, dst in (("batched", 1, d_eng), ("plain", 0, d_plain)):
        eng.set_option("block_engine", mode)
        flush.zero_()
        times[name] = _timed(stream, lambda: handler_calls(dst))
    eng.set_option("block_engine", 1)
    sc = float(checkerboard_share_cells(lens, share))
    result["plain_vs_batched"] = {"share": f"rank {share} of an {SHARES}-rank run: {len(blocks)} blocks, "
                                           f"{sc:.3g} cells, one block-handler call per block",
                                  "plain_gcups": round(sc / (times["plain"] * 1e-3) / 1e9, 2),
                                  "batched_gcups": round(sc / (times["batched"] * 1e-3) / 1e9, 2),
                                  "speedup": round(times["plain"] / times["batched"], 2),
                                  "identical": bool(torch.equal(d_plain, d_eng))}
    del d_plain, d_eng

    result["configs"] = run_configs(cs, 0, stream, flush, sets, picks, parity)
    result["configs"]["parity_workers_s"] = round(parity.close(), 1)
    result["serving"] = serving(cs, 0, a.serve_jobs, SERVE["load"])


if __name__ == "__main__":
    sys.exit(main())
