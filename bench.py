"""Benchmark: AN-coded star-join queries per second on one B200 (or N replicas).

Workload (one step = one batch): 64 seeded random star-join queries -- range
predicates on the codes of 1-4 dimension attributes (target selectivity
1e-4..0.1), group-by on 0-3 dimension attributes, a fact prefix drawn from
{1M, 6M, 60M, 600M} rows -- over an SSB-SF100-shaped AN-coded star schema
resident in HBM (lineorder 600,000,000 rows; date 2,556, customer 3,000,000,
part 1,400,000, supplier 200,000 rows) with 1,000 seeded single-bit flips in
the fact columns, continuous detection on every fetched value.  Data are
synthetic (seeded generators with the schema's shapes and value ranges).

Reported on one JSON line:
  value     queries/s of the fused batched path: K batches submitted through
            the C ABI (CUDA-graph replay, two batches in flight), timed with
            CUDA events on the launching stream, max over ranks;
  e2e       queries/s by wall clock through the public submit/wait API (two
            batches in flight; sync_calls_value: one synchronous call per batch) with host query
            descriptors in and host results out (copies in the timed region);
  plain     queries/s of the operator-at-a-time GPU path (one reference
            operator per launch sequence, composed in C++ through the C ABI;
            python_composition_value: the same composition driven from
            Python) on a sample of the same queries, plus a parity check of
            the fused results against both;
  roofline  the fact-table kernel: scan-equivalent bytes (rows scanned x the
            widths of the fact columns the batch references) over its CUDA-
            event time, against the measured HBM copy bandwidth;
  cpu_baseline  the reference's scalar operators (compiled from its sources),
            run as the same operator composition on host threads over an
            SF1-sized sample and scaled to the workload's mean fact size.

`--impl reference` prints the reference CPU arm alone (rank 0).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

SF100 = dict(fact=600_000_000, date=2556, customer=3_000_000, part=1_400_000, supplier=200_000)
SF1 = dict(fact=6_000_000, date=2556, customer=30_000, part=200_000, supplier=2_000)
FACT_SIZES = (1_000_000, 6_000_000, 60_000_000, 600_000_000)
BATCH = 64
FLIPS = 1000
METRIC = "AN-coded star-join queries/s (batched, continuous detection)"
UNIT = "queries/s"
CLOCK_FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def workload_config(args, fact_rows):
    return {"workload": "batched random star joins over an SF100-shaped AN-coded star schema",
            "fact_rows": fact_rows, "dims": {k: v for k, v in SF100.items() if k != "fact"},
            "queries_per_step": BATCH, "fact_prefixes": [s for s in FACT_SIZES if s <= fact_rows],
            "selectivity": "1e-4..0.1 target, predicates on 1-4 dimensions", "group_by": "0-3 attributes",
            "detection": "continuous", "bit_flips": args.flips, "seed": args.seed,
            "l2": "fact columns (~26 GB) far larger than L2; no flush needed"}


def make_batches(seed, nbatches, fact_rows):
    from ahead_b200.ssb import random_query
    rng = np.random.default_rng(seed)
    return [[random_query(rng, fact_sizes=FACT_SIZES, max_fact=fact_rows) for _ in range(BATCH)]
            for _ in range(nbatches)]


# ------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling every 100 ms from before the warm-up to the end of
    the timed loops; summary() keeps the samples taken inside the timed
    window (mark_start .. mark_end), by nvidia-smi's own timestamps."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None
        self.t0 = self.t1 = None

    def mark_start(self):
        # the sampler's start-up (driver queries) stays out of the timed region
        deadline = time.time() + 5.0
        while self.proc is not None and time.time() < deadline and os.path.getsize(self.file.name) == 0:
            time.sleep(0.05)
        self.t0 = datetime.datetime.now()

    def mark_end(self):
        self.t1 = datetime.datetime.now()

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            # line-buffered, so every sample reaches the file before the sampler is stopped
            pre = ["stdbuf", "-oL"] if shutil.which("stdbuf") else []
            self.proc = subprocess.Popen(pre + ["nvidia-smi", "-i", str(self.index), f"--query-gpu={CLOCK_FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.seek(0)
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for line in self.file.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f")
                rows.append((ts, float(f[2]), float(f[3]), f[6:10]))
            except ValueError:
                continue
        os.unlink(self.file.name)
        inside = [r for r in rows if self.t0 and self.t1 and self.t0 <= r[0] <= self.t1]
        window = "timed region"
        if not inside:  # no sample landed inside a short window: the ones around it
            inside, window = rows, "warm-up through timed region"
        reasons = sorted({n for r in inside for n, v in zip(names[1:], r[3]) if v.lower() == "active"})
        sm = [r[1] for r in inside]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(r[2] for r in inside) if inside else None,
                "reasons": reasons, "samples": len(sm), "window": window}


# ------------------------------------------------------------- CPU arms
REF_COLS = ("orderdate", "custkey", "partkey", "suppkey", "price", "discount")
# The reference's time for a 600M-row prefix over its time for the 60M-row
# prefix of the same query, measured on one host thread by `--ref-scaling`
# (two queries of the family: 9.887 and 9.891; profiles/reference_cpu_scaling.md).
REF_600M_OVER_60M = 9.89


def host_star_schema(fact_rows: int, seed: int, threads: int, flips: int):
    """The SF100-shaped star schema in host memory for the reference's CPU
    operators: the four dimensions at SF100 cardinalities (`generate`) and the
    lineorder columns a star join reads (four foreign keys, price, discount),
    generated in parallel row chunks, with `flips` seeded single-bit flips
    spread over those columns as on the device."""
    from concurrent.futures import ThreadPoolExecutor

    from ahead_b200.model import NP_DTYPE, WIDTH
    from ahead_b200.ssb import TYPES, _enc, col_bat, date_keys, generate
    s = generate(dict(SF100, fact=0), seed=seed)
    n = fact_rows
    dk = date_keys(SF100["date"])
    spec = {"orderdate": None, "custkey": (1, SF100["customer"] + 1), "partkey": (1, SF100["part"] + 1),
            "suppkey": (1, SF100["supplier"] + 1), "price": (90_000, 11_000_001), "discount": (0, 11)}
    cols = {c: np.empty(n, dtype=NP_DTYPE[WIDTH[TYPES[c]]]) for c in spec}
    chunk = 1 << 24

    def fill(i):
        lo, hi = i * chunk, min(n, (i + 1) * chunk)
        rng = np.random.default_rng([seed, i])
        for c, r in spec.items():
            v = dk[rng.integers(0, len(dk), hi - lo)] if r is None else rng.integers(r[0], r[1], hi - lo,
                                                                                    dtype=np.uint64)
            cols[c][lo:hi] = _enc(v, TYPES[c])

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(fill, range((n + chunk - 1) // chunk)))
    rng = np.random.default_rng(seed + 17)
    which = rng.integers(0, len(REF_COLS), flips)
    for ci, c in enumerate(REF_COLS):
        rows = np.unique(rng.integers(0, n, int((which == ci).sum())))
        a = cols[c]
        bits = rng.integers(0, 8 * a.dtype.itemsize, len(rows)).astype(a.dtype)
        a[rows] ^= np.left_shift(np.ones(len(rows), dtype=a.dtype), bits)
    s.tables["lineorder"] = {c: col_bat(c, a) for c, a in cols.items()}
    s.sizes["fact"] = n
    return s


def family_by_size(seed: int, sizes, per_size: int):
    """`per_size` queries of each prefix size, drawn in order from the bench's
    random query family (the same generator and seed scheme as the GPU arm)."""
    from ahead_b200.ssb import random_query
    rng = np.random.default_rng(seed)
    want = {z: [] for z in sizes}
    while any(len(v) < per_size for v in want.values()):
        q = random_query(rng, fact_sizes=FACT_SIZES)
        if q.fact_rows in want and len(want[q.fact_rows]) < per_size:
            want[q.fact_rows].append(q)
    return want


def cpu_run_batch(oracle, schema, queries, threads):
    """Wall seconds of `queries` on the reference's operators, `threads` at a
    time (ctypes releases the GIL inside the reference's code)."""
    from concurrent.futures import ThreadPoolExecutor

    from ahead_b200.pipelines import starjoin_continuous
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda q: starjoin_continuous(oracle, schema, q), queries))
    return time.perf_counter() - t0


def family_qps(per_query_s):
    """Queries/s of the family (prefix sizes equally likely) from the measured
    wall seconds per query of each size with every host thread busy (the sizes
    measured, when the lineorder is shorter than the largest prefix)."""
    return 1.0 / float(np.mean([t for t in per_query_s.values() if t == t]))


def cpu_reference_sample(seed: int, threads: int):
    """The bounded CPU baseline of the GPU line: the reference's scalar
    operators (oracle/_ref, compiled from its sources) on a host schema with
    SF100 dimensions and a 60M-row lineorder, `threads` queries of each prefix
    size 1M / 6M / 60M on `threads` host threads; the 600M prefix's time per
    query is taken as REF_600M_OVER_60M times the 60M one (the same hash
    tables, 10x the probed rows; `--ref-scaling` measured the ratio)."""
    from oracle.oracle import REF_LIB, Oracle
    kind = "reference" if os.path.exists(REF_LIB) else "port"
    o = Oracle(kind)
    sizes = FACT_SIZES[:3]
    s = host_star_schema(sizes[-1], seed, threads, FLIPS // 10)
    qs = family_by_size(seed + 1, sizes, threads)
    per = {}
    for z in sizes:
        per[z] = cpu_run_batch(o, s, qs[z], threads) / len(qs[z])
    per[FACT_SIZES[3]] = REF_600M_OVER_60M * per[FACT_SIZES[2]]
    desc = (f"measured on SF100 dims (customer 3,000,000, part 1,400,000, supplier 200,000, date 2,556) over a "
            f"60M-row lineorder: {threads} queries of each prefix 1M / 6M / 60M on {threads} host threads "
            f"(s/query at full load: " + ", ".join(f"{z // 1_000_000}M {per[z]:.3f}" for z in sizes) +
            f"); the 600M prefix taken as {REF_600M_OVER_60M}x the 60M time (the ratio --ref-scaling measured)")
    return family_qps(per), desc, kind, per


def cpu_reference_extrapolated(seed: int, threads: int, nqueries: int):
    """The earlier estimate, kept for comparison: the same composition on an
    SF1-sized schema with prefixes capped at 6M rows, scaled by fact rows to
    the family's mean prefix."""
    from concurrent.futures import ThreadPoolExecutor

    from ahead_b200.pipelines import starjoin_continuous
    from ahead_b200.ssb import generate, inject_flips, random_query
    from oracle.oracle import REF_LIB, Oracle
    o = Oracle("reference" if os.path.exists(REF_LIB) else "port")
    s = generate(SF1, seed=seed)
    for i, c in enumerate(("custkey", "suppkey", "partkey", "orderdate", "price", "discount", "quantity")):
        inject_flips(s, "lineorder", c, 10, seed=seed + 100 + i)
    rng = np.random.default_rng(seed + 1)
    family = [random_query(rng, fact_sizes=FACT_SIZES) for _ in range(max(nqueries, 1024))]
    qs = family[:nqueries]
    mean_rows = float(np.mean([q.fact_rows for q in family]))
    for q in qs:
        q.fact_rows = min(q.fact_rows, SF1["fact"])
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda q: starjoin_continuous(o, s, q), qs))
    dt = time.perf_counter() - t0
    return sum(q.fact_rows for q in qs) / dt / mean_rows


def _median_ms(fn, reps: int, sync):
    """Median wall time in ms of `reps` calls (each followed by `sync`)."""
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        sync()
        ts.append((time.perf_counter() - t0) * 1e3)
    return float(np.median(ts))


def _star_outcome(r, device: bool):
    """A star-join result as comparable host values (keys, sums, total, errors)."""
    from ahead_b200.gpu import err_to_host, to_host
    h = to_host if device else (lambda b: b)
    e = err_to_host if device else (lambda x: x)
    keys = [np.asarray(h(k).tail.data, dtype=np.uint64).tobytes() for k in r.keys]
    sums = None if r.sums is None else np.asarray(h(r.sums).tail.data, dtype=np.uint64).tobytes()
    errs = {c: (None if not e(v).present else np.asarray(e(v).values, np.uint64).tobytes())
            for c, v in sorted(r.fact_errors.items())}
    return keys, sums, r.total, errs


def configs_measure(gpu, seed: int):
    """The survey's first two configurations, each on one input, through the C
    ABI beside the reference's scalar operators (oracle/_ref) on the same
    input (one host thread, as the reference's programs run):
      config1: the single-column select + sum path (6,000,000-row u16 column,
               values uniform in [0, 10000), A = 233 into u32, select [1000,
               3000) on codes, fetch, checkAndDecode, AN-coded u64 sum, 10
               seeded flips);
      config2: one star join (config2_query: 3 dimension predicates, 280
               groups) on an SF1-shaped schema (6M-row lineorder; dimensions
               2,556 / 30,000 / 200,000 / 2,000) with 60 seeded flips, on the
               operator-at-a-time GPU path and on the fused engine.
    Latency = median wall time of synchronous calls after warm-up; parity =
    the GPU results equal the reference's."""
    import torch

    from ahead_b200.gpu import err_to_host, to_device, to_host
    from ahead_b200.model import RESSHORT, host_bat
    from ahead_b200.pipelines import select_sum_an, starjoin_continuous
    from ahead_b200.ssb import config2_query, generate, inject_flips
    from ahead_b200.starjoin import StarJoinEngine
    from oracle.oracle import REF_LIB, Oracle
    kind = "reference" if os.path.exists(REF_LIB) else "port"
    o = Oracle(kind)
    sync = torch.cuda.synchronize
    out = {}
    # config 1
    n = 6_000_000
    rng = np.random.default_rng(seed)
    v = rng.integers(0, 10_000, n, dtype=np.uint64)
    codes = (v * np.uint64(233)).astype(np.uint32)
    frng = np.random.default_rng(seed + 1)
    for r, bit in zip(frng.choice(n, size=10, replace=False), frng.integers(0, 32, 10)):
        codes[r] ^= np.uint32(1 << int(bit))
    col = host_bat(RESSHORT, codes, A=233)
    dcol = to_device(col)
    sync()

    def outcome1(r, device):
        h = to_host if device else (lambda b: b)
        e = err_to_host if device else (lambda x: x)
        oids = h(r.oids)
        errs = [e(r.select_errors)] + [e(x) for x in r.fetch_errors] + [e(x) for x in r.decode_errors]
        return (r.total, np.asarray(oids.head.data)[: oids.count].astype(np.uint64).tobytes(),
                tuple(None if not x.present else np.asarray(x.values, np.uint64).tobytes() for x in errs))

    ref1 = select_sum_an(o, col, 1000, 3000)
    cpu1 = _median_ms(lambda: select_sum_an(o, col, 1000, 3000), 3, lambda: None)
    for _ in range(3):
        select_sum_an(gpu, dcol, 1000, 3000)
    gpu1 = _median_ms(lambda: select_sum_an(gpu, dcol, 1000, 3000), 10, sync)
    same1 = outcome1(select_sum_an(gpu, dcol, 1000, 3000), True) == outcome1(ref1, False)
    out["config1"] = {"workload": "select+fetch+checkAndDecode+sum, 6,000,000-row u16 column, A=233, 10 flips",
                      "gpu_ms": gpu1, "cpu_ms": cpu1, "cpu_kind": kind, "cpu_cores": 1,
                      "speedup": cpu1 / gpu1, "parity_with_cpu": same1,
                      "selected": int(ref1.oids.count), "timing": "median wall ms of synchronous C-ABI calls"}
    # config 2
    s = generate(SF1, seed=seed)
    for i, c in enumerate(("custkey", "suppkey", "partkey", "orderdate", "price", "discount")):
        inject_flips(s, "lineorder", c, 10, seed=seed + 300 + i)
    ds = type(s)({t: {c: to_device(b) for c, b in cols.items()} for t, cols in s.tables.items()}, dict(s.sizes))
    sync()
    q = config2_query()
    ref2 = starjoin_continuous(o, s, q)
    cpu2 = _median_ms(lambda: starjoin_continuous(o, s, q), 3, lambda: None)
    for _ in range(2):
        starjoin_continuous(gpu, ds, q)
    plain2 = _median_ms(lambda: starjoin_continuous(gpu, ds, q), 5, sync)
    same_plain = _star_outcome(starjoin_continuous(gpu, ds, q), True) == _star_outcome(ref2, False)
    eng = StarJoinEngine(gpu, ds)
    fused = eng.run([q], graph=True)
    for _ in range(3):
        eng.run([q], graph=True)
    fused2 = _median_ms(lambda: eng.run([q], graph=True), 20, sync)
    same_fused = fused_vs_plain(fused[0], starjoin_continuous(gpu, ds, q))
    eng.close()
    out["config2"] = {"workload": "config2_query on an SF1-shaped schema (6M-row lineorder), 60 flips",
                      "fused_gpu_ms": fused2, "plain_gpu_ms": plain2, "cpu_ms": cpu2, "cpu_kind": kind,
                      "cpu_cores": 1, "speedup_fused": cpu2 / fused2, "speedup_plain": cpu2 / plain2,
                      "parity_plain_with_cpu": same_plain, "parity_fused_with_plain": same_fused,
                      "groups": int(ref2.ngroups), "timing": "median wall ms of synchronous C-ABI calls"}
    return out


def _fused_equals_composition(r, c) -> bool:
    """A fused result against the operator composition's (device BATs)."""
    from ahead_b200.gpu import err_to_host, to_host
    from ahead_b200.model import OK
    from ahead_b200.ssb import FACT_COLS
    if r.status != OK or len(r.keys) != len(c.keys):
        return False
    if c.sums is None:
        if r.total != c.total:
            return False
    else:
        for x, k in zip(r.keys, c.keys):
            if not np.array_equal(x, np.asarray(to_host(k).tail.data).astype(np.uint64)):
                return False
        if not np.array_equal(r.sums, np.asarray(to_host(c.sums).tail.data).astype(np.uint64)):
            return False
    for col in FACT_COLS:
        v = err_to_host(c.fact_errors[col]).values if col in c.fact_errors else None
        want = np.zeros(0, np.uint64) if v is None else np.asarray(v, dtype=np.uint64)
        if not np.array_equal(r.fact_errors[col], want):
            return False
    return True


def programs_fused_measure(gpu, eng, schema, fact_rows: int):
    """The 13 SSB programs as star queries of the fused engine (per-row
    strategy) at the full table: each alone (CUDA-event batch time of a
    second run), all 13 as one fused batch, and each result against the
    operator composition run operator by operator on the GPU (exact: group
    keys, AN-coded sums, error positions of every fact column).  The per-row
    kernel's shape is tuned per program (`ahead_sj_tune`) and the engine keeps
    the last one, so this section runs after the family's timing."""
    import torch

    from ahead_b200 import ssb_programs as P
    from ahead_b200.pipelines import starjoin_continuous
    names = ["q11", "q12", "q13", "q21", "q22", "q23", "q31", "q32", "q33", "q34", "q41", "q42", "q43"]
    qs = [P.program_query(n, fact_rows) for n in names]
    fused_ms, fact_ms, parity, comp_ms, shape = {}, {}, {}, {}, {}
    starjoin_continuous(gpu, schema, qs[0])  # untimed warm-up of the composition (kernels, allocator)
    for n, q in zip(names, qs):
        shape[n] = eng.tune([q])  # the per-row kernel's shape for this program (the family's may differ)
        eng.run([q])
        r = eng.run([q])[0]
        st = eng.last_stats()
        fused_ms[n] = float(st.batch_ms)
        fact_ms[n] = float(st.fact_ms)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c = starjoin_continuous(gpu, schema, q)
        torch.cuda.synchronize()
        comp_ms[n] = (time.perf_counter() - t0) * 1e3
        parity[n] = _fused_equals_composition(r, c)
        del c
    eng.tune(qs)
    eng.run(qs)
    rs = eng.run(qs)
    batch_ms = float(eng.last_stats().batch_ms)
    single = [eng.run([q])[0] for q in qs]
    batch_same = all(a.status == b.status and a.total == b.total and len(a.keys) == len(b.keys) and
                     all(np.array_equal(x, y) for x, y in zip(a.keys, b.keys)) and
                     (a.sums is None or np.array_equal(a.sums, b.sums)) and
                     all(np.array_equal(a.fact_errors[k], b.fact_errors[k]) for k in a.fact_errors)
                     for a, b in zip(rs, single))
    return {"fact_rows": fact_rows, "fused_ms": fused_ms, "fused_fact_region_ms": fact_ms, "per_row_shape": shape, "parity_with_composition": parity,
            "composition_gpu_ms": comp_ms, "all13_one_batch_ms": batch_ms, "all13_batch_equals_single": batch_same,
            "timing": "fused: CUDA-event batch time of the second run of each query (fact region: the "
                      "prefilter and the per-row pass, between the batch's two inner events); composition: "
                      "wall clock of the operator-at-a-time GPU run of the same query"}


def programs_measure(gpu, schema, fact_rows: int, seed: int, cpu_rows: int):
    """The reference's 13 SSB programs in the continuous placement through the
    GPU operators on the resident schema (one untimed run, then one timed run
    each), the same programs as the reference's DMR baseline (two unencoded
    replicas decoded from that schema, the normal placement on each, a vote),
    and the compiled reference's operators (oracle/_ref) on a
    `cpu_rows`-row sample of the same schema family, one host thread, scaled
    by fact rows to the GPU's table."""
    import torch

    from ahead_b200 import ssb_programs as P
    from ahead_b200.gpu import AheadError
    from ahead_b200.ssb import generate, inject_flips
    from oracle.oracle import REF_LIB, Oracle
    progs = [P.q11, P.q12, P.q13, P.q21, P.q22, P.q23, P.q31, P.q32, P.q33, P.q34, P.q41, P.q42, P.q43]

    def run(ops, sch, prog, placement="continuous", plain=None):
        try:
            prog(ops, sch, placement, plain) if plain is not None else prog(ops, sch, placement)
            return "ok"
        except AheadError as e:  # the reference's size-mismatch exception under bit flips
            return f"error {e.status}"
        except Exception as e:  # the oracle's form of the same
            return f"error {getattr(e, 'status', type(e).__name__)}"

    gpu_ms, outcome = {}, {}
    for prog in progs:
        run(gpu, schema, prog)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        outcome[prog.__name__] = run(gpu, schema, prog)
        torch.cuda.synchronize()
        gpu_ms[prog.__name__] = (time.perf_counter() - t0) * 1e3
    # the reference's DMR baseline on the same GPU: two unencoded replicas, the
    # normal placement on each, a vote
    from ahead_b200.ssb import decoded_device
    plains = [decoded_device(schema), decoded_device(schema), decoded_device(schema)]
    # the other detection placements of the same programs (the survey's third
    # configuration: early, late and re-encoding detection at this size)
    place_ms, place_outcome = {}, {}
    for pl in ("normal", "early", "late", "continuous_reenc"):
        place_ms[pl], place_outcome[pl] = {}, {}
        for prog in progs:
            plain = plains[0] if pl == "normal" else None
            run(gpu, schema, prog, pl, plain)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            place_outcome[pl][prog.__name__] = run(gpu, schema, prog, pl, plain)
            torch.cuda.synchronize()
            place_ms[pl][prog.__name__] = (time.perf_counter() - t0) * 1e3

    def voted(vote, reps):
        ms, outcome = {}, {}
        for prog in progs:
            def one():
                try:
                    vote(prog, gpu, reps)
                    return "ok"
                except P.ModularityError as e:
                    return str(e)
                except AheadError as e:  # the unencoded path on corrupt values: the reference's size mismatch
                    return f"error {e.status}"
            one()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            outcome[prog.__name__] = one()
            torch.cuda.synchronize()
            ms[prog.__name__] = (time.perf_counter() - t0) * 1e3
        return ms, outcome
    dmr_ms, dmr_outcome = voted(P.dmr, plains[:2])
    tmr_ms, tmr_outcome = voted(P.tmr, plains)  # three replicas, the reference's majority vote
    # the reference's `_mt` form: the two replicas at once, each on a context (stream) of its own
    from ahead_b200.gpu import GpuOps
    pair = [GpuOps(torch.cuda.current_device()), GpuOps(torch.cuda.current_device())]
    dmr_mt_ms, _ = voted(lambda prog, _ops, reps: P.dmr(prog, pair, reps, concurrent=True), plains[:2])
    for g in pair:
        g.close()
    del plains
    torch.cuda.empty_cache()
    kind = "reference" if os.path.exists(REF_LIB) else "port"
    o = Oracle(kind)
    s = generate(dict(SF1, fact=cpu_rows), seed=seed)
    for i, c in enumerate(("custkey", "suppkey", "partkey", "orderdate", "price", "discount", "quantity")):
        inject_flips(s, "lineorder", c, 2, seed=seed + 100 + i)
    cpu_ms = {}
    for prog in progs:
        t0 = time.perf_counter()
        run(o, s, prog)
        cpu_ms[prog.__name__] = (time.perf_counter() - t0) * 1e3 * fact_rows / cpu_rows
    ratio = [cpu_ms[k] / gpu_ms[k] for k in gpu_ms if gpu_ms[k] > 0]
    return {"placement": "continuous", "fact_rows": fact_rows, "gpu_ms": gpu_ms, "gpu_outcome": outcome,
            "other_placements_gpu_ms": place_ms, "other_placements_outcome": place_outcome,
            "dmr_gpu_ms": dmr_ms, "dmr_outcome": dmr_outcome, "dmr_concurrent_gpu_ms": dmr_mt_ms,
            "tmr_gpu_ms": tmr_ms, "tmr_outcome": tmr_outcome,
            "cpu_ms_scaled": cpu_ms, "cpu_kind": kind, "cpu_cores": 1,
            "cpu_sample": f"each program once on a {cpu_rows:,}-row lineorder with SF1-shaped dimensions, "
                          f"scaled by fact rows to {fact_rows:,}",
            "speedup_geomean": float(np.exp(np.mean(np.log(ratio)))) if ratio else None,
            "timing": "wall clock around each program (synchronized), operator-at-a-time GPU path"}


def ops_measure(gpu, schema, n: int, peak: float, steps: int = 10, warmup: int = 3):
    """The scan operators alone through the C ABI on device-resident columns,
    CUDA events on the library's stream over `steps` calls after `warmup`:
    selectAN (a range on codes, ~20 % selected), checkAndDecodeAN and checkAN
    of an n-row u16 column AN-coded with A = 233 into u32 (values uniform in
    [0, 10000), 10 single-bit flips), and aggregate_mul_sumAN over the fact
    table's price and discount.  Bytes are algorithmic: every input row once
    plus the outputs the call writes."""
    import ctypes

    import torch

    from ahead_b200.gpu import _in_bat, load_library
    from ahead_b200.model import AND, GE, LT, RESBIGINT, RESSHORT, CBat, CErrVec, Col, ainv, ccol, void_col
    lib = load_library()
    ctx = gpu.ctx
    stream = gpu.stream()
    U = ctypes.c_uint64
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    v = torch.randint(0, 10_000, (n,), generator=g, device="cuda", dtype=torch.int64)
    codes = (v * 233).to(torch.int32)
    del v
    rows = torch.randint(0, n, (10,), generator=g, device="cuda")
    bits = torch.randint(0, 31, (10,), generator=g, device="cuda", dtype=torch.int32)
    codes[rows] ^= torch.ones_like(bits) << bits
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    A, Ai = 233, ainv(233, 32)
    col = CBat(ccol(void_col(0), 0), ccol(Col(RESSHORT, None, A, Ai, 0xFFFF, 0), codes.data_ptr()), n)
    out_h = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
    out_t = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
    ebuf = [torch.empty(1 << 16, dtype=torch.int64, device="cuda") for _ in range(2)]

    def errvecs():
        e = (CErrVec * 2)()
        for i in range(2):
            e[i].data, e[i].capacity = ebuf[i].data_ptr(), 1 << 16
        return e

    def outbat():
        o = CBat()
        o.head.data, o.tail.data = out_h.data_ptr(), out_t.data_ptr()
        return o

    def timed(call):
        for _ in range(warmup):
            res = call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            res = call()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, res

    out = {}

    def sel():
        o, e = outbat(), errvecs()
        rc = lib.ahead_gpu_select_an(ctx, ctypes.byref(col), GE, U(1000 * A), LT, U(3000 * A), AND, U(16089),
                                     ctypes.byref(o), U(n), ctypes.byref(e[0]))
        return rc, int(o.count), int(e[0].count)
    ms, (rc, k, ne) = timed(sel)
    out["selectAN"] = dict(ms=ms, rows=n, selected=k, errors=ne, bytes=n * 4 + k * 8 + ne * 8, status=rc)

    def cad():
        o, e = outbat(), errvecs()
        rc = lib.ahead_gpu_check_and_decode_an(ctx, ctypes.byref(col), U(16089), ctypes.byref(o), U(n),
                                               ctypes.byref(e[0]), ctypes.byref(e[1]))
        return rc, int(o.count), int(e[1].count)
    ms, (rc, k, ne) = timed(cad)
    out["checkAndDecodeAN"] = dict(ms=ms, rows=n, decoded=k, errors=ne, bytes=n * 4 + k * 2 + ne * 8, status=rc)

    def chk():
        e = errvecs()
        rc = lib.ahead_gpu_check_an(ctx, ctypes.byref(col), U(Ai), U(0xFFFF), U(16089), ctypes.byref(e[0]))
        return rc, int(e[0].count)
    ms, (rc, ne) = timed(chk)
    out["checkAN"] = dict(ms=ms, rows=n, errors=ne, bytes=n * 4 + ne * 8, status=rc)

    price, disc = schema.tables["lineorder"]["price"], schema.tables["lineorder"]["discount"]
    pb, db = _in_bat(price), _in_bat(disc)
    m = price.count

    def mulsum():
        tot = U(0)
        e = errvecs()
        rc = lib.ahead_gpu_aggregate_mul_sum_an(ctx, ctypes.byref(pb), ctypes.byref(db), RESBIGINT, U(0), U(65117),
                                                U(ainv(65117, 64)), U(16089), ctypes.byref(tot), e)
        return rc, int(e[0].count) + int(e[1].count)
    ms, (rc, ne) = timed(mulsum)
    out["aggregate_mul_sumAN"] = dict(ms=ms, rows=m, errors=ne, bytes=m * 10 + ne * 8, status=rc)
    for r in out.values():
        r["gbs"] = r["bytes"] / (r["ms"] / 1e3) / 1e9
        r["frac"] = r["gbs"] / peak
    del codes, out_h, out_t, ebuf
    torch.cuda.empty_cache()
    return out


LINEORDER_AN = [("orderkey", "RESINT"), ("linenumber", "RESTINY"), ("custkey", "RESINT"), ("partkey", "RESINT"),
                ("suppkey", "RESINT"), ("orderdate", "RESINT"), ("orderpriority", "STRING:15"),
                ("shippriority", "CHAR"), ("quantity", "RESTINY"), ("extendedprice", "RESINT"),
                ("ordertotalprice", "RESINT"), ("discount", "RESTINY"), ("revenue", "RESINT"),
                ("supplycost", "RESINT"), ("tax", "RESTINY"), ("commitdate", "RESINT"), ("shipmode", "STRING")]


def lineorder_like(n: int, seed: int):
    """Columns with the reference's lineorderAN header (17 columns: 14 AN
    integers, two strings, a char) and SSB-shaped value ranges; the string
    fields are synthetic tokens."""
    from ahead_b200.ssb import date_keys
    rng = np.random.default_rng(seed)
    dk = date_keys().astype(np.int64)
    prio = np.array([f"PRIO-{i}".encode() for i in range(1, 6)])
    mode = np.array([f"MODE-{c}".encode() for c in "ABCDEFG"])
    cols = [np.arange(1, n + 1) // 4 + 1, rng.integers(1, 8, n), rng.integers(1, 30_001, n),
            rng.integers(1, 200_001, n), rng.integers(1, 2_001, n), dk[rng.integers(0, len(dk), n)],
            prio[rng.integers(0, 5, n)], np.full(n, b"0"), rng.integers(1, 51, n), rng.integers(90_000, 11_000_001, n),
            rng.integers(90_000, 50_000_001, n), rng.integers(0, 11, n), rng.integers(80_000, 11_000_001, n),
            rng.integers(1, 100_001, n), rng.integers(0, 9, n), dk[rng.integers(0, len(dk), n)],
            mode[rng.integers(0, 7, n)]]
    return [c for c, _ in LINEORDER_AN], [t for _, t in LINEORDER_AN], cols


def ingest_measure(gpu, peak: float, rows: int, reenc_rows: int, seed: int, cpu_lines: int = 500_000):
    """The table loader (include/ahead_ingest.h) on a lineorder-shaped table of
    `rows` rows written as `.tbl` text: a text load (the file in the page
    cache, streamed to the device and parsed there), the load that also
    writes the `.ahead` column files, a load from those files, and one with
    minimum bit-flip weight 2 (the 14 AN columns re-encoded on the
    device).  The re-encode kernel alone runs on `reenc_rows` resint codes
    (A 65117 <-> 16089), CUDA events on the library's stream; its bytes are
    a read and a write of every code.  The CPU line is the restatement of
    the reference's line loop (strtok / atol, one thread) on the first
    `cpu_lines` lines."""
    import ctypes

    import torch

    from ahead_b200 import ingest
    d = tempfile.mkdtemp(prefix="ahead_ingest_")
    out = {}
    try:
        names, types, cols = lineorder_like(rows, seed)
        path = os.path.join(d, "lineorderAN")
        t0 = time.perf_counter()
        ingest.write_tbl(path, names, types, cols)
        del cols
        text_bytes = os.path.getsize(path + ".tbl")
        out["workload"] = (f"lineorder-shaped table ({len(names)} columns of the reference's lineorderAN header, "
                           f"{rows:,} rows, {text_bytes / 1e6:.0f} MB of .tbl text), synthetic values")
        out["generate_s"] = time.perf_counter() - t0

        def run(**kw):
            t0 = time.perf_counter()
            t = ingest.load(gpu, path, **kw)
            ms = (time.perf_counter() - t0) * 1e3
            st = dict(t.stats)
            assert t.rows == rows
            del t
            return ms, st

        run(convert_table_files=False)  # warm-up: kernels loaded, text in the page cache
        ms, st = run(convert_table_files=False)
        out["text_load"] = {"ms": ms, "gbs": text_bytes / ms / 1e6, "rows_per_s": rows / ms * 1e3,
                            "parse_device_ms": st["parse_ms"], "parse_device_gbs": text_bytes / st["parse_ms"] / 1e6,
                            "file_ms": st["file_ms"], "blocks": st["blocks"]}
        ms, st = run()
        out["text_load_and_convert"] = {"ms": ms, "written_bytes": st["written_bytes"], "file_ms": st["file_ms"]}
        ms, st = run()
        out["binary_load"] = {"ms": ms, "bytes": st["binary_bytes"], "gbs": st["binary_bytes"] / ms / 1e6}
        ms, st = run(min_bfw=2)
        out["binary_load_minbfw2"] = {"ms": ms, "bytes": st["binary_bytes"], "gbs": st["binary_bytes"] / ms / 1e6,
                                      "reencoded": st["reencoded"], "reencode_device_ms": st["reencode_ms"]}
        cpu = None
        if cpu_lines:
            from oracle import tbl_oracle
            with open(path + ".tbl", "rb") as f:
                head = b"".join(f.readline() for _ in range(cpu_lines))
            hdr = ingest.read_header(path)
            kinds = [{ingest.STRING: 3, ingest.CHAR: 5}.get(t, 2) for _, t, _ in hdr]
            widths = [w for _, _, w in hdr]
            As = [tbl_oracle.LOAD_A.get(t, 0) for _, t, _ in hdr]
            t0 = time.perf_counter()
            rc, lines, _, _ = tbl_oracle.tbl_parse(head, kinds, widths, As)
            s = time.perf_counter() - t0
            cpu = {"value": lines / s, "unit": "rows/s", "gbs": len(head) / s / 1e9, "cores": 1, "kind": "port",
                   "sample": f"first {lines:,} lines ({len(head) / 1e6:.0f} MB), status {rc}"}
        out["cpu_baseline"] = cpu
    finally:
        shutil.rmtree(d, ignore_errors=True)

    lib = ingest._bind(gpu.lib)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    codes = torch.randint(0, 1 << 32, (reenc_rows,), generator=g, device="cuda", dtype=torch.int64) * 65117
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    stream = gpu.stream()
    pair = ((65117, 16089), (16089, 65117))
    for i in range(4):
        lib.ahead_gpu_reencode(gpu.ctx, codes.data_ptr(), reenc_rows, 8, *pair[i % 2])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k = 10
    e0.record(stream)
    for i in range(k):
        lib.ahead_gpu_reencode(gpu.ctx, codes.data_ptr(), reenc_rows, 8, *pair[i % 2])
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / k
    ok = bool(((codes * ingest_inverse(65117)) >> 32 == 0).all())  # still valid 65117-codes after an even count
    gbs = 16 * reenc_rows / ms / 1e6
    out["reencode_kernel"] = {"rows": reenc_rows, "width": 8, "ms": ms, "gbs": gbs, "peak": peak,
                              "frac": gbs / peak, "valid_after": ok,
                              "algorithmic_bytes": "16 B per value (read + write of a resint code)"}
    del codes
    torch.cuda.empty_cache()
    return out


def ingest_inverse(a: int) -> int:
    """A^-1 mod 2^64 as a signed int64 (torch multiplies in int64)."""
    v = pow(a, -1, 1 << 64)
    return v - (1 << 64) if v >= (1 << 63) else v


def reference_arm(args):
    """The reference's own CPU implementation of the path on the host's cores:
    its scalar AN operators compiled from its sources (oracle/_ref), composed
    as the star join, over a host schema with SF100 dimensions and a 60M-row
    lineorder (1,000 flips).  Each timed step runs one query per host thread,
    all threads at once, at one prefix size (1M and 6M in turn); after the
    steps, one query per thread at the 60M prefix, measured once.  The 600M
    prefix is taken as REF_600M_OVER_60M times the 60M time (measured by
    `--ref-scaling` on one thread): the reference materializes its
    intermediate BATs (about 155 B per joined fact row at peak), so one 600M
    query holds ~90 GB and one per host thread cannot run at once on the
    host, and a single one takes minutes (`--ref-scaling` measures the same
    queries at both prefixes on one thread to check the linear scaling).
    value = the family's queries/s (prefix sizes equally likely) from the
    seconds per query of each size; ms_per_step = the mean timed step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle.oracle import REF_LIB, Oracle
    if not os.path.exists(REF_LIB):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libahead_ref.so not built "
                          "(needs the reference sources at build time)"}))
        return 0
    threads = os.cpu_count() or 1
    o = Oracle("reference")
    t_gen = time.perf_counter()
    rows = min(args.fact_rows, FACT_SIZES[2])
    s = host_star_schema(rows, args.seed, threads, args.flips)
    t_gen = time.perf_counter() - t_gen
    sizes = [z for z in FACT_SIZES if z <= rows]
    small = [z for z in sizes if z < FACT_SIZES[2]] or sizes
    nsteps = args.warmup + args.steps
    qs = family_by_size(args.seed + 1, sizes, threads * (nsteps // len(small) + 1))
    used = {z: 0 for z in sizes}
    walls, nq = {z: 0.0 for z in sizes}, {z: 0 for z in sizes}
    step_ms = []
    for i in range(nsteps):
        z = small[(i - args.warmup) % len(small)]  # the timed steps start with the first size
        batch = qs[z][used[z]: used[z] + threads]
        used[z] += threads
        w = cpu_run_batch(o, s, batch, threads)
        if i >= args.warmup:
            step_ms.append(w * 1e3)
            walls[z] += w
            nq[z] += len(batch)
    big = [z for z in sizes if z not in small] + [z for z in small if not nq[z]]  # (fewer steps than sizes)
    for z in big:  # the 60M prefix: one query per thread, measured once
        walls[z] = cpu_run_batch(o, s, qs[z][:threads], threads)
        nq[z] = threads
    per = {z: walls[z] / nq[z] for z in sizes if nq[z]}
    if args.fact_rows >= FACT_SIZES[3] and FACT_SIZES[2] in per:
        per[FACT_SIZES[3]] = REF_600M_OVER_60M * per[FACT_SIZES[2]]
    for z in FACT_SIZES:
        per.setdefault(z, float("nan"))
    value = family_qps(per)
    sample = (f"measured on SF100 dims (customer 3,000,000, part 1,400,000, supplier 200,000, date 2,556) over a "
              f"{rows:,}-row lineorder with {args.flips} flips: steps of {threads} queries (one per host "
              f"thread) cycling prefixes " + "/".join(f"{z // 1_000_000}M" for z in small) +
              (f", then {threads} queries at the " + "/".join(f"{z // 1_000_000}M" for z in big) +
               " prefix" if big else "") +
              "; s/query at full load: " + ", ".join(f"{z // 1_000_000}M {per[z]:.3f}" for z in sizes) +
              (f"; the 600M prefix taken as {REF_600M_OVER_60M}x the 60M time (the ratio --ref-scaling measured "
               "on one thread; one 600M query holds ~90 GB of the reference's intermediates)"
               if args.fact_rows >= FACT_SIZES[3] else ""))
    extra = cpu_reference_extrapolated(args.seed, threads, threads)
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(step_ms)),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
           "data": "synthetic", "config": workload_config(args, args.fact_rows),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample,
                            "seconds_per_query": {str(z): per[z] for z in FACT_SIZES if per[z] == per[z]},
                            "generate_s": t_gen},
           "extrapolated": {"value": extra, "unit": UNIT,
                            "how": "the same composition on an SF1-sized schema with prefixes capped at 6M, "
                                   "scaled by fact rows to the family's mean prefix (the earlier estimate)"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def ref_scaling_arm(args):
    """The check behind the reference arm's 600M term: `--ref-queries`
    queries of the family's 600M prefix, each run on one host thread on the
    reference's operators over an SF100-shaped host schema with the full
    lineorder, at the 60M and at the 600M prefix; prints the seconds of each
    and their ratio (10 when the reference's time is linear in the prefix)."""
    from oracle.oracle import REF_LIB, Oracle
    from ahead_b200.pipelines import starjoin_continuous
    o = Oracle("reference" if os.path.exists(REF_LIB) else "port")
    threads = os.cpu_count() or 1
    s = host_star_schema(args.fact_rows, args.seed, threads, args.flips)
    big = FACT_SIZES[3] if args.fact_rows >= FACT_SIZES[3] else args.fact_rows
    small = big // 10
    qs = family_by_size(args.seed + 1, (FACT_SIZES[3],), args.ref_queries)[FACT_SIZES[3]]
    rows = []
    for q in qs:
        t = {}
        for n in (small, big):
            q.fact_rows = n
            t0 = time.perf_counter()
            starjoin_continuous(o, s, q)
            t[n] = time.perf_counter() - t0
        rows.append({"dims": [str(d) for d in q.dims()], "preds": len(q.preds), "groups": len(q.group),
                     "s_small": t[small], "s_big": t[big], "ratio": t[big] / t[small]})
    print(json.dumps({"ref_scaling": rows, "small_rows": small, "big_rows": big, "threads_used": 1,
                      "schema": f"SF100 dims, {args.fact_rows:,}-row lineorder, {args.flips} flips",
                      "mean_ratio": float(np.mean([r["ratio"] for r in rows]))}))
    return 0


# ------------------------------------------------------------- GPU arm
def fused_same(a, b):
    """Two FusedResults (the fused engine's, the C++ plain path's) are equal."""
    from ahead_b200.model import OK
    if a.status != OK or b.status != OK or a.total != b.total or len(a.keys) != len(b.keys):
        return False
    if (a.sums is None) != (b.sums is None) or (a.sums is not None and not np.array_equal(a.sums, b.sums)):
        return False
    if any(not np.array_equal(x, y) for x, y in zip(a.keys, b.keys)):
        return False
    return all(np.array_equal(a.fact_errors[c], b.fact_errors[c]) for c in a.fact_errors)


def fused_vs_plain(fused, plain):
    """Fused result (FusedResult) equals the plain path's StarResult."""
    from ahead_b200.gpu import err_to_host, to_host
    from ahead_b200.model import OK
    if fused.status != OK:
        return False
    if plain.sums is None:
        if fused.total != plain.total:
            return False
    else:
        keys = [np.asarray(to_host(k).tail.data, dtype=np.uint64) for k in plain.keys]
        sums = np.asarray(to_host(plain.sums).tail.data, dtype=np.uint64)
        if not np.array_equal(fused.sums, sums) or any(not np.array_equal(a, b) for a, b in zip(fused.keys, keys)):
            return False
    for c, e in plain.fact_errors.items():
        v = err_to_host(e).values
        v = np.zeros(0, np.uint64) if v is None else np.asarray(v, dtype=np.uint64)
        if not np.array_equal(fused.fact_errors[c], v):
            return False
    return all(len(v) == 0 for c, v in fused.fact_errors.items() if c not in plain.fact_errors)


def serve_measure(args, eng, gpu, schema, fact_rows, starjoin_continuous):
    """Serving: an open-loop Poisson stream of the same random query family
    through the C++ request loop (latency = results on the host - scheduled
    arrival); at a low rate also the plain operator-at-a-time path as a FIFO
    single server (its queueing latencies by the Lindley recursion over the
    service times measured for the same queries)."""
    import torch

    from ahead_b200.serving import StarJoinServer, poisson_arrivals
    from ahead_b200.ssb import random_query

    def run(rate, n, seed):
        rng = np.random.default_rng(seed)
        qs = [random_query(rng, fact_sizes=FACT_SIZES, max_fact=fact_rows) for _ in range(n)]
        arr = poisson_arrivals(rate, n, seed + 1)
        srv = StarJoinServer(eng, window_ms=args.window_ms, max_batch=BATCH, hbm_budget=150 << 30)
        ids = srv.replay(qs, arr)
        got = srv.collect(ids, timeout_s=600)
        st = srv.stats()
        srv.close()
        lat = np.array([got[i].latency_ms for i in ids])
        span = (max(got[i].done_us for i in ids) - min(got[i].arrival_us for i in ids)) / 1e6
        return qs, arr, lat, {"rate_qps": rate, "requests": n, "throughput_qps": n / span,
                              "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                              "mean_batch": st.mean_batch, "batches": int(st.batches),
                              "ok": int(sum(got[i].result.status == 0 for i in ids))}

    _, _, _, high = run(args.serve_rate, int(args.serve_rate * args.serve_seconds), args.seed + 7)
    qs, arr, _, low = run(args.low_rate, args.low_n, args.seed + 9)
    # the plain path as a FIFO server over the same arrivals
    svc = []
    for q in qs:
        torch.cuda.synchronize()
        t = time.perf_counter()
        starjoin_continuous(gpu, schema, q)
        torch.cuda.synchronize()
        svc.append((time.perf_counter() - t) * 1e6)
    free, plat = 0.0, []
    for a, sv in zip(arr, svc):
        start = max(a, free)
        free = start + sv
        plat.append((free - a) / 1e3)
    low["plain_p50_ms"] = float(np.percentile(plat, 50))
    low["plain_p99_ms"] = float(np.percentile(plat, 99))
    low["plain_mean_service_ms"] = float(np.mean(svc) / 1e3)
    return {"window_ms": args.window_ms, "hbm_budget_gb": 150, "high_rate": high, "low_rate": low,
            "latency": "results in host memory minus the scheduled arrival time"}


# the SF100 batches' signature count: 41 customer x 201 part x 41 supplier x 8 date codes
CUBE_CELLS = 41 * 201 * 41 * 8


def cube_roofs(lib, gpu, fact_rows, stats, fact_ms):
    """The cube scan's second roof: the measured rates of its column stream
    alone, of one random 64-bit L2 reduction per row alone and of both together
    (ahead_gpu_cube_roofs on synthetic rows of the scan's layout), and the
    scan's own rows per second as a fraction of the combined rate."""
    import ctypes
    rows = min(fact_rows, 200_000_000) // 512 * 512
    ms = (ctypes.c_float * 3)()
    lib.ahead_gpu_cube_roofs.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float)]
    if rows < 512 or lib.ahead_gpu_cube_roofs(gpu.ctx, rows, CUBE_CELLS, ms) != 0:
        return None
    scan = float(np.sum([s.fact_rows for s in stats]) / (np.sum(fact_ms) / 1e3))
    both = rows / (ms[2] / 1e3)
    return {"probe_rows": rows, "cells": CUBE_CELLS, "bytes_per_row": 50,
            "stream_rows_per_s": rows / (ms[0] / 1e3), "stream_gbs": rows * 50 / (ms[0] / 1e3) / 1e9,
            "reductions_per_s": rows / (ms[1] / 1e3), "stream_and_reductions_rows_per_s": both,
            "scan_rows_per_s": scan, "frac": scan / both,
            "command": "ahead_gpu_cube_roofs (include/ahead_gpu.h), median of five launches each"}


def scan_bytes_per_row(batch):
    dims = set()
    for q in batch:
        dims |= set(q.dims())
    return 8 * len(dims) + 8 + 2  # foreign keys (resint) + price (resint) + discount (restiny)


def gpu_arm(args):
    import torch

    from ahead_b200.gpu import GpuOps, load_library
    from ahead_b200.pipelines import starjoin_continuous
    from ahead_b200.ssb import generate_device
    from ahead_b200.starjoin import PACKED_SLOTS, StarJoinEngine

    from ahead_b200.replicas import Replicas
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    grp = Replicas("nccl")
    world, rank, local = grp.world, grp.rank, grp.local
    barrier, max_over_ranks = grp.barrier, grp.max

    fact_rows = args.fact_rows
    sizes = dict(SF100, fact=fact_rows)
    schema = generate_device(sizes, seed=args.seed, flips=args.flips, flip_seed=args.seed + 17)
    torch.cuda.synchronize()
    gpu = GpuOps(local)
    eng = StarJoinEngine(gpu, schema)
    if args.index_format != -1:
        eng.set_index(args.index_format)
    lib = load_library()
    stream = gpu.stream()  # the library's stream: the events below time its kernels
    batches = make_batches(grp.seed(args.seed), args.warmup + args.steps, fact_rows)

    with ClockSampler(local) as clk:  # sampling from before the warm-up on
        # warm-up: the tuner picks the fact-kernel shape, then the slots' graphs are captured
        variant = eng.tune(batches[0])
        if args.cube_variant >= 0:  # a fixed scan shape (e.g. for a launch list under a profiler)
            eng.set_cube_variant(args.cube_variant)
        for b in batches[: args.warmup]:
            eng.run(b, graph=True)

        # value: K batches, two in flight, CUDA events on the launching stream
        launches0 = lib.ahead_ctx_launches(gpu.ctx)
        timed = batches[args.warmup:]
        fact_ms, scan_bytes, stats = [], [], []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clk.mark_start()
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        pending = []
        for b in timed:
            pending.append((eng.submit(b, graph=True), b))
            if len(pending) == 2:
                t, bb = pending.pop(0)
                eng.wait(t)
                st = eng.last_stats()
                fact_ms.append(st.fact_ms)
                scan_bytes.append(st.fact_rows * scan_bytes_per_row(bb))
                stats.append(st)
        for t, bb in pending:
            eng.wait(t)
            st = eng.last_stats()
            fact_ms.append(st.fact_ms)
            scan_bytes.append(st.fact_rows * scan_bytes_per_row(bb))
            stats.append(st)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        launches = lib.ahead_ctx_launches(gpu.ctx) - launches0
        t_value = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        nq_total = BATCH * args.steps * world
        value = nq_total / t_value

        # e2e: wall clock through the public API (submit / wait, two batches in
        # flight), host descriptors in and host results out every batch
        barrier()
        torch.cuda.synchronize()
        h2d = d2h = 0
        t0 = time.perf_counter()
        pending = []
        for b in timed:
            pending.append(eng.submit(b, graph=True))
            if len(pending) == 2:
                eng.wait(pending.pop(0))
                st = eng.last_stats()
                h2d += st.h2d_bytes
                d2h += st.d2h_bytes
        for t in pending:
            eng.wait(t)
            st = eng.last_stats()
            h2d += st.h2d_bytes
            d2h += st.d2h_bytes
        torch.cuda.synchronize()
        t_e2e = max_over_ranks(time.perf_counter() - t0)
        e2e = nq_total / t_e2e
        # the same, one synchronous call per batch
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for b in timed:
            eng.run(b, graph=True)
        torch.cuda.synchronize()
        e2e_sync = nq_total / max_over_ranks(time.perf_counter() - t0)
        clk.mark_end()

    out = None
    if rank == 0:
        # plain operator-at-a-time GPU path on a sample of the first timed batch:
        # composed in C++ through the C ABI (ahead_plain_starjoin), and the same
        # composition driven from Python (pipelines.starjoin_continuous)
        sample = timed[0][: args.plain]
        fused = eng.run(sample, graph=False)
        for q in sample:  # untimed warm-up: first launches load kernels, the allocators reserve their memory
            eng.plain(q)
            starjoin_continuous(gpu, schema, q)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain_cpp = [eng.plain(q) for q in sample]
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - t0
        plain_qps = len(sample) / t_plain
        t0 = time.perf_counter()
        plain = [starjoin_continuous(gpu, schema, q) for q in sample]
        torch.cuda.synchronize()
        plain_py_qps = len(sample) / (time.perf_counter() - t0)
        parity = all(fused_vs_plain(f, p) for f, p in zip(fused, plain)) and \
            all(fused_same(f, c) for f, c in zip(fused, plain_cpp))
        del plain, plain_cpp

        peaks_path = os.path.join(HERE, "MEASURED_PEAKS.json")
        if os.path.exists(peaks_path):
            peak, peak_src = json.load(open(peaks_path))["hbm_gbs"], "measured"
        else:
            peak, peak_src = 6650.0, "fallback"
        achieved = sum(scan_bytes) / (sum(fact_ms) / 1e3) / 1e9
        traffic = None
        cube = all(st.strategy == 1 for st in stats)
        indexed = cube and all(eng.cube_variant_is_indexed(st.cube_variant) for st in stats)
        kernel = ("sj_cube_ix_kernel" if indexed else "sj_cube_kernel") if cube else "sj_fact_kernel"
        cube_variants = sorted({int(st.cube_variant) for st in stats})
        # index bytes per row the scan reads: 8 per slot word, 8 for the packed word
        ix_bytes = max((0 if not eng.cube_variant_reads_index(v) else
                        8 if eng.cube_variant_slots(v) in (1, PACKED_SLOTS) else 16) for v in cube_variants)
        tr_path = os.path.join(HERE, "profiles", f"{kernel}_traffic.txt")
        if os.path.exists(tr_path):
            # the captured figure for this index format (bytes per row), else the kernel's
            want = f"dram_bytes_per_scanned_row_index{ix_bytes}" if indexed else "dram_bytes_per_scanned_row"
            figures = {}
            for line in open(tr_path):
                if line.startswith("dram_bytes_per_scanned_row"):
                    figures[line.split("=")[0].strip()] = float(line.split("=")[1])
            per_row = figures.get(want, figures.get("dram_bytes_per_scanned_row"))
            if per_row is not None:
                traffic = per_row * float(np.mean([s.fact_rows for s in stats]))
        # the single-GPU sections run at N = 1 only: with more ranks every GPU of
        # the job would wait on rank 0 through them
        single = world == 1
        l2_roof = cube_roofs(lib, gpu, fact_rows, stats, fact_ms) if single and cube else None
        serving = serve_measure(args, eng, gpu, schema, fact_rows, starjoin_continuous) if single else None
        programs = None if args.no_programs or not single else programs_measure(gpu, schema, fact_rows, args.seed,
                                                                                 2_000_000)
        if programs is not None:
            programs["fused"] = programs_fused_measure(gpu, eng, schema, fact_rows)
        ops = None if args.no_programs or not single else ops_measure(gpu, schema, fact_rows, peak)
        ingest_out = None if args.no_ingest or not single else ingest_measure(gpu, peak, args.ingest_rows,
                                                                              args.reencode_rows, args.seed)
        configs = None if args.no_programs or not single else configs_measure(gpu, args.seed)
        cpu = None
        if not args.no_cpu and single:  # the CPU baseline: rank 0 at N = 1 only
            threads = os.cpu_count() or 1
            v, desc, kind, per = cpu_reference_sample(args.seed, threads)
            cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": kind, "sample": desc,
                   "seconds_per_query": {str(z): t for z, t in per.items()}}
        cfg = workload_config(args, fact_rows)
        cfg["parallelism"] = f"replicas{world}" if world > 1 else "single"
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_value / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": cfg,
            "clocks": clk.summary(),
            "e2e": {"value": e2e, "unit": UNIT, "sync_calls_value": e2e_sync, "h2d_bytes_per_step": h2d // len(timed),
                    "d2h_bytes_per_step": d2h // len(timed)},
            "gpu_launches": int(launches),
            "exception_rows_per_step": float(np.mean([s.exception_rows for s in stats])),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
                         "cube_variants": cube_variants,
                         "kernel_bytes_per_row": (scan_bytes_per_row(timed[0]) + ix_bytes) if indexed else None,
                         "index_bytes_per_row": ix_bytes if indexed else None,
                         "peak_source": peak_src,
                         "algorithmic_bytes": "rows scanned x (8 B per referenced foreign key + 8 B price + 2 B discount)",
                         "fact_kernel_variant": variant,
                         "fact_ms_mean": float(np.mean(fact_ms)), "batch_ms_mean": float(np.mean([s.batch_ms for s in stats])),
                         "l2": l2_roof},
            "parity": {"fused_vs_plain_600M": parity, "queries": len(sample)},
            "plain": {"value": plain_qps, "unit": UNIT, "queries": len(sample), "parity_with_fused": parity,
                      "host": "C++ (ahead_plain_starjoin)", "python_composition_value": plain_py_qps},
            "speedup_vs_plain": value / plain_qps,
            "serving": serving,
            "programs": programs,
            "operators": ops,
            "config1": None if configs is None else configs["config1"],
            "config2": None if configs is None else configs["config2"],
            "ingest": ingest_out,
            "cpu_baseline": cpu,
        }
    eng.close()
    grp.close()
    if out is not None:
        print(json.dumps(out))
        if not out["parity"]["fused_vs_plain_600M"]:
            print("parity failure: fused results differ from the operator-at-a-time path", file=sys.stderr)
            return 3
    return 0


def profile_arm(args):
    """A small, fixed invocation for ncu: build the schema, run
    --profile-batches batches of the query family without graphs (cube scan
    shape --cube-variant), print each batch's kernel times."""
    import torch

    from ahead_b200.gpu import GpuOps
    from ahead_b200.ssb import generate_device
    from ahead_b200.starjoin import StarJoinEngine
    torch.cuda.set_device(0)
    schema = generate_device(dict(SF100, fact=args.fact_rows), seed=args.seed, flips=args.flips,
                             flip_seed=args.seed + 17)
    eng = StarJoinEngine(GpuOps(0), schema)
    if args.index_format != -1:
        eng.set_index(args.index_format)
    if args.cube_variant >= 0:
        eng.set_cube_variant(args.cube_variant)
    eng.set_cube_split(args.cube_split)
    for b in make_batches(args.seed, args.profile_batches, args.fact_rows):
        eng.run(b, graph=False)
        st = eng.last_stats()
        print(json.dumps({"cube_variant": int(st.cube_variant), "cube_split": args.cube_split,
                          "batch_ms": st.batch_ms, "fact_ms": st.fact_ms, "rows": st.fact_rows,
                          "strategy": st.strategy, "exception_rows": st.exception_rows,
                          "unseen_sigs": st.unseen_sigs}))
    eng.close()
    return 0


def shard_arm(args):
    """Fact-sharded form (strong scaling): the same workload with lineorder's
    rows split into contiguous ranges, one per rank (every rank generates the
    same seeded table and keeps its range); per batch each rank's engine runs
    the local half over its rows, one exchange on the device combines the
    dense group tables and error logs of all ranks (all-reduce SUM / MIN /
    MAX and an all-gather over NCCL, ahead_b200/sharded.py), and each engine's
    final half orders the whole table's groups and errors.  Two batches in
    flight; time = CUDA events on the engine's stream, max over ranks."""
    import torch

    from ahead_b200.gpu import GpuOps, load_library
    from ahead_b200.replicas import Replicas
    from ahead_b200.sharded import EngineShardedStarJoin, shard_rows, shard_schema
    from ahead_b200.ssb import generate_device
    from ahead_b200.starjoin import StarJoinEngine
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    grp = Replicas("nccl")
    world, rank, local = grp.world, grp.rank, grp.local
    fact_rows = args.fact_rows
    full = generate_device(dict(SF100, fact=fact_rows), seed=args.seed, flips=args.flips, flip_seed=args.seed + 17)
    lo, n = shard_rows(fact_rows, world, rank)
    mine = shard_schema(full, lo, n)
    for b in mine.tables["lineorder"].values():  # keep only this rank's range in HBM
        b.tail.data = b.tail.data.clone()
    del full
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    gpu = GpuOps(local)
    eng = StarJoinEngine(gpu, mine)
    lib = load_library()
    batches = make_batches(args.seed, args.warmup + args.steps, fact_rows)  # one query stream for the job
    eng.tune(batches[0])  # (timed on the local rows, before the shard is declared)
    sj = EngineShardedStarJoin(eng, fact_rows, lo, group=grp if world > 1 else None)
    stream = gpu.stream()

    def run_all(bs):
        out = []
        for b in bs:
            r = sj.step(b)
            if r is not None:
                out.append(r)
        return out + sj.drain()

    with ClockSampler(local) as clk:
        run_all(batches[: args.warmup])
        launches0 = lib.ahead_ctx_launches(gpu.ctx)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clk.mark_start()
        grp.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        res = run_all(batches[args.warmup:])
        e1.record(stream)
        torch.cuda.synchronize()
        grp.barrier()
        t = grp.max(e0.elapsed_time(e1) / 1e3)
        clk.mark_end()
    launches = lib.ahead_ctx_launches(gpu.ctx) - launches0
    if rank == 0:
        cfg = workload_config(args, fact_rows)
        cfg.update(parallelism=f"fact-sharded{world}", shard_rows=n)
        nq = BATCH * args.steps
        print(json.dumps({
            "metric": METRIC, "value": nq / t, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": cfg,
            "clocks": clk.summary(), "gpu_launches": int(launches),
            "timing": "CUDA events on the engine's stream around the batches (local half, device exchange, "
                      "final half; two in flight), max over ranks",
            "statuses_ok": all(r.status == 0 for b in res for r in b)}))
    eng.close()
    grp.close()
    return 0


def ops_arm(args):
    """The scan operators alone on the bench's schema (also the invocation
    for an ncu launch list of their kernels): prints the `operators` object."""
    import torch

    from ahead_b200.gpu import GpuOps
    from ahead_b200.ssb import generate_device
    torch.cuda.set_device(0)
    peaks_path = os.path.join(HERE, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    schema = generate_device(dict(SF100, fact=args.fact_rows), seed=args.seed, flips=args.flips,
                             flip_seed=args.seed + 17)
    gpu = GpuOps(0)
    print(json.dumps(ops_measure(gpu, schema, args.fact_rows, peak)))
    gpu.close()
    return 0


def configs_arm(args):
    """The survey's configurations 1 and 2 alone: prints the `config1` and
    `config2` objects."""
    import torch

    from ahead_b200.gpu import GpuOps
    torch.cuda.set_device(0)
    gpu = GpuOps(0)
    out = configs_measure(gpu, args.seed)
    gpu.close()
    print(json.dumps(out))
    return 0 if all(v for c in out.values() for k, v in c.items() if k.startswith("parity")) else 3


def program_arm(args):
    """One SSB program (continuous placement) through the GPU operators on the
    bench's schema, one untimed and three timed runs (also the invocation for
    an ncu launch list of its kernels)."""
    import torch

    from ahead_b200 import ssb_programs as P
    from ahead_b200.gpu import GpuOps
    from ahead_b200.ssb import generate_device
    torch.cuda.set_device(0)
    schema = generate_device(dict(SF100, fact=args.fact_rows), seed=args.seed, flips=args.flips,
                             flip_seed=args.seed + 17)
    gpu = GpuOps(0)
    prog = getattr(P, args.program)
    ms = []
    for i in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        try:
            prog(gpu, schema, args.placement)
            status = "ok"
        except Exception as e:  # the reference's size-mismatch exception under bit flips
            status = f"error {getattr(e, 'status', type(e).__name__)}"
        torch.cuda.synchronize()
        ms.append((time.perf_counter() - t0) * 1e3)
    print(json.dumps({"program": args.program, "placement": args.placement, "fact_rows": args.fact_rows,
                      "ms": ms[1:], "status": status}))
    gpu.close()
    return 0


def programs_fused_arm(args):
    """The 13 SSB programs on the fused engine alone (the `programs.fused`
    object of the bench line), on the bench's schema."""
    import torch

    from ahead_b200.gpu import GpuOps
    from ahead_b200.ssb import generate_device
    from ahead_b200.starjoin import StarJoinEngine
    torch.cuda.set_device(0)
    schema = generate_device(dict(SF100, fact=args.fact_rows), seed=args.seed, flips=args.flips,
                             flip_seed=args.seed + 17)
    gpu = GpuOps(0)
    eng = StarJoinEngine(gpu, schema)
    print(json.dumps(programs_fused_measure(gpu, eng, schema, args.fact_rows)))
    eng.close()
    gpu.close()
    return 0


def ingest_arm(args):
    """The table loader's timing alone (also the small invocation for ncu):
    prints the `ingest` object of the bench line."""
    import torch

    from ahead_b200.gpu import GpuOps
    torch.cuda.set_device(0)
    peaks_path = os.path.join(HERE, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    gpu = GpuOps(0)
    print(json.dumps(ingest_measure(gpu, peak, args.ingest_rows, args.reencode_rows, args.seed,
                                    0 if args.no_cpu else 500_000)))
    gpu.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--fact-rows", type=int, default=SF100["fact"])
    ap.add_argument("--flips", type=int, default=FLIPS)
    ap.add_argument("--plain", type=int, default=16, help="queries timed on the plain GPU path")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--profile-batches", type=int, default=0,
                    help="only run this many batches without graphs (a small case for ncu) and exit")
    ap.add_argument("--index-format", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="join index: -1 packed when it fits (default), 0 none, 1 two words per row, 2 packed")
    ap.add_argument("--cube-variant", type=int, default=-1,
                    help="cube scan shape: with --profile-batches instead of the engine's default, "
                         "otherwise in place of the tuner's choice (-1: as chosen)")
    ap.add_argument("--no-programs", action="store_true", help="skip the 13 SSB programs' timing")
    ap.add_argument("--no-ingest", action="store_true", help="skip the table loader's timing")
    ap.add_argument("--ingest-only", action="store_true", help="time the table loader alone")
    ap.add_argument("--ops-only", action="store_true", help="time the scan operators alone")
    ap.add_argument("--configs-only", action="store_true", help="time the survey's configurations 1 and 2 alone")
    ap.add_argument("--ref-scaling", action="store_true",
                    help="reference operators: the same queries at the 60M and 600M prefixes on one host thread")
    ap.add_argument("--ref-queries", type=int, default=2, help="with --ref-scaling: queries to run")
    ap.add_argument("--program", default="", help="time one SSB program alone (q11 ... q43)")
    ap.add_argument("--programs-fused", action="store_true", help="the 13 SSB programs on the fused engine alone")
    ap.add_argument("--placement", default="continuous", help="with --program: detection placement")
    ap.add_argument("--shard", action="store_true",
                    help="fact-sharded form across the ranks (strong scaling) instead of replicas")
    ap.add_argument("--ingest-rows", type=int, default=SF1["fact"], help="rows of the loader's .tbl table")
    ap.add_argument("--reencode-rows", type=int, default=SF100["fact"], help="codes of the re-encode kernel timing")
    ap.add_argument("--cube-split", type=int, default=0,
                    help="with --profile-batches: rows of the cube scan's first phase (0: automatic)")
    ap.add_argument("--window-ms", type=float, default=2.0, help="serving: batching window")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="serving: Poisson arrival rate (queries/s)")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="serving: length of the arrival stream")
    ap.add_argument("--low-rate", type=float, default=20.0, help="serving: rate of the plain-path comparison")
    ap.add_argument("--low-n", type=int, default=48, help="serving: requests of the plain-path comparison")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.profile_batches:
        return profile_arm(args)
    if args.ingest_only:
        return ingest_arm(args)
    if args.ops_only:
        return ops_arm(args)
    if args.configs_only:
        return configs_arm(args)
    if args.ref_scaling:
        return ref_scaling_arm(args)
    if args.program:
        return program_arm(args)
    if args.programs_fused:
        return programs_fused_arm(args)
    if args.shard and args.impl != "reference":
        return shard_arm(args)
    return reference_arm(args) if args.impl == "reference" else gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
