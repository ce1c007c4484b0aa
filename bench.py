"""Benchmark: the plain one-plan execute() of the 4M x 64M equi-join.

Workload (one "step" = one execute of this plan):
  build  4,000,000 unique shuffled INT32 keys + INT64 payload
  probe  64,000,000 rows: INT32 foreign key Zipf(0.8) over the build keys,
         30% outside the build domain, 2% NULL; + FP64 payload
  output build key, build payload, probe key, probe payload
         (2 INT32 + INT64 + FP64), ~43.5M rows, paged
Seeded synthetic tables with these shapes stand in for the reference's JOB /
IMDB data (not available offline).

metric  probe rows/s of the whole job (all ranks).
value   inputs' pages resident in HBM when the timed region starts; each
        step decodes, builds, probes and writes the result pages in HBM.
        Device time of K steps from CUDA events on the library's stream,
        max over ranks. The inputs (~1.1 GB of pages) are larger than L2,
        so L2 is not flushed between steps.
e2e     the same plan through cj_execute with HOST page-locked input pages
        and a host result: page upload and result download inside the timed
        region; wall clock per step.
roofline dominant kernel's algorithmic bytes per launch / its mean
        event-timed duration, against the measured HBM copy bandwidth.
cpu_baseline the reference's own execute() (oracle/_ref, all host threads)
        on the same shape with INT32 payload stand-ins (the reference cannot
        emit INT64 / FP64 columns), rank 0 at N=1 only.

--impl reference runs only that CPU reference (rank 0; other ranks exit).
Multi-GPU (torchrun): independent replicas, one per GPU, no collective on
the data path ("scaling": "weak").

Other workloads (not the default line; --workload):
  c1  100K x 1M join (INT32 build payload, INT64 probe payload), same
      measurements as the default line.
  c2s C2 with the build keys spread 500x (unique multiples of 500): the
      open-addressing table instead of the direct-mapped one.
  c2h C2 with a non-unique build side (4M rows over 3M distinct keys): the
      unchained hash table; roofline of the hash path's kernels.
  c3  6-way left-deep join: a 36M-row fact table with 5 foreign keys into
      dimensions of 2.5K-4.2M rows (pre-filtered to 10-40 %), VARCHAR
      outputs (lengths log-normal, mean 20 B, 0.01 % long strings);
      metric fact rows/s.
  c4  256 seeded 2-4-way INT32 plans (builds log-uniform 10-1e6, probes
      1e3-1e7): plans/s through cj_execute_batch, beside a loop of
      cj_execute over the same plans and the reference's execute() on
      the host cores; host pages in, host pages out.
  c5  Poisson arrivals at several rates over a pool of 32 2-16-way plans
      (probes 1e4-1e7 rows) with INT32 / INT64 keys and 10 % VARCHAR
      outputs, over base tables resident in HBM (results to the host),
      served two ways over the same trace: the server
      (cj_server_*, 4 worker streams, 150 GB admission budget, continuous
      batching; a client thread takes and frees each result as it
      completes) and plain cj_execute one plan at a time in arrival order:
      p50 / p99 latency and plans/s per rate and arm.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "probe rows/s, 4M x 64M INT32 equi-join (plain execute)"
UNIT = "rows/s"
WORKLOAD = ("C2: build 4,000,000 unique shuffled INT32 keys + INT64 payload; probe 64,000,000 rows, "
            "INT32 FK Zipf(0.8) over build keys, 30% outside the build domain, 2% NULL, + FP64 payload; "
            "output build key, build INT64, probe key, probe FP64 (2 INT32 + INT64 + FP64)")
WORKLOADS = {
    "c2": {"metric": METRIC, "unit": UNIT, "desc": WORKLOAD, "units": "probe rows"},
    "c1": {"metric": "probe rows/s, 100K x 1M INT32 equi-join (plain execute)", "unit": UNIT,
           "desc": ("C1: build 100,000 unique shuffled INT32 keys + INT32 payload; probe 1,000,000 rows, INT32 FK "
                    "Zipf(1.0), 5% NULL, + INT64 payload; output build key, build payload, probe payload"),
           "units": "probe rows"},
    "c2s": {"metric": "probe rows/s, 4M x 64M INT32 equi-join, build keys spread 500x (plain execute)",
            "unit": UNIT,
            "desc": ("C2 with the 4,000,000 unique build keys spread over multiples of 500 below 2^31 (too wide "
                     "for a direct-mapped table: open-addressing table); probe and outputs as C2"),
            "units": "probe rows"},
    "c2h": {"metric": "probe rows/s, 4M x 64M INT32 equi-join, non-unique build keys (plain execute)",
            "unit": UNIT,
            "desc": ("C2 with a non-unique build side: 4,000,000 build rows over 3,000,000 distinct INT32 keys (a "
                     "third twice) + INT64 payload; probe 64,000,000 rows, FK Zipf(0.8) over the distinct keys, "
                     "30% outside, 2% NULL, + FP64 payload; the unchained hash table (radix-partitioned build, "
                     "Bloom-tag probe); about 58.5M output rows"),
            "units": "probe rows"},
    "c3": {"metric": "fact rows/s, 6-way join of a 36M-row fact table (plain execute)", "unit": UNIT,
           "desc": ("C3: fact 36,000,000 rows x 5 INT32 FKs (Zipf 0.5-1.2) into dimensions of 2,500 / 130,000 / "
                    "1,200,000 / 2,500,000 / 4,200,000 rows kept at 40/40/30/20/10 %; outputs the fact's first FK, "
                    "a fact VARCHAR and every dimension's VARCHAR (log-normal lengths, 0.01 % long strings)"),
           "units": "fact rows"},
}
C4_PLANS, C4_SEED = 256, 404
C5_RATES = (50, 200, 1000, 2000)
for _k, _v in WORKLOADS.items():
    _v["name"] = _k
WL = WORKLOADS["c2"]


def rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """One process per GPU (torchrun): each rank runs its own replica of the
    workload; the only collectives are the barriers around a timed region and
    the maximum over ranks of each measured time (no collective on the data
    path). With one rank every call is a no-op."""

    def __init__(self, backend: str = "nccl", device: str = "cpu", timeout_s: int = 120):
        self.rank, self.world, self.local = rank_info()
        self.device = device
        self.dist = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """The largest `x` over the ranks (every rank gets it)."""
        if not self.dist:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None


def whole_job_rate(units_per_rank: int, world: int, seconds_max: float) -> float:
    """Units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / seconds_max


class ClockSampler:
    """SM clock and clock-event-reason samples during the timed region.

    NVML is initialised in-process before the warm-up (start()), and a thread
    polls it every 5 ms; mark() brackets the timed region so only samples
    taken inside it count. Spawning nvidia-smi at the start of the timed
    region stalled CUDA host calls for tens of ms while it initialised, so
    the nvidia-smi line (same fields) is only the fallback when NVML is not
    importable, and it is started before the warm-up as well."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []  # (time, sm_mhz, max_mhz, set of reasons)
        self.proc = None
        self.stop_flag = threading.Event()
        self.thread = None
        self.source = None
        self.t0 = self.t1 = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.gpu)
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(props.uuid))
        except Exception:
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def poll():
                while not self.stop_flag.is_set():
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.rows.append((time.perf_counter(), float(sm), float(mx),
                                      {n for n, b in self.REASONS if bits & b}))
                    self.stop_flag.wait(0.005)
            self.source = "nvml"
        except Exception:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)

            def poll():
                names = [n for n, _ in self.REASONS]
                for line in self.proc.stdout:
                    r = [x.strip() for x in line.split(",")]
                    try:
                        self.rows.append((time.perf_counter(), float(r[1]), float(r[2]),
                                          {n for k, n in enumerate(names) if r[5 + k].lower() == "active"}))
                    except (ValueError, IndexError):
                        pass
            self.source = "nvidia-smi"
        self.thread = threading.Thread(target=poll, daemon=True)
        self.thread.start()
        deadline = time.time() + 10
        while not self.rows and time.time() < deadline:
            time.sleep(0.01)
        return self

    def mark(self, begin: bool):
        if begin:
            self.t0 = time.perf_counter()
        else:
            self.t1 = time.perf_counter()

    def stop(self):
        self.stop_flag.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        t0, t1 = self.t0 or 0.0, self.t1 or float("inf")
        inside = [r for r in self.rows if t0 <= r[0] <= t1]
        rows = inside
        if not rows and self.rows:  # region shorter than one poll: the samples either side
            before = [r for r in self.rows if r[0] < t0][-1:]
            after = [r for r in self.rows if r[0] > t1][:1]
            rows = before + after
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        reasons = set()
        for r in rows:
            reasons |= r[3]
        return {"sm_mhz": statistics.median(r[1] for r in rows), "sm_max_mhz": max(r[2] for r in rows),
                "reasons": sorted(reasons), "samples": len(inside), "source": self.source}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_table(workload: str):
    """Per-launch DRAM traffic of this workload's kernels, from the committed
    ncu summaries (keyed by workload, then by kernel)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(workload, {})
    except Exception:
        return {}


def algorithmic_bytes(kernel: str, st: dict, plan_info: dict):
    """Algorithmic HBM bytes of ONE launch of `kernel` in this workload
    (two-table workloads; None for the multi-join C3)."""
    if WL["name"] == "c3":
        return None
    nb, npr = plan_info["build_rows"], plan_info["probe_rows"]
    m = st["matches"]
    slots = plan_info["slots"]
    if kernel == "probe_hash":
        # probe keys (4 B + 1 validity bit per row), one pass over the hash
        # table (8 B tuples + 16 B directory entries for INT32 keys), per
        # match 2 x 4 B row ids and the 4 B key the probe emits for the
        # root's key columns
        return npr * (4 + 1 / 8) + nb * 8 + slots * 16 + m * 12
    if kernel == "probe_array":
        if not st.get("num_direct_joins"):
            return None  # the launch found the table unusable and returned at once
        # probe keys (4 B + validity bit), the direct-mapped table (4 B per
        # slot; the C2 build keys are a permutation of [0, rows), so slots =
        # build rows) once; per match 2 x 4 B row ids and the 4 B key the
        # probe emits for the root's key columns
        return npr * (4 + 1 / 8) + nb * 4 + m * 12
    if kernel == "probe_open":
        # probe keys (4 B + validity bit), the open-addressing table (8 B
        # slots, 2 per build row) once; per match 2 x 4 B row ids and the
        # 4 B key the probe emits for the root's key columns
        return npr * (4 + 1 / 8) + nb * 2 * 8 + m * 12
    if kernel == "write_pages_int32":
        # per output row: 4 B match row id + 4 B value + validity bit read; page bytes written
        pages = (m + 1983) // 1984
        return m * (4 + 4 + 1 / 8) + pages * 8192
    if kernel == "write_pages_8byte":
        pages = (m + 1006) // 1007
        return m * (4 + 8 + 1 / 8) + pages * 8192
    if kernel == "decode_int32":
        return plan_info["int32_pages"] * 8192 / plan_info["int32_cols"] + 0  # per launch: one column
    if kernel == "build":
        # keys read twice (histogram, scatter: 4 B + validity bit), tuples
        # written once by the scatter, read twice and written once by the
        # per-partition build; 16 B directory entries
        return nb * (2 * (4 + 1 / 8) + 8 + 16 + 8) + slots * 16
    return None


def gen_workload(pinned: bool, scale: float, int32_standin: bool = False, workload: str = None):
    from calamarijoins_b200.datagen import config_c1, config_c2, config_c3, join2
    from calamarijoins_b200 import DataType
    workload = workload or WL["name"]
    if workload == "c1":
        if int32_standin:
            return join2(max(int(100_000 * scale), 16), max(int(1_000_000 * scale), 16), seed=101, zipf=1.0,
                         probe_null=0.05, build_payload=(DataType.INT32,), probe_payload=(DataType.INT32,),
                         output=[0, 1, 3], pinned=pinned)
        return config_c1(scale=scale, pinned=pinned)
    if workload == "c3":  # INT32 keys, VARCHAR without NULLs: the reference runs it as it is
        return config_c3(scale=scale, pinned=pinned)
    if workload == "c2s":
        from calamarijoins_b200.datagen import config_c2s
        return config_c2s(scale=scale, pinned=pinned, int32_standin=int32_standin)
    if workload == "c2h":
        from calamarijoins_b200.datagen import config_c2h
        return config_c2h(scale=scale, pinned=pinned, int32_standin=int32_standin)
    if int32_standin:
        return join2(max(int(4_000_000 * scale), 16), max(int(64_000_000 * scale), 16), seed=202, zipf=0.8,
                     outside=0.30, probe_null=0.02, build_payload=(DataType.INT32,),
                     probe_payload=(DataType.INT32,), output=[0, 1, 2, 3], pinned=pinned)
    return config_c2(seed=202, scale=scale, pinned=pinned)


def work_units(plan) -> int:
    """Rows the metric counts: the probe side of the 2-table workloads, the
    fact table of C3."""
    return plan.inputs[0].num_rows if WL["name"] == "c3" else plan.inputs[1].num_rows


def plan_info(plan):
    import math
    nb = plan.inputs[0].num_rows
    npr = work_units(plan)
    i32 = [c for t in plan.inputs for c in t.columns if int(c.type) == 0]
    return {"build_rows": nb, "probe_rows": npr, "slots": 1 << max(11, math.ceil(math.log2(max(nb, 1)))),
            "int32_pages": sum(c.num_pages for c in i32), "int32_cols": max(len(i32), 1)}


def ref_threads():
    from oracle import oracle_api as oa
    avail = oa.ref_available()
    if not avail:
        return None, []
    n = os.cpu_count() or 1
    best = max([t for t in avail if t <= max(n, 8)] or [avail[0]])
    cands = sorted(set([best] + ([32] if 32 in avail else [])))
    return best, cands


def log(msg: str) -> None:
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def ref_worker(threads: int, scale: float, warmup: int, steps: int) -> None:
    """Child process: times one reference variant (one variant per process:
    every variant carries its own worker-pool singleton)."""
    from calamarijoins_b200 import PlanDescriptor
    from oracle import oracle_api as oa
    if WL["name"] == "c4":  # one pass = every plan of the batch, one after another
        from calamarijoins_b200.datagen import batch_plans
        descs = [PlanDescriptor(p) for p in batch_plans(C4_PLANS, seed=C4_SEED, scale=scale)]
        ms = []
        for i in range(max(warmup, 1) + steps):
            t0 = time.perf_counter()
            for d in descs:
                oa.ref_execute(d, threads)
            if i >= max(warmup, 1):
                ms.append((time.perf_counter() - t0) * 1e3)
        print(json.dumps({"threads": threads, "ms": statistics.median(ms), "probe_rows": len(descs), "build_rows": 0}))
        return
    plan = gen_workload(False, scale, int32_standin=True)
    d = PlanDescriptor(plan)
    units = work_units(plan)
    for _ in range(max(warmup, 1)):
        oa.ref_execute(d, threads)
    ms = []
    for _ in range(steps):
        _, w, _ = oa.ref_execute(d, threads)
        ms.append(w)
    print(json.dumps({"threads": threads, "ms": statistics.median(ms), "probe_rows": units,
                      "build_rows": plan.inputs[0].num_rows}))


def time_reference(scale: float, warmup: int, steps: int, timeout_s: float = 900):
    """Times oracle/_ref (the reference's execute()) on the host cores, each
    thread-count candidate in its own process."""
    best, cands = ref_threads()
    if best is None:
        return None
    results = {}
    info = {}
    for t in cands:
        log(f"reference: {t} threads, scale {scale}")
        res = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-worker", str(t), "--scale", str(scale),
                              "--warmup", str(warmup), "--steps", str(steps), "--workload", WL["name"]],
                             capture_output=True, text=True, timeout=timeout_s)
        if res.returncode != 0:
            log(f"reference variant {t} failed: {res.stderr[-500:]}")
            continue
        r = json.loads(res.stdout.strip().splitlines()[-1])
        results[t] = r["ms"]
        info = r
    if not results:
        return None
    t_best = min(results, key=results.get)
    return {"threads": t_best, "ms": results[t_best], "all_ms": results, "probe_rows": info["probe_rows"],
            "build_rows": info["build_rows"]}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    scale = args.scale
    r = time_reference(scale, args.warmup, args.steps)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference not compiled into oracle/_ref"}))
        return 0
    npr = r["probe_rows"]
    val = npr / (r["ms"] / 1000.0)
    sample = (f"{WL['name'].upper()} shape at scale {scale}: {r['build_rows']} x {npr} rows, INT32 stand-ins for "
              f"any INT64/FP64 payloads (the reference cannot emit them); median of {args.steps} runs after "
              f"{max(args.warmup, 1)} warm-up; best of thread counts {sorted(r['all_ms'])} on {os.cpu_count()} CPUs")
    line = {"impl": "reference", "metric": WL["metric"], "value": val, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": WL["desc"] + " [reference: INT32 stand-in payloads]", "parallelism": "cpu threads"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": r["threads"], "kind": "reference",
                             "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def check_parity(plan, resident, ctx, d_res):
    """Checker, outside every timed region: the row-multiset fingerprint of
    one device result of the benchmarked plan (copied back) against the
    fingerprint of the oracle's result for the same host pages."""
    import calamarijoins_b200 as cj
    from calamarijoins_b200 import _lib
    from oracle import oracle_api as oa
    res, _ = cj.execute_raw(resident, ctx, _lib.CJ_EXEC_RESULT_ON_DEVICE, d_res)
    try:
        got = oa.PagedResult.from_result(res)
    finally:
        res.free()
    ok_pages, msg = oa.validate(got)
    fp_gpu = oa.fingerprint(got)
    rows_gpu = got.num_rows
    del got
    t0 = time.perf_counter()
    want = oa.oracle_execute(cj.PlanDescriptor(plan))
    oracle_s = time.perf_counter() - t0
    fp_oracle = oa.fingerprint(want)
    return {"equal": bool(ok_pages and fp_gpu == fp_oracle and rows_gpu == want.num_rows),
            "pages_valid": bool(ok_pages), "page_error": msg or None,
            "rows": rows_gpu, "oracle_rows": want.num_rows,
            "fingerprint": f"{fp_gpu:016x}", "oracle_fingerprint": f"{fp_oracle:016x}",
            "method": ("order-insensitive fingerprint of the row multiset (values, NULLs, bytes) of one "
                       "device-resident execution against the oracle's (oracle/cj_oracle.c) on the same pages; "
                       f"oracle {oracle_s:.1f} s single-threaded")}


def run_ours(args):
    import ctypes as C
    import numpy as np
    import torch
    import calamarijoins_b200 as cj
    from calamarijoins_b200 import _lib

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    reps = Replicas("nccl", device=f"cuda:{local}")

    ctx = cj.Context(local)
    tuning = None
    if not args.no_tune:
        log("autotuning the hash build and probe")
        t0 = time.perf_counter()
        ctx.autotune()
        tuning = {"classes": ctx.tuning(), "seconds": round(time.perf_counter() - t0, 2),
                  "entry": "(log2 slots per radix partition, radix-pass CTAs/SM, probe CTAs/SM) per size class"}
    log("generating workload")
    plan = gen_workload(True, args.scale)
    log("uploading resident tables")
    info = plan_info(plan)
    resident = cj.Plan()
    resident.nodes, resident.root = plan.nodes, plan.root
    resident.inputs = [cj.ResidentTable(ctx, t) for t in plan.inputs]
    d_res = cj.PlanDescriptor(resident)
    d_host = cj.PlanDescriptor(plan)
    sp = C.c_void_p()
    _lib.check(_lib.lib().cj_context_stream(ctx.handle, C.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", local))

    def step_device():
        res, st = cj.execute_raw(resident, ctx, _lib.CJ_EXEC_RESULT_ON_DEVICE, d_res)
        res.free()
        return st

    # The workload generator leaves millions of Python objects behind; a
    # cyclic-GC pass over them in the middle of a step stalls the host for
    # tens of ms. Collect once and freeze them out of later passes.
    gc.collect()
    gc.freeze()
    clk = ClockSampler(local).start()
    log(f"clock sampler: {clk.source}")
    log("warm-up")
    for _ in range(args.warmup):
        st = step_device()
    log("timed device steps")
    reps.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches = 0
    clk.mark(True)
    ev[0].record(stream)
    for i in range(args.steps):
        st = step_device()
        launches += st.exec["kernel_launches"]
        ev[i + 1].record(stream)
    torch.cuda.synchronize()
    clk.mark(False)
    clk.stop()
    ms_total = ev[0].elapsed_time(ev[-1])
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    ms_total = reps.max(ms_total)
    reps.barrier()
    # per-kernel times (CUDA events around every launch) from a separate
    # pass over the same steps, so the headline steps carry no event records
    ctx.set_option(_lib.CJ_OPT_PROFILE_KERNELS, 1)
    step_device()
    ctx.profile_reset()
    for _ in range(args.steps):
        step_device()
    prof = ctx.profile()
    ctx.set_option(_lib.CJ_OPT_PROFILE_KERNELS, 0)
    ms_step = ms_total / args.steps
    value = whole_job_rate(info["probe_rows"], world, ms_step / 1000.0)

    # e2e through the public API with host buffers
    log("end-to-end steps")
    for _ in range(max(1, args.warmup)):
        res, st_h = cj.execute_raw(plan, ctx, 0, d_host)
        res.free()
    reps.barrier()
    walls = []
    h2d = d2h = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        res, st_h = cj.execute_raw(plan, ctx, 0, d_host)
        walls.append(time.perf_counter() - t0)
        res.free()
        h2d, d2h = st_h.exec["h2d_bytes"], st_h.exec["d2h_bytes"]
    e2e_s = statistics.mean(walls)
    e2e_steps = {"min": min(walls) * 1e3, "median": statistics.median(walls) * 1e3, "max": max(walls) * 1e3}
    e2e_s = reps.max(e2e_s)
    e2e_value = whole_job_rate(info["probe_rows"], world, e2e_s)

    parity = None
    if rank == 0 and not args.no_parity:
        log("parity: result fingerprint against the oracle's")
        parity = check_parity(plan, resident, ctx, d_res)
    log("cpu baseline")
    # roofline of the dominant kernel
    peak, peak_kind = measured_peaks()
    dom = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    roof = None
    if dom:
        name, (nl, tot_us) = dom
        avg_us = tot_us / max(nl, 1)
        ab = algorithmic_bytes(name, st.exec, info)
        tr = traffic_table(WL["name"]).get(name)
        achieved = (ab / (avg_us * 1e-6) / 1e9) if ab else None
        roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": (tr.get("bytes_per_launch") if tr else None), "peak_source": peak_kind,
                "launches_timed": nl, "avg_launch_us": avg_us, "algorithmic_bytes_per_launch": ab}

    kernels = {}
    total_prof = max(sum(x[1] for x in prof.values()), 1e-9)
    for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1]):
        e = {"launches": v[0], "total_us": v[1], "share": v[1] / total_prof}
        ab = algorithmic_bytes(k, st.exec, info)
        if ab:
            gbs = ab / (v[1] / max(v[0], 1) * 1e-6) / 1e9
            e.update({"algorithmic_bytes_per_launch": ab, "achieved_gbs": gbs, "frac_of_peak": gbs / peak})
        kernels[k] = e

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = time_reference(args.cpu_scale, 1, 3)
        if r is not None:
            snp = r["probe_rows"]
            cpu = {"value": snp / (r["ms"] / 1000.0), "unit": UNIT, "cores": r["threads"], "kind": "reference",
                   "sample": (f"reference execute() (oracle/_ref) on the {WL['name'].upper()} shape at scale "
                              f"{args.cpu_scale} "
                              f"({r['build_rows']} x {snp} rows) with INT32 stand-ins for the INT64/FP64 payloads; "
                              f"median of 3 runs after 1 warm-up; {r['threads']} threads (of {sorted(r['all_ms'])} "
                              f"tried) on {os.cpu_count()} host CPUs")}
    if rank == 0:
        line = {"metric": WL["metric"], "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "step_ms": {"min": min(step_ms), "median": statistics.median(step_ms), "max": max(step_ms)},
                "config": {"workload": WL["desc"], "scale": args.scale,
                           "inputs": "paged columns resident in HBM (device-resident cj_table)",
                           "l2": "inputs larger than L2 (1.1 GB of pages); no flush",
                           "parallelism": f"replicas x{world}",
                           "output_rows": st.exec["output_rows"], "output_pages": st.exec["output_pages"],
                           "tuning": tuning},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": e2e_s * 1000.0, "step_ms": e2e_steps},
                "roofline": roof, "cpu_baseline": cpu, "gpu_launches": launches, "parity": parity,
                "clocks": clk.summary(), "kernels": kernels,
                "phases_us": {k: st.exec[k] for k in ("decode_us", "build_us", "probe_us", "materialize_us")}}
        print(json.dumps(line))
    for t in resident.inputs:
        t.free()
    ctx.close()
    reps.close()
    return 0


def run_batch(args):
    """c4: plans/s of 256 plans, batched (cj_execute_batch) and looped
    (cj_execute), twice: with the inputs' pages resident in HBM and results
    left on the device, and with host pages in and host pages out; the
    reference's execute() over the same plans on the host cores."""
    import calamarijoins_b200 as cj
    from calamarijoins_b200 import _lib
    from calamarijoins_b200.datagen import batch_plans
    ctx = cj.Context(0)
    log("generating 256 plans")
    plans = batch_plans(C4_PLANS, seed=C4_SEED, scale=args.scale, pinned=True)
    descs = [cj.PlanDescriptor(p) for p in plans]
    rows = sum(p.inputs[0].num_rows for p in plans)
    log("uploading resident tables")
    rplans, tables = [], []
    for p in plans:
        rp = cj.Plan()
        rp.nodes, rp.root = p.nodes, p.root
        rp.inputs = [cj.ResidentTable(ctx, t) for t in p.inputs]
        tables.extend(rp.inputs)
        rplans.append(rp)
    rdescs = [cj.PlanDescriptor(p) for p in rplans]
    gc.collect()
    gc.freeze()

    def batched(ps, ds, flags):
        def fn():
            results, statuses, st = cj.execute_batch(ps, ctx, flags, descs=ds)
            assert all(x == 0 for x in statuses), statuses
            for r in results:
                r.free()
            return st
        return fn

    def looped(ps, ds, flags):
        def fn():
            for p, d in zip(ps, ds):
                r, _ = cj.execute_raw(p, ctx, flags, d)
                r.free()
        return fn

    dev = _lib.CJ_EXEC_RESULT_ON_DEVICE
    log("preparing the resident batch as one CUDA graph")
    t0 = time.perf_counter()
    prep = cj.PreparedBatch(rplans, ctx, dev, descs=rdescs)
    prepare_ms = (time.perf_counter() - t0) * 1e3

    def replay():
        results, st = prep.run()
        for r in results:
            r.free()
        return st

    arms = {"resident": {"graph": replay, "batched": batched(rplans, rdescs, dev),
                         "looped": looped(rplans, rdescs, dev)},
            "host": {"batched": batched(plans, descs, 0), "looped": looped(plans, descs, 0)}}
    out = {}
    for where, fns in arms.items():
        out[where] = {}
        for name, fn in fns.items():
            log(f"{where} {name}: warm-up")
            for _ in range(args.warmup):
                fn()
            walls = []
            for _ in range(args.steps):
                t0 = time.perf_counter()
                fn()
                walls.append(time.perf_counter() - t0)
            out[where][name] = {"plans_per_s": C4_PLANS / statistics.mean(walls),
                                "ms_per_pass": statistics.mean(walls) * 1e3,
                                "pass_ms": {"min": min(walls) * 1e3, "median": statistics.median(walls) * 1e3,
                                            "max": max(walls) * 1e3}}
        out[where]["batched_over_looped"] = out[where]["batched"]["plans_per_s"] / out[where]["looped"]["plans_per_s"]
    out["resident"]["graph_over_looped"] = out["resident"]["graph"]["plans_per_s"] / out["resident"]["looped"]["plans_per_s"]
    out["resident"]["graph"]["prepare_ms"] = prepare_ms
    st = arms["resident"]["batched"]()
    gst = replay()
    prep.close()
    ref = None
    if not args.no_cpu_baseline:
        r = time_reference(args.scale, 1, 3)
        if r is not None:
            ref = {"value": C4_PLANS / (r["ms"] / 1000.0), "unit": "plans/s", "cores": r["threads"],
                   "kind": "reference", "sample": (f"the reference's execute() over the same {C4_PLANS} plans one "
                                                   f"after another, median of 3 passes after 1 warm-up; best of "
                                                   f"thread counts {sorted(r['all_ms'])} on {os.cpu_count()} CPUs")}
    line = {"metric": "plans/s, 256 batched 2-4-way INT32 plans", "value": out["resident"]["graph"]["plans_per_s"],
            "unit": "plans/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out["resident"]["graph"]["ms_per_pass"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": ("C4: 256 seeded 2-4-way INT32 chain plans, builds log-uniform 10-1e6 rows, "
                                    "probes 1e3-1e7 rows; value: inputs resident in HBM, results on the device, "
                                    "the batch replayed as one captured CUDA graph (cj_batch_run)"),
                       "scale": args.scale, "fact_rows_total": rows},
            "resident": out["resident"], "host": out["host"],
            "e2e": {"value": out["host"]["batched"]["plans_per_s"], "unit": "plans/s",
                    "note": "host pages in, host pages out, through cj_execute_batch"},
            "batch_stats": {k: st[k] for k in ("num_levels", "num_joins", "kernel_launches", "syncs")},
            "graph_stats": {k: gst[k] for k in ("num_levels", "num_joins", "kernel_launches", "syncs")},
            "cpu_baseline": ref}
    print(json.dumps(line))
    for t in tables:
        t.free()
    ctx.close()
    return 0


def run_serve(args):
    """c5: Poisson arrivals over a pool of plans, at several rates, served
    two ways over the same arrival trace: the server (cj_server_*: worker
    streams, admission by estimated bytes, continuous batching), and the
    plain one-plan-at-a-time cj_execute in arrival order on one context
    (a plan waits for the one before it). Latency = completion - arrival;
    p50 / p99 and plans/s per rate and arm."""
    import queue
    import numpy as np
    import calamarijoins_b200 as cj
    from calamarijoins_b200 import DataType
    from calamarijoins_b200.datagen import chain_plan
    rng = np.random.default_rng(505)
    log("generating the plan pool")
    pool = []
    for i in range(32):
        ways = int(rng.integers(2, 17))
        nprobe = int(10 ** rng.uniform(4, 4 + 3 * max(min(args.scale, 1.0), 0.01) ** 0.25))
        pool.append(chain_plan(ways, nprobe, rng, max_build=max(int(1_000_000 * args.scale), 1000),
                               key_types=[DataType.INT32 if rng.random() < 0.7 else DataType.INT64
                                          for _ in range(ways - 1)],
                               varchar_frac=0.1, pinned=True))
    probe_rows = [p.inputs[0].num_rows for p in pool]
    # the pool's base tables live in HBM, as a serving system keeps them;
    # each request is a plan over them, its result goes to the host
    ctx = cj.Context(0)
    log("uploading the pool's tables")
    tables = []
    rpool = []
    for p in pool:
        rp = cj.Plan()
        rp.nodes, rp.root = p.nodes, p.root
        rp.inputs = [cj.ResidentTable(ctx, t) for t in p.inputs]
        tables.extend(rp.inputs)
        rpool.append(rp)
    pool = rpool
    descs = [cj.PlanDescriptor(p) for p in pool]
    gc.collect()
    gc.freeze()

    def pct(xs, q):
        xs = sorted(xs)
        return xs[min(len(xs) - 1, int(q * (len(xs) - 1) + 0.5))]

    def trace(lam):
        n = int(min(max(lam * 4, 100), 2000))
        return np.cumsum(rng.exponential(1.0 / lam, n)), rng.integers(0, len(descs), n)

    def served(srv, arrivals, order):
        q = queue.Queue()

        def consume():
            while True:
                t = q.get()
                if t is None:
                    return
                r, _ = srv.wait(t)
                r.free()
        th = threading.Thread(target=consume)
        th.start()
        t0 = time.perf_counter()
        for at, k in zip(arrivals, order):
            d = at - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            q.put(srv.submit(descs[k]))
        q.put(None)
        th.join()
        st = srv.stats(reset=True)
        return {"plans_per_s": st["plans_per_s"], "p50_ms": st["p50_us"] / 1e3, "p99_ms": st["p99_us"] / 1e3,
                "mean_ms": st["mean_us"] / 1e3, "max_ms": st["max_us"] / 1e3, "failed": st["failed"],
                "rejected": st["rejected"], "peak_admitted_gb": st["peak_admitted_bytes"] / 1e9,
                "batches": st["batches"], "mean_batch": st["mean_batch"], "skipped_ahead": st["skipped_ahead"],
                "batch_fallbacks": st["batch_fallbacks"], "pinned_allocs": st["pinned_allocs"],
                "pinned_alloc_mb": st["pinned_alloc_bytes"] / 1e6, "pool_high_gb": st["pool_high_bytes"] / 1e9}

    # device time of one execution: the sum of its phases' event intervals
    # on the kernel stream (an upper bound of the GPU's busy time for it)
    DEVICE_PHASES = ("decode_us", "build_us", "probe_us", "nested_loop_us", "intermediate_us", "materialize_us")

    def plain(ctx, arrivals, order, flags):
        lat = []
        dev_us = []
        t0 = time.perf_counter()
        last = t0
        for at, k in zip(arrivals, order):
            d = at - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            r, st_p = cj.execute_raw(pool[k], ctx, flags, descs[k])
            r.free()
            last = time.perf_counter()
            lat.append((last - t0) - at)
            dev_us.append(sum(st_p.exec[n] for n in DEVICE_PHASES))
        wall = last - (t0 + arrivals[0])
        dev_ms = statistics.mean(dev_us) / 1e3
        return {"plans_per_s": len(lat) / wall, "p50_ms": pct(lat, 0.5) * 1e3, "p99_ms": pct(lat, 0.99) * 1e3,
                "mean_ms": statistics.mean(lat) * 1e3, "max_ms": max(lat) * 1e3,
                "device_ms_per_plan": dev_ms, "device_bound_plans_per_s": 1e3 / dev_ms if dev_ms else None}

    from calamarijoins_b200 import _lib
    modes = {"host": 0, "device": _lib.CJ_EXEC_RESULT_ON_DEVICE}
    per_mode = {}
    result_bytes = []
    try:
        for mode, flags in modes.items():
            srv = cj.Server(device=0, slots=args.c5_slots, memory_budget=150 << 30, flags=flags,
                            max_batch=args.c5_max_batch,
                            host_cache_bytes=(8 << 30) if mode == "host" else 0, device_reserve_bytes=100 << 30)
            try:
                log(f"{mode} results: warm-up")
                for _ in range(2):  # every worker sees plans of every size: pinned and pool blocks exist
                    ts = [srv.submit(d) for d in descs for _ in range(2)]  # grouped executions
                    for t in ts:
                        r, _ = srv.wait(t)
                        r.free()
                    for d in descs:  # one plan at a time
                        r, _ = srv.wait(srv.submit(d))
                        r.free()
                srv.stats(reset=True)
                for i, (p, d) in enumerate(zip(pool, descs)):
                    r, _ = cj.execute_raw(p, ctx, flags, d)
                    if mode == "host":
                        result_bytes.append(sum(r.column_info(c)[1] for c in range(r.num_columns)) * 8192)
                    r.free()
                per_rate = []
                for lam in C5_RATES:
                    arrivals, order = trace(lam)
                    log(f"{mode} results, rate {lam}/s: {len(order)} plans, served")
                    sv = served(srv, arrivals, order)
                    log(f"{mode} results, rate {lam}/s: plain")
                    pl = plain(ctx, arrivals, order, flags)
                    per_rate.append({"rate": lam, "plans": len(order), "served": sv, "plain": pl,
                                     "served_over_plain": sv["plans_per_s"] / pl["plans_per_s"]})
                per_mode[mode] = per_rate
            finally:
                srv.close()
    finally:
        for t in tables:
            t.free()
        ctx.close()
    per_rate = per_mode["host"]
    mean_mb = statistics.mean(result_bytes) / 1e6
    best = max(per_rate, key=lambda x: x["served"]["plans_per_s"])
    plain_best = max(x["plain"]["plans_per_s"] for x in per_rate)

    def summary(rates):
        b = max(rates, key=lambda x: x["served"]["plans_per_s"])
        pb = max(x["plain"]["plans_per_s"] for x in rates)
        return {"served_best_plans_per_s": b["served"]["plans_per_s"], "plain_best_plans_per_s": pb,
                "served_over_plain_at_saturation": b["served"]["plans_per_s"] / pb}
    line = {"metric": "served plans/s (Poisson arrivals), p50 / p99 latency", "value": best["served"]["plans_per_s"],
            "unit": "plans/s", "n_gpus": 1, "steps": len(C5_RATES), "warmup": 1, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32/int64",
            "data": "synthetic",
            "config": {"workload": ("C5: pool of 32 seeded 2-16-way chain plans, 70 % INT32 / 30 % INT64 keys, "
                                    "10 % VARCHAR outputs, probes log-uniform 1e4-1e7 rows, dimensions 10-1e6 rows, "
                                    "base tables resident in HBM, results to host memory; Poisson arrivals, each "
                                    "plan drawn from the pool; served: "
                                    f"{args.c5_slots} worker streams, 150 GB admission budget, continuous batching "
                                    f"(at most {args.c5_max_batch} plans per grouped execution), 8 GB "
                                    "page-locked result cache and 100 GB of device pool reserved at creation; plain: "
                                    "cj_execute one plan at a time in arrival order"), "scale": args.scale,
                       "probe_rows": {"min": min(probe_rows), "max": max(probe_rows)}},
            "rates": per_rate,
            "plain_best_plans_per_s": plain_best,
            "served_over_plain_at_saturation": best["served"]["plans_per_s"] / plain_best,
            "result_mb_per_plan": mean_mb,
            "device_ms_per_plan": statistics.mean(x["plain"]["device_ms_per_plan"] for x in per_rate),
            "device_bound_plans_per_s": 1e3 / statistics.mean(x["plain"]["device_ms_per_plan"] for x in per_rate),
            "result_download_gbs_at_best": mean_mb * best["served"]["plans_per_s"] / 1e3,
            "device_results": {"rates": per_mode["device"], **summary(per_mode["device"]),
                               "note": "the same trace with results left in HBM (CJ_EXEC_RESULT_ON_DEVICE) in "
                                       "both arms: no result download"},
            "cpu_baseline": {"unavailable": "the reference joins INT32 keys only (30 % of the pool has INT64 keys) "
                                            "and has no serving front end"}}
    print(json.dumps(line))
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=float, default=1.0, help="row-count scale of the workload")
    ap.add_argument("--cpu-scale", type=float, default=1.0, help="scale of the CPU-baseline sample")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle fingerprint check")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (kernel defaults)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-worker", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--c5-slots", type=int, default=4, help="c5: the server's worker streams")
    ap.add_argument("--c5-max-batch", type=int, default=32, help="c5: plans per grouped execution, at most")
    ap.add_argument("--workload", choices=["c2", "c1", "c2s", "c2h", "c3", "c4", "c5"], default="c2",
                    help="c2 (default): the headline line; the others: see the module docstring")
    args = ap.parse_args(argv)
    global WL
    WL = WORKLOADS.get(args.workload, {"name": args.workload})
    if args.ref_worker:
        ref_worker(args.ref_worker, args.scale, args.warmup, args.steps)
        return 0
    import faulthandler
    faulthandler.dump_traceback_later(600, repeat=True, file=sys.stderr)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        if args.workload in ("c4", "c5"):
            print(json.dumps({"impl": "reference", "unavailable": "use --workload c2 (c4 and c5 report the "
                                                                   "reference inside their own line)"}))
            return 0
        return run_reference(args)
    if args.workload == "c4":
        return run_batch(args)
    if args.workload == "c5":
        return run_serve(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
