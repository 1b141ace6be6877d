"""Benchmark of the single-pass replace kernel on the 2 GiB / 1 GiB single-pair workload.

Workload (one "step"): three single-pair replaces, each one launch of the sm_100a kernel:
  (i)   2 GiB of b"a", b"aa" -> b"X"            (maximal self-overlap, 2**30 matches, shrink)
  (ii)  2 GiB of b"a", b"a" -> b"bcd"           (6 GiB output, 64-bit offsets, expand)
  (iii) 1 GiB i.i.d. uniform bytes, b"\\x00\\x00\\x01" -> b""  (embedded NULs, deletion)
Metric: GB/s of (input + output) bytes, 1 GB = 1e9 bytes.

value:  device-resident inputs (HBM), K steps timed with CUDA events on the launching
        stream; every input is larger than the 126 MB L2, so no flush is needed.
e2e:    the same step through the reference-facing C ABI call cuda_replace_unified with
        page-locked host inputs: H2D, kernel, D2H of the result inside the timed region.
cpu_baseline: CPython bytes.replace (single thread) on a bounded sample of the same cases.
batched: a sample of the 10,000-job workload through the request loop (segmented launches,
        CUDA graphs, HBM-budget admission): jobs/s closed loop and p50/p99 under Poisson
        arrivals, against the same jobs as per-job plain unified() calls (--no-batched skips).
--impl reference: the reference's CPU path (bytes.replace) alone, on all three cases.

Multi-GPU: the path does not shard across GPUs here (replicas only): under torchrun each
rank runs the same step on its own GPU, time = max over ranks, value = sum of bytes.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

GiB = 1 << 30
MiB = 1 << 20
SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
CASES = [("a-run aa->X", b"aa", b"X"), ("a-run a->bcd", b"a", b"bcd"), ("random 00 00 01->''", b"\x00\x00\x01", b"")]


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=float, default=1.0, help="input size multiplier (1.0 = full size)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cases", default="0,1,2", help="comma-separated subset of the three cases (profiling)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched/served jobs sample")
    ap.add_argument("--workload", choices=["single", "chain", "stream"], default="single",
                    help="single: the single-pair workload (default line); chain: 4 GiB text x 128 pairs "
                         "through apply_batch; stream: 16 GiB text x 8 pairs through gpu_replace_streaming")
    ap.add_argument("--gib", type=float, default=0.0, help="input GiB of the chain/stream workloads (0 = 4 / 16)")
    ap.add_argument("--jobs", type=int, default=500, help="jobs in the batched/served sample")
    ap.add_argument("--rates", default="0.25,0.5,0.75,0.9",
                    help="Poisson arrival rates of the served sample, as fractions of the closed-loop rate")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other workloads' figures (16 MiB one-shot, 4 GiB 128-pair chain, "
                         "16 GiB streaming, pageable-input unified)")
    return ap.parse_args(argv)


# ------------------------------------------------------------------ distributed plumbing
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend: str):
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float, device=None) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float, device=None) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def aggregate_replicas(bytes_per_rank: float, secs_per_rank: float, dist: Dist, device=None):
    """Replicas: total bytes over all ranks divided by the slowest rank's time."""
    total = dist.sum(bytes_per_rank, device)
    slowest = dist.max(secs_per_rank, device)
    return total, slowest


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={SMI_FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ inputs
def make_inputs(scale: float):
    import numpy as np

    from cuda_replace_b200 import workloads as WL
    n_run = int(2 * GiB * scale) // 16 * 16
    n_rand = int(1 * GiB * scale) // 16 * 16
    rand = np.random.default_rng(2).integers(0, 256, size=n_rand, dtype=np.uint8)
    return n_run, n_rand, rand, WL


def expected_lengths(n_run: int, rand_bytes: bytes):
    from oracle import oracle as O  # checker only
    n3, k3, _ = O.replace_len(rand_bytes, b"\x00\x00\x01", 0)
    return [(n_run // 2 + n_run % 2, n_run // 2), (3 * n_run, n_run), (n3, k3)]


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    p = REPO / "profiles" / "replace_super_c2_traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except json.JSONDecodeError:
            return None
    return None


# ------------------------------------------------------------------ CPU legs
def cpu_sample(rand_np, budget_scale: float = 1.0):
    """bytes.replace on a bounded sample of the three cases; returns (bytes, seconds, desc)."""
    sizes = [int(512 * MiB * budget_scale), int(256 * MiB * budget_scale), min(len(rand_np), int(GiB * budget_scale))]
    total_b, total_t = 0, 0.0
    srcs = [b"a" * sizes[0], b"a" * sizes[1], rand_np[:sizes[2]].tobytes()]
    for (name, pat, rep), src in zip(CASES, srcs):
        t0 = time.perf_counter()
        out = src.replace(pat, rep)
        dt = time.perf_counter() - t0
        total_b += len(src) + len(out)
        total_t += dt
        del out
    desc = (f"CPython bytes.replace, 1 thread: {sizes[0] >> 20} MiB a-run aa->X, {sizes[1] >> 20} MiB a-run a->bcd, "
            f"{sizes[2] >> 20} MiB random 00 00 01->'' (same generators as the GPU step)")
    return total_b, total_t, desc


def run_reference(args, dist: Dist):
    if dist.rank != 0:
        return 0
    import numpy as np
    rand = np.random.default_rng(2).integers(0, 256, size=int(GiB * min(args.scale, 1.0)), dtype=np.uint8)
    scale = 0.25 * min(args.scale, 1.0)
    for _ in range(args.warmup):
        cpu_sample(rand, scale)
    tb, tt = 0, 0.0
    desc = ""
    for _ in range(args.steps):
        b, t, desc = cpu_sample(rand, scale)
        tb += b
        tt += t
    value = tb / tt / 1e9
    line = {
        "impl": "reference", "metric": "GB/s (in+out), single-pair replace", "value": round(value, 4),
        "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(tt / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
        "config": {"workload": "2 GiB a-run aa->X + 2 GiB a-run a->bcd + 1 GiB random 00 00 01->'' "
                               "(each step a 1/4-size sample on the CPU)"},
        "cpu_baseline": {"value": round(value, 4), "unit": "GB/s", "cores": 1, "kind": "port",
                         "sample": desc + "; the reference's own CPU path (test/test.py:102-112)"},
        "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ main arm
def run_ours(args, dist: Dist):
    import numpy as np
    import torch

    from cuda_replace_b200 import build as B
    from cuda_replace_b200.cuda_replace_wrapper import CudaReplaceLib, Session

    torch.cuda.set_device(dist.local_rank)
    dev = torch.device("cuda", dist.local_rank)
    dist.init("nccl")
    lib = CudaReplaceLib(str(B.LIB_PATH))
    n_run, n_rand, rand_np, _ = make_inputs(args.scale)

    # device-resident inputs and outputs (pad 64 B: the kernel reads up to n rounded to 16)
    d_run = torch.full((n_run + 64,), ord("a"), dtype=torch.uint8, device=dev)
    d_rand = torch.empty(n_rand + 64, dtype=torch.uint8, device=dev)
    d_rand[:n_rand].copy_(torch.from_numpy(rand_np))
    outs = [torch.empty(n_run + 64, dtype=torch.uint8, device=dev),
            torch.empty(3 * n_run + 64, dtype=torch.uint8, device=dev),
            torch.empty(n_rand + 64, dtype=torch.uint8, device=dev)]
    caps = [n_run, 3 * n_run, n_rand]
    ins = [(d_run, n_run), (d_run, n_run), (d_rand, n_rand)]
    exp = expected_lengths(n_run, rand_np.tobytes()) if dist.rank == 0 else None
    sel = [int(c) for c in args.cases.split(",")]
    cases = [CASES[i] for i in sel]
    outs, caps, ins = [outs[i] for i in sel], [caps[i] for i in sel], [ins[i] for i in sel]
    if exp is not None:
        exp = [exp[i] for i in sel]
    stream = torch.cuda.Stream(device=dev)
    sessions = [Session(lib, b"") for _ in cases]

    def one_step(events=None):
        for i, ((name, pat, rep), (d_in, n), out, cap, s) in enumerate(zip(cases, ins, outs, caps, sessions)):
            if events is not None:
                events[i][0].record(stream)
            s.apply_device_async(d_in.data_ptr(), n, pat, rep, out.data_ptr(), cap, stream.cuda_stream)
            if events is not None:
                events[i][1].record(stream)

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 0)):
            one_step()
    torch.cuda.synchronize()
    # correctness of the warm-up outputs (lengths + kept counts) against the oracle
    results = [s.device_result() for s in sessions]
    if exp is not None:
        for (name, _, _), got, want in zip(cases, results, exp):
            if tuple(got) != tuple(want):
                raise SystemExit(f"bench self-check failed for {name}: got {got}, want {want}")
    bytes_per_step = sum(n + r[0] for (_, n), r in zip(ins, results))
    launches0 = sum(s.stats()[1] for s in sessions)

    per_launch = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in cases] for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(dist.local_rank)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    start.record(stream)
    for k in range(args.steps):
        one_step(per_launch[k])
    end.record(stream)
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    dist.barrier()
    secs = start.elapsed_time(end) / 1e3
    gpu_launches = sum(s.stats()[1] for s in sessions) - launches0
    total_bytes, slowest = aggregate_replicas(bytes_per_step * args.steps, secs, dist, dev)
    value = total_bytes / slowest / 1e9

    # roofline of the replace kernel: algorithmic (in+out) bytes / mean launch duration
    launch_ms = [[per_launch[k][i][0].elapsed_time(per_launch[k][i][1]) for k in range(args.steps)]
                 for i in range(len(cases))]
    case_bytes = [n + r[0] for (_, n), r in zip(ins, results)]
    achieved = sum(case_bytes) / (sum(statistics.mean(m) for m in launch_ms) / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic()

    # e2e through the reference-facing C ABI with page-locked host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, lib, n_run, rand_np, dist, dev, sel)

    batched = None
    if not args.no_batched:
        batched = run_batched(args, lib)

    extra = None
    if dist.rank == 0 and dist.world == 1 and not args.no_extra:
        del outs, d_run, d_rand
        torch.cuda.empty_cache()
        outs = d_run = d_rand = None
        extra = {"c1_one_shot": c1_figures(lib, dev),
                 "e2e_pageable": pageable_e2e(lib, n_run, rand_np),
                 "chain_128_pairs": chain_figures(lib, 4 * GiB if args.scale >= 1.0 else int(256 * MiB * args.scale) + MiB,
                                                  2, 1),
                 "stream_8_pairs": stream_figures(lib, 16 * GiB if args.scale >= 1.0 else int(GiB * args.scale) + MiB, 1),
                 "sparse_index": index_figures(lib, GiB if args.scale >= 1.0 else int(256 * MiB * args.scale) + MiB)}

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu:
        cb, ct, desc = cpu_sample(rand_np, min(args.scale, 1.0))
        cpu = {"value": round(cb / ct / 1e9, 4), "unit": "GB/s", "cores": 1, "kind": "port", "sample": desc}

    for s in sessions:
        s.close()
    if dist.rank == 0:
        line = {
            "metric": "GB/s (in+out), single-pair replace", "value": round(value, 2), "unit": "GB/s",
            "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(slowest / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
            "config": {
                "workload": (f"{n_run / GiB:g} GiB a-run aa->X + {n_run / GiB:g} GiB a-run a->bcd + "
                             f"{n_rand / GiB:g} GiB random 00 00 01->'' (one launch each)"),
                "bytes_in_plus_out_per_step": bytes_per_step, "l2": "inputs larger than L2 (126 MB), no flush",
                "parallelism": f"replicas x{dist.world}",
                "per_case_gbs": {c[0]: round(b / (statistics.mean(m) / 1e3) / 1e9, 1)
                                 for c, b, m in zip(cases, case_bytes, launch_ms)},
            },
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": traffic.get("bytes_per_step") if traffic else None,
                         "algorithmic_bytes": sum(case_bytes)},
            "gpu_launches": gpu_launches,
            "clocks": clock_info,
        }
        if e2e:
            line["e2e"] = e2e
        if batched:
            line["batched"] = batched
        if extra:
            line["extra"] = extra
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    del outs, d_run, d_rand
    dist.close()
    return 0


def run_batched(args, lib):
    """Batched/served jobs: the first --jobs jobs of the 10,000-job workload (same generator:
    sizes log-uniform 4 KiB-64 MiB, per-job alphabets of 4-64 symbols, 1-16 pairs with pattern
    1-32 B and replacement 0-64 B) through the request loop (cuda_replace_server_*), against the
    SAME jobs issued one by one as plain unified() calls (one call per pair). Each arm runs one
    untimed pass over all jobs first. Closed loop (all jobs submitted at once) gives jobs/s;
    Poisson arrivals at each rate of --rates (fractions of the closed-loop rate) give p50/p99
    latency from submit to result. Every result is compared with the unified() arm's."""
    import random

    from cuda_replace_b200 import workloads as WL
    from cuda_replace_b200.cuda_replace_wrapper import Server

    jobs = [WL.c5_job(i) for i in range(args.jobs)]
    n_bytes = sum(len(j.data) for j in jobs)
    out = {"jobs": len(jobs), "input_bytes": n_bytes}
    fracs = [float(x) for x in args.rates.split(",") if x]
    with Server(lib) as srv:
        # warm-up: one untimed pass over all jobs (tuning, graphs, staging, and the host pages
        # the results land in: first-touch page faults would otherwise dominate the figure)
        for t in [srv.submit(j.data, j.pairs) for j in jobs]:
            srv.wait(t)
        srv.reset_stats()
        t0 = time.perf_counter()
        tickets = [srv.submit(j.data, j.pairs) for j in jobs]
        outs = [srv.wait(t) for t in tickets]
        secs = time.perf_counter() - t0
        st = srv.stats()
        rate = len(jobs) / secs
        out.update({"jobs_per_s": round(rate, 2), "gbs_in": round(n_bytes / secs / 1e9, 3),
                    "closed_loop_p50_ms": round(st["p50_us"] / 1e3, 3), "closed_loop_p99_ms": round(st["p99_us"] / 1e3, 3),
                    "batches": st["batches"], "jobs_via_session": st["jobs_via_session"],
                    "tile_bytes": st["tile_bytes"], "grid_ctas": st["grid_ctas"]})
        # open loop: Poisson arrivals at fractions of the closed-loop rate
        sweep = []
        for frac in fracs:
            lam = frac * rate
            rng = random.Random(5)
            srv.reset_stats()
            t_start = time.perf_counter()
            t_next = t_start
            tickets = []
            for j in jobs:
                t_next += rng.expovariate(lam)
                d = t_next - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets.append(srv.submit(j.data, j.pairs))
            for t in tickets:
                srv.wait(t)
            span = time.perf_counter() - t_start
            st = srv.stats()
            sweep.append({"rate_frac": frac, "arrival_jobs_per_s": round(lam, 2),
                          "served_jobs_per_s": round(len(jobs) / span, 2),
                          "p50_ms": round(st["p50_us"] / 1e3, 3), "p99_ms": round(st["p99_us"] / 1e3, 3)})
        out["poisson"] = sweep
    # the same jobs as per-job plain unified() calls, after the same kind of warm pass
    def unified_all():
        res = []
        for j in jobs:
            d = j.data
            for p, r in j.pairs:
                d = lib.unified(d, p, r)
            res.append(d)
        return res
    base = unified_all()
    del base
    t0 = time.perf_counter()
    base = unified_all()
    ub = time.perf_counter() - t0
    bad = [j.job_id for j, a, b_ in zip(jobs, outs, base) if a != b_]
    if bad:
        raise SystemExit(f"batched self-check failed: jobs {bad[:8]} differ from per-job unified()")
    out["unified_jobs_per_s"] = round(len(jobs) / ub, 2)
    out["unified_same_jobs"] = True
    out["speedup_vs_unified"] = round(rate / (len(jobs) / ub), 2)
    golden = load_fullsize().get("c5", {}).get("jobs", [])
    checked = 0
    for j, o in zip(jobs, outs):
        if j.job_id < len(golden):
            g = golden[j.job_id]
            if len(o) != g["out_len"] or hashlib.sha256(o).hexdigest() != g["out_sha256"]:
                raise SystemExit(f"batched digest check failed for job {j.job_id}")
            checked += 1
    out["digests_checked"] = checked
    return out


def run_e2e(args, lib, n_run, rand_np, dist: Dist, dev, sel):
    import torch
    h_run = torch.full((n_run,), ord("a"), dtype=torch.uint8).pin_memory()
    h_rand = torch.from_numpy(rand_np).pin_memory()
    srcs = [[(h_run, n_run), (h_run, n_run), (h_rand, len(rand_np))][i] for i in sel]
    out_ptr = C.POINTER(C.c_uint8)()
    out_len = C.c_size_t()
    pats = [(C.create_string_buffer(p, len(p) or 1), len(p), C.create_string_buffer(r, len(r) or 1), len(r))
            for _, p, r in (CASES[i] for i in sel)]

    def step():
        h2d = d2h = 0
        for (h, n), (pb, pl, rb, rl) in zip(srcs, pats):
            rc = lib.lib.cuda_replace_unified(C.cast(h.data_ptr(), C.POINTER(C.c_uint8)), n,
                                              C.cast(pb, C.POINTER(C.c_uint8)), pl,
                                              C.cast(rb, C.POINTER(C.c_uint8)), rl, C.byref(out_ptr), C.byref(out_len))
            if rc != 0:
                raise RuntimeError(f"cuda_replace_unified rc={rc}")
            h2d += n
            d2h += out_len.value
            lib.lib.cuda_free_host(out_ptr)
        return h2d, d2h

    for _ in range(max(1, min(args.warmup, 2))):
        step()
    steps = max(1, min(args.steps, 5))
    dist.barrier()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for _ in range(steps):
        a, b = step()
        h2d += a
        d2h += b
    secs = time.perf_counter() - t0
    total, slowest = aggregate_replicas(h2d + d2h, secs, dist, dev)
    return {"value": round(total / slowest / 1e9, 3), "unit": "GB/s",
            "h2d_bytes_per_step": h2d // steps, "d2h_bytes_per_step": d2h // steps,
            "steps": steps, "api": "cuda_replace_unified (page-locked host input)"}


def load_fullsize() -> dict:
    """Digests of the chained bytes.replace output at full size (tests/golden/fullsize.json,
    made by tests/golden/make_fullsize.py)."""
    p = REPO / "tests" / "golden" / "fullsize.json"
    return json.loads(p.read_text()) if p.exists() else {}


def chain_figures(lib, total: int, steps: int, warmup: int) -> dict:
    """The 128-pair chain on tiled Zipf text (4 GiB at full size) with Session.apply_batch:
    lengths chained on the device, one read-back per chain. apply_batch runs each run of pairs
    that the planner proved independent in one pass (multi-pattern stages); the same chain with
    one pass per pair (CUDA_REPLACE_STAGES=0) is timed beside it. Device figure: the chain's
    algorithmic bytes, sum over the 128 pairs of (input + output), / the apply_batch call
    (input resident in HBM). End to end: host bytes in (reset) -> apply_batch -> host bytes out
    (result). The result's SHA-256 is checked against the full-size digest."""
    from cuda_replace_b200 import workloads as WL
    from cuda_replace_b200.cuda_replace_wrapper import Session
    txt, pairs = WL.c3_input(total, seed=3)
    res = {}
    with Session(lib, txt) as s:
        lens = [len(txt)]
        for p, r in pairs:  # pass lengths, for the algorithmic bytes (also a warm pass)
            lens.append(s.apply(p, r))
        algo = sum(lens[k] + lens[k + 1] for k in range(len(pairs)))
        out = None
        for arm, env in (("staged", None), ("per_pair", "0")):
            if env is None:
                os.environ.pop("CUDA_REPLACE_STAGES", None)
            else:
                os.environ["CUDA_REPLACE_STAGES"] = env
            dev_t, e2e_t, launches = [], [], 0
            nsteps = max(steps, 1) if arm == "staged" else 1
            for it in range(max(warmup, 1) + nsteps):
                t0 = time.perf_counter()
                s.reset(txt)
                t1 = time.perf_counter()
                _, l0 = s.stats()
                n = s.apply_batch(pairs)
                t2 = time.perf_counter()
                _, l1 = s.stats()
                o = s.result()
                t3 = time.perf_counter()
                if n != lens[-1] or len(o) != n:
                    raise SystemExit(f"chain self-check failed ({arm}): {n} != {lens[-1]}")
                if it >= max(warmup, 1):
                    dev_t.append(t2 - t1)
                    e2e_t.append(t3 - t0)
                    launches = l1 - l0
                if arm == "staged":
                    out = o
                else:
                    if o != out:
                        raise SystemExit("chain self-check failed: staged and per-pair results differ")
                del o
            res[arm] = (statistics.median(dev_t), statistics.median(e2e_t), launches, len(dev_t))
        os.environ.pop("CUDA_REPLACE_STAGES", None)
    g = load_fullsize().get("c3")
    digest = "not checked (size differs from the digest's)"
    if g and g["in_len"] == len(txt):
        if len(out) != g["out_len"] or hashlib.sha256(out).hexdigest() != g["out_sha256"]:
            raise SystemExit("chain digest check failed: output differs from the chained bytes.replace")
        digest = "sha256 equal to the chained bytes.replace"
    t, te, launches, nsteps = res["staged"]
    tp, tpe, lp, _ = res["per_pair"]
    return {"workload": f"{total / GiB:g} GiB tiled Zipf text x 128 entity pairs, Session.apply_batch",
            "gbs_sum_in_out": round(algo / t / 1e9, 2), "ms_per_chain": round(t * 1e3, 2),
            "passes": launches, "end_to_end_gbs": round((lens[0] + lens[-1]) / te / 1e9, 3),
            "end_to_end_ms": round(te * 1e3, 1),
            "per_pair": {"passes": lp, "ms_per_chain": round(tp * 1e3, 2),
                         "gbs_sum_in_out": round(algo / tp / 1e9, 2), "end_to_end_ms": round(tpe * 1e3, 1)},
            "launches_per_chain": launches, "final_len": lens[-1], "steps": nsteps, "check": digest,
            "timer": "host clock around the synchronous call"}


def stream_figures(lib, total: int, steps: int) -> dict:
    """Streaming: tiled Zipf text (16 GiB at full size) with a pattern planted across every
    256 MiB chunk boundary, 8 pairs, through gpu_replace_streaming (chunk-major: one
    host-link crossing each way). The result's SHA-256 is checked against the full-size
    digest."""
    from cuda_replace_b200 import workloads as WL
    from cuda_replace_b200.cuda_replace_wrapper import gpu_replace_streaming
    chunk = 256 * MiB
    buf, pairs, planted = WL.c4_input(total, chunk=chunk, seed=4)
    times, out = [], None
    for it in range(1 + max(steps, 1)):
        out = None
        t0 = time.perf_counter()
        out = gpu_replace_streaming(lib, buf, pairs, chunk_bytes=chunk)
        dt = time.perf_counter() - t0
        if it >= 1:
            times.append(dt)
    g = load_fullsize().get("c4")
    digest = "not checked (size differs from the digest's)"
    if g and g["in_len"] == len(buf):
        if len(out) != g["out_len"] or hashlib.sha256(out).hexdigest() != g["out_sha256"]:
            raise SystemExit("stream digest check failed: output differs from the chained bytes.replace")
        digest = "sha256 equal to the chained bytes.replace"
    t = statistics.median(times)
    return {"workload": f"{total / GiB:g} GiB tiled Zipf text x 8 pairs, chunk 256 MiB, "
                        f"{planted} patterns planted across chunk boundaries",
            "input_gbs": round(total / t / 1e9, 3), "ms": round(t * 1e3, 1),
            "h2d_bytes": total, "d2h_bytes": len(out), "host_link_gbs": round((total + len(out)) / t / 1e9, 3),
            "api": "gpu_replace_streaming (Python bytes in, Python bytes out)", "steps": len(times),
            "check": digest}


def index_figures(lib, total: int) -> dict:
    """A sparse pattern (64 planted NEEDLE tokens in tiled Zipf text, whose first byte occurs
    nowhere else) with and without the presence index (cuda_replace_build_index): apply time
    (host clock around the synchronous call, input resident), and the index build time."""
    from cuda_replace_b200 import workloads as WL
    from cuda_replace_b200.cuda_replace_wrapper import Session
    import random
    txt = bytearray(WL.tiled_text(total, seed=3))
    rng = random.Random(9)
    for _ in range(64):
        pos = rng.randrange(len(txt) - 8)
        txt[pos:pos + 6] = b"NEEDLE"
    txt = bytes(txt)
    want_len = len(txt) - 64 * 1 if txt.count(b"NEEDLE") == 64 else None
    res = {}
    with Session(lib, txt) as s:
        for arm in ("scan", "index"):
            t_apply, t_build = [], []
            for it in range(4):
                s.reset(txt)
                t0 = time.perf_counter()
                if arm == "index":
                    s.build_index()
                t1 = time.perf_counter()
                n = s.apply(b"NEEDLE", b"FOUND")
                t2 = time.perf_counter()
                if want_len is not None and n != want_len:
                    raise SystemExit(f"index self-check failed ({arm}): {n} != {want_len}")
                if it:
                    t_apply.append(t2 - t1)
                    t_build.append(t1 - t0)
            res[arm] = (statistics.median(t_apply), statistics.median(t_build))
    (ta, _), (ti, tb) = res["scan"], res["index"]
    return {"workload": f"{total / GiB:g} GiB tiled Zipf text, 64 x NEEDLE -> FOUND", "apply_ms": round(ta * 1e3, 3),
            "apply_ms_with_index": round(ti * 1e3, 3), "build_index_ms": round(tb * 1e3, 3),
            "gbs_in_out": round(2 * total / ta / 1e9, 1), "gbs_in_out_with_index": round(2 * total / ti / 1e9, 1),
            "timer": "host clock around the synchronous call (includes its 96-byte read-back)"}


def c1_figures(lib, dev) -> dict:
    """16 MiB one-shot ACGT -> N: launch-bound. Device: one launch on a resident input, CUDA
    events over 50 launches. Host: unified() from Python bytes to Python bytes."""
    import torch

    from cuda_replace_b200 import workloads as WL
    from cuda_replace_b200.cuda_replace_wrapper import Session
    src, pat, rep = WL.c1_acgt(16 * MiB, seed=1)
    want = src.replace(pat, rep)
    n = len(src)
    d_in = torch.empty(n + 64, dtype=torch.uint8, device=dev)
    d_in[:n].copy_(torch.frombuffer(bytearray(src), dtype=torch.uint8))
    d_out = torch.empty(n + 64, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    with Session(lib, b"") as s:
        for _ in range(5):
            s.apply_device_async(d_in.data_ptr(), n, pat, rep, d_out.data_ptr(), n, stream.cuda_stream)
        out_len, _ = s.device_result()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 50
        ev0.record(stream)
        for _ in range(reps):
            s.apply_device_async(d_in.data_ptr(), n, pat, rep, d_out.data_ptr(), n, stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        dev_us = ev0.elapsed_time(ev1) * 1e3 / reps
    if out_len != len(want) or bytes(d_out[:out_len].cpu().numpy()) != want:
        raise SystemExit("C1 self-check failed")
    for _ in range(3):
        lib.unified(src, pat, rep)
    t0 = time.perf_counter()
    calls = 20
    for _ in range(calls):
        got = lib.unified(src, pat, rep)
    host_us = (time.perf_counter() - t0) * 1e6 / calls
    if got != want:
        raise SystemExit("C1 unified self-check failed")
    return {"workload": "16 MiB i.i.d. ACGT, ACGT -> N (one launch)", "device_us": round(dev_us, 1),
            "device_gbs": round((n + out_len) / dev_us / 1e3, 1), "unified_us": round(host_us, 1),
            "unified_gbs": round((n + out_len) / host_us / 1e3, 2)}


def pageable_e2e(lib, n_run: int, rand_np) -> dict:
    """The single-pair step through the reference wrapper's call shape: CudaReplaceLib.unified
    on Python bytes (pageable host memory), result returned as Python bytes."""
    srcs = [b"a" * n_run, b"a" * n_run, rand_np.tobytes()]
    total = 0
    for (_, p, r), src in zip(CASES, srcs):  # warm pass
        total += len(src) + len(lib.unified(src, p, r))
    steps = 2
    t0 = time.perf_counter()
    for _ in range(steps):
        for (_, p, r), src in zip(CASES, srcs):
            out = lib.unified(src, p, r)
            del out
    secs = time.perf_counter() - t0
    return {"value": round(total * steps / secs / 1e9, 3), "unit": "GB/s", "steps": steps,
            "h2d_bytes_per_step": sum(len(x) for x in srcs), "d2h_bytes_per_step": total - sum(len(x) for x in srcs),
            "api": "CudaReplaceLib.unified(bytes) -> bytes (pageable host memory)"}


def run_chain(args):
    from cuda_replace_b200.cuda_replace_wrapper import CudaReplaceLib
    lib = CudaReplaceLib()
    total = int((args.gib or 4.0) * GiB)
    f = chain_figures(lib, total, args.steps, args.warmup)
    line = {"metric": "GB/s (sum over passes of in+out), 128-pair chain", "value": f["gbs_sum_in_out"],
            "unit": "GB/s", "n_gpus": 1, "steps": f["steps"], "warmup": max(args.warmup, 1),
            "ms_per_step": f["ms_per_chain"], "higher_is_better": True, "dtype": "u8",
            "data": "synthetic (Zipf text, 256 MiB generated block repeated)", "config": f,
            "gpu_launches_per_step": f["launches_per_chain"]}
    print(json.dumps(line), flush=True)
    return 0


def run_stream(args):
    from cuda_replace_b200.cuda_replace_wrapper import CudaReplaceLib
    lib = CudaReplaceLib()
    total = int((args.gib or 16.0) * GiB)
    f = stream_figures(lib, total, args.steps)
    line = {"metric": "GB/s of input, 8-pair streaming (host bytes in, host bytes out)",
            "value": f["input_gbs"], "unit": "GB/s", "n_gpus": 1, "steps": f["steps"], "warmup": 1,
            "ms_per_step": f["ms"], "higher_is_better": True, "dtype": "u8",
            "data": "synthetic (Zipf text, 256 MiB generated block repeated, matches planted at every chunk boundary)",
            "config": f}
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    args = parse_args(argv)
    dist = Dist()
    if args.impl == "reference":
        return run_reference(args, dist)
    if args.workload == "chain":
        return run_chain(args)
    if args.workload == "stream":
        return run_stream(args)
    return run_ours(args, dist)


if __name__ == "__main__":
    sys.exit(main())
