#!/usr/bin/env python3
"""Benchmark: imputed genotypes/s of the imputation step on the batched
dense-cohort workload (4,432 x 50,000 panel, 10,000 targets typed at 3,000
evenly spaced markers, L=8, Ne=20,000), one JSON line on rank 0.

A step = one pass of the hot path over the whole batch: per-marker L-state
selection from the resident PBWT index (1 launch), per-sample typed-marker
lists (3 launches), the anchor chain (1) and the parallel posterior pass with
dosage and argmax haplotypes (1), for all 10,000 chains. The PBWT index is
built once per panel before timing (reported as pbwt_build_ms).

  value  device-resident inputs/outputs, CUDA events on the launch stream,
         max over ranks; inputs (500 MB) exceed L2 so no flush is needed.
  e2e    the public C ABI call si_impute with pinned host buffers, H2D of the
         genotype codes and D2H of the results inside the timed region, for the
         reference's own output set (phased alleles, the GT it writes,
         imputer.cpp:393-400) in the compact host formats (2-bit codes in,
         haplotype bits out); e2e_with_dosage: byte codes in, f32 dosage and
         byte haplotypes out.

--impl reference times the reference's path on the host cores instead: the
reference has no CPU forward-backward, so its recurrences are run through the
FP64 C port (oracle/), threaded over samples, on a bounded sample per step.

Multi-GPU (torchrun): every rank imputes its own copy of the per-GPU batch
(independent chains, no data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    "dense-cohort": dict(M=50_000, N=4432, B=10_000, n_typed=3000, founders=100, L=8, ne=20000, seed=1),
    "plain-small": dict(M=1644, N=4432, B=444, every=5, founders=40, L=8, ne=10000, seed=0),
    # serving: an 8,000 x 120,000 panel (MAF ~ Beta(0.3, 0.6), switch 0.002); requests of 1-512 samples
    # (log-uniform) over 1,000-50,000 markers (log-uniform length, uniform start), typed every 20th
    # marker, L from {4, 8, 16}, Poisson arrivals
    "serving": dict(M=120_000, N=8000, founders=200, beta=(0.3, 0.6), switch=0.002, every=20, ne=20000, seed=4,
                    pool=1024, rate=200.0, seconds=10.0, hbm_budget=120 << 30),
}
LEGS = ["dense_map", "uneven_batch", "serving", "large_panel", "full_chain"]
ALGO_BYTES_PER_CELL = 7  # 1 B genotype code in, 4 B dosage + 2 B haplotype alleles out
POST_BYTES_PER_CELL = 6  # the posterior pass writes the outputs: 4 B dosage + 2 B alleles
KERNELS = ["select_kernel", "anchor_lists (count+scan+fill)", "anchor_chain_kernel", "anchor_posterior_kernel"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="dense-cohort")
    ap.add_argument("--samples", type=int, default=0, help="override the batch size B")
    ap.add_argument("--markers", type=int, default=0, help="override the marker count M")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-legs", action="store_true", help="skip the uneven-batch, large-panel and serving keys")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="serving key: length of the arrival window")
    ap.add_argument("--leg", choices=LEGS, default=None, help="run one extra key alone and print its JSON")
    ap.add_argument("--rate", type=float, default=0.0, help="serving: request arrivals per second")
    ap.add_argument("--seconds", type=float, default=0.0, help="serving: length of the arrival window")
    return ap.parse_args()


def make_workload(cfg):
    from swiftimpute_b200 import synth
    M, N, B = cfg["M"], cfg["N"], cfg["B"]
    panel, pos, _ = synth.make_panel(M, N, cfg["founders"], (0.5, 0.5), 0.01, 0.005, seed=cfg["seed"])
    typed = synth.typed_evenly(M, cfg["n_typed"]) if "n_typed" in cfg else synth.typed_every(M, cfg["every"])
    codes, truth, _ = synth.make_targets(panel, B, typed, seed=cfg["seed"] + 1000)
    return panel, pos, typed, codes, truth


class _NvmlSampler:
    """Reads SM clock, power and clock-event reasons every few ms from a thread
    (NVML; read-only), so that even a timed region of tens of ms is covered."""

    NAMES = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
             "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
             "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
             "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, device: int, period_s: float = 0.002):
        import threading
        import pynvml as nv
        self.nv = nv
        nv.nvmlInit()
        import os as _os
        vis = _os.environ.get("CUDA_VISIBLE_DEVICES")
        index = int(vis.split(",")[device]) if vis and vis.split(",")[device].isdigit() else device
        self.h = nv.nvmlDeviceGetHandleByIndex(index)
        self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
        self.rows = []
        self.stop_flag = threading.Event()
        self.period = period_s
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()

    def _run(self):
        nv = self.nv
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.rows.append((sm, pw, rs))
            except Exception:
                pass
            self.stop_flag.wait(self.period)

    def stop(self):
        self.stop_flag.set()
        self.th.join(timeout=5)
        nv = self.nv
        try:
            nv.nvmlShutdown()
        except Exception:
            pass
        if not self.rows:
            return None
        reasons = set()
        for _, _, rs in self.rows:
            for name, attr in self.NAMES.items():
                if rs & getattr(nv, attr):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(self.rows), "source": "nvml",
                "power_w_max": max(r[1] for r in self.rows)}


def clock_sampler_start(device: int):
    try:
        return _NvmlSampler(device)
    except Exception:
        return None


def clock_sampler_stop(handle):
    return handle.stop() if handle is not None else None


def peaks():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(kernel: str, config: str):
    """Per-launch DRAM bytes from the committed ncu summary of this kernel and workload, if any."""
    f = ROOT / "profiles" / f"{kernel}.{config}.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":", 1)[1].strip())
    return None


def cpu_model() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo), for the baseline records."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(panel, pos, codes, pairs, typed, cfg, seconds, gpu_dosage=None, gpu_haps=None):
    """The FP64 port of the reference recurrences on all host threads, on the
    first S samples of the workload (S sized to ~`seconds` of CPU work). With
    the device outputs of the same samples, also the parity of that sample."""
    import oracle
    threads = os.cpu_count() or 1
    M = codes.shape[1]
    s = max(1, threads)
    t0 = time.perf_counter()
    oracle.fb_batch(codes[:s], pairs, panel, pos, cfg["L"], cfg["ne"], threads=threads)
    dt = time.perf_counter() - t0
    S = int(min(codes.shape[0], max(s, round(s * seconds / max(dt, 1e-3)))))
    t0 = time.perf_counter()
    want = oracle.fb_batch(codes[:S], pairs, panel, pos, cfg["L"], cfg["ne"], threads=threads)
    dt = time.perf_counter() - t0
    imputed = S * (M - len(typed))
    out = {"value": imputed / dt, "unit": "imputed genotypes/s", "cores": threads, "cpu_model": cpu_model(),
           "kind": "port",
           "sample": f"first {S} of {codes.shape[0]} targets x {M} markers, FP64 log-space restatement of the "
                     f"reference recurrences, {dt:.1f} s"}
    parity = None
    if gpu_dosage is not None:
        d = np.abs(gpu_dosage[:S] - want["dosage"])
        masked = codes[:S] == 3
        x = gpu_dosage[:S][masked].astype(np.float64)
        y = want["dosage"][masked].astype(np.float64)
        r2 = float(np.corrcoef(x, y)[0, 1] ** 2) if x.size > 1 and x.std() > 0 and y.std() > 0 else None
        parity = {"targets": S, "max_abs_dosage_diff_vs_fp64_oracle": float(d.max()),
                  "mean_abs_dosage_diff": float(d.mean()), "dosage_r2_vs_fp64_oracle_masked": r2,
                  "argmax_haplotype_cells_differing": int((gpu_haps[:S] != want["haps_argmax"]).sum()),
                  "cells": int(S * M)}
    return out, parity


def pbwt_reference_time(panel):
    """The reference's own PBWTBuilder::build (compiled from its sources into
    oracle/_ref), single-threaded as the reference runs it, on the bench panel:
    the CPU path the device sweep replaces. Never fails the bench line."""
    import oracle
    if not oracle.ref_pbwt_available():
        return {"unavailable": "oracle/_ref/libref_pbwt.so is not built"}
    try:
        t0 = time.perf_counter()
        oracle.ref_pbwt_build(panel)
        dt = time.perf_counter() - t0
    except Exception as e:  # noqa: BLE001 - reported in the line instead
        return {"unavailable": f"{type(e).__name__}: {e}"}
    M, N = panel.shape
    return {"ms": dt * 1e3, "kind": "reference", "cores": 1, "cpu_model": cpu_model(),
            "sample": f"PBWTBuilder::build over the whole {N} x {M} panel, prefix and divergence arrays copied out"}


def workload_name(config: str, cfg: dict, M: int, B: int, n_typed: int) -> str:
    """The workload string both arms put in config.workload."""
    return (f"{config}: {cfg['N']} haplotypes x {M} markers, {B} targets typed at {n_typed} markers, "
            f"L={cfg['L']}, Ne={cfg['ne']}")


def run_reference(args, cfg):
    """Reference arm: the reference's recurrences on the host cores (rank 0)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    from swiftimpute_b200 import synth
    cfg = dict(cfg)
    panel, pos, typed, codes, truth = make_workload(cfg)
    pairs = oracle.select_pairs(oracle.pbwt_build_packed(synth.pack_panel(panel), cfg["N"])[0], cfg["L"])
    threads = os.cpu_count() or 1
    M = codes.shape[1]
    # each step: a bounded sample of the batch (~4 s of CPU work)
    t0 = time.perf_counter()
    oracle.fb_batch(codes[:threads], pairs, panel, pos, cfg["L"], cfg["ne"], threads=threads)
    per = (time.perf_counter() - t0) / threads
    S = int(max(threads, min(codes.shape[0], threads * round(4.0 / max(per * threads, 1e-3)))))
    for w in range(args.warmup):
        oracle.fb_batch(codes[:threads], pairs, panel, pos, cfg["L"], cfg["ne"], threads=threads)
    times = []
    for k in range(args.steps):
        rows = codes[(k * S) % max(1, codes.shape[0] - S):][:S]
        t0 = time.perf_counter()
        oracle.fb_batch(rows, pairs, panel, pos, cfg["L"], cfg["ne"], threads=threads)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    value = S * (M - len(typed)) / (ms / 1e3)
    unit = "imputed genotypes/s"
    line = {
        "impl": "reference", "metric": "imputed genotypes/s", "value": value, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, config shape)",
        "config": {"workload": workload_name(args.config, cfg, M, codes.shape[0], len(typed)), "markers": M,
                   "haplotypes": cfg["N"], "targets": codes.shape[0], "targets_per_step": S,
                   "typed_markers": int(len(typed)), "L": cfg["L"], "ne": cfg["ne"]},
        "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "cpu_model": cpu_model(), "kind": "port",
                         "sample": f"{S} targets x {M} markers per step; the reference has no CPU forward-backward, "
                                   "so its recurrences run through the FP64 C port"},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_serving(args, cfg):
    """Serving workload: Poisson arrivals submitted through the si_serve_* API
    on one GPU; latency percentiles from the server, throughput over the run."""
    import threading
    from swiftimpute_b200 import _native as N
    from swiftimpute_b200 import synth
    from swiftimpute_b200.engine import Engine, Server
    rank = int(os.environ.get("RANK", "0"))
    M, Nh = cfg["M"], cfg["N"]
    panel, pos, _ = synth.make_panel(M, Nh, cfg["founders"], cfg["beta"], cfg["switch"], 0.005, seed=cfg["seed"])
    pool, _, _ = synth.make_targets(panel, cfg["pool"], synth.typed_every(M, cfg["every"]), seed=cfg["seed"] + 1)
    rate = args.rate or cfg["rate"]
    seconds = args.seconds or cfg["seconds"]
    rng = np.random.default_rng(cfg["seed"] + 2)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * seconds * 1.5) + 16))
    arrivals = arrivals[arrivals < seconds]
    reqs = []
    for i in range(len(arrivals)):
        n = int(np.exp(rng.uniform(0, np.log(512))))
        length = int(np.exp(rng.uniform(np.log(1000), np.log(50_000))))
        m0 = int(rng.integers(0, M - length))
        rows = rng.integers(0, pool.shape[0], size=n)
        reqs.append((m0, m0 + length, int(rng.choice([4, 8, 16])), np.ascontiguousarray(pool[rows, m0:m0 + length])))
    cells = sum(r[3].size for r in reqs)
    # the clients' output buffers, allocated and touched before the run (a client reuses its buffers)
    outs = [{"dosage": np.full(r[3].shape, 0, np.float32), "haps": np.full((r[3].shape[0], 2, r[3].shape[1]), 0, np.uint8)}
            for r in reqs]
    eng = Engine(int(os.environ.get("LOCAL_RANK", "0")), hbm_budget_bytes=cfg["hbm_budget"])
    eng.upload_panel(panel)
    eng.set_map(pos)
    eng.pbwt_build()
    params = N.default_params(ne=cfg["ne"])
    # warm-up: a largest-size request per slot count, so tables, selections and the
    # per-launch scratch exist at full size before timing (as a server does at start-up)
    with Server(eng, params) as srv:
        for L in (4, 8, 16):
            srv.wait(srv.submit(0, 50_000, pool[:512, :50_000], num_states=L, index_origin=N.INDEX_GLOBAL))
    def run(max_batch_requests):
        """Replay the arrivals through a server; returns (statistics, wall seconds)."""
        srv = Server(eng, params, max_batch_requests=max_batch_requests)
        tickets = [None] * len(reqs)
        t0 = time.perf_counter()

        def submitter():
            for i, (a, b, L, codes) in enumerate(reqs):
                d = t0 + arrivals[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets[i] = srv.submit(a, b, codes, num_states=L, index_origin=N.INDEX_GLOBAL,
                                        sample_id_base=i << 10, out=outs[i])

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for t in tickets:
            srv.wait(t)
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.stop()
        return st, wall

    clocks = clock_sampler_start(int(os.environ.get("LOCAL_RANK", "0")))
    st, wall = run(0)
    clock_info = clock_sampler_stop(clocks)
    # the same arrivals served one request per launch (no batching)
    st1, wall1 = run(1)
    eng.close()
    if rank != 0:
        return
    busy_s = st["busy_ms"] / 1e3
    peak, peak_kind = peaks()
    line = {
        "metric": "imputed genotypes/s", "mode": "serving", "value": st["cells"] / wall,
        "unit": "cells/s over the run (samples x markers, typed included)", "n_gpus": 1,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded generator with the config's shape)",
        "config": {"workload": f"serving: {Nh} haplotypes x {M} markers, Poisson {rate:g} req/s for {seconds:g} s, "
                               f"1-512 samples x 1,000-50,000 markers per request, typed every {cfg['every']}th, "
                               "L in {4, 8, 16}, resident index", "requests": len(reqs), "cells": int(cells)},
        "offered_cells_per_s": cells / seconds,
        "latency_ms": {"p50": st["latency_p50_ms"], "p99": st["latency_p99_ms"], "max": st["latency_max_ms"]},
        "busy_fraction": busy_s / wall, "batches": st["batches"],
        "busy_cells_per_s": st["cells"] / busy_s if busy_s > 0 else None,
        "busy_roofline": {"bound": "hbm", "achieved": ALGO_BYTES_PER_CELL * st["cells"] / busy_s / 1e9 if busy_s else None,
                          "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
                          "note": "7 B per cell over busy intervals (host copies included)"},
        "completed": st["completed"], "failed": st["failed"],
        "hbm_budget_bytes": cfg["hbm_budget"],
        "one_request_per_launch": {"cells_per_s": st1["cells"] / wall1,
                                   "latency_ms": {"p50": st1["latency_p50_ms"], "p99": st1["latency_p99_ms"],
                                                  "max": st1["latency_max_ms"]},
                                   "busy_fraction": st1["busy_ms"] / 1e3 / wall1, "launches": st1["batches"]},
    }
    if clock_info:
        line["clocks"] = clock_info
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- extra legs (N = 1)
#
# The other BASELINE workloads, timed on the same GPU after the headline and
# added to the line as extra keys: the uneven batch in one graph-captured,
# autotuned plan launch; the large panel (PBWT build time and imputation);
# the serving loop at 200 requests/s for 60 s beside the reference's own path
# run one request at a time. Panels and targets are generated on the device
# (swiftimpute_b200.synth_device): a host generator would take minutes.

def _events_ms(fn, steps, stream):
    """Mean milliseconds of fn() over `steps` launches, CUDA events on `stream`."""
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def leg_dense_map(local, steps, peak, cpu_targets=1024):
    """The dense-cohort shape on a map with memory (markers 1 kb apart, so the
    transition is not the memoryless one of the 0.5 cM map): the step timed as
    the headline, and the first `cpu_targets` targets against the FP64 oracle."""
    import torch
    import oracle
    from swiftimpute_b200 import _native as N
    from swiftimpute_b200 import synth, synth_device
    from swiftimpute_b200.engine import Engine
    dev = torch.device("cuda", local)
    M, Nh, B, L, NE = 50_000, 4432, 10_000, 8, 20_000
    panel_d = synth_device.make_panel(M, Nh, 100, seed=11, device=dev)
    typed = synth.typed_evenly(M, 3000)
    codes = synth_device.make_targets(panel_d, B, typed=typed, seed=11)
    panel = panel_d.cpu().numpy()
    del panel_d
    pos = (1 + np.arange(M, dtype=np.uint64) * np.uint64(1000)).astype(np.uint64)
    with Engine(local) as eng:
        eng.upload_panel(panel)
        eng.set_map(pos)
        eng.pbwt_build()
        params = N.default_params(num_states=L, ne=NE)
        dos = torch.empty((B, M), dtype=torch.float32, device=dev)
        haps = torch.empty((B, 2, M), dtype=torch.uint8, device=dev)
        stream = torch.cuda.Stream(dev)
        kms = []

        def step():
            eng.impute_device(codes.data_ptr(), B, params, dos.data_ptr(), None, haps.data_ptr(), stream.cuda_stream)
            kms.append(eng.last_kernel_ms())
        step()
        kms.clear()
        ms = _events_ms(step, steps, stream)
        kavg = [sum(k[i] for k in kms) / len(kms) for i in range(4)]
        pairs = eng.select_states(L)
        c = codes[:cpu_targets].cpu().numpy()
        got_d, got_h = dos[:cpu_targets].cpu().numpy(), haps[:cpu_targets].cpu().numpy()
    del dos, haps, codes
    torch.cuda.empty_cache()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    want = oracle.fb_batch(c, pairs, panel, pos, L, float(NE), threads=threads)
    cpu_s = time.perf_counter() - t0
    masked = c == 3
    x, y = got_d[masked].astype(np.float64), want["dosage"][masked].astype(np.float64)
    post = POST_BYTES_PER_CELL * B * M / (kavg[3] / 1e3) / 1e9
    return {"workload": "dense cohort on a 1 kb map: 4432 haplotypes x 50000 markers, 10000 targets typed at "
                        "3000 markers, L=8, Ne=20000",
            "value": B * (M - len(typed)) / (ms / 1e3), "unit": "imputed genotypes/s", "ms_per_step": ms,
            "kernels_ms": dict(zip(KERNELS, kavg)),
            "roofline": {"bound": "hbm", "kernel": "anchor_posterior_kernel", "achieved": post, "peak": peak,
                         "unit": "GB/s", "frac": post / peak},
            "parity": {"targets": int(cpu_targets), "cells": int(c.size),
                       "max_abs_dosage_diff_vs_fp64_oracle": float(np.abs(got_d - want["dosage"]).max()),
                       "dosage_r2_vs_fp64_oracle_masked": float(np.corrcoef(x, y)[0, 1] ** 2),
                       "argmax_haplotype_cells_differing": int((got_h != want["haps_argmax"]).sum())},
            "cpu_port_imputed_genotypes_per_s": int(masked.sum()) / cpu_s}


def leg_full_chain(local, steps, peak, B=4000, check=64):
    """The per-gap-map path (SI_TRANS_PER_GAP: every gap its own transition, so
    the full-chain kernel steps every marker): the dense-cohort panel on a 1 kb
    map, B targets typed at 3,000 markers, timed, and the first `check` targets
    against the FP64 oracle with per-gap transitions."""
    import torch
    import oracle
    from swiftimpute_b200 import _native as N
    from swiftimpute_b200 import synth, synth_device
    from swiftimpute_b200.engine import Engine
    dev = torch.device("cuda", local)
    M, Nh, L, NE = 50_000, 4432, 8, 20_000
    panel_d = synth_device.make_panel(M, Nh, 100, seed=12, device=dev)
    typed = synth.typed_evenly(M, 3000)
    codes = synth_device.make_targets(panel_d, B, typed=typed, seed=12)
    panel = panel_d.cpu().numpy()
    del panel_d
    pos = (1 + np.arange(M, dtype=np.uint64) * np.uint64(1000)).astype(np.uint64)
    with Engine(local) as eng:
        eng.upload_panel(panel)
        eng.set_map(pos)
        eng.pbwt_build()
        params = N.default_params(num_states=L, ne=NE, transition_mode=N.TRANS_PER_GAP)
        dos = torch.empty((B, M), dtype=torch.float32, device=dev)
        haps = torch.empty((B, 2, M), dtype=torch.uint8, device=dev)
        stream = torch.cuda.Stream(dev)
        kms = []

        def step():
            eng.impute_device(codes.data_ptr(), B, params, dos.data_ptr(), None, haps.data_ptr(), stream.cuda_stream)
            kms.append(eng.last_kernel_ms())
        step()
        kms.clear()
        ms = _events_ms(step, steps, stream)
        kern = sum(k[3] for k in kms) / len(kms)
        pairs = eng.select_states(L)
        c = codes[:check].cpu().numpy()
        got_d = dos[:check].cpu().numpy()
    del dos, haps, codes
    torch.cuda.empty_cache()
    want = oracle.fb_batch(c, pairs, panel, pos, L, float(NE), per_gap=True, threads=os.cpu_count() or 1)
    ach = POST_BYTES_PER_CELL * B * M / (kern / 1e3) / 1e9
    return {"workload": f"per-gap map (full chain): 4432 haplotypes x 50000 markers on a 1 kb map, {B} targets typed "
                        "at 3000 markers, L=8, Ne=20000",
            "value": B * (M - len(typed)) / (ms / 1e3), "unit": "imputed genotypes/s", "ms_per_step": ms,
            "fb_chain_kernel_ms": kern,
            "roofline": {"bound": "hbm", "kernel": "fb_chain_kernel", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "note": "6 B per cell written"},
            "parity": {"targets": int(check), "max_abs_dosage_diff_vs_fp64_oracle":
                       float(np.abs(got_d - want["dosage"]).max())}}


def uneven_panel(local, seed=2):
    """The uneven-batch panel: 8,000 x 120,000, MAF ~ Beta(0.3, 0.6), switch 0.002, 0.5 cM map."""
    import torch
    from swiftimpute_b200 import synth_device
    M, Nh = 120_000, 8000
    panel = synth_device.make_panel(M, Nh, 200, (0.3, 0.6), 0.002, 0.005, seed=seed, device=torch.device("cuda", local))
    pos = (1 + np.arange(M, dtype=np.uint64) * np.uint64(500_000)).astype(np.uint64)
    return panel, pos


def leg_uneven(local, steps, peak, panel, pos):
    """4,096 targets over 64 regions (500-20,000 markers, log-uniform; uniform
    start), L in {4, 8, 16} per region, typed every 5th marker, each region
    indexed from its own first marker; one autotuned plan, graph-launched."""
    import torch
    from swiftimpute_b200 import _native as N
    from swiftimpute_b200 import synth_device
    from swiftimpute_b200.engine import Engine
    M = panel.shape[0]
    rng = np.random.default_rng(2)
    regions = []
    for _ in range(64):
        length = int(np.exp(rng.uniform(np.log(500), np.log(20_000))))
        m0 = int(rng.integers(0, M - length))
        regions.append((m0, m0 + length, int(rng.choice([4, 8, 16])), N.INDEX_REGION))
    assign = rng.integers(0, 64, size=4096)
    per_region = {}
    for r, (m0, m1, _, _) in enumerate(regions):
        n = int((assign == r).sum())
        if n:
            per_region[r] = synth_device.make_targets(panel[m0:m1].contiguous(), n, 5, seed=100 + r).cpu().numpy()
    jobs, seen = [], {r: 0 for r in per_region}
    for j, r in enumerate(assign):
        r = int(r)
        jobs.append((r, per_region[r][seen[r]], j))
        seen[r] += 1
    cells = sum(len(c) for _, c, _ in jobs)
    masked = sum(int((c == 3).sum()) for _, c, _ in jobs)
    with Engine(local) as eng:
        eng.upload_panel(panel.cpu().numpy())
        eng.set_map(pos)
        t0 = time.perf_counter()
        plan = eng.plan(regions, jobs, N.default_params(), autotune=True)
        create_s = time.perf_counter() - t0
        stream = torch.cuda.Stream(torch.device("cuda", local))
        plan.launch(graph=True, stream=stream.cuda_stream)
        ms = _events_ms(lambda: plan.launch(graph=True, stream=stream.cuda_stream), steps, stream)
        plan.check()
        info = plan.info()
        plan.destroy()
    achieved = ALGO_BYTES_PER_CELL * cells / (ms / 1e3) / 1e9
    return {"workload": "uneven batch: 8000 haplotypes x 120000 markers, 4096 targets over 64 regions of "
                        "500-20000 markers, L in {4, 8, 16}, typed every 5th, region-local index",
            "value": masked / (ms / 1e3), "unit": "imputed genotypes/s", "ms_per_launch": ms,
            "cells": int(cells), "imputed_cells": int(masked), "launch": "one CUDA graph (4 kernels), autotuned plan",
            "autotuned": info, "plan_create_s": create_s,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "note": "7 B per cell over the graph launch"}}


def leg_large_panel(local, steps, peak):
    """100,000 x 100,000 panel (1-bit packed on the device), 50,000 targets
    typed every 20th marker, L = 16, 0.5 cM map: PBWT build and imputation."""
    import torch
    from swiftimpute_b200 import _native as N
    from swiftimpute_b200 import synth_device
    from swiftimpute_b200.engine import Engine
    dev = torch.device("cuda", local)
    M = Nh = 100_000
    B, L = 50_000, 16
    panel = synth_device.make_panel(M, Nh, 500, (0.5, 0.5), 0.001, 0.005, seed=3, device=dev)
    words = synth_device.pack_panel(panel)
    codes = synth_device.make_targets(panel, B, 20, seed=3)
    del panel
    torch.cuda.empty_cache()
    pos = (1 + np.arange(M, dtype=np.uint64) * np.uint64(500_000)).astype(np.uint64)
    out = {}
    with Engine(local) as eng:
        eng.upload_packed(words, Nh)
        eng.set_map(pos)
        out["pbwt_build_ms"] = eng.pbwt_build()
        params = N.default_params(num_states=L, ne=10_000)
        dos = torch.empty((B, M), dtype=torch.float32, device=dev)
        haps = torch.empty((B, 2, M), dtype=torch.uint8, device=dev)
        stream = torch.cuda.Stream(dev)

        def step():
            eng.impute_device(codes.data_ptr(), B, params, dos.data_ptr(), None, haps.data_ptr(), stream.cuda_stream)
        step()
        torch.cuda.synchronize(dev)
        kms = []

        def timed():
            step()
            kms.append(eng.last_kernel_ms())
        ms = _events_ms(timed, steps, stream)
        kavg = [sum(k[i] for k in kms) / len(kms) for i in range(4)]
        typed = (M + 19) // 20
        masked = B * (M - typed)
        post = POST_BYTES_PER_CELL * B * M / (kavg[3] / 1e3) / 1e9
        out.update({
            "workload": "large panel: 100000 haplotypes x 100000 markers, 50000 targets typed every 20th, L=16",
            "value": masked / (ms / 1e3), "unit": "imputed genotypes/s", "ms_per_step": ms,
            "kernels_ms": dict(zip(KERNELS, kavg)),
            "roofline": {"bound": "hbm", "kernel": "anchor_posterior_kernel", "achieved": post, "peak": peak,
                         "unit": "GB/s", "frac": post / peak, "note": "6 B per cell written"},
            "step_roofline_frac": ALGO_BYTES_PER_CELL * B * M / (ms / 1e3) / 1e9 / peak})
        del dos, haps, codes
    torch.cuda.empty_cache()
    return out


def serving_requests(M, pool, rate, seconds, seed):
    """Poisson arrivals; each request 1-512 samples (log-uniform) over
    1,000-50,000 markers (log-uniform length, uniform start), L from {4, 8, 16}."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * seconds * 1.5) + 16))
    arrivals = arrivals[arrivals < seconds]
    reqs = []
    for _ in range(len(arrivals)):
        n = int(np.exp(rng.uniform(0, np.log(512))))
        length = int(np.exp(rng.uniform(np.log(1000), np.log(50_000))))
        m0 = int(rng.integers(0, M - length))
        rows = rng.integers(0, pool.shape[0], size=n)
        reqs.append((m0, m0 + length, int(rng.choice([4, 8, 16])), np.ascontiguousarray(pool[rows, m0:m0 + length])))
    return arrivals, reqs


def serve_replay(eng, params, arrivals, reqs, max_batch_requests=0):
    """Replay the arrivals through a server; returns (statistics, wall seconds)."""
    import threading
    from swiftimpute_b200 import _native as N
    from swiftimpute_b200.engine import Server
    outs = [{"dosage": np.zeros(r[3].shape, np.float32), "haps": np.zeros((r[3].shape[0], 2, r[3].shape[1]), np.uint8)}
            for r in reqs]
    srv = Server(eng, params, max_batch_requests=max_batch_requests)
    tickets = [None] * len(reqs)
    t0 = time.perf_counter()

    def submitter():
        for i, (a, b, L, codes) in enumerate(reqs):
            d = t0 + arrivals[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets[i] = srv.submit(a, b, codes, num_states=L, index_origin=N.INDEX_GLOBAL,
                                    sample_id_base=i << 10, out=outs[i])

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    for t in tickets:
        srv.wait(t)
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.stop()
    return st, wall


def reference_plain_serving(panel_host, pos, arrivals, reqs, ne, budget_s):
    """The reference's own path, one request at a time (Imputer::impute_batch
    steps with window_size = 0 on the request's region-sliced panel: CPU PBWT
    build, selection, emission, forward-backward, sampler), compiled from its
    sources (oracle/_ref). The first requests in arrival order are replayed
    sequentially until `budget_s` of work; latency = finish - arrival."""
    import oracle
    if not oracle.ref_gpu_available():
        return {"unavailable": "oracle/_ref/libref_gpu.so is not built"}
    done, lat, cells, masked = 0, [], 0, 0
    t_start = time.perf_counter()
    finish = 0.0
    for i, (m0, m1, L, codes) in enumerate(reqs):
        if time.perf_counter() - t_start > budget_s:
            break
        gl = oracle.codes_to_gl(codes)
        t0 = time.perf_counter()
        oracle.ref_gpu_impute(panel_host[m0:m1], pos[m0:m1], gl, L, ne, want_logpost=False)
        service = time.perf_counter() - t0
        finish = max(arrivals[i], finish) + service
        lat.append(finish - arrivals[i])
        cells += codes.size
        masked += int((codes == 3).sum())
        done += 1
    busy = time.perf_counter() - t_start
    lat_ms = np.array(lat) * 1e3
    return {"requests": done, "of": len(reqs), "imputed_genotypes_per_s": masked / busy,
            "cells_per_s": cells / busy,
            "latency_ms": {"p50": float(np.percentile(lat_ms, 50)), "p99": float(np.percentile(lat_ms, 99)),
                           "max": float(lat_ms.max())},
            "offered_load_fraction": (sum(r[3].size for r in reqs) / arrivals[-1]) / (cells / busy),
            "note": "sequential per-request runs of the reference's path on the same GPU; latencies of the first "
                    "requests in arrival order (a queue that never drains has latencies growing with the run)"}


def leg_serving(local, peak, panel, pos, rate=200.0, seconds=60.0, ref_budget_s=20.0):
    """Serving at `rate` requests/s for `seconds` over the uneven-batch panel
    with its resident index, under a 120 GB HBM budget."""
    from swiftimpute_b200 import _native as N
    from swiftimpute_b200 import synth_device
    from swiftimpute_b200.engine import Engine, Server
    M = panel.shape[0]
    pool = synth_device.make_targets(panel, 1024, 20, seed=5).cpu().numpy()
    panel_host = panel.cpu().numpy()
    arrivals, reqs = serving_requests(M, pool, rate, seconds, seed=6)
    cells = sum(r[3].size for r in reqs)
    masked = sum(int((r[3] == 3).sum()) for r in reqs)
    params = N.default_params(ne=20_000)
    with Engine(local, hbm_budget_bytes=120 << 30) as eng:
        eng.upload_panel(panel_host)
        eng.set_map(pos)
        eng.pbwt_build()
        with Server(eng, params) as srv:  # warm-up: tables, selections, scratch at full size
            for L in (4, 8, 16):
                srv.wait(srv.submit(0, 50_000, pool[:512, :50_000], num_states=L, index_origin=N.INDEX_GLOBAL))
        st, wall = serve_replay(eng, params, arrivals, reqs)
    busy_s = st["busy_ms"] / 1e3
    ref = reference_plain_serving(panel_host, pos, arrivals, reqs, 20_000, ref_budget_s)
    return {"workload": f"serving: 8000 haplotypes x {M} markers, resident index, Poisson {rate:g} req/s for "
                        f"{seconds:g} s, 1-512 samples x 1000-50000 markers, typed every 20th, L in {{4, 8, 16}}, "
                        "120 GB HBM budget",
            "requests": len(reqs), "completed": st["completed"], "failed": st["failed"],
            "imputed_genotypes_per_s": masked / wall, "cells_per_s": st["cells"] / wall,
            "offered_imputed_genotypes_per_s": masked / seconds,
            "latency_ms": {"p50": st["latency_p50_ms"], "p99": st["latency_p99_ms"], "max": st["latency_max_ms"]},
            "busy_fraction": busy_s / wall, "launches": st["batches"],
            "busy_roofline": {"bound": "hbm", "achieved": ALGO_BYTES_PER_CELL * st["cells"] / busy_s / 1e9,
                              "peak": peak, "unit": "GB/s",
                              "frac": ALGO_BYTES_PER_CELL * st["cells"] / busy_s / 1e9 / peak,
                              "note": "7 B per cell over the worker's busy time (host copies included)"},
            "reference_plain_per_request": ref}


def run_ours(args, cfg):
    import torch
    from swiftimpute_b200 import _native as N
    from swiftimpute_b200.engine import Engine
    from swiftimpute_b200.replicas import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    panel, pos, typed, codes, truth = make_workload(cfg)
    B, M = codes.shape
    eng = Engine(local)
    eng.upload_panel(panel)
    eng.set_map(pos)
    pbwt_ms = eng.pbwt_build()
    params = N.default_params(num_states=cfg["L"], ne=cfg["ne"], flags=N.IMPUTE_RESELECT)

    dev = torch.device("cuda", local)
    d_geno = torch.from_numpy(codes).to(dev)
    d_dos = torch.empty((B, M), dtype=torch.float32, device=dev)
    d_haps = torch.empty((B, 2, M), dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(dev)  # a real (non-legacy) stream: the events below bracket our kernels
    torch.cuda.synchronize(dev)

    def step():
        eng.impute_device(d_geno.data_ptr(), B, params, d_dos.data_ptr(), None, d_haps.data_ptr(), stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    # correctness spot-check of the device path against the host-buffer path is in tests; here only timing
    clocks = clock_sampler_start(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    kms = []
    t_start.record(stream)
    for k in range(args.steps):
        evs[k][0].record(stream)
        step()
        evs[k][1].record(stream)
        kms.append(eng.last_kernel_ms())  # waits for this step's last kernel (the step already waited mid-way)
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clock_info = clock_sampler_stop(clocks)
    total_ms = t_start.elapsed_time(t_end)
    kern_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(total_ms, dist, dev)
    ms_per_step = total_ms / args.steps
    imputed_per_gpu = B * (M - len(typed))
    value = world * imputed_per_gpu / (ms_per_step / 1e3)

    # end to end through the public C ABI with pinned host buffers
    from ctypes import byref, c_void_p
    from swiftimpute_b200.engine import pack_codes
    h_geno = torch.from_numpy(codes).pin_memory()
    h_dos = torch.empty((B, M), dtype=torch.float32).pin_memory()
    h_haps = torch.empty((B, 2, M), dtype=torch.uint8).pin_memory()
    h_codes2 = torch.from_numpy(pack_codes(codes)).pin_memory()
    Mw = (M + 31) // 32
    h_bits = torch.empty((B, 2, Mw), dtype=torch.int32).pin_memory()
    p_full = N.default_params(num_states=cfg["L"], ne=cfg["ne"], flags=N.IMPUTE_RESELECT)
    p_gt = N.default_params(num_states=cfg["L"], ne=cfg["ne"],
                            flags=N.IMPUTE_RESELECT | N.IMPUTE_CODES_2BIT | N.IMPUTE_HAPS_BITS)

    def e2e_full():
        eng._check(eng.lib.si_impute(eng.h, byref(p_full), c_void_p(h_geno.data_ptr()), B,
                                     c_void_p(h_dos.data_ptr()), None, c_void_p(h_haps.data_ptr())))

    def e2e_gt():
        eng._check(eng.lib.si_impute(eng.h, byref(p_gt), c_void_p(h_codes2.data_ptr()), B, None, None,
                                     c_void_p(h_bits.data_ptr())))

    def time_e2e(fn):
        fn()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            fn()
        return max_over_ranks((time.perf_counter() - t0) / args.e2e_steps, dist, dev)
    e2e_s = time_e2e(e2e_gt)
    e2e_value = world * imputed_per_gpu / e2e_s
    e2e_full_s = time_e2e(e2e_full)
    # quality vs truth on the device outputs (masked markers)
    dos = d_dos.cpu().numpy()
    masked = np.setdiff1d(np.arange(M), typed)
    sub = slice(0, min(B, 500))
    r2 = float(np.corrcoef(dos[sub][:, masked].ravel(), truth[sub][:, masked].ravel())[0, 1] ** 2)

    if rank != 0:
        eng.close()
        if dist:
            dist.destroy_process_group()
        return

    peak, peak_kind = peaks()
    avg_step = sum(kern_ms) / len(kern_ms)
    kavg = [sum(k[i] for k in kms) / len(kms) for i in range(4)]
    algo_step = ALGO_BYTES_PER_CELL * B * M
    algo_post = POST_BYTES_PER_CELL * B * M
    post_ms = kavg[3]
    achieved = algo_post / (post_ms / 1e3) / 1e9
    traffic = profile_traffic("anchor_posterior_kernel", args.config)
    line = {
        "metric": "imputed genotypes/s", "value": value, "unit": "imputed genotypes/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator with the config's shape; the reference's dataset is unavailable)",
        "config": {"workload": workload_name(args.config, cfg, M, B, len(typed)),
                   "markers": M, "haplotypes": cfg["N"], "targets": B, "typed_markers": int(len(typed)),
                   "L": cfg["L"], "ne": cfg["ne"], "l2": "inputs (B*M bytes) larger than L2, no flush",
                   "parallelism": f"replicas x{world} (independent chains)"},
        "roofline": {"bound": "hbm", "kernel": "anchor_posterior_kernel", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_launch": algo_post,
                     "algorithmic_bytes_note": "6 B per cell written (f32 dosage + 2 u8 alleles)",
                     "avg_launch_ms": post_ms},
        "step_roofline": {"achieved": algo_step / (avg_step / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                          "frac": algo_step / (avg_step / 1e3) / 1e9 / peak,
                          "algorithmic_bytes_per_step": algo_step, "avg_step_ms": avg_step,
                          "note": "7 B per cell (1 B code in, 6 B out) over the whole step"},
        "kernels_ms": dict(zip(KERNELS, kavg)),
        "e2e": {"value": e2e_value, "unit": "imputed genotypes/s", "h2d_bytes_per_step": int(h_codes2.numel()),
                "d2h_bytes_per_step": int(B * 2 * Mw * 4), "ms_per_step": e2e_s * 1e3,
                "outputs": "phased alleles (the GT the reference writes), haplotype bits; 2-bit codes in",
                "host_link_gbs": (h_codes2.numel() + B * 2 * Mw * 4) / e2e_s / 1e9},
        "e2e_with_dosage": {"value": world * imputed_per_gpu / e2e_full_s, "unit": "imputed genotypes/s",
                            "h2d_bytes_per_step": int(B * M), "d2h_bytes_per_step": int(B * M * 4 + B * 2 * M),
                            "ms_per_step": e2e_full_s * 1e3,
                            "outputs": "f32 dosage and byte haplotypes; byte codes in",
                            "host_link_gbs": (B * M + B * M * 4 + B * 2 * M) / e2e_full_s / 1e9},
        "gpu_launches": 6 * args.steps,
        "pbwt_build_ms": pbwt_ms,
        "dosage_r2_vs_truth": r2,
    }
    if clock_info:
        line["clocks"] = clock_info
    if not args.no_cpu_baseline and world == 1:
        import oracle
        pairs = eng.select_states(cfg["L"])
        line["cpu_baseline"], line["parity"] = cpu_baseline(panel, pos, codes, pairs, typed, cfg, args.cpu_seconds,
                                                            gpu_dosage=dos, gpu_haps=d_haps.cpu().numpy())
        line["pbwt_cpu_reference"] = pbwt_reference_time(panel)
    eng.close()
    if world == 1 and not args.no_legs and args.config == "dense-cohort":
        del d_geno, d_dos, d_haps, h_geno, h_dos, h_haps, h_codes2, h_bits
        torch.cuda.empty_cache()
        # each extra key in a process of its own: its memory is returned, and a
        # failure in one leaves the others and the headline standing
        import subprocess
        for name in LEGS:
            t0 = time.perf_counter()
            cmd = [sys.executable, str(Path(__file__).resolve()), "--leg", name, "--steps", str(args.steps),
                   "--serve-seconds", str(args.serve_seconds)]
            try:
                r = subprocess.run(cmd, capture_output=True, text=True, timeout=1200)
                last = [x for x in r.stdout.splitlines() if x.startswith("{")]
                line[name] = json.loads(last[-1]) if r.returncode == 0 and last else \
                    {"error": f"exit {r.returncode}: " + (r.stderr or r.stdout)[-600:]}
            except Exception as e:  # noqa: BLE001 - a failed leg is reported, the headline stands
                line[name] = {"error": f"{type(e).__name__}: {e}"}
            line[name]["leg_wall_s"] = time.perf_counter() - t0
            print(f"[bench] {name} done", file=sys.stderr, flush=True)
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_leg(args):
    """One extra key alone (a child of the headline run)."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    peak, _ = peaks()
    if args.leg == "dense_map":
        out = leg_dense_map(local, max(3, args.steps // 2), peak)
    elif args.leg == "large_panel":
        out = leg_large_panel(local, max(3, args.steps // 2), peak)
    elif args.leg == "full_chain":
        out = leg_full_chain(local, 3, peak)
    else:
        up = uneven_panel(local)
        out = leg_uneven(local, max(3, args.steps), peak, *up) if args.leg == "uneven_batch" else \
            leg_serving(local, peak, *up, seconds=args.serve_seconds)
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.leg:
        run_leg(args)
        return
    cfg = dict(CONFIGS[args.config])
    if args.samples:
        cfg["B"] = args.samples
    if args.markers:
        cfg["M"] = args.markers
        if "n_typed" in cfg:
            cfg["n_typed"] = max(1, round(cfg["n_typed"] * args.markers / CONFIGS[args.config]["M"]))
    if args.config == "serving":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "mode": "serving", "unavailable":
                              "the reference has no request queue; its CPU path is timed on the batch configs"}))
            return
        run_serving(args, cfg)
    elif args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
