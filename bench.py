#!/usr/bin/env python
"""K+KG assembly throughput of the OpenJFEM element hot path on B200.

One step = one stiffness assembly (K, with max_elem_stiff and orig_diag) and
one geometric-stiffness assembly (KG from a static displacement field) of the
whole model, i.e. the two calls SOL 105 makes per preload.  The workload is
the cylindrical barrel: R 2000 mm, L 6000 mm, 1440 x 696 cells with 10% of
them split into CTRIA3 pairs, I-section CBEAM rings every 500 mm, CBAR
longerons every 5 degrees and an RBE2 tying the loaded end to a centre node
(about 1.17M elements, 6.0M dof).  Synthetic, seeded inputs.

value: elements/s with all inputs resident in HBM (device-pointer C ABI).
e2e:   the same metric through the host-buffer C ABI calls (u in, K and KG
       values out, copies inside the timed region), with ordinary pageable
       host arrays as the Julia binding passes them; the pinned-memory figure
       is reported beside it.

--impl reference times the CPU restatement of the reference algorithm (the
reference itself is Julia and cannot run on this image) on the same barrel:
each step assembles K and KG of one axial band (1/24) of it, on its full node
set, and consecutive steps walk the bands.

Multi-GPU (torchrun): every rank assembles its own barrel replica (design
variants are independent units, no data-path collective); value is the sum
over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "K+KG assembly elements/s"
UNIT = "elements/s"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["barrel", "barrel_medium", "barrel_small", "panel", "plate", "serving", "variants",
                                          "group"], default="barrel")
    p.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    p.add_argument("--split", choices=["replicas", "rows"], default="replicas",
                   help="N>1: one model replica per GPU (weak scaling) or one model's row blocks over the GPUs (strong)")
    p.add_argument("--group-variants", type=int, default=4, help="group: design variants of every member per launch")
    p.add_argument("--rates", type=str, default="100,1000,5000", help="serving: Poisson arrival rates, req/s")
    p.add_argument("--requests", type=int, default=256, help="serving: requests per rate (server arms)")
    p.add_argument("--plain-requests", type=int, default=48, help="serving: requests per rate (plain arm)")
    p.add_argument("--max-batch", type=int, default=32, help="serving: batch limit per family")
    p.add_argument("--hbm-budget-gb", type=float, default=150.0, help="serving: device memory budget")
    p.add_argument("--variants", type=int, default=256, help="variants: design variants in one batch")
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    return p.parse_args()


def make_model(workload: str, seed: int):
    from jf_2026_05_19_b200 import decks
    if workload == "barrel":
        return decks.barrel_c4(seed=seed)
    if workload == "barrel_medium":
        return decks.barrel_c4(seed=seed, n_circ=720, n_axial=348, ring_every=29, longeron_every=10, name="barrel_720x348")
    if workload == "barrel_small":
        return decks.barrel_c4(seed=seed, n_circ=240, n_axial=96, ring_every=8, longeron_every=10, name="barrel_240x96")
    if workload == "panel":
        return decks.stiffened_panel_c2(seed=seed, stringer_offset=0.0, name="stiffened_panel_no_offset")
    return decks.plate_c1()


def workload_config(m, workload: str, world: int):
    c = m.counts()
    return {"workload": m.name if workload != "barrel" else
            "barrel R2000 L6000 1440x696 cells, 10% CTRIA3, CBEAM rings, CBAR longerons, RBE2 end",
            "elements_per_gpu": int(m.n_elements), "quad4": c["quad4"], "tria3": c["tria3"], "bar": c["bar"],
            "nodes": c["nodes"], "ndof": int(m.ndof), "rbe2_slaves": c["rbe2_slaves"],
            "replicas": world, "l2": "inputs and outputs larger than L2 (staging and CSR values are GBs)"}


CPU_BANDS = 24   # the barrel's 696 cell rows = 24 bands of 29 rows (~49k elements each)


def barrel_band(m, band: int, n_bands: int = CPU_BANDS):
    """Elements of one axial band of a barrel deck, in their deck order, on the
    full node set (so K and KG keep the whole barrel's dof numbering, pattern
    size and RBE2).  An element belongs to the band of its lowest cell row."""
    import dataclasses
    n_ring = m.n_nodes - (1 if m.rbe2_master.shape[0] else 0)
    z = m.coords[:, 2]
    rows_z = np.unique(np.round(z[:n_ring], 6))
    n_rows = rows_z.shape[0] - 1
    row_of = np.searchsorted(rows_z, np.round(z, 6))
    lo, hi = band * n_rows // n_bands, (band + 1) * n_rows // n_bands

    def pick(nodes):
        r = row_of[nodes].min(axis=1)
        return (r >= lo) & (r < hi)
    q, t, b = pick(m.q4_nodes), pick(m.t3_nodes), pick(m.bar_nodes)
    return dataclasses.replace(m, q4_nodes=m.q4_nodes[q], q4_prop=m.q4_prop[q], t3_nodes=m.t3_nodes[t],
                               t3_prop=m.t3_prop[t], bar_nodes=m.bar_nodes[b], bar_prop=m.bar_prop[b],
                               bar_pin=m.bar_pin[b], name=f"{m.name} band {band}/{n_bands}")


class CpuBands:
    """The CPU restatement of the reference assembly over bands of the bench barrel.

    Each call of step() assembles K (with max_elem_stiff and orig_diag) and KG
    of the next band, so consecutive steps walk the whole barrel; it returns
    the band's element count and records the time spent in the element loops
    and in the constraint redistribution + sparse() of each matrix."""

    def __init__(self, full, n_bands: int = CPU_BANDS):
        from jf_2026_05_19_b200 import decks
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O  # CPU restatement: the reported baseline and the reference arm
        self.O = O
        self.n_bands = n_bands
        # models other than the barrel are small enough to assemble whole per step
        self.bands = [barrel_band(full, b, n_bands) for b in range(n_bands)] if n_bands > 1 else [full]
        self.u = decks.smooth_displacement(full, seed=1)
        self.next = 0
        self.t_elem = self.t_sparse = 0.0

    def step(self) -> int:
        m = self.bands[self.next % self.n_bands]
        self.next += 1
        dk = self.O.assemble_k(m, detail=True)[5]
        dg = self.O.assemble_kg(m, self.u, detail=True)[3]
        self.t_elem += dk["t_elements"] + dg["t_elements"]
        self.t_sparse += dk["t_sparse"] + dg["t_sparse"]
        return m.n_elements

    def reset_phases(self):
        self.t_elem = self.t_sparse = 0.0

    def phases(self, steps: int) -> dict:
        return {"element_loops_s_per_step": self.t_elem / steps,
                "redistribution_and_sparse_s_per_step": self.t_sparse / steps,
                "note": "sparse() is serial in the reference (SparseArrays); element loops use every thread"}

    def sample_text(self, steps: int, n_el: int, seconds: float) -> str:
        if self.n_bands == 1:
            return f"{steps} steps, each K+KG of the whole model ({self.bands[0].name}); {n_el} elements in {seconds:.1f} s"
        return (f"{steps} steps, each K+KG of one axial band (1/{self.n_bands}, 29 of 696 cell rows, "
                f"~{n_el // max(steps, 1)} elements) of this barrel on its full 6.02M-dof node set, consecutive "
                f"bands per step; {n_el} elements in {seconds:.1f} s")


def time_cpu_oracle(full, seconds: float, steps_max: int = 24):
    """Reported CPU baseline: bands of the bench barrel for about `seconds`."""
    cpu = CpuBands(full)
    cpu.step()  # page in
    cpu.reset_phases()
    n_el, steps = 0, 0
    t0 = time.perf_counter()
    while True:
        n_el += cpu.step()
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= steps_max:
            break
    return n_el / el, cpu.O.num_threads(), cpu.sample_text(steps, n_el, el), cpu.phases(steps)


def cpu_sample_model(seed: int = 0):
    """A 480 x 96 barrel with the bench barrel's element mix (recovery baseline)."""
    from jf_2026_05_19_b200 import decks
    return decks.barrel_c4(seed=seed, n_circ=480, n_axial=96, ring_every=8, longeron_every=7, name="barrel_480x96")


def time_cpu_recovery(reps: int = 3):
    """Oracle SOL 101 output recovery on the same bounded sample (elements/s)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # CPU restatement: reported baseline only
    from jf_2026_05_19_b200 import decks
    m = cpu_sample_model()
    u = decks.smooth_displacement(m, seed=1)
    O.recover(m, u)
    t0 = time.perf_counter()
    for _ in range(reps):
        O.recover(m, u)
    el = time.perf_counter() - t0
    return m.n_elements * reps / el


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region.

    NVML is read every 5 ms from a background thread (read-only queries), so
    even a short timed region gets many samples; nvidia-smi at 200 ms is the
    fallback when the NVML bindings are missing.
    """
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, uuid=None, index=0, period_s=0.005):
        self.uuid, self.index, self.period = uuid, index, period_s
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.thread, self.proc, self.source = None, None, None

    def _nvml_loop(self, nv, h):
        bits = [(n, getattr(nv, attr)) for n, attr in self.REASONS]
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop_flag.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                r = get_reasons(h)
                for n, b in bits:
                    if r & b:
                        self.reasons.add(n)
            except Exception:
                pass
            self.stop_flag.wait(self.period)

    def start(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = None
            if self.uuid:
                try:
                    h = nv.nvmlDeviceGetHandleByUUID(self.uuid)
                except Exception:
                    h = None
            if h is None:
                h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop_flag = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
            self.source = "nvml 5 ms"
            return
        except Exception:
            self.thread = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.path = tempfile.mktemp(suffix=".csv")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi 200 ms"
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            sm = self.samples
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(self.reasons), "samples": len(sm), "source": self.source}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                if int(parts[0]) != self.index:
                    continue
                sm.append(float(parts[1])); mx.append(float(parts[2]))
            except ValueError:
                continue
            for (n, _), v in zip(self.REASONS, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": self.source}


def device_uuid(torch, dev):
    """NVML UUID string of a torch CUDA device, or None."""
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


def measure_fp64_peak(torch, dev):
    """Dense FP64 GEMM throughput on this GPU (cuBLAS DGEMM via torch), TFLOP/s."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(3):
        s = torch.cuda.Event(enable_timing=True); e = torch.cuda.Event(enable_timing=True)
        s.record(); torch.matmul(a, b); e.record(); e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / best / 1e12


def load_traffic():
    """Per-launch DRAM traffic of the dominant kernels from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(path):
        try:
            return json.load(open(path))
        except Exception:
            return {}
    return {}


def max_over_ranks(seconds: float, dist, device) -> float:
    """The slowest rank's time (every rank gets it); the value itself without a process group."""
    if dist is None:
        return seconds
    import torch
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args):
    """The reference algorithm on the host cores (C++ restatement, OpenMP over
    elements, serial sparse like the reference), on the GPU arm's workload:
    each step is K+KG of one axial band of the same barrel."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "variants":
        from jf_2026_05_19_b200 import decks
        full = decks.panel_variant_c3(0, seed=0, no_offset=True)
    else:
        full = make_model(args.workload, seed=0)
    cpu = CpuBands(full, CPU_BANDS if args.workload == "barrel" else 1)
    for _ in range(max(args.warmup, 1)):
        cpu.step()
    cpu.reset_phases()
    n_el = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        n_el += cpu.step()
    el = time.perf_counter() - t0
    v = n_el / el
    threads = cpu.O.num_threads()
    config = dict(workload_config(full, args.workload, args.gpus), parallelism=f"replicas x{args.gpus}")
    if args.workload == "variants":
        config = {"workload": "stiffened-panel design variants, one variant's K+KG per step"}
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded barrel deck)",
            "config": config,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": cpu.sample_text(args.steps, n_el, el), "phases": cpu.phases(args.steps),
                             "same_config": True,
                             "note": "reference is Julia 1.12 (absent here); C++ restatement of its algorithm"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


SERVE_METRIC = "served K+KG requests/s, mixed 8-family stream (p50/p99 latency beside)"


def serving_setup(seed: int = 0):
    """Eight families (1.6k-596k elements), their u fields and per-family thickness pools."""
    from jf_2026_05_19_b200 import decks
    fams = decks.serving_families(seed=seed)
    us = [decks.smooth_displacement(m, seed=20 + i) for i, m in enumerate(fams)]
    rng = np.random.default_rng(seed + 1)
    pools = []
    for m in fams:
        base = np.concatenate([m.q4_prop[:, 0], m.t3_prop[:, 0]])
        pools.append([base * np.exp(0.1 * rng.standard_normal(base.shape[0])) for _ in range(4)])
    return fams, us, pools


def serving_stream(rate: float, n: int, n_fam: int, seed: int):
    """Poisson arrivals: (arrival s, family, pool index); identical for every arm at one rate."""
    rng = np.random.default_rng(1000 + seed + int(rate))
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    return [(float(t[i]), int(rng.integers(n_fam)), int(rng.integers(4))) for i in range(n)]


def latency_summary(lat, t_first, t_last, n):
    lat = np.asarray(lat)
    return {"requests": int(n), "throughput_req_s": n / max(t_last - t_first, 1e-9),
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3)}


def run_server_stream(native, srv, stream, pools):
    """Submit at the arrival times (open loop); a collector waits, reads times and releases."""
    import queue
    import threading
    q = queue.Queue()
    rec = []

    def collect():
        while True:
            t = q.get()
            if t is None:
                return
            srv.wait(t, -1.0)
            rec.append(srv.result(t)[3])
            srv.release(t)

    th = threading.Thread(target=collect)
    th.start()
    t0 = time.perf_counter()
    lag = 0.0
    for (ta, f, k) in stream:
        while True:
            now = time.perf_counter() - t0
            if now >= ta:
                break
            if ta - now > 2e-4:
                time.sleep(min(ta - now - 1e-4, 0.01))
        lag = max(lag, time.perf_counter() - t0 - ta)
        q.put(srv.submit(f, pools[f][k], keep=False))
    q.put(None)
    th.join()
    ts = np.array(rec)
    out = latency_summary(ts[:, 2] - ts[:, 0], ts[:, 0].min(), ts[:, 2].max(), len(rec))
    out["max_submit_lag_ms"] = lag * 1e3
    return out


def run_plain_stream(native, torch, fams, us_dev, pools, stream, nz_bufs):
    """The plain one-deck-per-launch GPU path: per request, build the model on the GPU
    (pattern and maps), assemble K and KG into device buffers, wait, free it."""
    t0 = time.perf_counter()
    lat, done = [], []
    for (ta, f, k) in stream:
        while time.perf_counter() - t0 < ta:
            time.sleep(1e-4)
        m = fams[f]
        h = pools[f][k]
        nq = m.q4_nodes.shape[0]
        with native.GpuModel(m.with_thickness(h[:nq], h[nq:])) as g:
            nzk, nzg = nz_bufs[f]
            g.assemble_k_device(nzk.data_ptr())
            g.assemble_kg_device(us_dev[f].data_ptr(), nzg.data_ptr())
            torch.cuda.synchronize()
        t = time.perf_counter() - t0
        lat.append(t - ta)
        done.append(t)
    return latency_summary(lat, stream[0][0], max(done), len(stream))


def run_serving(args):
    import torch
    from jf_2026_05_19_b200 import native
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(0)
    rates = [float(r) for r in args.rates.split(",")]
    fams, us, pools = serving_setup()
    sizes = [m.n_elements for m in fams]
    models = [native.GpuModel(m) for m in fams]
    launches_per_batch = [2 * (sum(1 for c in ("quad4", "tria3", "bar") if m.counts()[c]) + 1 +
                               (2 if m.rbe2_master.shape[0] else 0)) for m in fams]
    # families under 64k elements share one group handle, so their requests
    # share launches; the large families keep their own handles
    small = [i for i, n in enumerate(sizes) if n < 64_000]
    large = [i for i in range(len(fams)) if i not in small]
    group = native.GpuGroup([fams[i] for i in small])
    g_units = [group] + [models[i] for i in large]
    g_u = [np.concatenate([us[i] for i in small])] + [us[i] for i in large]
    g_map = [None] * len(fams)
    for k, i in enumerate(small):
        g_map[i] = (0, k)
    for k, i in enumerate(large):
        g_map[i] = (1 + k, -1)
    arms = {}
    clocks = ClockSampler(uuid=device_uuid(torch, torch.device("cuda", 0)), index=0)
    clocks.start()
    for name, policy, units, uu, fmap in (
            ("batched", native.SERVE_BATCHED, g_units, g_u, g_map),
            ("batched_per_family", native.SERVE_BATCHED, models, us, None),
            ("serial_resident", native.SERVE_SERIAL, models, us, None)):
        with native.Server(units, uu, hbm_budget_bytes=int(args.hbm_budget_gb * 1e9), max_batch=args.max_batch,
                           policy=policy, family_map=fmap) as srv:
            warm = [srv.submit(f, pools[f][0], keep=False) for f in range(len(fams))]
            for t in warm:
                srv.wait(t, -1.0); srv.release(t)
            # warm-up stream at the top rate (another seed), so batches of every size the
            # measured streams form have run once before the timing
            run_server_stream(native, srv, serving_stream(max(rates), 64, len(fams), 1), pools)
            res = {}
            b0 = srv.stats()["batches"]
            for r in rates:
                res[f"{r:g}"] = run_server_stream(native, srv, serving_stream(r, args.requests, len(fams), 0), pools)
            st = srv.stats()
            res["batches"] = st["batches"] - b0
            res["largest_batch"] = st["max_batch"]
            res["pool_peak_gb"] = st["pool_peak_bytes"] / 1e9
            res["batch_limits"] = [srv.batch_limit(f) for f in range(len(fams))]
            arms[name] = res
    for g in models:
        g.close()
    group.close()
    torch.cuda.synchronize()
    us_dev = [torch.from_numpy(u).cuda() for u in us]
    nz_bufs = []
    for m in fams:
        with native.GpuModel(m) as g:
            nz_bufs.append((torch.empty(g.nnz, dtype=torch.float64, device="cuda"),
                            torch.empty(g.nnz, dtype=torch.float64, device="cuda")))
    plain = {}
    for r in rates:
        plain[f"{r:g}"] = run_plain_stream(native, torch, fams, us_dev, pools,
                                           serving_stream(r, args.plain_requests, len(fams), 0), nz_bufs)
    arms["plain_one_deck_per_launch"] = plain
    clk = clocks.stop()
    top = f"{max(rates):g}"
    v = arms["batched"][top]["throughput_req_s"]
    mean_shell = float(np.mean([p[0].shape[0] for p in pools]))
    line = {"metric": SERVE_METRIC, "value": v, "unit": "req/s", "n_gpus": 1, "steps": args.requests,
            "warmup": len(fams), "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded plate/panel/barrel families, Poisson arrivals, lognormal(0.1) thickness vectors",
            "config": {"workload": "serving: 8 device-resident families, K+KG per request, uniform family choice",
                       "family_elements": sizes, "rates_req_s": rates, "hbm_budget_gb": args.hbm_budget_gb,
                       "max_batch": args.max_batch, "value_at_rate": float(top),
                       "grouped_families": small,
                       "admission": "one device pool of the budget; batches take workspace and results as they form"},
            "serving": arms,
            "speedup_at_top_rate": {
                "vs_plain_one_deck_per_launch": v / arms["plain_one_deck_per_launch"][top]["throughput_req_s"],
                "vs_serial_resident": v / arms["serial_resident"][top]["throughput_req_s"],
                "vs_batched_per_family": v / arms["batched_per_family"][top]["throughput_req_s"]},
            "e2e": {"value": v, "unit": "req/s", "h2d_bytes_per_step": 8 * mean_shell, "d2h_bytes_per_step": 0,
                    "note": "submit-to-done wall clock through the server's C ABI; thickness vectors copied in, "
                            "K and KG stay on the device"},
            "gpu_launches": int(arms["batched"]["batches"] * float(np.mean(launches_per_batch))),
            "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def run_variants(args):
    """256 stiffened-panel design variants (own thickness vector and stringer section each)
    assembled as one batch: K and KG for every variant per graph replay."""
    import torch
    from jf_2026_05_19_b200 import decks, native, roofline
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    nv = args.variants
    ms = [decks.panel_variant_c3(v, no_offset=True) for v in range(nv)]
    base = ms[0]
    u = decks.smooth_displacement(base, seed=1)
    H = np.stack([np.concatenate([m.q4_prop[:, 0], m.t3_prop[:, 0]]) for m in ms])
    BP = np.stack([m.bar_prop for m in ms])
    g = native.GpuModel(base)
    g.batch_reserve(nv)
    s = torch.cuda.Stream()
    g.set_stream(s.cuda_stream)
    Hd, BPd, ud = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (H, BP, u))
    nzk = torch.empty(nv, g.nnz, dtype=torch.float64, device=dev)
    nzg = torch.empty_like(nzk)
    mx = torch.zeros(nv, dtype=torch.float64, device=dev)

    def call():
        g.assemble_batch_device(nv, Hd.data_ptr(), BPd.data_ptr(), ud.data_ptr(), 0, nzk.data_ptr(), mx.data_ptr(), 0,
                                nzg.data_ptr())

    torch.cuda.synchronize()
    for _ in range(2):
        call()
    s.synchronize()
    # per-kernel split from timed direct calls
    g.timing_accumulated("k", reset=True); g.timing_accumulated("kg", reset=True)
    for _ in range(3):
        call()
    s.synchronize()
    kt, kn = g.timing_accumulated("k", reset=True)
    gt, gn = g.timing_accumulated("kg", reset=True)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        call()
    for _ in range(max(args.warmup, 3)):
        graph.replay()
    torch.cuda.synchronize()
    clocks = ClockSampler(uuid=device_uuid(torch, dev), index=0)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    with torch.cuda.stream(s):
        for _ in range(args.steps):
            graph.replay()
    e1.record(s)
    e1.synchronize()
    clk = clocks.stop()
    el = e0.elapsed_time(e1) / 1e3 / args.steps
    # one launch sequence per variant (no batching, no graph)
    p0 = torch.cuda.Event(enable_timing=True); p1 = torch.cuda.Event(enable_timing=True)
    p0.record(s)
    for v in range(nv):
        g.assemble_batch_device(1, Hd[v].data_ptr(), BPd[v].data_ptr(), ud.data_ptr(), 0, nzk[v].data_ptr(),
                                mx[v:].data_ptr(), 0, nzg[v].data_ptr())
    p1.record(s)
    p1.synchronize()
    per_variant = p0.elapsed_time(p1) / 1e3
    # end to end: inputs from pinned host memory, graph replay, per-variant max read back
    Hp = torch.from_numpy(H).pin_memory(); BPp = torch.from_numpy(BP).pin_memory()
    mxp = torch.empty(nv, dtype=torch.float64).pin_memory()
    q0 = torch.cuda.Event(enable_timing=True); q1 = torch.cuda.Event(enable_timing=True)
    q0.record(s)
    with torch.cuda.stream(s):
        for _ in range(args.e2e_steps):
            Hd.copy_(Hp, non_blocking=True); BPd.copy_(BPp, non_blocking=True)
            graph.replay()
            mxp.copy_(mx, non_blocking=True)
    q1.record(s)
    q1.synchronize()
    e2e_el = q0.elapsed_time(q1) / 1e3 / args.e2e_steps
    # parity of two variants against their own handles
    for v in (0, nv - 1):
        with native.GpuModel(ms[v]) as gv:
            assert np.array_equal(gv.assemble_k()[0], nzk[v].cpu().numpy()), f"variant {v} K differs"
            assert np.array_equal(gv.assemble_kg(u), nzg[v].cpu().numpy()), f"variant {v} KG differs"
    del graph
    g.set_stream(0)
    n_el = nv * base.n_elements
    counts = {k: nv * c for k, c in base.counts().items()}
    per_kernel = {}
    for tag, tt, nn in (("k", kt, kn), ("kg", gt, gn)):
        for name in ("quad4", "tria3", "bar", "dof_reduce", "block_reduce"):
            per_kernel[f"{name}_{tag}"] = tt[name] / max(nn, 1)
    dom = max(per_kernel, key=per_kernel.get)
    fp64 = measure_fp64_peak(torch, dev)
    roof = {"bound": "tensor", "unit": "TFLOP/s", "kernel": dom, "peak": fp64, "traffic": None,
            "peak_source": "FP64 DGEMM (torch.matmul float64 8192^3) measured in this run"}
    if dom.startswith(("quad4", "tria3", "bar")):
        roof["achieved"] = roofline.kernel_flops(dom, counts[dom.split("_")[0]]) / (per_kernel[dom] / 1e3) / 1e12
    else:
        st = g.stats()
        mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
        hbm = json.load(open(mp))["hbm_gbs"] if os.path.exists(mp) else 6650.0
        roof = {"bound": "hbm", "unit": "GB/s", "kernel": dom, "peak": hbm, "traffic": None,
                "achieved": nv * (8 * st["staging_values"] + 20 * st["n_blocks"] + 8 * st["nnz"]) / (per_kernel[dom] / 1e3) / 1e9}
    roof["frac"] = roof["achieved"] / roof["peak"]
    roof["launch_ms"] = per_kernel[dom]
    g.close()
    line = {"metric": METRIC, "value": n_el / el, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: 256 seeded stiffened-panel variants (lognormal thickness, stringer height U[15,25])",
            "config": {"workload": f"{nv} stiffened-panel design variants, K+KG of all in one CUDA-graph replay",
                       "elements_per_variant": int(base.n_elements), "variants": nv, "elements_per_step": int(n_el),
                       "nnz_per_variant": int(nzk.shape[1]),
                       "l2": "outputs larger than L2", "parallelism": "one GPU, variants batched on blockIdx.y"},
            "variants": {"graph_replay_ms": el * 1e3, "one_launch_sequence_per_variant_ms": per_variant * 1e3,
                         "speedup_vs_per_variant_launches": per_variant / el,
                         "kernel_ms_direct_call": per_kernel},
            "roofline": roof,
            "e2e": {"value": n_el / e2e_el, "unit": UNIT, "h2d_bytes_per_step": int(H.nbytes + BP.nbytes),
                    "d2h_bytes_per_step": 8 * nv},
            "gpu_launches": args.steps * 2 * (sum(1 for c in ("quad4", "tria3", "bar") if base.counts()[c]) + 1 +
                                              (2 if base.rbe2_master.shape[0] else 0)),
            "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def run_group(args):
    """Mixed-model batch: the eight serving-stream families (plate, stiffened panel and
    barrel meshes of 1.6k to 596k elements, CQUAD4/CTRIA3/CBAR/CBEAM, RBE2) in one group
    handle, each with --group-variants thickness variants, K and KG of every member and
    variant in one CUDA-graph replay; against one launch sequence per member and variant
    on the members' own handles."""
    import torch
    from jf_2026_05_19_b200 import decks, native
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    fams = decks.serving_families(seed=0)
    nv = max(1, args.group_variants)
    rng = np.random.default_rng(3)
    hv = [[np.concatenate([m.q4_prop[:, 0], m.t3_prop[:, 0]]) * np.exp(0.1 * rng.standard_normal(m.q4_nodes.shape[0] + m.t3_nodes.shape[0]))
           for m in fams] for _ in range(nv)]
    nq = [m.q4_nodes.shape[0] for m in fams]
    H = np.stack([np.concatenate([np.concatenate([hv[v][i][:nq[i]] for i in range(len(fams))]),
                                  np.concatenate([hv[v][i][nq[i]:] for i in range(len(fams))])]) for v in range(nv)])
    us = [decks.smooth_displacement(m, seed=20 + i) for i, m in enumerate(fams)]
    g = native.GpuGroup(fams)
    tuned = g.launch_config() if args.no_autotune else g.autotune()
    g.batch_reserve(nv)
    s = torch.cuda.Stream()
    g.set_stream(s.cuda_stream)
    Hd = torch.from_numpy(H).to(dev)
    ud = torch.from_numpy(np.concatenate(us)).to(dev)
    nzk = torch.empty(nv, g.nnz, dtype=torch.float64, device=dev)
    nzg = torch.empty_like(nzk)

    def call():
        g.assemble_batch_device(nv, Hd.data_ptr(), 0, ud.data_ptr(), 0, nzk.data_ptr(), 0, 0, nzg.data_ptr())

    torch.cuda.synchronize()
    call(); call()
    s.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        call()
    for _ in range(max(args.warmup, 3)):
        graph.replay()
    torch.cuda.synchronize()
    clocks = ClockSampler(uuid=device_uuid(torch, dev), index=0)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    with torch.cuda.stream(s):
        for _ in range(args.steps):
            graph.replay()
    e1.record(s)
    e1.synchronize()
    clk = clocks.stop()
    el = e0.elapsed_time(e1) / 1e3 / args.steps
    # the same work as one launch sequence per member and variant, on the members' own handles
    own = [native.GpuModel(m) for m in fams]
    bufs = []
    for i, gm in enumerate(own):
        gm.set_stream(s.cuda_stream)
        gm.batch_reserve(1)
        h1 = torch.from_numpy(np.stack([hv[v][i] for v in range(nv)])).to(dev)
        u1 = torch.from_numpy(us[i]).to(dev)
        bufs.append((h1, u1, torch.empty(gm.nnz, dtype=torch.float64, device=dev), torch.empty(gm.nnz, dtype=torch.float64, device=dev)))

    def per_model():
        for gm, (h1, u1, k1, kg1) in zip(own, bufs):
            for v in range(nv):
                gm.assemble_batch_device(1, h1[v].data_ptr(), 0, u1.data_ptr(), 0, k1.data_ptr(), 0, 0, kg1.data_ptr())

    per_model()
    s.synchronize()
    p0 = torch.cuda.Event(enable_timing=True); p1 = torch.cuda.Event(enable_timing=True)
    p0.record(s)
    for _ in range(args.steps):
        per_model()
    p1.record(s)
    p1.synchronize()
    sep = p0.elapsed_time(p1) / 1e3 / args.steps
    for gm in own:
        gm.close()
    n_el = nv * sum(m.n_elements for m in fams)
    line = {"metric": METRIC, "value": n_el / el, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: the eight seeded serving families, lognormal(0.1) thickness variants",
            "config": {"workload": f"mixed-model group: {len(fams)} meshes x {nv} variants, K+KG of all in one CUDA-graph replay",
                       "members_elements": [int(m.n_elements) for m in fams], "variants": nv,
                       "elements_per_step": int(n_el), "nnz_group": int(g.nnz), "l2": "outputs larger than L2",
                       "parallelism": "one GPU; members side by side in each launch, variants on blockIdx.y"},
            "group": {"graph_replay_ms": el * 1e3, "launch_sequence_per_member_and_variant_ms": sep * 1e3,
                      "speedup_vs_per_member_launches": sep / el, "launch_config": tuned},
            "gpu_launches": args.steps * 2 * (3 + 2 + 1),  # element kernels, RBE2 path, block reduction
            "clocks": clk}
    g.close()
    print(json.dumps(line), flush=True)
    return 0


def run_reference_serving(args):
    """Oracle port, one request at a time: elements/s on the bounded barrel sample,
    converted with the stream's mean request size."""
    from jf_2026_05_19_b200 import decks
    v_el, threads, sample, _ = time_cpu_oracle(make_model("barrel", seed=0), args.cpu_seconds)
    fams = decks.serving_families()
    mean_el = float(np.mean([m.n_elements for m in fams]))
    v = v_el / mean_el
    line = {"metric": SERVE_METRIC, "value": v, "unit": "req/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded families)",
            "config": {"workload": "serving: 8 families, uniform family choice", "mean_request_elements": mean_el},
            "cpu_baseline": {"value": v, "unit": "req/s", "cores": threads, "kind": "port",
                             "sample": sample + f"; req/s = elements/s / {mean_el:.0f} mean elements per request"},
            "e2e": {"value": v, "unit": "req/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    if args.workload == "variants":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        if args.impl == "reference":
            return run_reference(args)
        return run_variants(args)
    if args.workload == "group":
        if int(os.environ.get("RANK", "0")) != 0 or args.impl == "reference":
            return 0
        return run_group(args)
    if args.workload == "serving":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0  # one GPU serves; other ranks have nothing to do
        return run_reference_serving(args) if args.impl == "reference" else run_serving(args)
    if args.impl == "reference":
        return run_reference(args)
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (the CPU oracle is only the reference arm)")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    from jf_2026_05_19_b200 import decks, native, roofline

    fp64_peak = measure_fp64_peak(torch, dev)
    m = make_model(args.workload, seed=rank)
    part = full = None
    if args.split == "rows" and world > 1:
        # one model over the GPUs: this rank assembles the elements of its row block
        from jf_2026_05_19_b200 import partition
        full = make_model(args.workload, seed=0)
        part = partition.part_of(full, rank, world)
        m = part.model
    g = native.GpuModel(m)
    t_tune = time.perf_counter()
    launch_cfg = g.launch_config() if args.no_autotune else g.autotune()
    t_tune = time.perf_counter() - t_tune
    # a dedicated (non-default) stream shared by the library and the timing events
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    g.set_stream(stream.cuda_stream)
    u_host = decks.smooth_displacement(m, seed=1 + rank)
    u_dev = torch.from_numpy(u_host).to(dev)
    nz_k = torch.empty(g.nnz, dtype=torch.float64, device=dev)
    nz_kg = torch.empty(g.nnz, dtype=torch.float64, device=dev)
    diag = torch.empty(g.ndof, dtype=torch.float64, device=dev)
    mx = torch.zeros(1, dtype=torch.float64, device=dev)

    def step():
        g.assemble_k_device(nz_k.data_ptr(), mx.data_ptr(), diag.data_ptr())
        g.assemble_kg_device(u_dev.data_ptr(), nz_kg.data_ptr())

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    g.timing_accumulated("k", reset=True)
    g.timing_accumulated("kg", reset=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(uuid=device_uuid(torch, dev), index=local)
    clocks.start()
    start = torch.cuda.Event(enable_timing=True); end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        step()
    end.record(stream)
    end.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    elapsed = start.elapsed_time(end) / 1e3
    elapsed = max_over_ranks(elapsed, dist, dev)
    kt, kn = g.timing_accumulated("k", reset=True)
    gt, gn = g.timing_accumulated("kg", reset=True)

    # end-to-end through the host-buffer C ABI: ordinary pageable host arrays,
    # as the Julia binding passes Vector{Float64}; pinned arrays beside it
    e2e_steps = max(1, min(args.e2e_steps, args.steps))

    def e2e_time(u_h, nzk_h, nzg_h, dg_h):
        g.assemble_k(nzk_h, want_diag=True, diag_out=dg_h); g.assemble_kg(u_h, nzg_h)  # warm, pages in
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        s2 = torch.cuda.Event(enable_timing=True); e2 = torch.cuda.Event(enable_timing=True)
        s2.record(stream)
        for _ in range(e2e_steps):
            g.assemble_k(nzk_h, want_diag=True, diag_out=dg_h)
            g.assemble_kg(u_h, nzg_h)
        e2.record(stream)
        e2.synchronize()
        return max_over_ranks(s2.elapsed_time(e2) / 1e3, dist, dev)

    e2e_el = e2e_time(u_host.copy(), np.empty(g.nnz), np.empty(g.nnz), np.empty(g.ndof))
    pin = [torch.from_numpy(u_host).pin_memory()] + [torch.empty(n, dtype=torch.float64).pin_memory()
                                                     for n in (g.nnz, g.nnz, g.ndof)]
    e2e_pinned_el = e2e_time(*[t.numpy() for t in pin])
    del pin

    # SOL 101 output recovery of the same model and displacement, timed on its
    # own after the step (it follows the static solve, not the assembly)
    counts = m.counts()
    rec_sh = torch.empty((counts["quad4"] + counts["tria3"], 48), dtype=torch.float64, device=dev)
    rec_bar = torch.empty((max(counts["bar"], 1), 18), dtype=torch.float64, device=dev)

    def recover():
        g.recover_stresses_device(u_dev.data_ptr(), None, 0, rec_sh.data_ptr(), rec_bar.data_ptr() if counts["bar"] else None)

    for _ in range(3):
        recover()
    torch.cuda.synchronize()
    s3 = torch.cuda.Event(enable_timing=True); e3 = torch.cuda.Event(enable_timing=True)
    s3.record(stream)
    for _ in range(5):
        recover()
    e3.record(stream)
    e3.synchronize()
    rec_ms = s3.elapsed_time(e3) / 5

    n_el = m.n_elements
    value = (full.n_elements if part else world * n_el) * args.steps / elapsed
    gather_ms = None
    if part is not None:
        # the one exchange of the split: every rank's owned K columns to every rank
        cp, _ = g.pattern()
        a, b = int(cp[part.dof_lo] - 1), int(cp[part.dof_hi] - 1)
        n_own = torch.tensor([b - a], device=dev)
        n_all = [torch.zeros_like(n_own) for _ in range(world)]
        dist.all_gather(n_all, n_own)
        width = int(max(int(x.item()) for x in n_all))
        send = torch.zeros(width, dtype=torch.float64, device=dev)
        send[:b - a] = nz_k[a:b]
        recv = torch.empty(world * width, dtype=torch.float64, device=dev)
        dist.all_gather_into_tensor(recv, send)
        torch.cuda.synchronize()
        dist.barrier()
        ga = torch.cuda.Event(enable_timing=True); gb = torch.cuda.Event(enable_timing=True)
        ga.record(stream)
        with torch.cuda.stream(stream):
            dist.all_gather_into_tensor(recv, send)
        gb.record(stream)
        gb.synchronize()
        gather_ms = max_over_ranks(ga.elapsed_time(gb) / 1e3, dist, dev) * 1e3
        del send, recv
    e2e_value = (full.n_elements if part else world * n_el) * e2e_steps / e2e_el
    e2e_pinned_value = world * n_el * e2e_steps / e2e_pinned_el
    # dominant kernel over the timed region
    per_kernel = {}
    for tag, tt, nn in (("k", kt, kn), ("kg", gt, gn)):
        for name in ("quad4", "tria3", "bar", "dof_reduce", "block_reduce", "diag"):
            if tag == "kg" and name == "diag":
                continue
            per_kernel[f"{name}_{tag}"] = tt[name] / max(nn, 1)
    dominant = max(per_kernel, key=per_kernel.get)
    traffic = load_traffic()
    st = g.stats()
    if "reduce" in dominant or dominant.startswith("diag"):
        # block reduction: staging read, block metadata, one write per nonzero
        alg_bytes = 8 * st["staging_values"] + 20 * st["n_blocks"] + 8 * st["nnz"]
        mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
        peak = json.load(open(mp))["hbm_gbs"] if os.path.exists(mp) else 6650.0
        roof = {"bound": "hbm", "unit": "GB/s",
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if os.path.exists(mp) else "fallback 6.65 TB/s"}
        achieved = alg_bytes / (per_kernel[dominant] / 1e3) / 1e9
    else:
        etype = dominant.split("_")[0]
        alg = roofline.kernel_flops(dominant, counts[etype])
        achieved = alg / (per_kernel[dominant] / 1e3) / 1e12
        peak = fp64_peak
        roof = {"bound": "tensor", "unit": "TFLOP/s",
                "peak_source": "FP64 DGEMM (torch.matmul float64 8192^3, best of 3) measured in this run"}
    roof.update({"kernel": dominant, "achieved": achieved, "peak": peak, "frac": achieved / peak,
                 "traffic": traffic.get(dominant), "launch_ms": per_kernel[dominant]})
    if roof["bound"] == "tensor":
        # hardware use: the FP64 flops the kernel executes (ncu counters), not the
        # reference's dense products that `achieved` counts
        ex = roofline.kernel_executed_flops(dominant, counts[dominant.split("_")[0]])
        if ex is not None:
            roof["executed_tflops"] = ex / (per_kernel[dominant] / 1e3) / 1e12
            roof["executed_frac"] = roof["executed_tflops"] / peak
            roof["note"] = ("achieved/frac count the canonical dense-product flops; executed_* count the "
                            "DFMA/DADD/DMUL the closed-form kernel issues (ncu counters, roofline.EXECUTED_FLOPS)")
    ms_step = elapsed / args.steps * 1e3
    h2d = 8 * m.ndof
    kg_live = g.kg_transfer_entries()       # KG entries moved by the pageable call (-1: the whole pattern)
    d2h = 8 * g.nnz + 8 * (kg_live if kg_live >= 0 else g.nnz) + 8 * m.ndof + 8
    launches_per_step = (sum(1 for t in ("quad4", "tria3", "bar") if counts[t] > 0) * 2
                         + 2 * (1 if st["dof_contribs"] else 0) + 2 + 1)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong" if part else "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded deck generator; smooth seeded displacement for KG)",
            "config": (dict(workload_config(m, args.workload, world), parallelism=f"replicas x{world}", nnz=g.nnz)
                       if part is None else
                       dict(workload_config(full, args.workload, 1), parallelism=f"row blocks x{world}",
                            part_elements_rank0=int(n_el), halo_elements=int(sum(
                                partition.part_of(full, r, world).model.n_elements for r in range(world))
                                - full.n_elements))),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "host_memory": "pageable (numpy arrays, as a Julia Vector{Float64})",
                    "kg_live_entries": kg_live, "note": "pageable copies run through a pinned ring with host threads "
                    "writing non-temporal stores; KG sends only its live entries (d2h_bytes_per_step counts them) "
                    "and the host threads expand them; pinned_value: caller-pinned arrays, one DMA each",
                    "pinned_value": e2e_pinned_value},
            "roofline": roof, "gpu_launches": launches_per_step * args.steps, "clocks": clk,
            "kernel_ms": per_kernel, "fp64_dgemm_tflops": fp64_peak, "model_stats": st,
            "launch_config": dict(launch_cfg, autotuned=not args.no_autotune, tune_s=round(t_tune, 3)),
            **({"row_split": {"gather_owned_k_ms": gather_ms, "note": "NCCL all-gather of every rank's owned K "
                              "columns, timed once after the step; the assembly itself has no collective"}}
               if part is not None else {}),
            "whole_step_roofline": {"flops": roofline.flops_per_step(counts), "bytes": roofline.bytes_per_step(counts, g.nnz)},
            "recovery": {"ms": rec_ms, "elements_per_s": n_el / rec_ms * 1e3, "timed_calls": 5,
                         "output_bytes": 8 * (rec_sh.numel() + (rec_bar.numel() if counts["bar"] else 0)),
                         "note": "jfg_recover_stresses_device on the same model and u, outside the timed step"}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "barrel":
        v, thr, sample, phases = time_cpu_oracle(m, args.cpu_seconds)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample,
                                "phases": phases, "same_config": True}
        line["recovery"]["cpu_port_elements_per_s"] = time_cpu_recovery()
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
